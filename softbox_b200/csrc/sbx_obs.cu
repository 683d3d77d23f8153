// sbx_obs.cu — per-network observables of dense networks (single or packed): the filament
// RMS extent (FullSystemDemoHarness.filRms, FullSystemDemoHarness.java:1047-1055), the
// largest-cluster fraction, and the mean in-plane network stress.
//
// Reductions are deterministic: one block per network, thread t sums items t, t+256, ...
// of its network in index order in FP64, then a fixed shared-memory tree (strides 128 ..
// 1). The oracle restates this order, so results are bit-identical to it (and equal the
// reference's serial sums to ~1e-13 relative).
//
// Clusters: nodes are the segments and the backbones; edges are chain links, ACTIVE
// crosslinks and bound heads (segment -- the head's backbone). Roots hook onto the smaller
// root with atomicMin and paths are compressed every round; the final label of a node is
// the smallest node id of its component, so the labelling does not depend on the order in
// which edges are processed.
#include <cuda_runtime.h>

#include "../../include/softbox_b200.h"
#include "sbx_internal.cuh"

namespace {

constexpr int OBS_THREADS = 256;
constexpr int OBS_MAX_FIND = 1 << 20;

__device__ __forceinline__ void tree_sum(double* sh, int w) {
    for (int s = OBS_THREADS / 2; s > 0; s >>= 1) {
        __syncthreads();
        if (threadIdx.x < s)
            for (int k = 0; k < w; k++) sh[k * OBS_THREADS + threadIdx.x] += sh[k * OBS_THREADS + threadIdx.x + s];
    }
    __syncthreads();
}

__device__ __forceinline__ double seg_c(const float* c, const double* c64, int n, int i, int k) {
    return c64 ? c64[(int64_t)k * n + i] : (double)c[(int64_t)k * n + i];
}

// out[2*net] = RMS extent (um), out[2*net+1] = active segment count
__global__ void __launch_bounds__(OBS_THREADS) k_extent(int n, const int* segBase, const float* coord,
                                                        const double* coord64, const int* filState, double* out) {
    __shared__ double sh[4 * OBS_THREADS];
    __shared__ double mean[4];
    int net = blockIdx.x, t = threadIdx.x;
    int b0 = segBase[net], b1 = segBase[net + 1];
    double cnt = 0, sx = 0, sy = 0, sz = 0;
    for (int i = b0 + t; i < b1; i += OBS_THREADS) {
        if (filState && filState[i] < 0) continue;
        cnt += 1.0;
        sx += seg_c(coord, coord64, n, i, 0);
        sy += seg_c(coord, coord64, n, i, 1);
        sz += seg_c(coord, coord64, n, i, 2);
    }
    sh[t] = cnt; sh[OBS_THREADS + t] = sx; sh[2 * OBS_THREADS + t] = sy; sh[3 * OBS_THREADS + t] = sz;
    tree_sum(sh, 4);
    if (t == 0) {
        double c = sh[0];
        mean[0] = c;
        mean[1] = c > 0 ? sh[OBS_THREADS] / c : 0.0;
        mean[2] = c > 0 ? sh[2 * OBS_THREADS] / c : 0.0;
        mean[3] = c > 0 ? sh[3 * OBS_THREADS] / c : 0.0;
    }
    __syncthreads();
    double mx = mean[1], my = mean[2], mz = mean[3], s2 = 0;
    for (int i = b0 + t; i < b1; i += OBS_THREADS) {
        if (filState && filState[i] < 0) continue;
        double dx = seg_c(coord, coord64, n, i, 0) - mx;
        double dy = seg_c(coord, coord64, n, i, 1) - my;
        double dz = seg_c(coord, coord64, n, i, 2) - mz;
        s2 += dx * dx + dy * dy + dz * dz;
    }
    sh[t] = s2;
    tree_sum(sh, 1);
    if (t == 0) {
        double c = mean[0];
        out[2 * net] = c > 0 ? sqrt(sh[0] / c) : 0.0;
        out[2 * net + 1] = c;
    }
}

// virial of the link and bond payloads: out[net] = -(sum r_x F_x + r_y F_y) / (2 V), Pa
__global__ void __launch_bounds__(OBS_THREADS) k_stress(
    int nSeg, const float* fC, const float* fU, const float* fE1, const float* fLen, const int* linkBase,
    const int* linkA, const int* linkB, const int* linkState, const float* loc1, const float* loc2, const float* xd,
    int nB, const int* motBase, const float* mC, const float* mU, const int* boundSeg, const float* bindArc,
    const float* bd, double headLen, const float* volume, double* out) {
    __shared__ double sh[OBS_THREADS];
    int net = blockIdx.x, t = threadIdx.x;
    double w = 0;
    if (linkBase)
        for (int k = linkBase[net] + t; k < linkBase[net + 1]; k += OBS_THREADS) {
            if (linkState[k] < 0) continue;
            int a = linkA[k], b = linkB[k];
            if (a < 0 || b < 0) continue;
            double l1 = loc1[k], l2 = loc2[k];
            double rx = (fE1[a] + l1 * fU[a]) - (fE1[b] + l2 * fU[b]);
            double ry = (fE1[nSeg + a] + l1 * fU[nSeg + a]) - (fE1[nSeg + b] + l2 * fU[nSeg + b]);
            w += 1.0e-6 * rx * xd[12 * (int64_t)k] + 1.0e-6 * ry * xd[12 * (int64_t)k + 1];
        }
    if (motBase)
        for (int m = motBase[net] + t; m < motBase[net + 1]; m += OBS_THREADS) {
            int s = boundSeg[m];
            if (s < 0) continue;
            int h = 3 * m + 2;
            double hx = mC[h] + 0.5 * headLen * mU[h], hy = mC[nB + h] + 0.5 * headLen * mU[nB + h];
            double off = (double)bindArc[m] - 0.5 * fLen[s];
            double ax = fC[s] + off * fU[s], ay = fC[nSeg + s] + off * fU[nSeg + s];
            w += 1.0e-6 * (hx - ax) * bd[13 * (int64_t)m] + 1.0e-6 * (hy - ay) * bd[13 * (int64_t)m + 1];
        }
    sh[t] = w;
    tree_sum(sh, 1);
    if (t == 0) out[net] = -sh[0] / (2.0 * volume[net] * 1.0e-18);
}

// ---------------------------------------------------------------- clusters
__device__ __forceinline__ int find_root(const int* label, int x) {
    for (int it = 0; it < OBS_MAX_FIND; it++) {
        int p = label[x];
        if (p == x) return x;
        x = p;
    }
    return x;
}

__global__ void k_cl_init(int nSeg, int nNode, const int* filState, int* label, int* size, int* flags, int rounds) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nNode) {
        label[i] = (i < nSeg && filState && filState[i] < 0) ? -1 : i;
        size[i] = 0;
    }
    if (i <= rounds) flags[i] = 0;
}

// one hooking pass over every edge kind; flags[r] = 1 when anything changed
__global__ void k_cl_hook(int r, int nSeg, const int* e2, int nLinks, const int* linkA, const int* linkB,
                          const int* linkState, int nM, const int* boundSeg, const int* motorBackbone, int* label,
                          int* flags) {
    if (r > 0 && flags[r - 1] == 0) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int u = -1, v = -1;
    if (i < nSeg) {
        u = i;
        v = e2[i];
    } else if (i < nSeg + nLinks) {
        int k = i - nSeg;
        if (linkState[k] >= 0) { u = linkA[k]; v = linkB[k]; }
    } else if (i < nSeg + nLinks + nM) {
        int m = i - nSeg - nLinks;
        int s = boundSeg[m];
        if (s >= 0 && motorBackbone[m] >= 0) { u = s; v = nSeg + motorBackbone[m]; }
    }
    if (u < 0 || v < 0 || u == v || label[u] < 0 || label[v] < 0) return;
    int ru = find_root(label, u), rv = find_root(label, v);
    if (ru == rv) return;
    int hi = ru > rv ? ru : rv, lo = ru > rv ? rv : ru;
    if (atomicMin(&label[hi], lo) > lo) flags[r] = 1;
}

__global__ void k_cl_compress(int r, int nNode, int* label, int* flags) {
    if (r > 0 && flags[r - 1] == 0) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nNode || label[i] < 0) return;
    int root = find_root(label, i);
    if (label[i] != root) {
        label[i] = root;
        flags[r] = 1;
    }
}

__global__ void k_cl_size(int nSeg, const int* label, int* size) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nSeg && label[i] >= 0) atomicAdd(&size[label[i]], 1);
}

// out[2*net] = largest component size (segments), out[2*net+1] = active segments
__global__ void __launch_bounds__(OBS_THREADS) k_cl_largest(const int* segBase, const int* label, const int* size,
                                                            int* out) {
    __shared__ int shMax[OBS_THREADS], shCnt[OBS_THREADS];
    int net = blockIdx.x, t = threadIdx.x;
    int best = 0, cnt = 0;
    for (int i = segBase[net] + t; i < segBase[net + 1]; i += OBS_THREADS) {
        int l = label[i];
        if (l < 0) continue;
        cnt++;
        int s = size[l];
        best = s > best ? s : best;
    }
    shMax[t] = best; shCnt[t] = cnt;
    for (int s = OBS_THREADS / 2; s > 0; s >>= 1) {
        __syncthreads();
        if (t < s) {
            shMax[t] = max(shMax[t], shMax[t + s]);
            shCnt[t] += shCnt[t + s];
        }
    }
    if (t == 0) { out[2 * net] = shMax[0]; out[2 * net + 1] = shCnt[0]; }
}

}  // namespace

extern "C" sbx_status sbx_obs_extent(sbx_ctx* ctx, int32_t nNet, const int32_t* segBase, int32_t nSeg,
                                     const float* coord, const double* coord64, const int32_t* filState,
                                     double* out) {
    SBX_REQUIRE(ctx && nNet >= 0 && nSeg >= 0 && (nNet == 0 || (segBase && (coord || coord64) && out)));
    if (nNet == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_extent, nNet, OBS_THREADS, nSeg, segBase, coord, coord64, filState, out);
    return check_launch(ctx, "sbx_obs_extent");
}

extern "C" sbx_status sbx_obs_stress(sbx_ctx* ctx, int32_t nNet, int32_t nSeg, const float* coord, const float* uVec,
                                     const float* end1, const float* segLength, const int32_t* linkBase,
                                     const int32_t* linkFilA, const int32_t* linkFilB, const int32_t* linkState,
                                     const float* loc1, const float* loc2, const float* xlinkData, int32_t nMotors,
                                     const int32_t* motBase, const float* motCoord, const float* motUVec,
                                     const int32_t* boundSeg, const float* bindArc, const float* bondData,
                                     double headLen, const float* volume, double* out) {
    SBX_REQUIRE(ctx && nNet >= 0 && nSeg >= 0 && nMotors >= 0);
    if (nNet == 0) return SBX_OK;
    SBX_REQUIRE(coord && uVec && end1 && segLength && volume && out &&
                (!linkBase || (linkFilA && linkFilB && linkState && loc1 && loc2 && xlinkData)) &&
                (!motBase || (motCoord && motUVec && boundSeg && bindArc && bondData)));
    SBX_LAUNCH(ctx, k_stress, nNet, OBS_THREADS, nSeg, coord, uVec, end1, segLength, linkBase, linkFilA, linkFilB,
               linkState, loc1, loc2, xlinkData, 3 * nMotors, motBase, motCoord, motUVec, boundSeg, bindArc, bondData,
               headLen, volume, out);
    return check_launch(ctx, "sbx_obs_stress");
}

extern "C" sbx_status sbx_obs_clusters(sbx_ctx* ctx, int32_t nNet, const int32_t* segBase, int32_t nSeg,
                                       const int32_t* filState, const int32_t* end2NbrSlot, int32_t nLinks,
                                       const int32_t* linkFilA, const int32_t* linkFilB, const int32_t* linkState,
                                       int32_t nMotors, const int32_t* boundSeg, const int32_t* motorBackbone,
                                       int32_t nBackbones, int32_t rounds, int32_t* label, int32_t* size,
                                       int32_t* flags, int32_t* out) {
    SBX_REQUIRE(ctx && nNet >= 0 && nSeg >= 0 && nLinks >= 0 && nMotors >= 0 && nBackbones >= 0 && rounds >= 1);
    if (nNet == 0) return SBX_OK;
    SBX_REQUIRE(segBase && end2NbrSlot && label && size && flags && out && (nLinks == 0 || (linkFilA && linkFilB &&
                linkState)) && (nMotors == 0 || (boundSeg && motorBackbone)));
    int nNode = nSeg + nBackbones;
    int nInit = nNode > rounds + 1 ? nNode : rounds + 1;
    SBX_LAUNCH(ctx, k_cl_init, blocks(nInit), 256, nSeg, nNode, filState, label, size, flags, rounds);
    int nEdge = nSeg + nLinks + nMotors;
    for (int r = 0; r < rounds; r++) {
        SBX_LAUNCH(ctx, k_cl_hook, blocks(nEdge > 0 ? nEdge : 1), 256, r, nSeg, end2NbrSlot, nLinks, linkFilA,
                   linkFilB, linkState, nMotors, boundSeg, motorBackbone, label, flags);
        SBX_LAUNCH(ctx, k_cl_compress, blocks(nNode > 0 ? nNode : 1), 256, r, nNode, label, flags);
    }
    SBX_LAUNCH(ctx, k_cl_size, blocks(nSeg > 0 ? nSeg : 1), 256, nSeg, label, size);
    SBX_LAUNCH(ctx, k_cl_largest, nNet, OBS_THREADS, segBase, label, size, out);
    return check_launch(ctx, "sbx_obs_clusters");
}
