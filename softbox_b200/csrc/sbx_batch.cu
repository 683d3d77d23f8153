// sbx_batch.cu — many independent dense networks packed into one set of store arrays.
//
// Network k owns a contiguous index range in every store (segments, motors, backbones,
// links) and its own grid cells [gridDims[4k+3], +nX*nY*nZ), so one launch per step phase
// advances every network. Only the kernels whose result depends on more than the item's
// own indices need the network: the RNG draws (keyed by the item's LOCAL index and its
// network's seed, exactly as the network run alone), the grid cell of a body and the
// motor's stencil walk (the network's own grid), and the walls (the network's own box).
// Every other kernel of the step is the single-network one over the packed arrays, whose
// cross-store indices the packer offsets. A packed run therefore equals, bit for bit, each
// network run alone.
#include <cuda_runtime.h>

#include "../../include/softbox_b200.h"
#include "sbx_internal.cuh"
#include "sbx_physics.cuh"

using namespace sbx;

namespace {

__device__ __forceinline__ void ld3(const float* a, int n, int i, float v[3]) {
    v[0] = a[i]; v[1] = a[n + i]; v[2] = a[2 * n + i];
}
__device__ __forceinline__ void st3(float* a, int n, int i, const float v[3]) {
    a[i] = v[0]; a[n + i] = v[1]; a[2 * n + i] = v[2];
}

// key[i] = (network, local index); motor bodies use their motor's key (3 bodies per motor)
__device__ __forceinline__ int2 item_key(const int* key, int i, int per) {
    int m = per == 3 ? i / 3 : i;
    int2 k = make_int2(key[2 * m], key[2 * m + 1]);
    if (per == 3) k.y = 3 * k.y + (i - 3 * m);
    return k;
}

__global__ void k_brownian_b(int n, int per, float* rF, float* rT, const float* bTG, const float* bRG,
                             const float* tSc, const float* rSc, const float* params, const int* counts,
                             const int* key, const int* seeds, int seedCol) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int2 k = item_key(key, i, per);
    float g[6];
    gauss6_wang(k.y, counts[1], seeds[3 * k.x + seedCol], g);
    float gT[3] = {bTG[i], bTG[n + i], bTG[2 * n + i]};
    float gR[3] = {bRG[i], bRG[n + i], bRG[2 * n + i]};
    float rf[3], rt[3];
    brownian_amplitudes(g, tSc[i], rSc[i], params[1], gT, gR, rf, rt);
    for (int c = 0; c < 3; c++) { rF[c * n + i] = rf[c]; rT[c * n + i] = rt[c]; }
}

__global__ void k_release_b(int nM, int* boundSeg, const float* fdf, const float* fm, int* cooldown, int* stats,
                            int* capStats, const float* kp, const int* counts, const int* key, const int* seeds) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nM) return;
    int2 k = item_key(key, m, 1);
    int bs = boundSeg[m], cd = cooldown[m], sb = stats[2 * m], sr = stats[2 * m + 1], cs = capStats[m];
    release_one(k.y, bs, cd, sb, sr, cs, fdf[m], fm[m], kp, counts[1], seeds[3 * k.x]);
    boundSeg[m] = bs; cooldown[m] = cd; stats[2 * m] = sb; stats[2 * m + 1] = sr; capStats[m] = cs;
}

__global__ void k_cycle_b(int nM, int* state, const int* boundSeg, const float* hist, const float* np,
                          const int* counts, const int* key, const int* seeds) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nM) return;
    int2 k = item_key(key, m, 1);
    state[m] = cycle_one(k.y, state[m], boundSeg[m] >= 0, hist + 10 * m, np, counts[1], seeds[3 * k.x]);
}

__global__ void k_xl_unbind_b(int nSeg, const float* fU, const float* fE1, int nLinks, const int* A, const int* B,
                              const float* loc1, const float* loc2, int* state, float* hist, int* place,
                              const float* op, const int* counts, const int* key, const int* seeds) {
    int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nLinks || state[l] < 0) return;
    int2 k = item_key(key, l, 1);
    // unbind_one keys its draw by the link index and indexes the strain ring by it: shift the
    // ring pointers so that the local index addresses this link's own ring
    int off = l - k.y;
    if (unbind_one(k.y, nSeg, fU, fE1, A[l], B[l], loc1[l], loc2[l], hist + (int64_t)off * STRAIN_WIN, place + off,
                   op, counts[1], seeds[3 * k.x]))
        state[l] = LINK_FREE;
}

// body view: slots [0, nSeg) are segments, [nSeg, S) motor heads
__global__ void k_body_cell_b(int cap, const float* center, const int* counts, int* bodyCell, int nSeg,
                              const int* segKey, const int* motKey, const float* gpTab, const int* gdTab) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cap) return;
    int S = counts[1];
    if (i >= S) { bodyCell[i] = -1; return; }
    int net = i < nSeg ? segKey[2 * i] : motKey[2 * (i - nSeg)];
    const float* gp = gpTab + 6 * net;
    const int* gd = gdTab + 4 * net;
    int nX = gd[0], nY = gd[1], nZ = gd[2];
    int ix = cell_coord(center[i], gp[0], gp[4], nX);
    int iy = cell_coord(center[cap + i], gp[1], gp[4], nY);
    int iz = cell_coord(center[2 * cap + i], gp[2], gp[4], nZ);
    bodyCell[i] = gd[3] + ix + iy * nX + iz * (nX * nY);
}

__global__ void k_grid_reachable_b(int nM, const float* head, const float* uVec, const float* rodUVec, int nSeg,
                                   const float* e1, const float* e2, const int* offsets, const int* contents,
                                   const int* ownerStore, const int* ownerSlot, int* reachSeg, int* reachCount,
                                   const float* kp, const int* motKey, const float* gpTab, const int* gdTab) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nM) return;
    int net = motKey[2 * m];
    const int* gd = gdTab + 4 * net;
    reachCount[m] = grid_reach_walk(m, nM, head, uVec, rodUVec, nSeg, e1, e2, gpTab + 6 * net, gd, offsets + gd[3],
                                    contents, ownerStore, ownerSlot, reachSeg + (int64_t)m * MAX_CAND, kp[7], kp[8]);
}

__global__ void k_grid_reachable_cells_b(int nM, const float* head, const float* uVec, const float* rodUVec,
                                         const int* offsets, const float4* cellE1, const float4* cellE2,
                                         int* reachSeg, int* reachCount, const float* kp, const int* motKey,
                                         const float* gpTab, const int* gdTab) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nM) return;
    int net = motKey[2 * m];
    const int* gd = gdTab + 4 * net;
    reachCount[m] = grid_reach_walk_cells(m, nM, head, uVec, rodUVec, gpTab + 6 * net, gd, offsets + gd[3], cellE1,
                                          cellE2, reachSeg + (int64_t)m * MAX_CAND, kp[7], kp[8]);
}

__global__ void k_confine_b(int n, const float* coord, const float* uVec, const float* segLength, const float* bTG,
                            float* F, float* T, const float* bpTab, const int* counts, const int* key) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    BoxParams bx = box_params(bpTab + 8 * key[2 * i], counts[1]);
    if (!bx.active) return;
    float c[3], u[3], f[3], t[3];
    ld3(coord, n, i, c); ld3(uVec, n, i, u); ld3(F, n, i, f); ld3(T, n, i, t);
    if (confine_one(bx, c, u, segLength[i], bTG[i], f, t)) {
        st3(F, n, i, f);
        st3(T, n, i, t);
    }
}

}  // namespace

#define SBX_DONE(name) return check_launch(ctx, name)

extern "C" sbx_status sbx_brownian_force_batched(sbx_ctx* ctx, int32_t n, int32_t perKey, float* rF, float* rT,
                                                 const float* bTG, const float* bRG, const float* tSc,
                                                 const float* rSc, const float* params, const int32_t* counts,
                                                 const int32_t* key, const int32_t* seeds, int32_t seedCol) {
    SBX_REQUIRE(ctx && n >= 0 && (perKey == 1 || perKey == 3) && seedCol >= 0 && seedCol < 3 &&
                (n == 0 || (rF && rT && bTG && bRG && tSc && rSc && params && counts && key && seeds)));
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_brownian_b, blocks(n), 256, n, perKey, rF, rT, bTG, bRG, tSc, rSc, params, counts, key, seeds,
               seedCol);
    SBX_DONE("sbx_brownian_force_batched");
}

extern "C" sbx_status sbx_nucleotide_release_batched(sbx_ctx* ctx, int32_t nM, int32_t* boundSeg, const float* fdf,
                                                     const float* fm, int32_t* cooldown, int32_t* stats,
                                                     int32_t* capStats, const float* kp, const int32_t* counts,
                                                     const int32_t* motKey, const int32_t* seeds) {
    SBX_REQUIRE(ctx && nM >= 0 && (nM == 0 || (boundSeg && fdf && fm && cooldown && stats && capStats && kp &&
                                               counts && motKey && seeds)));
    if (nM == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_release_b, blocks(nM), 256, nM, boundSeg, fdf, fm, cooldown, stats, capStats, kp, counts,
               motKey, seeds);
    SBX_DONE("sbx_nucleotide_release_batched");
}

extern "C" sbx_status sbx_nucleotide_cycle_batched(sbx_ctx* ctx, int32_t nM, int32_t* state, const int32_t* boundSeg,
                                                   const float* hist, const float* np, const int32_t* counts,
                                                   const int32_t* motKey, const int32_t* seeds) {
    SBX_REQUIRE(ctx && nM >= 0 && (nM == 0 || (state && boundSeg && hist && np && counts && motKey && seeds)));
    if (nM == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_cycle_b, blocks(nM), 256, nM, state, boundSeg, hist, np, counts, motKey, seeds);
    SBX_DONE("sbx_nucleotide_cycle_batched");
}

extern "C" sbx_status sbx_xlink_unbind_batched(sbx_ctx* ctx, int32_t nSeg, const float* fU, const float* fE1,
                                               int32_t nLinks, const int32_t* A, const int32_t* B, const float* loc1,
                                               const float* loc2, int32_t* state, float* hist, int32_t* place,
                                               const float* op, const int32_t* counts, const int32_t* linkKey,
                                               const int32_t* seeds) {
    SBX_REQUIRE(ctx && nLinks >= 0 && (nLinks == 0 || (fU && fE1 && A && B && loc1 && loc2 && state && hist && place &&
                                                       op && counts && linkKey && seeds)));
    if (nLinks == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_xl_unbind_b, blocks(nLinks), 256, nSeg, fU, fE1, nLinks, A, B, loc1, loc2, state, hist, place,
               op, counts, linkKey, seeds);
    SBX_DONE("sbx_xlink_unbind_batched");
}

extern "C" sbx_status sbx_grid_body_cell_batched(sbx_ctx* ctx, int32_t cap, const float* center,
                                                 const int32_t* counts, int32_t* bodyCell, int32_t nSeg,
                                                 const int32_t* segKey, const int32_t* motKey, const float* gpTab,
                                                 const int32_t* gdTab) {
    SBX_REQUIRE(ctx && cap >= 0 && nSeg >= 0 &&
                (cap == 0 || (center && counts && bodyCell && segKey && motKey && gpTab && gdTab)));
    if (cap == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_body_cell_b, blocks(cap), 256, cap, center, counts, bodyCell, nSeg, segKey, motKey, gpTab,
               gdTab);
    SBX_DONE("sbx_grid_body_cell_batched");
}

extern "C" sbx_status sbx_binding_grid_reachable_batched(sbx_ctx* ctx, const float* head, const float* uVec,
                                                         const float* rodUVec, int32_t nSeg, const float* e1,
                                                         const float* e2, const int32_t* offsets,
                                                         const int32_t* contents, const int32_t* ownerStore,
                                                         const int32_t* ownerSlot, int32_t* reachSeg,
                                                         int32_t* reachCount, const float* kp, int32_t nM,
                                                         const int32_t* motKey, const float* gpTab,
                                                         const int32_t* gdTab) {
    SBX_REQUIRE(ctx && nM >= 0 && (nM == 0 || (head && uVec && rodUVec && e1 && e2 && offsets && contents &&
                                               ownerStore && ownerSlot && reachSeg && reachCount && kp && motKey &&
                                               gpTab && gdTab)));
    if (nM == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_grid_reachable_b, blocks(nM, 128), 128, nM, head, uVec, rodUVec, nSeg, e1, e2, offsets,
               contents, ownerStore, ownerSlot, reachSeg, reachCount, kp, motKey, gpTab, gdTab);
    SBX_DONE("sbx_binding_grid_reachable_batched");
}

extern "C" sbx_status sbx_fusion_grid_reachable_batched(sbx_ctx* ctx, const float* head, const float* uVec,
                                                        const float* rodUVec, const int32_t* gridCellOffsets,
                                                        const float* cellEnd1, const float* cellEnd2,
                                                        int32_t* reachSeg, int32_t* reachCount, const float* kp,
                                                        int32_t nM, const int32_t* motKey, const float* gpTab,
                                                        const int32_t* gdTab) {
    SBX_REQUIRE(ctx && nM >= 0 && (nM == 0 || (head && uVec && rodUVec && gridCellOffsets && cellEnd1 && cellEnd2 &&
                                               reachSeg && reachCount && kp && motKey && gpTab && gdTab)));
    if (nM == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_grid_reachable_cells_b, blocks(nM, 128), 128, nM, head, uVec, rodUVec, gridCellOffsets,
               reinterpret_cast<const float4*>(cellEnd1), reinterpret_cast<const float4*>(cellEnd2), reachSeg,
               reachCount, kp, motKey, gpTab, gdTab);
    SBX_DONE("sbx_fusion_grid_reachable_batched");
}

extern "C" sbx_status sbx_confine_batched(sbx_ctx* ctx, int32_t n, const float* coord, const float* uVec,
                                          const float* segLength, const float* bTG, float* F, float* T,
                                          const float* boxTab, const int32_t* counts, const int32_t* key) {
    SBX_REQUIRE(ctx && n >= 0 && (n == 0 || (coord && uVec && segLength && bTG && F && T && boxTab && counts && key)));
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_confine_b, blocks(n), 256, n, coord, uVec, segLength, bTG, F, T, boxTab, counts, key);
    SBX_DONE("sbx_confine_batched");
}
