// sbx_sort.cu — the stable counting sort behind the spatial grid and every CSR-inverse.
//
// Replaces SpatialGrid.gridHistogram/gridScanLocal/gridScanChunks/gridScanAdd/
// gridScatter (SpatialGrid.java:87-182) and CrossBridgeSystem.csrHistogram/csrScan/
// csrScatter (CrossBridgeSystem.java:190-217), plus their chunk-matrix variants, with:
//   1. atomic histogram of the keys (integer atomics: the counts are order-free);
//   2. exclusive scan in SCAN_CHUNK = 512 tiles: per-tile block scan, one-block scan of
//      the tile sums (chunkSum, with the grand total in chunkSum[numChunks]), tile add
//      that also resets the counts to zero (the reference's write cursor);
//   3. unordered atomic scatter into a scratch list;
//   4. rank pass: each item's position inside its row = the number of row members with a
//      smaller index, which reproduces the reference's ascending-index order exactly.
// Results (offsets, lists, counts, chunkSum) equal the serial reference bit for bit.
#include <cuda_runtime.h>

#include "sbx_internal.cuh"

namespace {

__device__ __forceinline__ int item_count(const int* nDev, int useDevN, int nBound) {
    if (!useDevN) return nBound;
    int n = nDev[1];
    return n < nBound ? n : nBound;
}

// a key names a row: keys < 0 are unbound items (skipped, as the reference does); a key at
// or past the row count would index past the row arrays, so the item is skipped and the
// caller's error word is set
__device__ __forceinline__ bool key_ok(int c, int nRows, int* errFlag) {
    if (c < nRows) return c >= 0;
    if (errFlag) *(volatile int*)errFlag = 1;
    return false;
}

__global__ void k_cs_hist(const int* keys, const int* nDev, int useDevN, int nBound, int nRows, int* rowCount,
                          int* errFlag) {
    int n = item_count(nDev, useDevN, nBound);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int c = keys[i];
        if (key_ok(c, nRows, errFlag)) atomicAdd(&rowCount[c], 1);
    }
}

// block-wide exclusive scan of one int per thread; returns the exclusive prefix, *total = sum
template <int NT>
__device__ __forceinline__ int block_exclusive_scan(int v, int* total) {
    __shared__ int warp_sums[NT / 32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = (lane < NT / 32) ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < NT / 32) warp_sums[lane] = w;
    }
    __syncthreads();
    int warp_prefix = warp > 0 ? warp_sums[warp - 1] : 0;
    *total = warp_sums[NT / 32 - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

// SpatialGrid.gridScanLocal (SpatialGrid.java:99-117), one block per 512-row tile
__global__ void __launch_bounds__(256) k_scan_local(const int* rowCount, int nRows, int* offsets, int* chunkSum) {
    int base = blockIdx.x * SCAN_CHUNK;
    int i0 = base + 2 * threadIdx.x, i1 = i0 + 1;
    int v0 = i0 < nRows ? rowCount[i0] : 0;
    int v1 = i1 < nRows ? rowCount[i1] : 0;
    int total;
    int ex = block_exclusive_scan<256>(v0 + v1, &total);
    if (i0 < nRows) offsets[i0] = ex;
    if (i1 < nRows) offsets[i1] = ex + v0;
    if (threadIdx.x == 0) chunkSum[blockIdx.x] = total;
}

// SpatialGrid.gridScanChunks (SpatialGrid.java:121-133) as a one-block scan with carry,
// eight consecutive tile sums per thread per pass
__global__ void __launch_bounds__(1024) k_scan_chunks(int* chunkSum, int numChunks) {
    constexpr int PER = 8;
    int carry = 0;
    for (int t0 = 0; t0 < numChunks; t0 += 1024 * PER) {
        int base = t0 + threadIdx.x * PER;
        int v[PER];
        int sum = 0;
#pragma unroll
        for (int j = 0; j < PER; j++) {
            v[j] = base + j < numChunks ? chunkSum[base + j] : 0;
            sum += v[j];
        }
        int total;
        int ex = block_exclusive_scan<1024>(sum, &total);
        int run = carry + ex;
#pragma unroll
        for (int j = 0; j < PER; j++) {
            if (base + j < numChunks) chunkSum[base + j] = run;
            run += v[j];
        }
        carry += total;
    }
    if (threadIdx.x == 0) chunkSum[numChunks] = carry;
}

// The counting sort's exclusive scan (SpatialGrid.gridScanLocal / gridScanChunks / gridScanAdd,
// SpatialGrid.java:99-160, with the same outputs) as reduce-then-scan over tiles of
// SCAN_TILE_ROWS = 8 scan chunks: k_tile_reduce writes each tile's sum; k_tile_scan adds the
// sums of the preceding tiles itself (a strided block reduction, no single-block pass and no
// inter-block wait), scans its tile through shared memory and writes offsets, the chunk
// prefixes chunkSum[c] (chunkSum[numChunks] = the total), offsets[nRows] = min(total, listCap),
// and resets the counts to zero (the scatter cursor).
constexpr int SCAN_TILE_ROWS = 8 * SCAN_CHUNK;
constexpr int TILE_PER_THREAD = SCAN_TILE_ROWS / 256;

__device__ __forceinline__ int tile_slot(int r) { return r + (r >> 5); }     // padded: no bank conflicts

__global__ void __launch_bounds__(256) k_tile_reduce(const int* rowCount, int nRows, int* tileSum) {
    const int base = blockIdx.x * SCAN_TILE_ROWS;
    int s = 0;
#pragma unroll
    for (int k = 0; k < TILE_PER_THREAD; k++) {
        int r = base + threadIdx.x + 256 * k;
        if (r < nRows) s += rowCount[r];
    }
    int total;
    block_exclusive_scan<256>(s, &total);
    if (threadIdx.x == 0) tileSum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(256) k_tile_scan(int* rowCount, int nRows, int* offsets, int* chunkSum, int numChunks,
                                                   const int* tileSum, int listCap) {
    __shared__ int sv[SCAN_TILE_ROWS + SCAN_TILE_ROWS / 32];
    const int tile = blockIdx.x, base = tile * SCAN_TILE_ROWS;
    int p = 0;
    for (int k = threadIdx.x; k < tile; k += 256) p += tileSum[k];
    int prefix;
    block_exclusive_scan<256>(p, &prefix);
#pragma unroll
    for (int k = 0; k < TILE_PER_THREAD; k++) {
        int r = threadIdx.x + 256 * k, g = base + r;
        sv[tile_slot(r)] = g < nRows ? rowCount[g] : 0;
    }
    __syncthreads();
    int v[TILE_PER_THREAD], s = 0;
#pragma unroll
    for (int k = 0; k < TILE_PER_THREAD; k++) {
        v[k] = sv[tile_slot(TILE_PER_THREAD * threadIdx.x + k)];
        s += v[k];
    }
    int tot;
    int run = block_exclusive_scan<256>(s, &tot);
#pragma unroll
    for (int k = 0; k < TILE_PER_THREAD; k++) {
        sv[tile_slot(TILE_PER_THREAD * threadIdx.x + k)] = run;
        run += v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < TILE_PER_THREAD; k++) {
        int r = threadIdx.x + 256 * k, g = base + r;
        if (g < nRows) {
            offsets[g] = prefix + sv[tile_slot(r)];
            rowCount[g] = 0;
        }
    }
    if (threadIdx.x < SCAN_TILE_ROWS / SCAN_CHUNK) {
        int c = tile * (SCAN_TILE_ROWS / SCAN_CHUNK) + threadIdx.x;
        if (c < numChunks) chunkSum[c] = prefix + sv[tile_slot(threadIdx.x * SCAN_CHUNK)];
    }
    if (tile == gridDim.x - 1 && threadIdx.x == 0) {
        int total = prefix + tot;
        chunkSum[numChunks] = total;
        offsets[nRows] = total < listCap ? total : listCap;
    }
}

__global__ void k_cs_scatter(const int* keys, const int* nDev, int useDevN, int nBound, int nRows,
                             const int* offsets, int* rowCount, int* tmp) {
    int n = item_count(nDev, useDevN, nBound);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int c = keys[i];
        if (c < 0 || c >= nRows) continue;
        tmp[offsets[c] + atomicAdd(&rowCount[c], 1)] = i;
    }
}

__global__ void k_cs_rank(const int* keys, const int* nDev, int useDevN, int nBound, int nRows, const int* offsets,
                          const int* tmp, int* rowList, int listCap, const float* payload, int pStride, int pOff,
                          const int* guard, float* rowPayload) {
    int n = item_count(nDev, useDevN, nBound);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int c = keys[i];
        if (c < 0 || c >= nRows) continue;
        int start = offsets[c], end = offsets[c + 1];
        int rank = 0;
        for (int j = start; j < end; j++) rank += tmp[j] < i;
        int pos = start + rank;
        if (pos >= listCap) continue;
        rowList[pos] = i;
        if (rowPayload) {
            // 6 floats at pos: a row's items end up contiguous, so a gather reads them in order
            float v[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            if (!guard || guard[i] >= 0) {
                const float* q = payload + (int64_t)i * pStride + pOff;
                for (int j = 0; j < 6; j++) v[j] = q[j];
            }
            float2* o = reinterpret_cast<float2*>(rowPayload + 6 * (int64_t)pos);
            o[0] = make_float2(v[0], v[1]);
            o[1] = make_float2(v[2], v[3]);
            o[2] = make_float2(v[4], v[5]);
        }
    }
}

// exclusive_scan's tile add: out += tile prefix; the input optionally reset (csrScan's
// cursor side effect); out[n] = total
__global__ void __launch_bounds__(256) k_scan_add_plain(int* out, int n, const int* chunkSum, int numChunks, int* in,
                                                        int zeroIn) {
    int b = chunkSum[blockIdx.x];
    int base = blockIdx.x * SCAN_CHUNK;
    for (int k = threadIdx.x; k < SCAN_CHUNK; k += blockDim.x) {
        int c = base + k;
        if (c < n) {
            out[c] += b;
            if (zeroIn) in[c] = 0;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = chunkSum[numChunks];
}

}  // namespace

sbx_status exclusive_scan(sbx_ctx* ctx, int* in, int n, int* out, bool zeroIn, int* chunkSum, const char* what) {
    int numChunks = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;
    if (numChunks == 0) {
        if (cudaMemsetAsync(out, 0, sizeof(int), ctx->stream) != cudaSuccess)
            return fail(ctx, SBX_ECUDA, std::string(what) + ": memset");
        return SBX_OK;
    }
    SBX_LAUNCH(ctx, k_scan_local, numChunks, 256, in, n, out, chunkSum);
    SBX_LAUNCH(ctx, k_scan_chunks, 1, 1024, chunkSum, numChunks);
    SBX_LAUNCH(ctx, k_scan_add_plain, numChunks, 256, out, n, chunkSum, numChunks, in, zeroIn ? 1 : 0);
    return check_launch(ctx, what);
}

sbx_status counting_sort(sbx_ctx* ctx, const CountingSort& cs, const char* what) {
    if (!cs.tileSum) return fail(ctx, SBX_EINVAL, std::string(what) + ": no tile-sum scratch");
    int numChunks = (cs.nRows + SCAN_CHUNK - 1) / SCAN_CHUNK;
    int itemBlocks = blocks(cs.nBound);
    if (itemBlocks > 148 * 16) itemBlocks = 148 * 16;
    if (cudaMemsetAsync(cs.rowCount, 0, sizeof(int) * (size_t)cs.nRows, ctx->stream) != cudaSuccess)
        return fail(ctx, SBX_ECUDA, std::string(what) + ": memset");
    if (cs.nBound > 0)
        SBX_LAUNCH(ctx, k_cs_hist, itemBlocks, 256, cs.keys, cs.nDev, cs.useDevN, cs.nBound, cs.nRows, cs.rowCount,
                   cs.errFlag ? cs.errFlag : ctx->err_dev);
    int numTiles = (int)scan_tile_words(cs.nRows);
    SBX_LAUNCH(ctx, k_tile_reduce, numTiles, 256, cs.rowCount, cs.nRows, cs.tileSum);
    SBX_LAUNCH(ctx, k_tile_scan, numTiles, 256, cs.rowCount, cs.nRows, cs.rowOffsets, cs.chunkSum, numChunks,
               cs.tileSum, cs.listCap);
    if (cs.nBound > 0) {
        SBX_LAUNCH(ctx, k_cs_scatter, itemBlocks, 256, cs.keys, cs.nDev, cs.useDevN, cs.nBound, cs.nRows,
                   cs.rowOffsets, cs.rowCount, cs.tmp);
        SBX_LAUNCH(ctx, k_cs_rank, itemBlocks, 256, cs.keys, cs.nDev, cs.useDevN, cs.nBound, cs.nRows, cs.rowOffsets,
                   cs.tmp, cs.rowList, cs.listCap, cs.payload, cs.pStride, cs.pOff, cs.guard, cs.rowPayload);
    }
    return check_launch(ctx, what);
}
