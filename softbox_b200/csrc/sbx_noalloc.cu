// sbx_noalloc.cu — sbx_csr_build_noalloc: the CSR-inverse build without any device allocation.
//
// sbx_csr_build keeps its scan tile sums and its unordered-scatter list in the context's
// grow-only scratch; the first call that needs more scratch than the context holds
// synchronises the stream and calls cudaMalloc. Some callers cannot allow that: a host
// that owns the device heap under a fixed budget (a JVM harness whose arrays were all
// allocated up front) or a step sequence that must not stall on a device synchronisation
// in the middle. This variant takes its scratch from one file-scope __device__ array of
// fixed size instead, so it calls no cudaMalloc, cudaFree or allocating library routine.
//
// Contract:
//  * Limits: nItems <= SBX_CSR_NOALLOC_MAX_ITEMS and nRows <= SBX_CSR_NOALLOC_MAX_ROWS;
//    larger inputs are rejected with SBX_EINVAL before anything is launched.
//  * Nothing has to start at zero: rowCount is cleared by the call itself, the tile sums
//    are written before they are read, and the scatter list is read only where this call
//    wrote it.
//  * The scratch is one array per device, shared by every context and stream on it. Two
//    calls whose executions overlap on one device (different streams, or different host
//    threads with different streams) race on it and give wrong results; calls on one
//    stream run one after another and are safe.
//  * The first call on each device resolves the scratch address (cudaGetSymbolAddress with
//    that device current); make that first call before any stream capture begins.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/softbox_b200.h"
#include "sbx_internal.cuh"

namespace {

// tile-sum region: ceil(MAX_ROWS / SCAN_CHUNK) + 1 ints, rounded up to 256 bytes
constexpr int NOALLOC_CHUNK_INTS =
    ((SBX_CSR_NOALLOC_MAX_ROWS / SCAN_CHUNK + 1) + 63) / 64 * 64;
constexpr int MAX_DEVICES = 64;

// scan tile sums: scan_tile_words(MAX_ROWS) ints, rounded up to 256 bytes
constexpr int NOALLOC_TILE_INTS = (SBX_CSR_NOALLOC_MAX_ROWS / (8 * SCAN_CHUNK) + 1 + 63) / 64 * 64;

static __device__ __align__(256) int g_csr_scratch[NOALLOC_CHUNK_INTS + NOALLOC_TILE_INTS +
                                                   SBX_CSR_NOALLOC_MAX_ITEMS];

std::mutex g_setup_mutex;
int* g_scratch_addr[MAX_DEVICES] = {};

// once per device: the device address of g_csr_scratch, resolved with that device current
sbx_status scratch_for_device(sbx_ctx* ctx, int** out) {
    if (ctx->device < 0 || ctx->device >= MAX_DEVICES)
        return fail(ctx, SBX_EINVAL, "sbx_csr_build_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[ctx->device]) {
        int prev = -1;
        cudaError_t e = cudaGetDevice(&prev);
        if (e == cudaSuccess && prev != ctx->device) e = cudaSetDevice(ctx->device);
        void* p = nullptr;
        if (e == cudaSuccess) e = cudaGetSymbolAddress(&p, g_csr_scratch);
        if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
        if (e != cudaSuccess || !p)
            return fail(ctx, SBX_ECUDA,
                        std::string("sbx_csr_build_noalloc: scratch set-up failed: ") + cudaGetErrorString(e));
        g_scratch_addr[ctx->device] = (int*)p;
    }
    *out = g_scratch_addr[ctx->device];
    return SBX_OK;
}

}  // namespace

extern "C" sbx_status sbx_csr_build_noalloc(sbx_ctx* ctx, const int32_t* keys, int32_t nItems, int32_t nRows,
                                            int32_t* rowCount, int32_t* rowOffsets, int32_t* rowList) {
    SBX_REQUIRE(ctx && nItems >= 0 && nRows > 0 && rowCount && rowOffsets && (nItems == 0 || (keys && rowList)));
    if (nItems > SBX_CSR_NOALLOC_MAX_ITEMS)
        return fail(ctx, SBX_EINVAL,
                    "sbx_csr_build_noalloc: nItems " + std::to_string(nItems) + " exceeds the static scratch limit " +
                        std::to_string(SBX_CSR_NOALLOC_MAX_ITEMS) + " (use sbx_csr_build)");
    if (nRows > SBX_CSR_NOALLOC_MAX_ROWS)
        return fail(ctx, SBX_EINVAL,
                    "sbx_csr_build_noalloc: nRows " + std::to_string(nRows) + " exceeds the static scratch limit " +
                        std::to_string(SBX_CSR_NOALLOC_MAX_ROWS) + " (use sbx_csr_build)");
    int* s = nullptr;
    sbx_status st = scratch_for_device(ctx, &s);
    if (st) return st;
    CountingSort cs{keys, nullptr, 0, nItems, nRows, rowCount, s, rowOffsets, rowList, nItems,
                    s + NOALLOC_CHUNK_INTS + NOALLOC_TILE_INTS};
    cs.tileSum = s + NOALLOC_CHUNK_INTS;
    return counting_sort(ctx, cs, "sbx_csr_build_noalloc");
}
