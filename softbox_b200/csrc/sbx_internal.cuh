// sbx_internal.cuh — library-internal context, launch helpers and the counting sort.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "../../include/softbox_b200.h"

struct sbx_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;
    int64_t launches = 0;
    void* scratch = nullptr;          // grow-only device scratch for scans / unordered scatters
    size_t scratch_bytes = 0;
    int* host_flag = nullptr;         // pinned word for device -> host status flags
    // mapped pinned word that kernels set when an input breaks a documented range (a CSR key
    // >= its row count); sbx_ctx_sync reports and clears it. err_dev is its device address.
    int* err_host = nullptr;
    int* err_dev = nullptr;
    // stream markers of sbx_ctx_mark / sbx_ctx_wait_mark (created on first use)
    static constexpr int kMarks = 8;
    cudaEvent_t marks[kMarks] = {};
    // the copy stream of sbx_download_async_side and the event that orders its copies after
    // the work queued on `stream` (both created on first use)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copy_after = nullptr;
};

sbx_status fail(sbx_ctx* ctx, sbx_status code, const std::string& msg);
sbx_status check_launch(sbx_ctx* ctx, const char* what);
sbx_status ensure_scratch(sbx_ctx* ctx, size_t bytes);
sbx_status any_nonfinite(sbx_ctx* ctx, const float* a, int64_t n, bool* out);

static inline int blocks(int64_t n, int bs = 256) {
    int64_t b = (n + bs - 1) / bs;
    return (int)(b > 0 ? b : 1);
}

#define SBX_REQUIRE(cond)                                                              \
    do {                                                                               \
        if (!(cond)) return fail(ctx, SBX_EINVAL, std::string(__func__) + ": invalid argument"); \
    } while (0)

#define SBX_LAUNCH(ctx, kernel, grid, block, ...)                       \
    do {                                                                \
        kernel<<<(grid), (block), 0, (ctx)->stream>>>(__VA_ARGS__);     \
        (ctx)->launches++;                                              \
    } while (0)

// ---------------------------------------------------------------- index checks (debug build)
// Built with -DSBX_CHECK (python -m softbox_b200.build --check: libsoftbox_b200_check.so),
// the kernels test every data-dependent index they follow (a chain neighbour, a bound
// segment, a link end, a CSR list entry, a grid cell, a motor slot, a reach-walk entry)
// against the length of the array it indexes. A bad index is counted, the first one's site
// and value are kept, and the access is skipped; sbx_check_report returns them. In the
// normal build every test is the constant `true` and compiles away.
enum SbxCheckSite {
    CK_NEIGHBOUR = 1, CK_BOUND_SEG = 2, CK_LINK_END = 3, CK_LIST_ENTRY = 4, CK_CELL = 5, CK_MOTOR_SLOT = 6,
    CK_REACH_ENTRY = 7, CK_CSR_POS = 8
};
#ifdef SBX_CHECK
static __device__ unsigned long long sbx_check_count;   // per translation unit
static __device__ unsigned long long sbx_check_first;   // (site << 32) | index of the first bad index
__device__ __forceinline__ bool sbx_idx_ok(long long i, long long n, int site) {
    if (i >= 0 && i < n) return true;
    if (atomicAdd(&sbx_check_count, 1ULL) == 0ULL)
        sbx_check_first = ((unsigned long long)(unsigned)site << 32) | (unsigned long long)(unsigned)i;
    return false;
}
#define SBX_IDX_OK(i, n, site) sbx_idx_ok((long long)(i), (long long)(n), (site))
// each translation unit with checked kernels exports its counters
#define SBX_CHECK_EXPORT(tu)                                                                        \
    extern "C" int sbx_check_collect_##tu(unsigned long long* count, unsigned long long* first,     \
                                          int reset) {                                              \
        if (cudaMemcpyFromSymbol(count, sbx_check_count, sizeof(*count)) != cudaSuccess ||          \
            cudaMemcpyFromSymbol(first, sbx_check_first, sizeof(*first)) != cudaSuccess)           \
            return -1;                                                                              \
        if (reset) {                                                                                \
            const unsigned long long z = 0;                                                         \
            if (cudaMemcpyToSymbol(sbx_check_count, &z, sizeof(z)) != cudaSuccess ||                \
                cudaMemcpyToSymbol(sbx_check_first, &z, sizeof(z)) != cudaSuccess)                  \
                return -1;                                                                          \
        }                                                                                           \
        return 0;                                                                                   \
    }
#else
#define SBX_IDX_OK(i, n, site) true
#define SBX_CHECK_EXPORT(tu)
#endif
// an index that may be negative (meaning "none") or must lie in [0, n)
#define SBX_IDX_OK_OR_NONE(i, n, site) ((i) < 0 || SBX_IDX_OK((i), (n), (site)))

// ---------------------------------------------------------------- counting sort
// Stable counting sort of items [0, n) by key (keys < 0 are skipped; keys >= nRows are
// skipped and set *errFlag) into row CSR form:
// rowCount (atomic histogram, left equal to the row lengths), rowOffsets[0..nRows]
// (exclusive scan over SCAN_CHUNK tiles with the tile sums in chunkSum, terminator
// clamped to listCap), rowList (items in ascending index within each row).
// n = min(*nDev, nBound) when useDevN (SpatialGrid reads S from counts[1]), else nBound.
constexpr int SCAN_CHUNK = 512;

struct CountingSort {
    const int* keys;
    const int* nDev;      // optional device pointer to the item count
    int useDevN;          // read n from nDev[1] (the reference's counts[1] slot)
    int nBound;
    int nRows;
    int* rowCount;
    int* chunkSum;        // ceil(nRows/SCAN_CHUNK)+1 ints
    int* rowOffsets;      // nRows+1
    int* rowList;         // listCap
    int listCap;
    int* tmp;             // unordered scatter buffer, >= nBound ints
    // optional: the items' 6-float payloads copied in list order (rowPayload[6 pos + j] =
    // payload[item * pStride + pOff + j], zeros where guard[item] < 0)
    const float* payload = nullptr;
    int pStride = 0, pOff = 0;
    const int* guard = nullptr;
    float* rowPayload = nullptr;
    // the scan's per-tile sums: scan_tile_words(nRows) ints
    int* tileSum = nullptr;
    // set to 1 when a key is >= nRows (the item is skipped); may be null
    int* errFlag = nullptr;
};

// tiles of the counting sort's scan (8 scan chunks each)
static inline size_t scan_tile_words(int nRows) { return (size_t)(nRows + 8 * SCAN_CHUNK - 1) / (8 * SCAN_CHUNK); }

sbx_status counting_sort(sbx_ctx* ctx, const CountingSort& cs, const char* what);

// Exclusive prefix sum of in[0..n) into out[0..n), total into out[n]; zeroIn resets in[]
// (CrossBridgeSystem.csrScan's cursor side effect). chunkSum: ceil(n/SCAN_CHUNK)+1 ints.
sbx_status exclusive_scan(sbx_ctx* ctx, int* in, int n, int* out, bool zeroIn, int* chunkSum, const char* what);
