// sbx_systems.cu — context, memory and the per-system entry points of the C ABI.
//
// One entry point per public static method of the reference's System classes; each
// launches sm_100a kernels on the context stream. Per-slot systems are one thread per
// slot (the reference's @Parallel loop index). The reference's atomic-free chunked
// counting sorts (SpatialGrid.java:237-331, CrossBridgeSystem.java:232-298) and its
// single-thread scans are replaced by an atomic histogram, a two-level parallel scan
// and a rank pass that restores the stable (ascending index) order, so the CSR arrays
// come out bit-identical to the reference's serial build.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/softbox_b200.h"
#include "sbx_internal.cuh"
#include "sbx_physics.cuh"

using namespace sbx;

// ============================================================================ context
extern "C" sbx_status sbx_ctx_create(int device, void* stream, sbx_ctx** out) {
    if (!out) return SBX_EINVAL;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return SBX_ECUDA;
    sbx_ctx* ctx = new sbx_ctx();
    ctx->device = device;
    if (stream) {
        ctx->stream = (cudaStream_t)stream;
        ctx->own_stream = false;
    } else {
        // a blocking stream: it stays ordered against work on the legacy default stream
        if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamDefault) != cudaSuccess) {
            delete ctx;
            return SBX_ECUDA;
        }
        ctx->own_stream = true;
    }
    // the input-range error word: mapped pinned host memory, so that a kernel can set it
    // and sbx_ctx_sync can read it without a copy
    if (cudaHostAlloc(&ctx->err_host, sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess ||
        cudaHostGetDevicePointer(&ctx->err_dev, ctx->err_host, 0) != cudaSuccess) {
        if (ctx->err_host) cudaFreeHost(ctx->err_host);
        if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        cudaGetLastError();
        return SBX_ENOMEM;
    }
    *ctx->err_host = 0;
    *out = ctx;
    return SBX_OK;
}

extern "C" sbx_status sbx_ctx_destroy(sbx_ctx* ctx) {
    if (!ctx) return SBX_EINVAL;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->host_flag) cudaFreeHost(ctx->host_flag);
    if (ctx->err_host) cudaFreeHost(ctx->err_host);
    if (ctx->copy_stream) {
        cudaStreamSynchronize(ctx->copy_stream);
        cudaStreamDestroy(ctx->copy_stream);
    }
    if (ctx->copy_after) cudaEventDestroy(ctx->copy_after);
    for (cudaEvent_t e : ctx->marks)
        if (e) cudaEventDestroy(e);
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return SBX_OK;
}

extern "C" const char* sbx_ctx_last_error(sbx_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

extern "C" sbx_status sbx_ctx_set_stream(sbx_ctx* ctx, void* stream) {
    if (!ctx) return SBX_EINVAL;
    if (ctx->own_stream) {
        cudaStreamSynchronize(ctx->stream);
        cudaStreamDestroy(ctx->stream);
        ctx->own_stream = false;
    }
    ctx->stream = (cudaStream_t)stream;
    return SBX_OK;
}

extern "C" void* sbx_ctx_stream(sbx_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

extern "C" sbx_status sbx_ctx_sync(sbx_ctx* ctx) {
    if (!ctx) return SBX_EINVAL;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess && ctx->copy_stream) e = cudaStreamSynchronize(ctx->copy_stream);
    if (e != cudaSuccess) return fail(ctx, SBX_ECUDA, std::string("sync: ") + cudaGetErrorString(e));
    if (ctx->err_host && *(volatile int*)ctx->err_host) {
        const int w = *(volatile int*)ctx->err_host;
        *(volatile int*)ctx->err_host = 0;
        if (w == 2) return fail(ctx, SBX_ETIMEOUT, "a staged reach walk's bulk copies did not complete in time");
        return fail(ctx, SBX_EINVAL, "a CSR key was >= its row count (the item was skipped)");
    }
    return SBX_OK;
}

extern "C" int64_t sbx_ctx_launch_count(sbx_ctx* ctx) { return ctx ? ctx->launches : -1; }

extern "C" int64_t sbx_ctx_scratch_bytes(sbx_ctx* ctx) { return ctx ? (int64_t)ctx->scratch_bytes : -1; }

#ifdef SBX_CHECK
extern "C" int sbx_check_collect_systems(unsigned long long*, unsigned long long*, int);
extern "C" int sbx_check_collect_fused(unsigned long long*, unsigned long long*, int);
#endif

extern "C" int32_t sbx_check_build(void) {
#ifdef SBX_CHECK
    return 1;
#else
    return 0;
#endif
}

extern "C" sbx_status sbx_check_report(int64_t* count, int32_t* site, int64_t* index, int32_t reset) {
    if (!count || !site || !index) return SBX_EINVAL;
    *count = 0;
    *site = 0;
    *index = 0;
#ifdef SBX_CHECK
    // the translation units with checked kernels, each with its own counters
    int (*collect[])(unsigned long long*, unsigned long long*, int) = {sbx_check_collect_systems,
                                                                      sbx_check_collect_fused};
    for (auto fn : collect) {
        unsigned long long c = 0, f = 0;
        if (fn(&c, &f, reset) != 0) return SBX_ECUDA;
        if (c && *count == 0) {
            *site = (int32_t)(f >> 32);
            *index = (int64_t)(int32_t)(unsigned)(f & 0xffffffffULL);
        }
        *count += (int64_t)c;
    }
#else
    (void)reset;
#endif
    return SBX_OK;
}

sbx_status fail(sbx_ctx* ctx, sbx_status code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

sbx_status check_launch(sbx_ctx* ctx, const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ctx, SBX_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return SBX_OK;
}

static size_t align8(size_t b) { return (b + 7) & ~(size_t)7; }

sbx_status ensure_scratch(sbx_ctx* ctx, size_t bytes) {
    if (bytes <= ctx->scratch_bytes) return SBX_OK;
    cudaStreamSynchronize(ctx->stream);
    if (ctx->scratch) cudaFree(ctx->scratch);
    ctx->scratch = nullptr;
    ctx->scratch_bytes = 0;
    size_t want = std::max(bytes, (size_t)1 << 20);
    if (cudaMalloc(&ctx->scratch, want) != cudaSuccess) return fail(ctx, SBX_ENOMEM, "scratch allocation failed");
    ctx->scratch_bytes = want;
    return SBX_OK;
}

extern "C" sbx_status sbx_malloc(sbx_ctx* ctx, size_t bytes, void** dptr) {
    if (!ctx || !dptr) return SBX_EINVAL;
    cudaSetDevice(ctx->device);
    if (cudaMalloc(dptr, bytes ? bytes : 1) != cudaSuccess) return fail(ctx, SBX_ENOMEM, "cudaMalloc failed");
    return SBX_OK;
}
extern "C" sbx_status sbx_free(sbx_ctx* ctx, void* dptr) {
    if (!ctx) return SBX_EINVAL;
    cudaStreamSynchronize(ctx->stream);
    if (cudaFree(dptr) != cudaSuccess) return fail(ctx, SBX_ECUDA, "cudaFree failed");
    return SBX_OK;
}
extern "C" sbx_status sbx_upload(sbx_ctx* ctx, void* dst, const void* src, size_t bytes) {
    if (!ctx || (!dst && bytes) || (!src && bytes)) return SBX_EINVAL;
    if (cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
        return fail(ctx, SBX_ECUDA, "upload failed");
    return SBX_OK;
}
extern "C" sbx_status sbx_download(sbx_ctx* ctx, void* dst, const void* src, size_t bytes) {
    if (!ctx || (!dst && bytes) || (!src && bytes)) return SBX_EINVAL;
    if (cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess)
        return fail(ctx, SBX_ECUDA, "download failed");
    return sbx_ctx_sync(ctx);
}
extern "C" sbx_status sbx_download_async(sbx_ctx* ctx, void* dst, const void* src, size_t bytes) {
    if (!ctx || (!dst && bytes) || (!src && bytes)) return SBX_EINVAL;
    if (cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess)
        return fail(ctx, SBX_ECUDA, "download failed");
    return SBX_OK;
}
extern "C" sbx_status sbx_ctx_mark(sbx_ctx* ctx, int32_t slot) {
    if (!ctx || slot < 0 || slot >= sbx_ctx::kMarks) return SBX_EINVAL;
    if (!ctx->marks[slot] && cudaEventCreateWithFlags(&ctx->marks[slot], cudaEventDisableTiming) != cudaSuccess)
        return fail(ctx, SBX_ECUDA, "sbx_ctx_mark: event");
    if (cudaEventRecord(ctx->marks[slot], ctx->stream) != cudaSuccess) return fail(ctx, SBX_ECUDA, "sbx_ctx_mark: record");
    return SBX_OK;
}
// the copy stream's copies start after everything queued on the context's stream so far;
// the context's stream itself moves on at once
extern "C" sbx_status sbx_download_async_side(sbx_ctx* ctx, void* dst, const void* src, size_t bytes) {
    if (!ctx || (!dst && bytes) || (!src && bytes)) return SBX_EINVAL;
    if (!ctx->copy_stream && cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(ctx, SBX_ECUDA, "sbx_download_async_side: stream");
    if (!ctx->copy_after && cudaEventCreateWithFlags(&ctx->copy_after, cudaEventDisableTiming) != cudaSuccess)
        return fail(ctx, SBX_ECUDA, "sbx_download_async_side: event");
    if (cudaEventRecord(ctx->copy_after, ctx->stream) != cudaSuccess ||
        cudaStreamWaitEvent(ctx->copy_stream, ctx->copy_after, 0) != cudaSuccess)
        return fail(ctx, SBX_ECUDA, "sbx_download_async_side: order");
    if (cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->copy_stream) != cudaSuccess)
        return fail(ctx, SBX_ECUDA, "sbx_download_async_side: copy");
    return SBX_OK;
}
extern "C" sbx_status sbx_ctx_mark_side(sbx_ctx* ctx, int32_t slot) {
    if (!ctx || slot < 0 || slot >= sbx_ctx::kMarks || !ctx->copy_stream) return SBX_EINVAL;
    if (!ctx->marks[slot] && cudaEventCreateWithFlags(&ctx->marks[slot], cudaEventDisableTiming) != cudaSuccess)
        return fail(ctx, SBX_ECUDA, "sbx_ctx_mark_side: event");
    if (cudaEventRecord(ctx->marks[slot], ctx->copy_stream) != cudaSuccess)
        return fail(ctx, SBX_ECUDA, "sbx_ctx_mark_side: record");
    return SBX_OK;
}
extern "C" sbx_status sbx_ctx_stream_wait_mark(sbx_ctx* ctx, int32_t slot) {
    if (!ctx || slot < 0 || slot >= sbx_ctx::kMarks || !ctx->marks[slot]) return SBX_EINVAL;
    if (cudaStreamWaitEvent(ctx->stream, ctx->marks[slot], 0) != cudaSuccess)
        return fail(ctx, SBX_ECUDA, "sbx_ctx_stream_wait_mark");
    return SBX_OK;
}
extern "C" sbx_status sbx_ctx_wait_mark(sbx_ctx* ctx, int32_t slot) {
    if (!ctx || slot < 0 || slot >= sbx_ctx::kMarks || !ctx->marks[slot]) return SBX_EINVAL;
    cudaError_t e = cudaEventSynchronize(ctx->marks[slot]);
    if (e != cudaSuccess) return fail(ctx, SBX_ECUDA, std::string("wait: ") + cudaGetErrorString(e));
    if (ctx->err_host && *(volatile int*)ctx->err_host) {
        const int w = *(volatile int*)ctx->err_host;
        *(volatile int*)ctx->err_host = 0;
        if (w == 2) return fail(ctx, SBX_ETIMEOUT, "a staged reach walk's bulk copies did not complete in time");
        return fail(ctx, SBX_EINVAL, "a CSR key was >= its row count (the item was skipped)");
    }
    return SBX_OK;
}
extern "C" sbx_status sbx_memset(sbx_ctx* ctx, void* dst, int value, size_t bytes) {
    if (!ctx || (!dst && bytes)) return SBX_EINVAL;
    if (cudaMemsetAsync(dst, value, bytes, ctx->stream) != cudaSuccess) return fail(ctx, SBX_ECUDA, "memset failed");
    return SBX_OK;
}

// ============================================================================ drag
__device__ void d_rod_drag_si(double lengthUm, double radiusUm, double aeta, double g[6]) {
    const double PI = PI_D;
    double LM = 1.0e-6 * lengthUm;
    double RM = radiusUm * 1.0e-6;
    double logT = sbxm::log(LM / (2 * RM));
    g[0] = (2 * PI * aeta * LM) / (logT + -0.20);
    g[1] = (4 * PI * aeta * LM) / (logT + 0.84);
    g[2] = g[1];
    g[3] = 4 * PI * aeta * RM * RM * LM;
    g[4] = (PI * aeta * (LM * LM * LM)) / (3 * (logT + -0.662));
    g[5] = g[4];
}

__device__ void d_store_drag(int n, int i, const double g[6], float* bTG, float* bRG, float* bTD, float* bRD) {
    const double KT = 1.380662e-23 * 298.15;
    for (int k = 0; k < 3; k++) {
        bTG[k * n + i] = (float)g[k];
        bRG[k * n + i] = (float)g[3 + k];
        bTD[k * n + i] = (float)(KT / g[k]);
        bRD[k * n + i] = (float)(KT / g[3 + k]);
    }
}

__global__ void k_drag_filament(int n, const int* monomerCount, const int* e1, const int* e2, double aeta,
                                float* segLength, float* bTG, float* bRG, float* bTD, float* bRD) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double halfmono = 0.0054 / 2.0;
    double length = (monomerCount[i] + 1) * halfmono;
    segLength[i] = (float)length;
    double minLength = (e1[i] == -1 || e2[i] == -1) ? 32 * halfmono : 30 * halfmono;
    double asIf = length < minLength ? minLength : length;
    double g[6];
    d_rod_drag_si(asIf, 0.007 / 2.0, aeta, g);
    d_store_drag(n, i, g, bTG, bRG, bTD, bRD);
}

__global__ void k_drag_motor(int nM, double aeta, float* segLength, float* bTG, float* bRG, float* bTD, float* bRD) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    int n = 3 * nM;
    if (s >= n) return;
    int role = s % 3;
    double g[6];
    if (role == 0) { d_rod_drag_si(0.080, 0.003, aeta, g); segLength[s] = (float)0.080; }
    else if (role == 1) { d_rod_drag_si(0.008, 0.002, aeta, g); segLength[s] = (float)0.008; }
    else {
        double RM = 0.010 * 1.0e-6;
        double bt = 6 * PI_D * aeta * RM, br = 8 * PI_D * aeta * (RM * RM * RM);
        g[0] = g[1] = g[2] = bt;
        g[3] = g[4] = g[5] = br;
        segLength[s] = (float)0.020;
    }
    d_store_drag(n, s, g, bTG, bRG, bTD, bRD);
}

__global__ void k_drag_backbone(int nBb, double bbLen, double aeta, float* segLength, float* bTG, float* bRG,
                                float* bTD, float* bRD, float* inv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nBb) return;
    double g[6];
    d_rod_drag_si(bbLen, 0.005, aeta, g);
    segLength[i] = (float)bbLen;
    d_store_drag(nBb, i, g, bTG, bRG, bTD, bRD);
    inv[i] = (float)(1.0 / g[1]);
    inv[nBb + i] = (float)(1.0 / g[4]);
}

extern "C" sbx_status sbx_drag_run_filament(sbx_ctx* ctx, int32_t n, const int32_t* mc, const int32_t* e1,
                                            const int32_t* e2, double aeta, float* segLength, float* bTG,
                                            float* bRG, float* bTD, float* bRD) {
    SBX_REQUIRE(ctx && n >= 0 && (n == 0 || (mc && e1 && e2 && segLength && bTG && bRG && bTD && bRD)));
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_drag_filament, blocks(n), 256, n, mc, e1, e2, aeta, segLength, bTG, bRG, bTD, bRD);
    return check_launch(ctx, "sbx_drag_run_filament");
}

extern "C" sbx_status sbx_drag_run_motor(sbx_ctx* ctx, int32_t nM, double aeta, float* segLength, float* bTG,
                                         float* bRG, float* bTD, float* bRD) {
    SBX_REQUIRE(ctx && nM >= 0 && (nM == 0 || (segLength && bTG && bRG && bTD && bRD)));
    if (nM == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_drag_motor, blocks(3 * nM), 256, nM, aeta, segLength, bTG, bRG, bTD, bRD);
    return check_launch(ctx, "sbx_drag_run_motor");
}

extern "C" sbx_status sbx_drag_run_backbone(sbx_ctx* ctx, int32_t nBb, double bbLen, double aeta, float* segLength,
                                            float* bTG, float* bRG, float* bTD, float* bRD, float* inv) {
    SBX_REQUIRE(ctx && nBb >= 0 && (nBb == 0 || (segLength && bTG && bRG && bTD && bRD && inv)));
    if (nBb == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_drag_backbone, blocks(nBb), 256, nBb, bbLen, aeta, segLength, bTG, bRG, bTD, bRD, inv);
    return check_launch(ctx, "sbx_drag_run_backbone");
}

// ============================================================================ Brownian
template <int MODE>   // 0 wang, 1 philox, 2 supplied
__global__ void k_brownian(int n, float* rF, float* rT, const float* bTG, const float* bRG, const float* tSc,
                           const float* rSc, const float* params, const int* counts, uint64_t seed64,
                           const float* noise) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float g[6];
    if (MODE == 0) gauss6_wang(i, counts[1], counts[2], g);
    else if (MODE == 1) gauss6_philox(i, counts[1], seed64, g);
    else for (int k = 0; k < 6; k++) g[k] = noise[(int64_t)k * n + i];
    float gT[3] = {bTG[i], bTG[n + i], bTG[2 * n + i]};
    float gR[3] = {bRG[i], bRG[n + i], bRG[2 * n + i]};
    float rf[3], rt[3];
    brownian_amplitudes(g, tSc[i], rSc[i], params[1], gT, gR, rf, rt);
    for (int k = 0; k < 3; k++) { rF[k * n + i] = rf[k]; rT[k * n + i] = rt[k]; }
}

__global__ void k_check_finite(const float* a, int64_t n, int* flag) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (!isfinite(a[i])) { *flag = 1; return; }
}

#define BROWNIAN_REQ SBX_REQUIRE(ctx && n >= 0 && (n == 0 || (rF && rT && bTG && bRG && tSc && rSc && params)))

extern "C" sbx_status sbx_brownian_force(sbx_ctx* ctx, int32_t n, float* rF, float* rT, const float* bTG,
                                         const float* bRG, const float* tSc, const float* rSc, const float* params,
                                         const int32_t* counts) {
    BROWNIAN_REQ;
    SBX_REQUIRE(n == 0 || counts);
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_brownian<0>, blocks(n), 256, n, rF, rT, bTG, bRG, tSc, rSc, params, counts, 0ull, nullptr);
    return check_launch(ctx, "sbx_brownian_force");
}

extern "C" sbx_status sbx_brownian_force_philox(sbx_ctx* ctx, int32_t n, float* rF, float* rT, const float* bTG,
                                                const float* bRG, const float* tSc, const float* rSc,
                                                const float* params, const int32_t* counts, uint64_t seed) {
    BROWNIAN_REQ;
    SBX_REQUIRE(n == 0 || counts);
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_brownian<1>, blocks(n), 256, n, rF, rT, bTG, bRG, tSc, rSc, params, counts, seed, nullptr);
    return check_launch(ctx, "sbx_brownian_force_philox");
}

sbx_status any_nonfinite(sbx_ctx* ctx, const float* a, int64_t n, bool* out) {
    if (!ctx->host_flag) {
        if (cudaMallocHost(&ctx->host_flag, sizeof(int)) != cudaSuccess) return fail(ctx, SBX_ENOMEM, "pinned flag");
    }
    sbx_status st = ensure_scratch(ctx, 256);
    if (st) return st;
    int* dflag = (int*)ctx->scratch;
    cudaMemsetAsync(dflag, 0, sizeof(int), ctx->stream);
    int nb = (int)std::min<int64_t>((n + 255) / 256, 4 * 148);
    SBX_LAUNCH(ctx, k_check_finite, nb > 0 ? nb : 1, 256, a, n, dflag);
    cudaMemcpyAsync(ctx->host_flag, dflag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if ((st = sbx_ctx_sync(ctx))) return st;
    *out = *ctx->host_flag != 0;
    return SBX_OK;
}

extern "C" sbx_status sbx_brownian_force_supplied(sbx_ctx* ctx, int32_t n, float* rF, float* rT, const float* bTG,
                                                  const float* bRG, const float* tSc, const float* rSc,
                                                  const float* params, const float* noise) {
    BROWNIAN_REQ;
    SBX_REQUIRE(n == 0 || noise);
    if (n == 0) return SBX_OK;
    bool bad = false;
    sbx_status st = any_nonfinite(ctx, noise, 6 * (int64_t)n, &bad);
    if (st) return st;
    if (bad) return fail(ctx, SBX_ENONFINITE, "sbx_brownian_force_supplied: noise holds NaN/Inf");
    SBX_LAUNCH(ctx, k_brownian<2>, blocks(n), 256, n, rF, rT, bTG, bRG, tSc, rSc, params, nullptr, 0ull, noise);
    return check_launch(ctx, "sbx_brownian_force_supplied");
}

__global__ void k_zero_acc(int n, float* F, float* T) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < 3; k++) { F[k * n + i] = 0.f; T[k * n + i] = 0.f; }
}

extern "C" sbx_status sbx_zero_accumulators(sbx_ctx* ctx, int32_t n, float* F, float* T) {
    SBX_REQUIRE(ctx && n >= 0 && (n == 0 || (F && T)));
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_zero_acc, blocks(n), 256, n, F, T);
    return check_launch(ctx, "sbx_zero_accumulators");
}

// ============================================================================ integrate / derive / confine
__device__ __forceinline__ void load3(const float* a, int n, int i, float v[3]) {
    v[0] = a[i]; v[1] = a[n + i]; v[2] = a[2 * n + i];
}
__device__ __forceinline__ void store3(float* a, int n, int i, const float v[3]) {
    a[i] = v[0]; a[n + i] = v[1]; a[2 * n + i] = v[2];
}

// integrate one slot in place; writes coord (and coord64 when given), uVec, yVec
// integration of slot i with its force and torque sums already in registers
__device__ __forceinline__ void integrate_slot_ft(int n, int i, float* coord, double* coord64, float* uVec,
                                                  float* yVec, const float f[3], const float t[3], const float* rF,
                                                  const float* rT, const float* bTG, const float* bRG, float dt,
                                                  Pose& q) {
    Pose p;
    load3(coord, n, i, p.c); load3(uVec, n, i, p.u); load3(yVec, n, i, p.y);
    float rf[3], rt[3], gT[3], gR[3], dc[3];
    load3(rF, n, i, rf); load3(rT, n, i, rt);
    load3(bTG, n, i, gT); load3(bRG, n, i, gR);
    integrate_pose(p, f, t, rf, rt, gT, gR, dt, q, dc);
    if (coord64) {
        for (int k = 0; k < 3; k++) {
            double c = coord64[k * n + i] + (double)dc[k];
            coord64[k * n + i] = c;
            q.c[k] = (float)c;
        }
    }
    store3(coord, n, i, q.c); store3(uVec, n, i, q.u); store3(yVec, n, i, q.y);
}

__device__ __forceinline__ void integrate_slot(int n, int i, float* coord, double* coord64, float* uVec, float* yVec,
                                               const float* F, const float* T, const float* rF, const float* rT,
                                               const float* bTG, const float* bRG, float dt, Pose& q) {
    float f[3], t[3];
    load3(F, n, i, f); load3(T, n, i, t);
    integrate_slot_ft(n, i, coord, coord64, uVec, yVec, f, t, rF, rT, bTG, bRG, dt, q);
}

__global__ void k_integrate(int n, float* coord, double* coord64, float* uVec, float* yVec, const float* F,
                            const float* T, const float* rF, const float* rT, const float* bTG, const float* bRG,
                            const float* params) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Pose q;
    integrate_slot(n, i, coord, coord64, uVec, yVec, F, T, rF, rT, bTG, bRG, params[0], q);
}

__global__ void k_derive(int n, const float* coord, const float* uVec, float* yVec, float* zVec, float* end1,
                         float* end2, const float* segLength) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float c[3], u[3], y[3], z[3], e1[3], e2[3];
    load3(coord, n, i, c); load3(uVec, n, i, u); load3(yVec, n, i, y);
    derive_pose(c, u, y, z, e1, e2, segLength[i]);
    store3(zVec, n, i, z); store3(yVec, n, i, y); store3(end1, n, i, e1); store3(end2, n, i, e2);
}

__global__ void k_confine(int n, const float* coord, const float* uVec, const float* segLength, const float* bTG,
                          float* F, float* T, const float* boxParams, const int* counts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    BoxParams bx = box_params(boxParams, counts[1]);
    if (!bx.active) return;
    float c[3], u[3], f[3], t[3];
    load3(coord, n, i, c); load3(uVec, n, i, u); load3(F, n, i, f); load3(T, n, i, t);
    if (confine_one(bx, c, u, segLength[i], bTG[i], f, t)) {
        store3(F, n, i, f);
        store3(T, n, i, t);
    }
}

// MechanicsFusion.forceBuild / integDerive / integDeriveConfined (MechanicsFusion.java:52-338)
__global__ void k_force_build(int n, float* F, float* T, float* rF, float* rT, const float* bTG, const float* bRG,
                              const float* tSc, const float* rSc, const float* params, const int* counts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < 3; k++) { F[k * n + i] = 0.f; T[k * n + i] = 0.f; }
    float g[6];
    gauss6_wang(i, counts[1], counts[2], g);
    float gT[3], gR[3], rf[3], rt[3];
    load3(bTG, n, i, gT); load3(bRG, n, i, gR);
    brownian_amplitudes(g, tSc[i], rSc[i], params[1], gT, gR, rf, rt);
    store3(rF, n, i, rf); store3(rT, n, i, rt);
}

template <bool CONFINED>
__global__ void __launch_bounds__(256, 4) k_integ_derive(int n, float* coord, double* coord64, float* uVec, float* yVec, float* zVec,
                               const float* segLength, float* end1, float* end2, float* F, float* T, const float* rF,
                               const float* rT, const float* bTG, const float* bRG, const float* params,
                               const int* counts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float dt;
    if (CONFINED) {
        BoxParams bx = box_params(params, counts[1]);
        dt = params[7];
        if (bx.active) {
            float c[3], u[3], f[3], t[3];
            load3(coord, n, i, c); load3(uVec, n, i, u); load3(F, n, i, f); load3(T, n, i, t);
            if (confine_one(bx, c, u, segLength[i], bTG[i], f, t)) {     // most rods touch no wall
                store3(F, n, i, f);
                store3(T, n, i, t);
            }
        }
    } else {
        dt = params[0];
    }
    Pose q;
    integrate_slot(n, i, coord, coord64, uVec, yVec, F, T, rF, rT, bTG, bRG, dt, q);
    float z[3], e1[3], e2[3];
    derive_pose(q.c, q.u, q.y, z, e1, e2, segLength[i]);
    store3(zVec, n, i, z); store3(yVec, n, i, q.y); store3(end1, n, i, e1); store3(end2, n, i, e2);
}

extern "C" sbx_status sbx_integrate(sbx_ctx* ctx, int32_t n, float* coord, double* coord64, float* uVec,
                                    float* yVec, const float* F, const float* T, const float* rF, const float* rT,
                                    const float* bTG, const float* bRG, const float* params) {
    SBX_REQUIRE(ctx && n >= 0 && (n == 0 || (coord && uVec && yVec && F && T && rF && rT && bTG && bRG && params)));
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_integrate, blocks(n), 256, n, coord, coord64, uVec, yVec, F, T, rF, rT, bTG, bRG, params);
    return check_launch(ctx, "sbx_integrate");
}

extern "C" sbx_status sbx_derive(sbx_ctx* ctx, int32_t n, const float* coord, const float* uVec, float* yVec,
                                 float* zVec, float* end1, float* end2, const float* segLength) {
    SBX_REQUIRE(ctx && n >= 0 && (n == 0 || (coord && uVec && yVec && zVec && end1 && end2 && segLength)));
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_derive, blocks(n), 256, n, coord, uVec, yVec, zVec, end1, end2, segLength);
    return check_launch(ctx, "sbx_derive");
}

extern "C" sbx_status sbx_confine(sbx_ctx* ctx, int32_t n, const float* coord, const float* uVec,
                                  const float* segLength, const float* bTG, float* F, float* T,
                                  const float* boxParams, const int32_t* counts) {
    SBX_REQUIRE(ctx && n >= 0 && (n == 0 || (coord && uVec && segLength && bTG && F && T && boxParams && counts)));
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_confine, blocks(n), 256, n, coord, uVec, segLength, bTG, F, T, boxParams, counts);
    return check_launch(ctx, "sbx_confine");
}

extern "C" sbx_status sbx_fusion_force_build(sbx_ctx* ctx, int32_t n, float* F, float* T, float* rF, float* rT,
                                             const float* bTG, const float* bRG, const float* tSc, const float* rSc,
                                             const float* params, const int32_t* counts) {
    SBX_REQUIRE(ctx && n >= 0 && (n == 0 || (F && T && rF && rT && bTG && bRG && tSc && rSc && params && counts)));
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_force_build, blocks(n), 256, n, F, T, rF, rT, bTG, bRG, tSc, rSc, params, counts);
    return check_launch(ctx, "sbx_fusion_force_build");
}

extern "C" sbx_status sbx_fusion_integ_derive(sbx_ctx* ctx, int32_t n, float* coord, double* coord64, float* uVec,
                                              float* yVec, float* zVec, const float* segLength, float* end1,
                                              float* end2, const float* F, const float* T, const float* rF,
                                              const float* rT, const float* bTG, const float* bRG,
                                              const float* params) {
    SBX_REQUIRE(ctx && n >= 0 && (n == 0 || (coord && uVec && yVec && zVec && segLength && end1 && end2 && F && T &&
                                             rF && rT && bTG && bRG && params)));
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_integ_derive<false>, blocks(n), 256, n, coord, coord64, uVec, yVec, zVec, segLength, end1, end2,
               (float*)F, (float*)T, rF, rT, bTG, bRG, params, nullptr);
    return check_launch(ctx, "sbx_fusion_integ_derive");
}

extern "C" sbx_status sbx_fusion_integ_derive_confined(sbx_ctx* ctx, int32_t n, float* coord, double* coord64,
                                                       float* uVec, float* yVec, float* zVec, const float* segLength,
                                                       float* end1, float* end2, float* F, float* T, const float* rF,
                                                       const float* rT, const float* bTG, const float* bRG,
                                                       const float* boxParams, const int32_t* counts) {
    SBX_REQUIRE(ctx && n >= 0 && (n == 0 || (coord && uVec && yVec && zVec && segLength && end1 && end2 && F && T &&
                                             rF && rT && bTG && bRG && boxParams && counts)));
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_integ_derive<true>, blocks(n), 256, n, coord, coord64, uVec, yVec, zVec, segLength, end1, end2,
               F, T, rF, rT, bTG, bRG, boxParams, counts);
    return check_launch(ctx, "sbx_fusion_integ_derive_confined");
}


// ============================================================================ chain
// ChainBendingForceSystem.chainForces (ChainBendingForceSystem.java:105-331), one thread per
// rod. Each joint's costly scalars (chain_joint) are computed once by its lower-slot rod and
// shared through shared memory with the partner when both rods are in the block and the
// partner's neighbour entries point back consistently; otherwise the rod computes the joint
// from its own side, which gives the same bits. The rod geometry is loaded where each part
// needs it (the joint, then the apply step re-reads the few values it uses) so that no full
// geometry set stays live across the barrier: fewer registers, more resident warps to hide
// the FP64 and load latencies.
//
// With GATHER the same pass then adds the filament-side CSR gathers of the step, in the
// reference's order: CrosslinkerSystem.segGatherA (:129-150), segGatherB (:153-173) and
// CrossBridgeSystem.segGather (:302-320). Each reads a row-ordered payload (sbx_csr_build_payload:
// row s's items at rows [offsets[s], offsets[s+1]) of 6 floats), sums the row in FP64 in list
// order and adds it to the float accumulators; a guarded-out item holds zeros, which leave the
// sum's bits unchanged (the sum starts at +0.0 and so is never -0.0). The accumulators are read
// and written once for chain and gathers, and the gathers' loads overlap the joint arithmetic.
constexpr int CHAIN_THREADS = 256;

struct RowGathers {
    const int* offA; const float* payA;
    const int* offB; const float* payB;
    const int* offM; const float* payM;
};

struct RowSum {
    int k0, k1;
    float2 q[3];
};

SBX_DEV void row_begin(RowSum& r, int s, const int* off) {
    r.k0 = r.k1 = 0;
    if (off) { r.k0 = off[s]; r.k1 = off[s + 1]; }
}

SBX_DEV void row_first(RowSum& r, const float* pay) {
    if (r.k0 < r.k1) {
        const float2* q = reinterpret_cast<const float2*>(pay + 6 * (int64_t)r.k0);
        r.q[0] = q[0]; r.q[1] = q[1]; r.q[2] = q[2];
    }
}

SBX_DEV void row_finish(const RowSum& r, const float* pay, float Fv[3], float Tv[3]) {
    double f[3] = {0.0, 0.0, 0.0}, t[3] = {0.0, 0.0, 0.0};
    if (r.k0 < r.k1) {
        f[0] += r.q[0].x; f[1] += r.q[0].y; f[2] += r.q[1].x;
        t[0] += r.q[1].y; t[1] += r.q[2].x; t[2] += r.q[2].y;
        for (int k = r.k0 + 1; k < r.k1; k++) {
            const float* q = pay + 6 * (int64_t)k;
            f[0] += q[0]; f[1] += q[1]; f[2] += q[2];
            t[0] += q[3]; t[1] += q[4]; t[2] += q[5];
        }
    }
    for (int k = 0; k < 3; k++) {
        Fv[k] = (float)(Fv[k] + f[k]);
        Tv[k] = (float)(Tv[k] + t[k]);
    }
}

template <bool GATHER>
__global__ void __launch_bounds__(CHAIN_THREADS, 3) k_chain(int n, const float* coord, const float* uVec,
                                                            const float* segLength, const int* e2s, const int* e2d,
                                                            const int* e1s, const int* e1d, const float* bTG,
                                                            const float* bRG, float* F, float* T,
                                                            const float* chainParams, RowGathers g) {
    __shared__ ChainJoint js[2 * CHAIN_THREADS];
    const int tid = threadIdx.x, lo = blockIdx.x * blockDim.x;
    const int hi = min(lo + (int)blockDim.x, n);
    const int i = lo + tid;
    int s2 = -1, d2 = 0, s1 = -1, d1 = 0;
    if (i < n) {
        s2 = e2s[i]; d2 = e2d[i]; s1 = e1s[i]; d1 = e1d[i];
        if (!SBX_IDX_OK_OR_NONE(s2, n, CK_NEIGHBOUR)) s2 = -1;
        if (!SBX_IDX_OK_OR_NONE(s1, n, CK_NEIGHBOUR)) s1 = -1;
        if (s2 > i) {
            ChainParams cp = chain_params(chainParams);
            js[2 * tid] = chain_joint(cp, i, 0, s2, d2, load_rod(n, i, coord, uVec, segLength, bTG, bRG),
                                      load_rod(n, s2, coord, uVec, segLength, bTG, bRG));
        }
        if (s1 > i) {
            ChainParams cp = chain_params(chainParams);
            js[2 * tid + 1] = chain_joint(cp, i, 1, s1, d1, load_rod(n, i, coord, uVec, segLength, bTG, bRG),
                                          load_rod(n, s1, coord, uVec, segLength, bTG, bRG));
        }
    }
    __syncthreads();
    if (i >= n) return;
    float Fv[3], Tv[3];
    for (int k = 0; k < 3; k++) { Fv[k] = F[k * n + i]; Tv[k] = T[k * n + i]; }
    RowSum ra, rb, rm;
    if (GATHER) {
        row_begin(ra, i, g.offA);
        row_begin(rb, i, g.offB);
        row_begin(rm, i, g.offM);
    }
    double f[3] = {0.0, 0.0, 0.0}, t[3] = {0.0, 0.0, 0.0};
    // side `side` of rod i: the joint from its own slot, the partner's slot, or recomputed
    for (int side = 0; side < 2; side++) {
        int slot = side == 0 ? s2 : s1, nside = side == 0 ? d2 : d1;
        if (slot < 0) continue;
        ChainParams cp = chain_params(chainParams);
        RodGeom r = load_rod(n, i, coord, uVec, segLength, bTG, bRG);
        RodGeom nb = load_rod(n, slot, coord, uVec, segLength, bTG, bRG);
        ChainJoint J;
        bool have = false;
        if (slot > i) {
            J = js[2 * tid + side];
            have = true;
        } else if (slot >= lo && slot < hi && (nside == 0 || nside == 1)) {
            int ps = 1 - nside;                                  // the partner's side facing rod i
            int back = ps == 0 ? e2s[slot] : e1s[slot], backSide = ps == 0 ? e2d[slot] : e1d[slot];
            if (back == i && backSide == 1 - side) {
                J = js[2 * (slot - lo) + ps];
                have = true;
            }
        }
        if (!have) J = chain_joint(cp, i, side, slot, nside, r, nb);
        chain_apply(cp, i, side, slot, nside, r, nb, J, f, t);
    }
    for (int k = 0; k < 3; k++) {
        Fv[k] = (float)(Fv[k] + f[k]);
        Tv[k] = (float)(Tv[k] + t[k]);
    }
    if (GATHER) {
        row_first(ra, g.payA);
        row_first(rb, g.payB);
        row_first(rm, g.payM);
        if (g.offA) row_finish(ra, g.payA, Fv, Tv);
        if (g.offB) row_finish(rb, g.payB, Fv, Tv);
        if (g.offM) row_finish(rm, g.payM, Fv, Tv);
    }
    for (int k = 0; k < 3; k++) { F[k * n + i] = Fv[k]; T[k * n + i] = Tv[k]; }
}

extern "C" sbx_status sbx_chain_forces(sbx_ctx* ctx, int32_t n, const float* coord, const float* uVec,
                                       const float* segLength, const int32_t* e2s, const int32_t* e2d,
                                       const int32_t* e1s, const int32_t* e1d, const float* bTG, const float* bRG,
                                       float* F, float* T, const float* chainParams) {
    SBX_REQUIRE(ctx && n >= 0 && (n == 0 || (coord && uVec && segLength && e2s && e2d && e1s && e1d && bTG && bRG &&
                                             F && T && chainParams)));
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_chain<false>, blocks(n, CHAIN_THREADS), CHAIN_THREADS, n, coord, uVec, segLength, e2s, e2d,
               e1s, e1d, bTG, bRG, F, T, chainParams, RowGathers{});
    return check_launch(ctx, "sbx_chain_forces");
}

static bool aligned8(const void* p) { return ((uintptr_t)p & 7u) == 0; }

extern "C" sbx_status sbx_fusion_chain_gathers(sbx_ctx* ctx, int32_t n, const float* coord, const float* uVec,
                                               const float* segLength, const int32_t* e2s, const int32_t* e2d,
                                               const int32_t* e1s, const int32_t* e1d, const float* bTG,
                                               const float* bRG, float* F, float* T, const float* chainParams,
                                               const int32_t* segOffsetsA, const float* rowPayloadA,
                                               const int32_t* segOffsetsB, const float* rowPayloadB,
                                               const int32_t* segMotorOffsets, const float* rowPayloadM) {
    SBX_REQUIRE(ctx && n >= 0 && (n == 0 || (coord && uVec && segLength && e2s && e2d && e1s && e1d && bTG && bRG &&
                                             F && T && chainParams)) &&
                (!segOffsetsA || (rowPayloadA && aligned8(rowPayloadA))) &&
                (!segOffsetsB || (rowPayloadB && aligned8(rowPayloadB))) &&
                (!segMotorOffsets || (rowPayloadM && aligned8(rowPayloadM))));
    if (n == 0) return SBX_OK;
    RowGathers g{segOffsetsA, rowPayloadA, segOffsetsB, rowPayloadB, segMotorOffsets, rowPayloadM};
    SBX_LAUNCH(ctx, k_chain<true>, blocks(n, CHAIN_THREADS), CHAIN_THREADS, n, coord, uVec, segLength, e2s, e2d,
               e1s, e1d, bTG, bRG, F, T, chainParams, g);
    return check_launch(ctx, "sbx_fusion_chain_gathers");
}

// ============================================================================ publishing
__global__ void k_fil_publish(int n, const float* coord, const float* segLength, int cap, float* center, float* R,
                              int* ownerStore, int* ownerSlot, const float* viewParams, const int* filState) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    center[i] = coord[i];
    center[cap + i] = coord[n + i];
    center[2 * cap + i] = coord[2 * n + i];
    R[i] = 0.5f * segLength[i] + viewParams[0];
    ownerStore[i] = (filState && filState[i] < 0) ? STORE_NONE : STORE_FILAMENT;
    ownerSlot[i] = i;
}

__global__ void k_mot_publish_head(int nM, const float* bc, const float* bu, const float* bl, float* head, float* uVec,
                                   float* rodUVec) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nM) return;
    int nB = 3 * nM, h = 3 * m + 2, r = 3 * m;
    float hl = bl[h];
    for (int k = 0; k < 3; k++) {
        head[k * nM + m] = bc[k * nB + h] + 0.5f * hl * bu[k * nB + h];
        uVec[k * nM + m] = bu[k * nB + h];
        rodUVec[k * nM + m] = bu[k * nB + r];
    }
}

__global__ void k_mot_publish(int nM, const float* head, const float* reach, int cap, float* center, float* R,
                              int* ownerStore, int* ownerSlot, const int* publishParams) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nM) return;
    int b = publishParams[0] + m;
    center[b] = head[m];
    center[cap + b] = head[nM + m];
    center[2 * cap + b] = head[2 * nM + m];
    R[b] = reach[m];
    ownerStore[b] = STORE_MOTOR;
    ownerSlot[b] = m;
}

extern "C" sbx_status sbx_filament_publish(sbx_ctx* ctx, int32_t n, const float* coord, const float* segLength,
                                           int32_t cap, float* center, float* R, int32_t* ownerStore,
                                           int32_t* ownerSlot, const float* viewParams, const int32_t* filState) {
    SBX_REQUIRE(ctx && n >= 0 && cap >= n && (n == 0 || (coord && segLength && center && R && ownerStore &&
                                                           ownerSlot && viewParams)));
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_fil_publish, blocks(n), 256, n, coord, segLength, cap, center, R, ownerStore, ownerSlot,
               viewParams, filState);
    return check_launch(ctx, "sbx_filament_publish");
}

extern "C" sbx_status sbx_motor_publish_head(sbx_ctx* ctx, int32_t nM, const float* bc, const float* bu,
                                             const float* bl, float* head, float* uVec, float* rodUVec) {
    SBX_REQUIRE(ctx && nM >= 0 && (nM == 0 || (bc && bu && bl && head && uVec && rodUVec)));
    if (nM == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_mot_publish_head, blocks(nM), 256, nM, bc, bu, bl, head, uVec, rodUVec);
    return check_launch(ctx, "sbx_motor_publish_head");
}

extern "C" sbx_status sbx_motor_publish(sbx_ctx* ctx, int32_t nM, const float* head, const float* reach, int32_t cap,
                                        float* center, float* R, int32_t* ownerStore, int32_t* ownerSlot,
                                        const int32_t* publishParams) {
    SBX_REQUIRE(ctx && nM >= 0 && (nM == 0 || (head && reach && center && R && ownerStore && ownerSlot &&
                                               publishParams)));
    if (nM == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_mot_publish, blocks(nM), 256, nM, head, reach, cap, center, R, ownerStore, ownerSlot,
               publishParams);
    return check_launch(ctx, "sbx_motor_publish");
}

// ============================================================================ grid
__global__ void k_body_cell(int cap, const float* center, const float* gp, const int* gd, const int* counts,
                            int* bodyCell) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cap) return;
    int S = counts[1];
    if (i >= S) { bodyCell[i] = -1; return; }
    int nX = gd[0], nY = gd[1], nZ = gd[2];
    int ix = cell_coord(center[i], gp[0], gp[4], nX);
    int iy = cell_coord(center[cap + i], gp[1], gp[4], nY);
    int iz = cell_coord(center[2 * cap + i], gp[2], gp[4], nZ);
    bodyCell[i] = ix + iy * nX + iz * (nX * nY);
}

extern "C" sbx_status sbx_grid_body_cell(sbx_ctx* ctx, int32_t cap, const float* center, const float* gp,
                                         const int32_t* gd, const int32_t* counts, int32_t* bodyCell) {
    SBX_REQUIRE(ctx && cap >= 0 && (cap == 0 || (center && gp && gd && counts && bodyCell)));
    if (cap == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_body_cell, blocks(cap), 256, cap, center, gp, gd, counts, bodyCell);
    return check_launch(ctx, "sbx_grid_body_cell");
}

extern "C" sbx_status sbx_grid_build(sbx_ctx* ctx, int32_t cap, const int32_t* bodyCell, const int32_t* counts,
                                     int32_t totalCells, int32_t* cellCount, int32_t* chunkSum, int32_t* offsets,
                                     int32_t* contents, int32_t contentsCap) {
    SBX_REQUIRE(ctx && cap >= 0 && totalCells > 0 && bodyCell && counts && cellCount && chunkSum && offsets &&
                contents);
    if (contentsCap < cap) return fail(ctx, SBX_EINVAL, "sbx_grid_build: contentsCap < cap");
    size_t tmpBytes = align8(sizeof(int) * (size_t)std::max(cap, 1));
    sbx_status st = ensure_scratch(ctx, tmpBytes + sizeof(int) * scan_tile_words(totalCells));
    if (st) return st;
    CountingSort cs{bodyCell, counts, 1, cap, totalCells, cellCount, chunkSum, offsets, contents, contentsCap,
                    (int*)ctx->scratch};
    cs.tileSum = reinterpret_cast<int*>(static_cast<char*>(ctx->scratch) + tmpBytes);
    return counting_sort(ctx, cs, "sbx_grid_build");
}

__global__ void k_broad_phase(int cap, const float* center, const float* R, const int* bodyCell, const int* offsets,
                              const int* contents, const int* gd, const float* gp, const int* counts, int* candPartner,
                              int* candCount) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cap) return;
    candCount[i] = 0;
    int S = counts[1];
    if (i >= S) return;
    int c = bodyCell[i];
    if (c < 0) return;
    int nX = gd[0], nY = gd[1], nZ = gd[2], nXY = nX * nY;
    float cutoff = gp[5];
    int cz = c / nXY, rem = c - cz * nXY, cy = rem / nX, cx = rem - cy * nX;
    float icx = center[i], icy = center[cap + i], icz = center[2 * cap + i], ri = R[i];
    int x0 = max(cx - 1, 0), x1 = min(cx + 1, nX - 1);
    int y0 = max(cy - 1, 0), y1 = min(cy + 1, nY - 1);
    int z0 = max(cz - 1, 0), z1 = min(cz + 1, nZ - 1);
    int cnt = 0;
    for (int zz = z0; zz <= z1; zz++)
        for (int yy = y0; yy <= y1; yy++)
            for (int xx = x0; xx <= x1; xx++) {
                int cc = xx + yy * nX + zz * nXY;
                int start = offsets[cc], end = offsets[cc + 1];
                for (int idx = start; idx < end; idx++) {
                    int j = contents[idx];
                    if (j <= i) continue;
                    float dx = icx - center[j];
                    float dy = icy - center[cap + j];
                    float dz = icz - center[2 * cap + j];
                    float distSq = dx * dx + dy * dy + dz * dz;
                    float reach = ri + R[j] + cutoff;
                    if (distSq <= reach * reach) {
                        if (cnt < MAX_CAND) candPartner[(int64_t)i * MAX_CAND + cnt] = j;
                        cnt++;
                    }
                }
            }
    candCount[i] = cnt;
}

extern "C" sbx_status sbx_grid_broad_phase(sbx_ctx* ctx, int32_t cap, const float* center, const float* R,
                                           const int32_t* bodyCell, const int32_t* offsets, const int32_t* contents,
                                           const int32_t* gd, const float* gp, const int32_t* counts,
                                           int32_t* candPartner, int32_t* candCount) {
    SBX_REQUIRE(ctx && cap >= 0 && (cap == 0 || (center && R && bodyCell && offsets && contents && gd && gp && counts &&
                                                 candPartner && candCount)));
    if (cap == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_broad_phase, blocks(cap, 128), 128, cap, center, R, bodyCell, offsets, contents, gd, gp, counts,
               candPartner, candCount);
    return check_launch(ctx, "sbx_grid_broad_phase");
}

__global__ void k_brute_force(int cap, const float* center, const float* R, const float* gp, const int* counts,
                              int* partner, int* count) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cap) return;
    count[i] = 0;
    int S = counts[1];
    if (i >= S) return;
    float cutoff = gp[5];
    float icx = center[i], icy = center[cap + i], icz = center[2 * cap + i], ri = R[i];
    int cnt = 0;
    for (int j = i + 1; j < S; j++) {
        float dx = icx - center[j];
        float dy = icy - center[cap + j];
        float dz = icz - center[2 * cap + j];
        float distSq = dx * dx + dy * dy + dz * dz;
        float reach = ri + R[j] + cutoff;
        if (distSq <= reach * reach) {
            if (cnt < MAX_CAND) partner[(int64_t)i * MAX_CAND + cnt] = j;
            cnt++;
        }
    }
    count[i] = cnt;
}

extern "C" sbx_status sbx_grid_brute_force(sbx_ctx* ctx, int32_t cap, const float* center, const float* R,
                                           const float* gp, const int32_t* counts, int32_t* partner, int32_t* count) {
    SBX_REQUIRE(ctx && cap >= 0 && (cap == 0 || (center && R && gp && counts && partner && count)));
    if (cap == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_brute_force, blocks(cap, 128), 128, cap, center, R, gp, counts, partner, count);
    return check_launch(ctx, "sbx_grid_brute_force");
}

// ============================================================================ binding
__global__ void k_grid_reachable(int nM, const float* head, const float* uVec, const float* rodUVec, int nSeg,
                                 const float* e1, const float* e2, const float* gp, const int* gd, const int* offsets,
                                 const int* contents, const int* ownerStore, const int* ownerSlot, int* reachSeg,
                                 int* reachCount, const float* kp) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nM) return;
    reachCount[m] = grid_reach_walk(m, nM, head, uVec, rodUVec, nSeg, e1, e2, gp, gd, offsets, contents, ownerStore,
                                    ownerSlot, reachSeg + (int64_t)m * MAX_CAND, kp[7], kp[8]);
}

extern "C" sbx_status sbx_binding_grid_reachable(sbx_ctx* ctx, const float* head, const float* uVec,
                                                 const float* rodUVec, int32_t nSeg, const float* e1, const float* e2,
                                                 const float* gp, const int32_t* gd, const int32_t* offsets,
                                                 const int32_t* contents, const int32_t* ownerStore,
                                                 const int32_t* ownerSlot, int32_t* reachSeg, int32_t* reachCount,
                                                 const float* kp, int32_t nM) {
    SBX_REQUIRE(ctx && nM >= 0 && (nM == 0 || (head && uVec && rodUVec && e1 && e2 && gp && gd && offsets &&
                                               contents && ownerStore && ownerSlot && reachSeg && reachCount && kp)));
    if (nM == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_grid_reachable, blocks(nM, 128), 128, nM, head, uVec, rodUVec, nSeg, e1, e2, gp, gd, offsets,
               contents, ownerStore, ownerSlot, reachSeg, reachCount, kp);
    return check_launch(ctx, "sbx_binding_grid_reachable");
}

// The endpoints of every grid entry in cell order (for grid_reach_walk_cells): one pass over
// the contents after the grid build, entries past offsets[C] untouched.
__global__ void k_cell_endpoints(int C, const int* offsets, const int* contents, const int* ownerStore,
                                 const int* ownerSlot, int nSeg, const float* e1, const float* e2, float4* cellE1,
                                 float4* cellE2) {
    int total = offsets[C];
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
        int j = contents[idx];
        float4 a = make_float4(0.f, 0.f, 0.f, __int_as_float(-1)), b = make_float4(0.f, 0.f, 0.f, 0.f);
        if (ownerStore[j] == STORE_FILAMENT) {
            int s = ownerSlot[j];
            a = make_float4(e1[s], e1[nSeg + s], e1[2 * nSeg + s], __int_as_float(s));
            b = make_float4(e2[s], e2[nSeg + s], e2[2 * nSeg + s], 0.f);
        }
        cellE1[idx] = a;
        cellE2[idx] = b;
    }
}

extern "C" sbx_status sbx_grid_cell_endpoints(sbx_ctx* ctx, int32_t cap, int32_t totalCells,
                                              const int32_t* gridCellOffsets, const int32_t* gridCellContents,
                                              const int32_t* ownerStore, const int32_t* ownerSlot, int32_t nSeg,
                                              const float* e1, const float* e2, float* cellEnd1, float* cellEnd2) {
    SBX_REQUIRE(ctx && cap >= 0 && totalCells > 0 && nSeg >= 0 && gridCellOffsets &&
                (cap == 0 || (gridCellContents && ownerStore && ownerSlot && cellEnd1 && cellEnd2 &&
                              ((uintptr_t)cellEnd1 & 15u) == 0 && ((uintptr_t)cellEnd2 & 15u) == 0)) &&
                (nSeg == 0 || (e1 && e2)));
    if (cap == 0) return SBX_OK;
    int nb = blocks(cap);
    if (nb > 148 * 16) nb = 148 * 16;
    SBX_LAUNCH(ctx, k_cell_endpoints, nb, 256, totalCells, gridCellOffsets, gridCellContents, ownerStore, ownerSlot,
               nSeg, e1, e2, reinterpret_cast<float4*>(cellEnd1), reinterpret_cast<float4*>(cellEnd2));
    return check_launch(ctx, "sbx_grid_cell_endpoints");
}

__global__ void k_grid_reachable_cells(int nM, const float* head, const float* uVec, const float* rodUVec,
                                       const float* gp, const int* gd, const int* offsets, const float4* cellE1,
                                       const float4* cellE2, int* reachSeg, int* reachCount, const float* kp) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nM) return;
    reachCount[m] = grid_reach_walk_cells(m, nM, head, uVec, rodUVec, gp, gd, offsets, cellE1, cellE2,
                                          reachSeg + (int64_t)m * MAX_CAND, kp[7], kp[8]);
}

extern "C" sbx_status sbx_fusion_grid_reachable(sbx_ctx* ctx, const float* head, const float* uVec,
                                                const float* rodUVec, const float* gp, const int32_t* gd,
                                                const int32_t* gridCellOffsets, const float* cellEnd1,
                                                const float* cellEnd2, int32_t* reachSeg, int32_t* reachCount,
                                                const float* kp, int32_t nM) {
    SBX_REQUIRE(ctx && nM >= 0 && (nM == 0 || (head && uVec && rodUVec && gp && gd && gridCellOffsets && cellEnd1 &&
                                               cellEnd2 && reachSeg && reachCount && kp)));
    if (nM == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_grid_reachable_cells, blocks(nM, 128), 128, nM, head, uVec, rodUVec, gp, gd, gridCellOffsets,
               reinterpret_cast<const float4*>(cellEnd1), reinterpret_cast<const float4*>(cellEnd2), reachSeg,
               reachCount, kp);
    return check_launch(ctx, "sbx_fusion_grid_reachable");
}

// ---------------------------------------------------------------- reach walk over staged cell rows
// BindingDetectionSystem.gridReachable (BindingDetectionSystem.java:161-227) for the heads
// binned in one tile of the grid (REACH_TILE_X consecutive x-cells of one y-row, every z),
// with the tile's neighbourhood staged in shared memory: the cell offsets of the 3 nZ rows
// around it (coalesced loads) and their cell-ordered endpoint pairs (cp.async.bulk, one
// copy per row and array, completion on an mbarrier; no multicast, source in this GPU's
// memory). Each head's walk then reads shared memory only, in the order of
// grid_reach_walk_cells (the same rows, cells and entries): the same lists and counts. A
// tile whose neighbourhood exceeds the staging capacity, a head past the tile's head list
// and a head that is not binned (the blocks after the tiles look for those) take
// grid_reach_walk_cells itself. A bulk-copy wait longer than one second sets bit 1 of the
// context's error word (reported as SBX_ETIMEOUT by sbx_ctx_sync), waits once more for the
// copies and leaves the tile's heads to the global walk.
constexpr int REACH_TILE_X = 64, REACH_ZMAX = 16, REACH_CAP_E = 768, REACH_HCAP = 256;
constexpr unsigned long long REACH_WAIT_NS = 1000000000ULL;

static size_t reach_tile_smem(int nZ) {
    return 2 * sizeof(float4) * REACH_CAP_E + sizeof(int) * ((size_t)3 * nZ * (REACH_TILE_X + 3) + 3 * nZ + 1) +
           sizeof(int) * REACH_HCAP;
}

__device__ __forceinline__ bool reach_bulk_wait(unsigned long long* mbar, unsigned phase) {
    unsigned mb = (unsigned)__cvta_generic_to_shared(mbar);
    unsigned done = 0, it = 0;
    unsigned long long t0 = 0;
    while (!done) {
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(done) : "r"(mb), "r"(phase) : "memory");
        if (!done && (++it & 15u) == 0) {
            unsigned long long now;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
            if (t0 == 0) t0 = now;
            else if (now - t0 > REACH_WAIT_NS) break;
        }
    }
    return done != 0;
}

__global__ void __launch_bounds__(128) k_reach_tiles(int nM, const float* head, const float* uVec,
                                                     const float* rodUVec, const float* gp, const int* gd, int nX,
                                                     int nY, int nZ, const int* offsets, const int* contents,
                                                     const int* ownerStore, const int* ownerSlot,
                                                     const int* bodyCell, int cap, const int* publishParams,
                                                     const float4* cellE1, const float4* cellE2, int* reachSeg,
                                                     int* reachCount, const float* kp, int* errWord) {
    extern __shared__ __align__(16) unsigned char rsm[];
    float4* sE1 = reinterpret_cast<float4*>(rsm);
    float4* sE2 = sE1 + REACH_CAP_E;
    const int W = REACH_TILE_X + 3, R = 3 * nZ;
    int* sOff = reinterpret_cast<int*>(sE2 + REACH_CAP_E);   // [R][W]: the staged rows' cell offsets
    int* sBase = sOff + R * W;                                 // [R + 1]: each row's first staged entry
    int* sHead = sBase + R + 1;                                // the tile's heads
    __shared__ int sNHead, sStaged;
    __shared__ __align__(8) unsigned long long mbar;
    const float tol = kp[7], align = kp[8];
    const int tilesX = (nX + REACH_TILE_X - 1) / REACH_TILE_X, nTiles = tilesX * nY;
    if ((int)blockIdx.x >= nTiles) {
        // heads that are in no grid cell: the global walk
        const int m = ((int)blockIdx.x - nTiles) * blockDim.x + threadIdx.x;
        if (m >= nM) return;
        const int b = publishParams[0] + m;
        if (b >= 0 && b < cap && bodyCell[b] >= 0) return;
        reachCount[m] = grid_reach_walk_cells(m, nM, head, uVec, rodUVec, gp, gd, offsets, cellE1, cellE2,
                                              reachSeg + (int64_t)m * MAX_CAND, tol, align);
        return;
    }
    const int ty = blockIdx.x / tilesX, tx0 = (blockIdx.x - ty * tilesX) * REACH_TILE_X;
    const int tx1 = min(tx0 + REACH_TILE_X, nX) - 1;             // the tile's last x-cell
    const int xa = max(tx0 - 1, 0), xb = min(tx1 + 1, nX - 1);    // staged x-cells
    const int nc = xb - xa + 2;                                   // offsets per staged row
    const int nXY = nX * nY;
    // (1) the staged rows' cell offsets (rows outside the grid hold zeros: no entries), eight
    // loads per thread in flight together
    for (int q0 = 0; q0 < R * nc; q0 += 8 * 128) {
        int v[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int q = q0 + j * 128 + (int)threadIdx.x;
            const int r = q / nc, k = q - r * nc;
            const int yy = ty - 1 + r / nZ, zz = r - (r / nZ) * nZ;
            v[j] = (q < R * nc && yy >= 0 && yy < nY) ? offsets[xa + k + yy * nX + zz * nXY] : 0;
        }
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int q = q0 + j * 128 + (int)threadIdx.x;
            if (q < R * nc) sOff[(q / nc) * W + (q - (q / nc) * nc)] = v[j];
        }
    }
    if (threadIdx.x == 0) {
        sNHead = 0;
        unsigned mb = (unsigned)__cvta_generic_to_shared(&mbar);
        asm volatile("mbarrier.init.shared.b64 [%0], 1;\n" :: "r"(mb) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    // (2) where each row lands in the staging buffer; the expected bytes before any copy
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int r = 0; r < R; r++) {
            sBase[r] = acc;
            acc += sOff[r * W + nc - 1] - sOff[r * W];
        }
        sBase[R] = acc;
        const bool staged = acc > 0 && acc <= REACH_CAP_E;
        sStaged = staged;
        if (staged) {
            unsigned mb = (unsigned)__cvta_generic_to_shared(&mbar);
            asm volatile("mbarrier.arrive.expect_tx.shared.b64 _, [%0], %1;\n" :: "r"(mb), "r"((unsigned)acc * 32u)
                         : "memory");
        }
    }
    __syncthreads();
    const bool staged = sStaged != 0;
    // (3) one bulk copy per staged row and array
    if (staged) {
        for (int q = threadIdx.x; q < 2 * R; q += blockDim.x) {
            const int r = q >> 1, n = sOff[r * W + nc - 1] - sOff[r * W];
            if (n <= 0) continue;
            float4* dst = ((q & 1) ? sE2 : sE1) + sBase[r];
            const float4* src = ((q & 1) ? cellE2 : cellE1) + sOff[r * W];
            unsigned d = (unsigned)__cvta_generic_to_shared(dst), mb = (unsigned)__cvta_generic_to_shared(&mbar);
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                         :: "r"(d), "l"(src), "r"((unsigned)n * 16u), "r"(mb) : "memory");
        }
    }
    // (4) meanwhile, the heads binned in the tile's own cells (staged rows y = ty): the rows'
    // entries as one sequence, four per thread in flight together
    int ePre[REACH_ZMAX + 1];
    ePre[0] = 0;
    for (int z = 0; z < nZ; z++) {
        const int r = nZ + z;
        ePre[z + 1] = ePre[z] + sOff[r * W + (tx1 + 1 - xa)] - sOff[r * W + (tx0 - xa)];
    }
    const int nOwn = ePre[nZ];
    for (int i0 = 0; i0 < nOwn; i0 += 4 * 128) {
        int slot[4], own[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int i = i0 + j * 128 + (int)threadIdx.x;
            slot[j] = -1;
            if (i < nOwn) {
                int z = 0;
                while (i >= ePre[z + 1]) z++;
                slot[j] = contents[sOff[(nZ + z) * W + (tx0 - xa)] + (i - ePre[z])];
            }
        }
#pragma unroll
        for (int j = 0; j < 4; j++) own[j] = slot[j] >= 0 ? ownerStore[slot[j]] : STORE_NONE;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (own[j] != STORE_MOTOR) continue;
            const int m = ownerSlot[slot[j]];
            const int h = atomicAdd(&sNHead, 1);
            if (h < REACH_HCAP) {
                sHead[h] = m;
            } else {
                reachCount[m] = grid_reach_walk_cells(m, nM, head, uVec, rodUVec, gp, gd, offsets, cellE1, cellE2,
                                                      reachSeg + (int64_t)m * MAX_CAND, tol, align);
            }
        }
    }
    bool ok = true;
    if (staged) {
        ok = __syncthreads_or(reach_bulk_wait(&mbar, 0)) != 0;
        if (!ok && threadIdx.x == 0) {
            *(volatile int*)errWord = 2;
            reach_bulk_wait(&mbar, 0);     // the copies may still be landing: one more bounded wait
        }
    }
    __syncthreads();
    // (5) the walks: the staged rows when the tile is staged, else the global walk
    const int nh = min(sNHead, REACH_HCAP);
    for (int h = threadIdx.x; h < nh; h += blockDim.x) {
        const int m = sHead[h];
        int* outSlice = reachSeg + (int64_t)m * MAX_CAND;
        const float hx = head[m], hy = head[nM + m];
        const int hcx = cell_coord(hx, gp[0], gp[4], nX), hcy = cell_coord(hy, gp[1], gp[4], nY);
        // (a head binned here lies in the tile's cells; anything else takes the global walk)
        if (!staged || !ok || hcy != ty || hcx < tx0 || hcx > tx1) {
            reachCount[m] = grid_reach_walk_cells(m, nM, head, uVec, rodUVec, gp, gd, offsets, cellE1, cellE2,
                                                  outSlice, tol, align);
            continue;
        }
        const float mx = head[m], my = head[nM + m], mz = head[2 * nM + m];
        const float mux = uVec[m], muy = uVec[nM + m], muz = uVec[2 * nM + m];
        const float rux = rodUVec[m], ruy = rodUVec[nM + m], ruz = rodUVec[2 * nM + m];
        const int cx = cell_coord(mx, gp[0], gp[4], nX), cy = cell_coord(my, gp[1], gp[4], nY),
                  cz = cell_coord(mz, gp[2], gp[4], nZ);
        const int x0 = max(cx - 1, 0), x1 = min(cx + 1, nX - 1);
        const int y0 = max(cy - 1, 0), y1 = min(cy + 1, nY - 1);
        const int z0 = max(cz - 1, 0), z1 = min(cz + 1, nZ - 1);
        int out = 0;
        for (int rr = 0; rr < 9; rr++) {
            const int zz = z0 + rr / 3, yy = y0 + rr % 3;
            if (zz > z1 || yy > y1) continue;
            const int r = (yy - (ty - 1)) * nZ + zz;           // the staged row (cy == ty)
            const int* ro = sOff + r * W;
            const int b0 = ro[x0 - xa], b1 = ro[x1 + 1 - xa];
            const int base = sBase[r] - ro[0];
            for (int e = b0; e < b1; e++) {
                const float4 a1 = sE1[base + e], a2 = sE2[base + e];
                const int sg = __float_as_int(a1.w);
                if (sg < 0) continue;
                const float d = reach_test_dist_sq(mx, my, mz, mux, muy, muz, rux, ruy, ruz, a1.x, a1.y, a1.z, a2.x,
                                                   a2.y, a2.z, tol, align);
                if (d >= 0.f) {
                    if (out < MAX_CAND) outSlice[out] = sg;
                    out++;
                }
            }
        }
        reachCount[m] = out;
    }
}

extern "C" sbx_status sbx_fusion_grid_reachable_staged(
    sbx_ctx* ctx, const float* head, const float* uVec, const float* rodUVec, const float* gp, const int32_t* gd,
    int32_t nX, int32_t nY, int32_t nZ, const int32_t* gridCellOffsets, const int32_t* gridCellContents,
    const int32_t* ownerStore, const int32_t* ownerSlot, const int32_t* bodyCell, int32_t cap,
    const int32_t* publishParams, const float* cellEnd1, const float* cellEnd2, int32_t* reachSeg,
    int32_t* reachCount, const float* kp, int32_t nM) {
    SBX_REQUIRE(ctx && nM >= 0 && nX > 0 && nY > 0 && nZ > 0 && cap >= 0 &&
                (nM == 0 || (head && uVec && rodUVec && gp && gd && gridCellOffsets && gridCellContents && ownerStore &&
                             ownerSlot && bodyCell && publishParams && cellEnd1 && cellEnd2 && reachSeg &&
                             reachCount && kp)));
    if (nM == 0) return SBX_OK;
    if (nZ > REACH_ZMAX)
        return sbx_fusion_grid_reachable(ctx, head, uVec, rodUVec, gp, gd, gridCellOffsets, cellEnd1, cellEnd2,
                                         reachSeg, reachCount, kp, nM);
    const size_t smem = reach_tile_smem(nZ);
    if (cudaFuncSetAttribute(k_reach_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return fail(ctx, SBX_ECUDA, "sbx_fusion_grid_reachable_staged: shared memory attribute");
    const int64_t tiles = (int64_t)((nX + REACH_TILE_X - 1) / REACH_TILE_X) * nY;
    const int64_t grid = tiles + (nM + 127) / 128;
    if (grid > 0x7fffffff) return fail(ctx, SBX_EINVAL, "sbx_fusion_grid_reachable_staged: grid too large");
    k_reach_tiles<<<(unsigned)grid, 128, smem, ctx->stream>>>(
        nM, head, uVec, rodUVec, gp, gd, nX, nY, nZ, gridCellOffsets, gridCellContents, ownerStore, ownerSlot, bodyCell,
        cap, publishParams, reinterpret_cast<const float4*>(cellEnd1), reinterpret_cast<const float4*>(cellEnd2),
        reachSeg, reachCount, kp, ctx->err_dev);
    ctx->launches++;
    return check_launch(ctx, "sbx_fusion_grid_reachable_staged");
}

__global__ void k_brute_reachable(int nM, const float* head, const float* uVec, const float* rodUVec, int nSeg,
                                  const float* e1, const float* e2, int* reachSeg, int* reachCount, const float* kp) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nM) return;
    float mx = head[m], my = head[nM + m], mz = head[2 * nM + m];
    float mux = uVec[m], muy = uVec[nM + m], muz = uVec[2 * nM + m];
    float rux = rodUVec[m], ruy = rodUVec[nM + m], ruz = rodUVec[2 * nM + m];
    float tol = kp[7], align = kp[8];
    int out = 0;
    for (int s = 0; s < nSeg; s++) {
        float d = reach_test_dist_sq(mx, my, mz, mux, muy, muz, rux, ruy, ruz, e1[s], e1[nSeg + s], e1[2 * nSeg + s],
                                     e2[s], e2[nSeg + s], e2[2 * nSeg + s], tol, align);
        if (d >= 0.f) {
            if (out < MAX_CAND) reachSeg[(int64_t)m * MAX_CAND + out] = s;
            out++;
        }
    }
    reachCount[m] = out;
}

extern "C" sbx_status sbx_binding_brute_reachable(sbx_ctx* ctx, const float* head, const float* uVec,
                                                  const float* rodUVec, int32_t nSeg, const float* e1, const float* e2,
                                                  int32_t* reachSeg, int32_t* reachCount, const float* kp, int32_t nM) {
    SBX_REQUIRE(ctx && nM >= 0 && (nM == 0 || (head && uVec && rodUVec && e1 && e2 && reachSeg && reachCount && kp)));
    if (nM == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_brute_reachable, blocks(nM, 128), 128, nM, head, uVec, rodUVec, nSeg, e1, e2, reachSeg,
               reachCount, kp);
    return check_launch(ctx, "sbx_binding_brute_reachable");
}

__global__ void k_bind_nearest(int nM, const float* head, const float* uVec, const float* rodUVec, int nSeg,
                               const float* e1, const float* e2, const int* candSeg, const int* candCount,
                               int* boundSeg, float* bindArc, const float* kp) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nM) return;
    if (boundSeg[m] != FREE_BINDABLE) return;
    int best;
    float arc;
    if (bind_nearest_scan(m, nM, head, uVec, rodUVec, nSeg, e1, e2, candSeg + (int64_t)m * MAX_CAND, candCount[m],
                          kp[7], kp[8], &best, &arc)) {
        boundSeg[m] = best;
        bindArc[m] = arc;
    }
}

extern "C" sbx_status sbx_binding_bind_nearest(sbx_ctx* ctx, const float* head, const float* uVec,
                                               const float* rodUVec, int32_t nSeg, const float* e1, const float* e2,
                                               const int32_t* candSeg, const int32_t* candCount, int32_t* boundSeg,
                                               float* bindArc, const float* kp, int32_t nM) {
    SBX_REQUIRE(ctx && nM >= 0 && (nM == 0 || (head && uVec && rodUVec && e1 && e2 && candSeg && candCount &&
                                               boundSeg && bindArc && kp)));
    if (nM == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_bind_nearest, blocks(nM, 128), 128, nM, head, uVec, rodUVec, nSeg, e1, e2, candSeg, candCount,
               boundSeg, bindArc, kp);
    return check_launch(ctx, "sbx_binding_bind_nearest");
}

__global__ void k_release(int nM, int* boundSeg, const float* fdf, const float* fm, int* cooldown, int* stats,
                          int* capStats, const float* kp, const int* counts) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nM) return;
    int bs = boundSeg[m], cd = cooldown[m], sb = stats[2 * m], sr = stats[2 * m + 1], cs = capStats[m];
    release_one(m, bs, cd, sb, sr, cs, fdf[m], fm[m], kp, counts[1], counts[2]);
    boundSeg[m] = bs; cooldown[m] = cd; stats[2 * m] = sb; stats[2 * m + 1] = sr; capStats[m] = cs;
}

extern "C" sbx_status sbx_nucleotide_release(sbx_ctx* ctx, int32_t nM, int32_t* boundSeg, const float* fdf,
                                             const float* fm, int32_t* cooldown, int32_t* stats, int32_t* capStats,
                                             const float* kp, const int32_t* counts) {
    SBX_REQUIRE(ctx && nM >= 0 && (nM == 0 || (boundSeg && fdf && fm && cooldown && stats && capStats && kp && counts)));
    if (nM == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_release, blocks(nM), 256, nM, boundSeg, fdf, fm, cooldown, stats, capStats, kp, counts);
    return check_launch(ctx, "sbx_nucleotide_release");
}

__global__ void k_cycle(int nM, int* state, const int* boundSeg, const float* hist, const float* np, const int* counts) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nM) return;
    state[m] = cycle_one(m, state[m], boundSeg[m] >= 0, hist + 10 * m, np, counts[1], counts[2]);
}

extern "C" sbx_status sbx_nucleotide_cycle(sbx_ctx* ctx, int32_t nM, int32_t* state, const int32_t* boundSeg,
                                           const float* hist, const float* np, const int32_t* counts) {
    SBX_REQUIRE(ctx && nM >= 0 && (nM == 0 || (state && boundSeg && hist && np && counts)));
    if (nM == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_cycle, blocks(nM), 256, nM, state, boundSeg, hist, np, counts);
    return check_launch(ctx, "sbx_nucleotide_cycle");
}

// ============================================================================ cross-bridge
__global__ void k_bond(int nB, const float* mC, const float* mU, const float* mY, const float* mBRG, int nSeg,
                       const float* fC, const float* fU, const float* fY, const float* fBRG, const float* fLen,
                       const int* boundSeg, const float* bindArc, const int* nuc, float* bondData, const float* xb) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nB / 3) return;
    float out[XB_STRIDE];
    int s = boundSeg[m];
    if (!SBX_IDX_OK_OR_NONE(s, nSeg, CK_BOUND_SEG)) s = -1;
    bond_one(m, nB, mC, mU, mY, mBRG, nSeg, fC, fU, fY, fBRG, fLen, s, bindArc[m], nuc[m], xb, out);
    for (int k = 0; k < XB_STRIDE; k++) bondData[m * XB_STRIDE + k] = out[k];
}

extern "C" sbx_status sbx_xbridge_bond_forces(sbx_ctx* ctx, int32_t nB, const float* mC, const float* mU,
                                              const float* mY, const float* mBRG, int32_t nSeg, const float* fC,
                                              const float* fU, const float* fY, const float* fBRG, const float* fLen,
                                              const int32_t* boundSeg, const float* bindArc, const int32_t* nuc,
                                              float* bondData, const float* xb) {
    SBX_REQUIRE(ctx && nB >= 0 && (nB < 3 || (mC && mU && mY && mBRG && fC && fU && fY && fBRG && fLen && boundSeg &&
                                              bindArc && nuc && bondData && xb)));
    if (nB < 3) return SBX_OK;
    SBX_LAUNCH(ctx, k_bond, blocks(nB / 3), 256, nB, mC, mU, mY, mBRG, nSeg, fC, fU, fY, fBRG, fLen, boundSeg, bindArc,
               nuc, bondData, xb);
    return check_launch(ctx, "sbx_xbridge_bond_forces");
}

__global__ void k_apply_head(int nB, const float* bondData, float* F, float* T) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nB / 3) return;
    int h = 3 * m + 2, d = m * XB_STRIDE;
    for (int k = 0; k < 3; k++) {
        F[k * nB + h] = F[k * nB + h] + bondData[d + k];
        T[k * nB + h] = T[k * nB + h] + bondData[d + 3 + k];
    }
}

extern "C" sbx_status sbx_xbridge_apply_head_force(sbx_ctx* ctx, int32_t nB, const float* bondData, float* F,
                                                   float* T) {
    SBX_REQUIRE(ctx && nB >= 0 && (nB < 3 || (bondData && F && T)));
    if (nB < 3) return SBX_OK;
    SBX_LAUNCH(ctx, k_apply_head, blocks(nB / 3), 256, nB, bondData, F, T);
    return check_launch(ctx, "sbx_xbridge_apply_head_force");
}

__global__ void k_register(int nM, const float* bondData, const int* boundSeg, float* fdf, float* fm, float* hist,
                           int* place) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nM) return;
    register_force_dot_one(m, bondData, boundSeg[m] >= 0, fdf, fm, hist, place);
}

extern "C" sbx_status sbx_xbridge_register_force_dot(sbx_ctx* ctx, int32_t nM, const float* bondData,
                                                     const int32_t* boundSeg, float* fdf, float* fm, float* hist,
                                                     int32_t* place) {
    SBX_REQUIRE(ctx && nM >= 0 && (nM == 0 || (bondData && boundSeg && fdf && fm && hist && place)));
    if (nM == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_register, blocks(nM), 256, nM, bondData, boundSeg, fdf, fm, hist, place);
    return check_launch(ctx, "sbx_xbridge_register_force_dot");
}

extern "C" sbx_status sbx_csr_build(sbx_ctx* ctx, const int32_t* keys, int32_t nItems, int32_t nRows,
                                    int32_t* rowCount, int32_t* rowOffsets, int32_t* rowList) {
    SBX_REQUIRE(ctx && nItems >= 0 && nRows > 0 && rowCount && rowOffsets && (nItems == 0 || (keys && rowList)));
    size_t chunks = (size_t)(nRows + SCAN_CHUNK - 1) / SCAN_CHUNK + 1;
    size_t intBytes = align8(sizeof(int) * (chunks + (size_t)std::max(nItems, 1)));
    sbx_status st = ensure_scratch(ctx, intBytes + sizeof(int) * scan_tile_words(nRows));
    if (st) return st;
    int* s = (int*)ctx->scratch;
    CountingSort cs{keys, nullptr, 0, nItems, nRows, rowCount, s, rowOffsets, rowList, nItems, s + chunks};
    cs.tileSum = reinterpret_cast<int*>(static_cast<char*>(ctx->scratch) + intBytes);
    return counting_sort(ctx, cs, "sbx_csr_build");
}

extern "C" sbx_status sbx_csr_build_payload(sbx_ctx* ctx, const int32_t* keys, int32_t nItems, int32_t nRows,
                                            int32_t* rowCount, int32_t* rowOffsets, int32_t* rowList,
                                            const float* payload, int32_t payloadStride, int32_t payloadOffset,
                                            const int32_t* guard, float* rowPayload) {
    SBX_REQUIRE(ctx && nItems >= 0 && nRows > 0 && rowCount && rowOffsets && payloadStride >= 6 &&
                payloadOffset >= 0 && payloadOffset + 6 <= payloadStride &&
                (nItems == 0 || (keys && rowList && payload && rowPayload && aligned8(rowPayload))));
    size_t chunks = (size_t)(nRows + SCAN_CHUNK - 1) / SCAN_CHUNK + 1;
    size_t intBytes = align8(sizeof(int) * (chunks + (size_t)std::max(nItems, 1)));
    sbx_status st = ensure_scratch(ctx, intBytes + sizeof(int) * scan_tile_words(nRows));
    if (st) return st;
    int* s = (int*)ctx->scratch;
    CountingSort cs{keys, nullptr, 0, nItems, nRows, rowCount, s, rowOffsets, rowList, nItems, s + chunks};
    cs.tileSum = reinterpret_cast<int*>(static_cast<char*>(ctx->scratch) + intBytes);
    cs.payload = payload;
    cs.pStride = payloadStride;
    cs.pOff = payloadOffset;
    cs.guard = guard;
    cs.rowPayload = rowPayload;
    return counting_sort(ctx, cs, "sbx_csr_build_payload");
}

__global__ void k_csr_gather(int nRows, const int* offsets, const int* list, const float* payload, int stride, int off,
                             const int* guard, float* F, float* T) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nRows) return;
    double f[3], t[3];
    csr_gather_row(s, offsets, list, payload, stride, off, guard, f, t);
    for (int k = 0; k < 3; k++) {
        F[k * nRows + s] = (float)(F[k * nRows + s] + f[k]);
        T[k * nRows + s] = (float)(T[k * nRows + s] + t[k]);
    }
}

extern "C" sbx_status sbx_xbridge_seg_gather(sbx_ctx* ctx, int32_t nSeg, const int32_t* offsets, const int32_t* list,
                                             const float* bondData, float* F, float* T) {
    SBX_REQUIRE(ctx && nSeg >= 0 && (nSeg == 0 || (offsets && list && bondData && F && T)));
    if (nSeg == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_csr_gather, blocks(nSeg), 256, nSeg, offsets, list, bondData, XB_STRIDE, 6, nullptr, F, T);
    return check_launch(ctx, "sbx_xbridge_seg_gather");
}

__global__ void k_xb_brute_gather(int nSeg, int nM, const int* boundSeg, const float* bd, float* F, float* T) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nSeg) return;
    double f[3] = {0, 0, 0}, t[3] = {0, 0, 0};
    for (int m = 0; m < nM; m++) {
        if (boundSeg[m] != s) continue;
        int d = m * XB_STRIDE;
        for (int k = 0; k < 3; k++) { f[k] += bd[d + 6 + k]; t[k] += bd[d + 9 + k]; }
    }
    for (int k = 0; k < 3; k++) { F[k * nSeg + s] = (float)f[k]; T[k * nSeg + s] = (float)t[k]; }
}

extern "C" sbx_status sbx_xbridge_brute_gather(sbx_ctx* ctx, int32_t nSeg, int32_t nM, const int32_t* boundSeg,
                                               const float* bd, float* F, float* T) {
    SBX_REQUIRE(ctx && nSeg >= 0 && nM >= 0 && (nSeg == 0 || (boundSeg && bd && F && T)));
    if (nSeg == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_xb_brute_gather, blocks(nSeg), 256, nSeg, nM, boundSeg, bd, F, T);
    return check_launch(ctx, "sbx_xbridge_brute_gather");
}

// ============================================================================ crosslinkers
__global__ void k_xl_count(int nLinks, int nSeg, const int* state, const int* A, const int* B, int* count) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nLinks || state[k] < 0) return;
    if (!SBX_IDX_OK(A[k], nSeg, CK_LINK_END) || !SBX_IDX_OK(B[k], nSeg, CK_LINK_END)) return;
    atomicAdd(&count[A[k]], 1);
    atomicAdd(&count[B[k]], 1);
}

extern "C" sbx_status sbx_xlink_count_active(sbx_ctx* ctx, int32_t nLinks, const int32_t* state, const int32_t* A,
                                             const int32_t* B, int32_t nSeg, int32_t* count) {
    SBX_REQUIRE(ctx && nLinks >= 0 && nSeg >= 0 && (nSeg == 0 || count) && (nLinks == 0 || (state && A && B)));
    if (nSeg > 0 && cudaMemsetAsync(count, 0, sizeof(int) * nSeg, ctx->stream) != cudaSuccess)
        return fail(ctx, SBX_ECUDA, "sbx_xlink_count_active: memset");
    if (nLinks == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_xl_count, blocks(nLinks), 256, nLinks, nSeg, state, A, B, count);
    return check_launch(ctx, "sbx_xlink_count_active");
}

__global__ void k_xl_forces(int nSeg, const float* fC, const float* fU, const float* fE1, const float* fBTG,
                            int nLinks, const int* A, const int* B, const float* loc1, const float* loc2,
                            const int* ct, float* xd, const float* xp) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nLinks) return;
    if (!SBX_IDX_OK_OR_NONE(A[k], nSeg, CK_LINK_END) || !SBX_IDX_OK_OR_NONE(B[k], nSeg, CK_LINK_END)) return;
    float out[XL_STRIDE];
    link_forces_one(k, nSeg, fC, fU, fE1, fBTG, A[k], B[k], loc1[k], loc2[k], ct, xp, out);
    for (int j = 0; j < XL_STRIDE; j++) xd[k * XL_STRIDE + j] = out[j];
}

extern "C" sbx_status sbx_xlink_forces(sbx_ctx* ctx, int32_t nSeg, const float* fC, const float* fU, const float* fE1,
                                       const float* fBTG, int32_t nLinks, const int32_t* A, const int32_t* B,
                                       const float* loc1, const float* loc2, const int32_t* ct, float* xd,
                                       const float* xp) {
    SBX_REQUIRE(ctx && nLinks >= 0 && (nLinks == 0 || (fC && fU && fE1 && fBTG && A && B && loc1 && loc2 && ct && xd &&
                                                       xp)));
    if (nLinks == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_xl_forces, blocks(nLinks), 256, nSeg, fC, fU, fE1, fBTG, nLinks, A, B, loc1, loc2, ct, xd, xp);
    return check_launch(ctx, "sbx_xlink_forces");
}

__global__ void k_xl_torsion(int nSeg, const float* fU, int nLinks, const int* A, const int* B, const int* state,
                             const int* orient, float* hist, int* place, float* xd, const float* tp) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nLinks) return;
    if (tp[1] < 0.5f) return;
    if (!SBX_IDX_OK_OR_NONE(A[k], nSeg, CK_LINK_END) || !SBX_IDX_OK_OR_NONE(B[k], nSeg, CK_LINK_END)) return;
    link_torsion_one(k, nSeg, fU, A[k], B[k], state[k], orient[k], hist, place, xd, tp[0]);
}

extern "C" sbx_status sbx_xlink_torsion(sbx_ctx* ctx, int32_t nSeg, const float* fU, int32_t nLinks, const int32_t* A,
                                        const int32_t* B, const int32_t* state, const int32_t* orient, float* hist,
                                        int32_t* place, float* xd, const float* tp) {
    SBX_REQUIRE(ctx && nLinks >= 0 && (nLinks == 0 || (fU && A && B && state && orient && hist && place && xd && tp)));
    if (nLinks == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_xl_torsion, blocks(nLinks), 256, nSeg, fU, nLinks, A, B, state, orient, hist, place, xd, tp);
    return check_launch(ctx, "sbx_xlink_torsion");
}

extern "C" sbx_status sbx_xlink_seg_gather(sbx_ctx* ctx, int32_t side, int32_t nSeg, const int32_t* offsets,
                                           const int32_t* list, const float* xd, const int32_t* state, float* F,
                                           float* T) {
    SBX_REQUIRE(ctx && (side == 0 || side == 1) && nSeg >= 0 && (nSeg == 0 || (offsets && list && xd && state && F &&
                                                                              T)));
    if (nSeg == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_csr_gather, blocks(nSeg), 256, nSeg, offsets, list, xd, XL_STRIDE, side == 0 ? 0 : 6, state, F,
               T);
    return check_launch(ctx, "sbx_xlink_seg_gather");
}

__global__ void k_xl_brute_gather(int nSeg, int nLinks, const int* A, const int* B, const float* xd, const int* state,
                                  float* F, float* T) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nSeg) return;
    double f[3] = {0, 0, 0}, t[3] = {0, 0, 0};
    for (int k = 0; k < nLinks; k++) {
        if (state[k] < 0) continue;
        int d = k * XL_STRIDE;
        if (A[k] == s) for (int j = 0; j < 3; j++) { f[j] += xd[d + j]; t[j] += xd[d + 3 + j]; }
        if (B[k] == s) for (int j = 0; j < 3; j++) { f[j] += xd[d + 6 + j]; t[j] += xd[d + 9 + j]; }
    }
    for (int j = 0; j < 3; j++) { F[j * nSeg + s] = (float)f[j]; T[j * nSeg + s] = (float)t[j]; }
}

extern "C" sbx_status sbx_xlink_brute_gather(sbx_ctx* ctx, int32_t nSeg, int32_t nLinks, const int32_t* A,
                                             const int32_t* B, const float* xd, const int32_t* state, float* F,
                                             float* T) {
    SBX_REQUIRE(ctx && nSeg >= 0 && nLinks >= 0 && (nSeg == 0 || (A && B && xd && state && F && T)));
    if (nSeg == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_xl_brute_gather, blocks(nSeg), 256, nSeg, nLinks, A, B, xd, state, F, T);
    return check_launch(ctx, "sbx_xlink_brute_gather");
}

__global__ void k_xl_unbind(int nSeg, const float* fU, const float* fE1, int nLinks, const int* A, const int* B,
                            const float* loc1, const float* loc2, int* state, float* hist, int* place,
                            const float* op, const int* counts) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nLinks) return;
    if (state[k] < 0) return;
    if (!SBX_IDX_OK_OR_NONE(A[k], nSeg, CK_LINK_END) || !SBX_IDX_OK_OR_NONE(B[k], nSeg, CK_LINK_END)) return;
    if (unbind_one(k, nSeg, fU, fE1, A[k], B[k], loc1[k], loc2[k], hist, place, op, counts[1], counts[2]))
        state[k] = LINK_FREE;
}

extern "C" sbx_status sbx_xlink_unbind(sbx_ctx* ctx, int32_t nSeg, const float* fU, const float* fE1, int32_t nLinks,
                                       const int32_t* A, const int32_t* B, const float* loc1, const float* loc2,
                                       int32_t* state, float* hist, int32_t* place, const float* op,
                                       const int32_t* counts) {
    SBX_REQUIRE(ctx && nLinks >= 0 && (nLinks == 0 || (fU && fE1 && A && B && loc1 && loc2 && state && hist && place &&
                                                       op && counts)));
    if (nLinks == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_xl_unbind, blocks(nLinks), 256, nSeg, fU, fE1, nLinks, A, B, loc1, loc2, state, hist, place, op,
               counts);
    return check_launch(ctx, "sbx_xlink_unbind");
}

// ============================================================================ myosin structure
// MotorJointSystem.joints (MotorJointSystem.java:72-197): one thread per motor evaluates its
// two joints once and accumulates them into its rod, lever and head in the reference order.
__global__ void k_joints(int nB, const float* coord, const float* uVec, const float* segLength, const float* bTG,
                         const float* bRG, float* F, float* T, const int* nuc, const float* jp) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nB / 3) return;
    int st = nuc[m];
    MotorJoint J2 = motor_joint(m, 0, nB, coord, uVec, segLength, bTG, bRG, jp);
    MotorJoint J1 = motor_joint(m, 1, nB, coord, uVec, segLength, bTG, bRG, jp);
    for (int role = 0; role < 3; role++) {
        int s = 3 * m + role;
        double f[3] = {0.0, 0.0, 0.0}, t[3] = {0.0, 0.0, 0.0};
        if (role == 0 || role == 1) motor_joint_apply(J2, 0, role == 1, st, s, nB, uVec, segLength, jp, f, t);
        if (role == 1 || role == 2) motor_joint_apply(J1, 1, role == 2, st, s, nB, uVec, segLength, jp, f, t);
        for (int k = 0; k < 3; k++) {
            F[k * nB + s] = (float)(F[k * nB + s] + f[k]);
            T[k * nB + s] = (float)(T[k * nB + s] + t[k]);
        }
    }
}

extern "C" sbx_status sbx_motor_joints(sbx_ctx* ctx, int32_t nB, const float* coord, const float* uVec,
                                       const float* segLength, const float* bTG, const float* bRG, float* F, float* T,
                                       const int32_t* nuc, const float* jp) {
    SBX_REQUIRE(ctx && nB >= 0 && nB % 3 == 0 && (nB == 0 || (coord && uVec && segLength && bTG && bRG && F && T &&
                                                              nuc && jp)));
    if (nB == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_joints, blocks(nB / 3, 128), 128, nB, coord, uVec, segLength, bTG, bRG, F, T, nuc, jp);
    return check_launch(ctx, "sbx_motor_joints");
}

__global__ void k_couple(int nB, const float* coord, const float* uVec, const float* segLength, const float* bTG,
                         const float* bRG, float* F, float* T, int nD, const int* mA, const int* mB, const int* par,
                         const float* dp, const int* boundSeg) {
    int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= nD) return;
    couple_one(nB, coord, uVec, segLength, bTG, bRG, GlobalAcc{F, T, nB}, mA[d], mB[d], par[d] != 0, dp, boundSeg);
}

extern "C" sbx_status sbx_dimer_couple(sbx_ctx* ctx, int32_t nB, const float* coord, const float* uVec,
                                       const float* segLength, const float* bTG, const float* bRG, float* F, float* T,
                                       int32_t nD, const int32_t* mA, const int32_t* mB, const int32_t* par,
                                       const float* dp, const int32_t* boundSeg) {
    SBX_REQUIRE(ctx && nD >= 0 && (nD == 0 || (coord && uVec && segLength && bTG && bRG && F && T && mA && mB && par &&
                                               dp && boundSeg)));
    if (nD == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_couple, blocks(nD), 256, nB, coord, uVec, segLength, bTG, bRG, F, T, nD, mA, mB, par, dp,
               boundSeg);
    return check_launch(ctx, "sbx_dimer_couple");
}

__global__ void k_tether(int nMB, const float* mC, const float* mU, const float* mL, const float* mBTG,
                         const float* mBRG, float* mF, float* mT, int nBb, const float* bbC, const float* bbU,
                         const float* inv, int nD, const int* hbs, const int* mA, const float* ax, float* miniData,
                         const float* mp) {
    int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= nD) return;
    tether_one(d, nMB, mC, mU, mL, mBTG, mBRG, GlobalAcc{mF, mT, nMB}, nBb, bbC, bbU, inv, hbs[d], mA[d], ax[d], miniData, mp);
}

extern "C" sbx_status sbx_mini_tether(sbx_ctx* ctx, int32_t nMB, const float* mC, const float* mU, const float* mL,
                                      const float* mBTG, const float* mBRG, float* mF, float* mT, int32_t nBb,
                                      const float* bbC, const float* bbU, const float* inv, int32_t nD,
                                      const int32_t* hbs, const int32_t* mA, const float* ax, float* miniData,
                                      const float* mp) {
    SBX_REQUIRE(ctx && nD >= 0 && (nD == 0 || (mC && mU && mL && mBTG && mBRG && mF && mT && bbC && bbU && inv && hbs &&
                                               mA && ax && miniData && mp)));
    if (nD == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_tether, blocks(nD), 256, nMB, mC, mU, mL, mBTG, mBRG, mF, mT, nBb, bbC, bbU, inv, nD, hbs, mA, ax,
               miniData, mp);
    return check_launch(ctx, "sbx_mini_tether");
}

extern "C" sbx_status sbx_mini_backbone_gather(sbx_ctx* ctx, int32_t nBb, const int32_t* offsets, const int32_t* list,
                                               const float* miniData, float* F, float* T) {
    SBX_REQUIRE(ctx && nBb >= 0 && (nBb == 0 || (offsets && list && miniData && F && T)));
    if (nBb == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_csr_gather, blocks(nBb), 256, nBb, offsets, list, miniData, MINI_STRIDE, 0, nullptr, F, T);
    return check_launch(ctx, "sbx_mini_backbone_gather");
}

// ThermostatDiag.torsionalRestore (ThermostatDiag.java:127-145); statistical diagnostic
__global__ void k_torsional_restore(int nMotors, const float* uVec, const float* bRG, float* T, double coeff,
                                    double dt) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nMotors) return;
    int nB = 3 * nMotors, rod = 3 * m;
    double ux = uVec[rod], uy = uVec[nB + rod], uz = uVec[2 * nB + rod];
    double axx = uy, axy = -ux, axz = 0.0;
    double am2 = axx * axx + axy * axy + axz * axz;
    if (am2 <= 1.0e-30) return;
    double im = 1.0 / sqrt(am2);
    axx *= im; axy *= im; axz *= im;
    double dot = uz;
    if (dot > 1) dot = 1;
    if (dot < -1) dot = -1;
    double angDeg = acos(dot) * 180.0 / PI_D;
    double invBRG = 1.0 / bRG[nB + rod];
    double tmag = coeff * (PI_D / 180.0) * angDeg / (invBRG * dt);
    T[rod] = (float)(T[rod] + axx * tmag);
    T[nB + rod] = (float)(T[nB + rod] + axy * tmag);
    T[2 * nB + rod] = (float)(T[2 * nB + rod] + axz * tmag);
}

extern "C" sbx_status sbx_thermostat_torsional_restore(sbx_ctx* ctx, int32_t nMotors, const float* uVec,
                                                       const float* bRG, float* T, double coeff, double dt) {
    SBX_REQUIRE(ctx && nMotors >= 0 && (nMotors == 0 || (uVec && bRG && T)));
    if (nMotors == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_torsional_restore, blocks(nMotors), 256, nMotors, uVec, bRG, T, coeff, dt);
    return check_launch(ctx, "sbx_thermostat_torsional_restore");
}

// ============================================================================ deflection support
// DeflectionSupport.seedAccumulators (DeflectionSupport.java:24-33): forceSum = load * extForce
// with load = (float)counts[3], torqueSum = 0
__global__ void k_seed_accumulators(int n, float* F, float* T, const float* ext, const int* counts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float load = (float)counts[3];
    for (int k = 0; k < 3; k++) {
        F[k * n + i] = load * ext[k * n + i];
        T[k * n + i] = 0.f;
    }
}

extern "C" sbx_status sbx_deflection_seed_accumulators(sbx_ctx* ctx, int32_t n, float* forceSum, float* torqueSum,
                                                       const float* extForce, const int32_t* counts) {
    SBX_REQUIRE(ctx && n >= 0 && (n == 0 || (forceSum && torqueSum && extForce && counts)));
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_seed_accumulators, blocks(n), 256, n, forceSum, torqueSum, extForce, counts);
    return check_launch(ctx, "sbx_deflection_seed_accumulators");
}

// DeflectionSupport.pinEndpoints (DeflectionSupport.java:40-58): pin p translates segment
// pinSeg[p] so that its end pinEnd[p] (1 = end1, else end2) sits on pinAnchor[3p..3p+2]
__global__ void k_pin_endpoints(int n, float* coord, const float* uVec, const float* segLength, int P,
                                const int* pinSeg, const int* pinEnd, const float* anchor) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    int s = pinSeg[p];
    if (s < 0 || s >= n) return;
    float c[3] = {coord[s], coord[n + s], coord[2 * n + s]};
    float u[3] = {uVec[s], uVec[n + s], uVec[2 * n + s]};
    float half = 0.5f * segLength[s];
    float sgn = pinEnd[p] == 1 ? -1.f : 1.f;
    for (int k = 0; k < 3; k++) {
        float e = sgn < 0.f ? c[k] - half * u[k] : c[k] + half * u[k];
        float d = anchor[3 * p + k] - e;
        coord[k * n + s] = c[k] + d;
    }
}

extern "C" sbx_status sbx_deflection_pin_endpoints(sbx_ctx* ctx, int32_t n, float* coord, const float* uVec,
                                                   const float* segLength, int32_t nPins, const int32_t* pinSeg,
                                                   const int32_t* pinEnd, const float* pinAnchor) {
    SBX_REQUIRE(ctx && n >= 0 && nPins >= 0 && (nPins == 0 || (coord && uVec && segLength && pinSeg && pinEnd &&
                                                               pinAnchor)));
    if (nPins == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_pin_endpoints, blocks(nPins), 256, n, coord, uVec, segLength, nPins, pinSeg, pinEnd, pinAnchor);
    return check_launch(ctx, "sbx_deflection_pin_endpoints");
}

SBX_CHECK_EXPORT(systems)
