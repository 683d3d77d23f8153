// sbx_mlp.cu — the surrogate ensemble's kernels: BF16 GEMMs on the 5th-generation tensor
// cores (tcgen05.mma, FP32 accumulators in tensor memory) with fused bias / GELU / transpose
// epilogues, and the small elementwise kernels of training (loss gradient, GELU backward,
// bias gradients, Adam).
//
// GEMM: C[M x N] = A[M x K] . B[N x K]^T, A and B row-major BF16 (K contiguous, "K-major"),
// K <= 256. One CTA (16 warps) per SM keeps its B tile (up to 256 columns) in shared memory
// and loops over 128-row tiles of C, staging the next tile's A while the current tile's
// epilogue runs: the A and B tiles are staged in shared memory in the
// canonical no-swizzle K-major layout (8 x 16-byte core matrices; core matrix (row group g,
// k group c) at ((g * Kp/8) + c) * 128 bytes), one thread issues K/16 MMAs (M = 128, N = the
// tile width) into TMEM and commits them to an mbarrier, and the epilogue reads the
// accumulators back with tcgen05.ld: warp w takes TMEM lanes (rows) 32 (w mod 4) .. +31 and
// every fourth 16-column chunk from chunk w / 4, adds the bias, applies GELU and writes each
// row's 16 values with vector stores (the transposed output by lanes along the rows).
// blockIdx.z selects an independent problem (an ensemble member) by strides.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/softbox_b200.h"
#include "sbx_internal.cuh"

namespace {

constexpr int MT = 128;              // rows of a C tile (the MMA's M)
constexpr int NT = 256;              // max columns of a C tile (the MMA's N)
constexpr int KMAX = 256;            // max contraction length
constexpr int GEMM_THREADS = 512;   // 16 warps: 4 TMEM lane quarters x 4 column groups
constexpr int COL_GROUPS = GEMM_THREADS / 128;
constexpr long long WAIT_NS = 1000000000LL;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ long long gtimer() {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// canonical K-major no-swizzle shared-memory descriptor (sm_100 version bits = 1)
__device__ __forceinline__ unsigned long long kmajor_desc(unsigned addr, unsigned lbo, unsigned sbo) {
    return (unsigned long long)((addr >> 4) & 0x3FFFu) | ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: F32 accumulate, BF16 A and B, both K-major, M x N
__host__ __device__ constexpr unsigned idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(N >> 3) << 17) | ((unsigned)(M >> 4) << 24);
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

struct GemmArgs {
    int M, N, K;
    const __nv_bfloat16* A; int lda; long long sA;
    const __nv_bfloat16* B; int ldb; long long sB;
    const float* bias; long long sBias;
    int act;
    __nv_bfloat16* out; int ldo; long long sOut;
    __nv_bfloat16* outT; int ldt; long long sOutT;
    float* outF; int ldf; long long sOutF;
    int* err;
};

// rows [r0, r0 + rows) x [0, Kp) of a row-major BF16 matrix into the core-matrix layout;
// rows past `rowsValid` and columns past K are zero. Aligned 16-byte pieces go by cp.async
// (every thread keeps all its copies in flight), the rest by plain loads; the caller waits
// with cp_async_wait_all() before the block barrier.
__device__ void stage(char* dst, const __nv_bfloat16* src, int ld, int r0, int rows, int rowsValid, int K, int Kp,
                      bool vec) {
    int kg = Kp >> 3;
    for (int u = threadIdx.x; u < rows * kg; u += GEMM_THREADS) {
        int r = u / kg, c = u - r * kg;
        int gr = r0 + r, k0 = c * 8;
        char* d = dst + ((r >> 3) * kg + c) * 128 + (r & 7) * 16;
        if (gr < rowsValid && vec && k0 + 8 <= K) {
            const __nv_bfloat16* p = src + (long long)gr * ld + k0;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(d)), "l"(p));
            continue;
        }
        uint4 v = make_uint4(0, 0, 0, 0);
        if (gr < rowsValid) {
            const __nv_bfloat16* p = src + (long long)gr * ld + k0;
            unsigned short h[8];
            for (int j = 0; j < 8; j++) h[j] = (k0 + j < K) ? __bfloat16_as_ushort(p[j]) : (unsigned short)0;
            v = make_uint4(h[0] | (unsigned)h[1] << 16, h[2] | (unsigned)h[3] << 16, h[4] | (unsigned)h[5] << 16,
                           h[6] | (unsigned)h[7] << 16);
        }
        *reinterpret_cast<uint4*>(d) = v;
    }
}

__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// One CTA keeps its B tile (up to 256 x 256 BF16) in shared memory and loops over M tiles
// blockIdx.x, blockIdx.x + gridDim.x, ...: per tile it stages A, issues the MMA chain into
// TMEM, waits for the tile's commit (mbarrier phase = tile iteration parity) and runs the
// epilogue, then syncs before the next tile's MMAs overwrite the accumulators.
__global__ void __launch_bounds__(GEMM_THREADS, 1) k_gemm(GemmArgs g) {
    extern __shared__ __align__(1024) char smem[];
    const int z = blockIdx.z;
    const int n0 = blockIdx.y * NT;
    const int nCols = min(NT, g.N - n0);
    const int Np = (nCols + 15) & ~15;             // MMA N: a multiple of 16 for M = 128
    const int Kp = (g.K + 15) & ~15;
    const int tilesM = (g.M + MT - 1) / MT;
    char* sA = smem;
    char* sB = smem + MT * Kp * 2;
    unsigned long long* mbar = reinterpret_cast<unsigned long long*>(sB + NT * Kp * 2);
    unsigned* tmemSlot = reinterpret_cast<unsigned*>(mbar + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned ncolsAlloc = 32;
    while ((int)ncolsAlloc < Np) ncolsAlloc <<= 1;

    if (threadIdx.x == 0)
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmemSlot)),
                     "r"(ncolsAlloc));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    const __nv_bfloat16* A = g.A + z * g.sA;
    const __nv_bfloat16* B = g.B + z * g.sB;
    bool vecA = (g.lda % 8 == 0) && (((uintptr_t)A & 15) == 0);
    bool vecB = (g.ldb % 8 == 0) && (((uintptr_t)B & 15) == 0);
    stage(sB, B, g.ldb, n0, Np, g.N, g.K, Kp, vecB);
    const float* bias = g.bias ? g.bias + z * g.sBias : nullptr;
    __nv_bfloat16* out = g.out ? g.out + z * g.sOut : nullptr;
    __nv_bfloat16* outT = g.outT ? g.outT + z * g.sOutT : nullptr;
    float* outF = g.outF ? g.outF + z * g.sOutF : nullptr;
    // 16-byte row stores where every row start is 16-byte aligned
    const bool vecOut = out && (g.ldo % 8 == 0) && (((uintptr_t)out & 15) == 0);
    const bool vecOutF = outF && (g.ldf % 4 == 0) && (((uintptr_t)outF & 15) == 0);
    const int quarter = warp & 3, cgroup = warp >> 2;
    bool ok = true;
    unsigned tmem = 0;

    int iter = 0;
    if ((int)blockIdx.x < tilesM) stage(sA, A, g.lda, (int)blockIdx.x * MT, MT, g.M, g.K, Kp, vecA);
    for (int tile = blockIdx.x; tile < tilesM && ok; tile += gridDim.x, iter++) {
        const int m0 = tile * MT;
        // this tile's A was staged before the previous tile's epilogue (or above)
        cp_async_wait_all();
        asm volatile("fence.proxy.async.shared::cta;");
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
        tmem = *tmemSlot;
        if (threadIdx.x == 0) {
            const unsigned idesc = idesc_bf16(MT, Np);
            const unsigned aBase = smem_u32(sA), bBase = smem_u32(sB);
            const unsigned sbo = (unsigned)(Kp >> 3) * 128u;
            for (int kk = 0; kk < Kp / 16; kk++) {
                unsigned long long ad = kmajor_desc(aBase + kk * 256u, 128u, sbo);
                unsigned long long bd = kmajor_desc(bBase + kk * 256u, 128u, sbo);
                unsigned acc = kk > 0 ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(mbar)));
        }
        // bounded wait for this tile's MMAs: phase `iter` of the barrier
        {
            const unsigned parity = (unsigned)(iter & 1);
            bool done_ok = false;
            long long t0 = gtimer();
            for (;;) {
                unsigned done;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                    "selp.u32 %0, 1, 0, p;\n\t}"
                    : "=r"(done)
                    : "r"(smem_u32(mbar)), "r"(parity));
                if (done) { done_ok = true; break; }
                if (gtimer() - t0 > WAIT_NS) break;
            }
            ok = __syncthreads_and(done_ok ? 1 : 0) != 0;   // one verdict for the whole CTA
        }
        if (!ok && threadIdx.x == 0 && g.err) atomicOr(g.err, 1);
        asm volatile("tcgen05.fence::after_thread_sync;");
        // the MMAs have read A: stage the next tile's A while this tile's epilogue runs
        if (ok && tile + (int)gridDim.x < tilesM)
            stage(sA, A, g.lda, (tile + (int)gridDim.x) * MT, MT, g.M, g.K, Kp, vecA);
        if (ok) {
            const int row = m0 + quarter * 32 + lane;
            for (int c0 = cgroup * 16; c0 < Np; c0 += COL_GROUPS * 16) {
                unsigned r[16];
                unsigned taddr = tmem + ((unsigned)(quarter * 32) << 16) + (unsigned)c0;
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                      "=r"(r[15])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;");
                const int nb = n0 + c0;                    // this chunk's first column
                float v[16], a[16];
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    v[j] = __uint_as_float(r[j]);
                    if (bias && nb + j < g.N) v[j] += bias[nb + j];
                    a[j] = g.act ? gelu(v[j]) : v[j];
                }
                if (outT) {
#pragma unroll
                    for (int j = 0; j < 16; j++)
                        if (row < g.M && nb + j < g.N) outT[(long long)(nb + j) * g.ldt + row] = __float2bfloat16_rn(a[j]);
                }
                if (row < g.M) {
                    const bool full = nb + 16 <= g.N;
                    if (out) {
                        __nv_bfloat16* o = out + (long long)row * g.ldo + nb;
                        if (vecOut && full) {
                            unsigned w[8];
#pragma unroll
                            for (int j = 0; j < 8; j++) {
                                __nv_bfloat162 h = __floats2bfloat162_rn(a[2 * j], a[2 * j + 1]);
                                w[j] = *reinterpret_cast<unsigned*>(&h);
                            }
                            reinterpret_cast<uint4*>(o)[0] = make_uint4(w[0], w[1], w[2], w[3]);
                            reinterpret_cast<uint4*>(o)[1] = make_uint4(w[4], w[5], w[6], w[7]);
                        } else {
                            for (int j = 0; j < 16; j++)
                                if (nb + j < g.N) o[j] = __float2bfloat16_rn(a[j]);
                        }
                    }
                    if (outF) {
                        float* o = outF + (long long)row * g.ldf + nb;
                        if (vecOutF && full) {
#pragma unroll
                            for (int j = 0; j < 4; j++)
                                reinterpret_cast<float4*>(o)[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2],
                                                                              v[4 * j + 3]);
                        } else {
                            for (int j = 0; j < 16; j++)
                                if (nb + j < g.N) o[j] = v[j];
                        }
                    }
                }
            }
        }
        // every warp is done with sA and the accumulators before the next tile
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
    }
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        tmem = *tmemSlot;
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncolsAlloc));
    }
}

// dZ = dA * GELU'(Z) (or dA when Z is NULL) -> BF16 row-major and transposed; M x N, per z
__global__ void k_gelu_back(int M, int N, const float* dA, const float* Z, long long sMN, __nv_bfloat16* g,
                            __nv_bfloat16* gT, long long sG, long long sGT) {
    int z = blockIdx.y;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)M * N) return;
    int row = (int)(i / N), n = (int)(i - (long long)row * N);
    float d = dA[z * sMN + i];
    if (Z) d *= gelu_grad(Z[z * sMN + i]);
    __nv_bfloat16 h = __float2bfloat16_rn(d);
    g[z * sG + i] = h;
    gT[z * sGT + (long long)n * M + row] = h;
}

// column sums over rows (bias gradients), fixed row order: out[n] = sum_r in[r*N + n]
__global__ void k_colsum_bf16(int M, int N, const __nv_bfloat16* in, long long sIn, float* out, long long sOut) {
    int z = blockIdx.y, n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    for (int r = 0; r < M; r++) s += __bfloat162float(in[z * sIn + (long long)r * N + n]);
    out[z * sOut + n] = s;
}

// MSE gradient on the first `nOut` of Np output columns: g = 2 (y - t) / (M nOut) (0 on padding)
__global__ void k_mse_grad(int M, int Np, int nOut, const float* y, long long sY, const float* t, long long sT,
                           float* g, long long sG, float* loss) {
    int z = blockIdx.y;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)M * Np) return;
    int row = (int)(i / Np), n = (int)(i - (long long)row * Np);
    float v = 0.f;
    if (n < nOut) {
        float d = y[z * sY + i] - t[z * sT + (long long)row * nOut + n];
        v = 2.0f * d / (float)(M * nOut);
        if (loss) atomicAdd(&loss[z], d * d / (float)(M * nOut));
    }
    g[z * sG + i] = v;
}

// Adam on FP32 master weights W[N x K] (per z); writes the BF16 copies W (N x K) and W^T (K x N)
__global__ void k_adam(int N, int K, float* w, const float* gw, float* m, float* v, long long s, float lr, float b1,
                       float b2, float eps, float c1, float c2, __nv_bfloat16* wb, __nv_bfloat16* wbT, long long sb,
                       long long sbT) {
    int z = blockIdx.y;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)N * K) return;
    long long o = z * s + i;
    float gg = gw[o];
    float mm = b1 * m[o] + (1.0f - b1) * gg;
    float vv = b2 * v[o] + (1.0f - b2) * gg * gg;
    m[o] = mm;
    v[o] = vv;
    float ww = w[o] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    w[o] = ww;
    if (wb) {
        __nv_bfloat16 h = __float2bfloat16_rn(ww);
        wb[z * sb + i] = h;
        if (wbT) {
            int n = (int)(i / K), k = (int)(i - (long long)n * K);
            wbT[z * sbT + (long long)k * N + n] = h;
        }
    }
}

}  // namespace

#define SBX_LAUNCH_SMEM(ctx, kernel, grid, block, smem, ...)                \
    do {                                                                  \
        kernel<<<(grid), (block), (smem), (ctx)->stream>>>(__VA_ARGS__);  \
        (ctx)->launches++;                                                \
    } while (0)

extern "C" sbx_status sbx_mlp_gemm_bf16(sbx_ctx* ctx, int32_t nz, int32_t M, int32_t N, int32_t K,
                                        const void* A, int32_t lda, int64_t strideA, const void* B, int32_t ldb,
                                        int64_t strideB, const float* bias, int64_t strideBias, int32_t act,
                                        void* out, int32_t ldo, int64_t strideOut, void* outT, int32_t ldt,
                                        int64_t strideOutT, float* outF, int32_t ldf, int64_t strideOutF,
                                        int32_t* errFlag) {
    SBX_REQUIRE(ctx && nz >= 1 && M >= 0 && N >= 1 && K >= 1 && K <= KMAX && A && B && lda >= K && ldb >= K &&
                (act == 0 || act == 1) && (out || outT || outF) && (!out || ldo >= N) && (!outT || ldt >= M) &&
                (!outF || ldf >= N) && nz <= 65535);
    if (M == 0) return SBX_OK;
    static bool attr = false;
    const int Kp = (K + 15) & ~15;
    size_t smem = (size_t)(MT + NT) * Kp * 2 + 16;
    if (!attr) {
        cudaFuncSetAttribute(k_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (MT + NT) * KMAX * 2 + 16);
        attr = true;
    }
    GemmArgs g{M, N, K, (const __nv_bfloat16*)A, lda, strideA, (const __nv_bfloat16*)B, ldb, strideB, bias,
               strideBias, act, (__nv_bfloat16*)out, ldo, strideOut, (__nv_bfloat16*)outT, ldt, strideOutT, outF, ldf,
               strideOutF, errFlag};
    // one wave of CTAs (1 per SM, shared memory bound), each looping over its M tiles with
    // its B tile resident
    int sms = 148;
    {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    const int tilesM = (M + MT - 1) / MT, tilesN = (N + NT - 1) / NT;
    int gx = sms / (tilesN * nz);                  // a single wave: no SM runs two of them
    gx = gx < 1 ? 1 : (gx > tilesM ? tilesM : gx);
    dim3 grid(gx, tilesN, nz);
    SBX_LAUNCH_SMEM(ctx, k_gemm, grid, GEMM_THREADS, smem, g);
    return check_launch(ctx, "sbx_mlp_gemm_bf16");
}

extern "C" sbx_status sbx_mlp_gelu_backward(sbx_ctx* ctx, int32_t nz, int32_t M, int32_t N, const float* dA,
                                            const float* Z, int64_t strideMN, void* g, void* gT, int64_t strideG,
                                            int64_t strideGT) {
    SBX_REQUIRE(ctx && nz >= 1 && M >= 0 && N >= 1 && dA && g && gT);
    if (M == 0) return SBX_OK;
    long long n = (long long)M * N;
    dim3 grid((unsigned)((n + 255) / 256), nz);
    SBX_LAUNCH_SMEM(ctx, k_gelu_back, grid, 256, 0, M, N, dA, Z, strideMN, (__nv_bfloat16*)g, (__nv_bfloat16*)gT,
               strideG, strideGT);
    return check_launch(ctx, "sbx_mlp_gelu_backward");
}

extern "C" sbx_status sbx_mlp_colsum_bf16(sbx_ctx* ctx, int32_t nz, int32_t M, int32_t N, const void* in,
                                          int64_t strideIn, float* out, int64_t strideOut) {
    SBX_REQUIRE(ctx && nz >= 1 && M >= 0 && N >= 1 && in && out);
    dim3 grid((N + 127) / 128, nz);
    SBX_LAUNCH_SMEM(ctx, k_colsum_bf16, grid, 128, 0, M, N, (const __nv_bfloat16*)in, strideIn, out, strideOut);
    return check_launch(ctx, "sbx_mlp_colsum_bf16");
}

extern "C" sbx_status sbx_mlp_mse_grad(sbx_ctx* ctx, int32_t nz, int32_t M, int32_t Np, int32_t nOut, const float* y,
                                       int64_t strideY, const float* t, int64_t strideT, float* g, int64_t strideG,
                                       float* loss) {
    SBX_REQUIRE(ctx && nz >= 1 && M >= 1 && Np >= nOut && nOut >= 1 && y && t && g);
    long long n = (long long)M * Np;
    dim3 grid((unsigned)((n + 255) / 256), nz);
    SBX_LAUNCH_SMEM(ctx, k_mse_grad, grid, 256, 0, M, Np, nOut, y, strideY, t, strideT, g, strideG, loss);
    return check_launch(ctx, "sbx_mlp_mse_grad");
}

extern "C" sbx_status sbx_mlp_adam(sbx_ctx* ctx, int32_t nz, int32_t N, int32_t K, float* w, const float* gw,
                                   float* m, float* v, int64_t stride, float lr, float beta1, float beta2, float eps,
                                   int32_t stepNumber, void* wBf16, void* wBf16T, int64_t strideB, int64_t strideBT) {
    SBX_REQUIRE(ctx && nz >= 1 && N >= 1 && K >= 1 && w && gw && m && v && stepNumber >= 1);
    float c1 = 1.0f - powf(beta1, (float)stepNumber), c2 = 1.0f - powf(beta2, (float)stepNumber);
    long long n = (long long)N * K;
    dim3 grid((unsigned)((n + 255) / 256), nz);
    SBX_LAUNCH_SMEM(ctx, k_adam, grid, 256, 0, N, K, w, gw, m, v, stride, lr, beta1, beta2, eps, c1, c2,
               (__nv_bfloat16*)wBf16, (__nv_bfloat16*)wBf16T, strideB, strideBT);
    return check_launch(ctx, "sbx_mlp_adam");
}
