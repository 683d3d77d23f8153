// sbx_free.cu — free Brownian rods: the DiffusionHarness.cpuStepFdt step
// (DiffusionHarness.java:161-169: brownianForce -> integrate -> derive) advanced for many
// steps in ONE launch. Free rods do not interact, so each thread keeps its rod's pose in
// registers across steps and touches HBM only to load the rod once and store it once;
// the per-step work is the counter-keyed RNG, Box-Muller and the Langevin update. The
// arrays written at the end (pose, derived geometry, the last step's randForce /
// randTorque) equal running the three systems step by step.
#include <cuda_runtime.h>

#include "../../include/softbox_b200.h"
#include "sbx_internal.cuh"
#include "sbx_physics.cuh"
#include "sbx_trace.h"

using namespace sbx;

namespace {

template <int MODE>   // 0 wang, 1 philox, 2 supplied
__global__ void __launch_bounds__(128) k_free_rods(int n, float* coord, double* coord64, float* uVec, float* yVec,
                                                   float* zVec, float* end1, float* end2, const float* segLength,
                                                   const float* F, const float* T, float* rF, float* rT,
                                                   const float* bTG, const float* bRG, const float* tSc,
                                                   const float* rSc, const float* params, int* counts, int t0,
                                                   int nsteps, uint64_t seed64, const float* noise) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Pose p;
    float f[3], t[3], gT[3], gR[3], rf[3] = {0, 0, 0}, rt[3] = {0, 0, 0};
    double c64[3];
    for (int k = 0; k < 3; k++) {
        p.c[k] = coord[k * n + i]; p.u[k] = uVec[k * n + i]; p.y[k] = yVec[k * n + i];
        f[k] = F[k * n + i]; t[k] = T[k * n + i];
        gT[k] = bTG[k * n + i]; gR[k] = bRG[k * n + i];
        if (coord64) c64[k] = coord64[k * n + i];
    }
    float tS = tSc[i], rS = rSc[i], mag = params[1], dt = params[0], L = segLength[i];
    int seed = counts[2];
    float z[3] = {0, 0, 0}, e1[3] = {0, 0, 0}, e2[3] = {0, 0, 0};
    for (int s = 0; s < nsteps; s++) {
        int step = t0 + s;
        float g[6];
        if (MODE == 0) gauss6_wang(i, step, seed, g);
        else if (MODE == 1) gauss6_philox(i, step, seed64, g);
        else for (int k = 0; k < 6; k++) g[k] = noise[((int64_t)s * 6 + k) * n + i];
        brownian_amplitudes(g, tS, rS, mag, gT, gR, rf, rt);
        Pose q;
        float dc[3];
        integrate_pose(p, f, t, rf, rt, gT, gR, dt, q, dc);
        if (coord64)
            for (int k = 0; k < 3; k++) { c64[k] = c64[k] + (double)dc[k]; q.c[k] = (float)c64[k]; }
        derive_pose(q.c, q.u, q.y, z, e1, e2, L);
        p = q;
    }
    for (int k = 0; k < 3; k++) {
        coord[k * n + i] = p.c[k]; uVec[k * n + i] = p.u[k]; yVec[k * n + i] = p.y[k];
        zVec[k * n + i] = z[k]; end1[k * n + i] = e1[k]; end2[k * n + i] = e2[k];
        rF[k * n + i] = rf[k]; rT[k * n + i] = rt[k];
        if (coord64) coord64[k * n + i] = c64[k];
    }
    if (i == 0) counts[1] = t0 + nsteps - 1;
}

}  // namespace

extern "C" sbx_status sbx_free_rods_run(sbx_ctx* ctx, sbx_filament_store* fil, int32_t t0, int32_t nsteps,
                                        int32_t noise_mode, uint64_t philox_seed, const float* noise) {
    SBX_TRACE("sbx.free.run");
    if (!ctx || !fil || nsteps < 0 || noise_mode < 0 || noise_mode > 2) return SBX_EINVAL;
    const sbx_rigid_body& b = fil->body;
    int n = b.n;
    if (n <= 0 || nsteps == 0) return SBX_OK;
    if (!b.coord || !b.uVec || !b.yVec || !b.zVec || !b.end1 || !b.end2 || !b.segLength || !b.forceSum ||
        !b.torqueSum || !b.randForce || !b.randTorque || !b.bTransGam || !b.bRotGam || !b.brownTransScale ||
        !b.brownRotScale || !fil->params || !fil->counts)
        return fail(ctx, SBX_EINVAL, "sbx_free_rods_run: null array");
    if (noise_mode == 2) {
        if (!noise) return fail(ctx, SBX_EINVAL, "sbx_free_rods_run: supplied noise is null");
        bool bad = false;
        sbx_status st = any_nonfinite(ctx, noise, (int64_t)nsteps * 6 * n, &bad);
        if (st) return st;
        if (bad) return fail(ctx, SBX_ENONFINITE, "sbx_free_rods_run: noise holds NaN/Inf");
    }
#define FREE_ARGS n, b.coord, b.coord64, b.uVec, b.yVec, b.zVec, b.end1, b.end2, b.segLength, b.forceSum, b.torqueSum, \
                  b.randForce, b.randTorque, b.bTransGam, b.bRotGam, b.brownTransScale, b.brownRotScale, fil->params, \
                  fil->counts, t0, nsteps, philox_seed, noise
    if (noise_mode == 0) SBX_LAUNCH(ctx, k_free_rods<0>, blocks(n, 128), 128, FREE_ARGS);
    else if (noise_mode == 1) SBX_LAUNCH(ctx, k_free_rods<1>, blocks(n, 128), 128, FREE_ARGS);
    else SBX_LAUNCH(ctx, k_free_rods<2>, blocks(n, 128), 128, FREE_ARGS);
#undef FREE_ARGS
    return check_launch(ctx, "sbx_free_rods_run");
}
