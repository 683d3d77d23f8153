// sbx_dense.cu — the dense contractile step (DenseContractileHarness.cpuStep,
// DenseContractileHarness.java:350-429) as (a) the per-system call sequence and (b) a
// plan whose step is captured once into a CUDA graph and replayed.
//
// The step index lives in device memory (plan->d_step): the first kernel of a step
// writes every counts array from it and the last kernel advances it, so one captured
// graph replays any number of consecutive steps with the right RNG keys and
// containment cadence.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/softbox_b200.h"
#include "sbx_fused.cuh"
#include "sbx_internal.cuh"
#include "sbx_physics.cuh"
#include "sbx_trace.h"

#include <vector>

using namespace sbx;

namespace {

// MotorStore.setCounts / MiniFilamentStore.setBackboneCounts / counts.set(1, t) /
// CrosslinkerStore.setCounts (DenseContractileHarness.java:353)
__global__ void k_dense_set_counts(const int* d_step, int t_host, int* motCounts, int nM, int nSeg, int seed,
                                   int* bbCounts, int nBb, int seedBb, int* filCounts, int* xlCounts) {
    int t = d_step ? *d_step : t_host;
    motCounts[0] = nM; motCounts[1] = t; motCounts[2] = seed; motCounts[3] = nSeg;
    bbCounts[0] = nBb; bbCounts[1] = t; bbCounts[2] = seedBb; bbCounts[3] = nBb;
    filCounts[1] = t;
    if (xlCounts) { xlCounts[1] = t; xlCounts[2] = seed; }
}

__global__ void k_step_set(int* d_step, int t) { *d_step = t; }

// MechanicsFusion.forceBuild (zero + BrownianForceSystem.brownianForce) in supplied-noise
// mode: the step's six Gaussians of slot i are noise[counts[1] - t0][k][i]. A step outside
// the supplied range (the host rejects such runs before launching) draws zeros and sets *err.
__global__ void k_force_build_supplied(int n, float* F, float* T, float* rF, float* rT, const float* bTG,
                                       const float* bRG, const float* tSc, const float* rSc, const float* params,
                                       const int* counts, const float* noise, int t0, int nsteps, int* err) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < 3; k++) { F[k * n + i] = 0.f; T[k * n + i] = 0.f; }
    int s = counts[1] - t0;
    bool in = s >= 0 && s < nsteps;
    if (!in && i == 0) atomicOr(err, 1);
    const float* q = noise + (int64_t)(in ? s : 0) * 6 * n + i;
    float g[6];
    for (int k = 0; k < 6; k++) g[k] = in ? q[(int64_t)k * n] : 0.f;
    float gT[3] = {bTG[i], bTG[n + i], bTG[2 * n + i]};
    float gR[3] = {bRG[i], bRG[n + i], bRG[2 * n + i]};
    float rf[3], rt[3];
    brownian_amplitudes(g, tSc[i], rSc[i], params[1], gT, gR, rf, rt);
    for (int k = 0; k < 3; k++) { rF[k * n + i] = rf[k]; rT[k * n + i] = rt[k]; }
}

// the noise of one store for the step's force build (null: the Wang-hash draws)
struct StoreNoise {
    const float* noise;
    int t0, nsteps;
    int* err;
};

sbx_status force_build(sbx_ctx* ctx, int n, float* F, float* T, float* rF, float* rT, const float* bTG,
                       const float* bRG, const float* tSc, const float* rSc, const float* params,
                       const int* counts, const StoreNoise& nz) {
    if (!nz.noise)
        return sbx_fusion_force_build(ctx, n, F, T, rF, rT, bTG, bRG, tSc, rSc, params, counts);
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_force_build_supplied, blocks(n), 256, n, F, T, rF, rT, bTG, bRG, tSc, rSc, params, counts,
               nz.noise, nz.t0, nz.nsteps, nz.err);
    return check_launch(ctx, "dense step: supplied-noise force build");
}
__global__ void k_step_advance(int* d_step) { *d_step += 1; }

#define CHK(x)                      \
    do {                            \
        sbx_status _s = (x);        \
        if (_s != SBX_OK) return _s; \
    } while (0)

// the reference step order over the per-system entry points
// Context scratch of one dense step: the counting sorts' temporaries first, then the
// row-ordered payload copies of the three filament-side CSRs (crosslinker A and B sides,
// motors; 6 floats per item), then the reach walk's cell-ordered endpoints.
size_t dense_sort_bytes(const sbx_dense_scene* sc) {
    auto rows = [](int n) { return (size_t)(n + SCAN_CHUNK - 1) / SCAN_CHUNK + 1; };
    auto csr = [&](int nRows, int nItems) {           // sbx_csr_build's layout: ints, then tile sums
        return ((sizeof(int) * (rows(nRows) + (size_t)std::max(nItems, 1)) + 7) & ~(size_t)7) +
               sizeof(int) * scan_tile_words(nRows);
    };
    int nSeg = sc->fil.body.n;
    size_t need = ((sizeof(int) * (size_t)std::max(sc->grid.cap, 1) + 7) & ~(size_t)7) +
                  sizeof(int) * scan_tile_words(sc->grid.totalCells);
    need = std::max(need, csr(sc->mini.backbone.n, sc->mini.nDimers));
    need = std::max(need, csr(nSeg, sc->mot.nMotors));
    need = std::max(need, csr(nSeg, sc->xl.nLinks));
    return need;
}

size_t dense_row_payload_offset(const sbx_dense_scene* sc) { return (dense_sort_bytes(sc) + 255) & ~(size_t)255; }

size_t dense_row_payload_bytes(const sbx_dense_scene* sc) {
    return sizeof(float) * 6 * (2 * (size_t)std::max(sc->xl.nLinks, 0) + (size_t)std::max(sc->mot.nMotors, 0));
}

// then the cell-ordered endpoints of the reach walk (two float4 per grid entry)
size_t dense_cell_endpoints_offset(const sbx_dense_scene* sc) {
    return (dense_row_payload_offset(sc) + dense_row_payload_bytes(sc) + 255) & ~(size_t)255;
}

float* dense_row_payload(sbx_ctx* ctx, const sbx_dense_scene* sc) {
    return reinterpret_cast<float*>(static_cast<char*>(ctx->scratch) + dense_row_payload_offset(sc));
}

float* dense_cell_endpoints(sbx_ctx* ctx, const sbx_dense_scene* sc) {
    return reinterpret_cast<float*>(static_cast<char*>(ctx->scratch) + dense_cell_endpoints_offset(sc));
}

// A second stream for the filament-side work of a step (owned by a plan): the fork and join
// events and that stream's own sort scratch, so that its CSR builds and the minifilament
// CSR build on the main stream never share temporaries.
struct SideStream {
    cudaStream_t stream;
    cudaEvent_t fork, join;      // filament-side head of the step
    cudaEvent_t fork2, join2;    // motor-side tail of the step
    void* scratch;
    size_t scratchBytes;
};

// Moves the context's launches (and its sort scratch) to the side stream for a scope, after
// the side stream waits for the work already on the main stream; at scope end the side
// stream records the join event and the context is restored.
struct SideScope {
    sbx_ctx* ctx;
    const SideStream* side;
    cudaEvent_t join = nullptr;
    cudaStream_t savedStream = nullptr;
    void* savedScratch = nullptr;
    size_t savedBytes = 0;
    sbx_status status = SBX_OK;
    SideScope(sbx_ctx* c, const SideStream* s, bool tail = false) : ctx(c), side(s) {
        if (!side) return;
        cudaEvent_t fork = tail ? side->fork2 : side->fork;
        join = tail ? side->join2 : side->join;
        if (cudaEventRecord(fork, ctx->stream) != cudaSuccess ||
            cudaStreamWaitEvent(side->stream, fork, 0) != cudaSuccess) {
            status = fail(ctx, SBX_ECUDA, "dense step: side-stream fork");
            side = nullptr;
            return;
        }
        savedStream = ctx->stream;
        savedScratch = ctx->scratch;
        savedBytes = ctx->scratch_bytes;
        ctx->stream = side->stream;
        ctx->scratch = side->scratch;
        ctx->scratch_bytes = side->scratchBytes;
    }
    ~SideScope() {
        if (!side) return;
        cudaEventRecord(join, side->stream);
        ctx->stream = savedStream;
        ctx->scratch = savedScratch;
        ctx->scratch_bytes = savedBytes;
    }
};

sbx_status side_join(sbx_ctx* ctx, const SideStream* side, bool tail = false) {
    if (cudaStreamWaitEvent(ctx->stream, tail ? side->join2 : side->join, 0) != cudaSuccess)
        return fail(ctx, SBX_ECUDA, "dense step: side-stream join");
    return SBX_OK;
}

// the supplied noise of a plan (sbx_dense_plan_set_noise) as the step sees it
struct StepNoise {
    sbx_dense_noise nz;
    int* err;
    StoreNoise store(const float* p) const { return StoreNoise{p, nz.t0, nz.nsteps, err}; }
};

sbx_status dense_sequence(sbx_ctx* ctx, const sbx_dense_scene* sc, const int* d_step, int t,
                          const sbx_batch* bt = nullptr, const SideStream* side = nullptr,
                          const StepNoise* noise = nullptr) {
    const sbx_filament_store& f = sc->fil;
    const sbx_motor_store& mot = sc->mot;
    const sbx_dimer_store& dim = sc->dim;
    const sbx_minifilament_store& mini = sc->mini;
    const sbx_crosslinker_store& xl = sc->xl;
    const sbx_grid_state& g = sc->grid;
    const sbx_rigid_body& b = mot.body;
    const sbx_rigid_body& bb = mini.backbone;
    const sbx_rigid_body& fb = f.body;
    const int nSeg = fb.n, nM = mot.nMotors, nB = b.n, nBb = bb.n, nD = dim.nDimers;
    const bool xlOn = sc->xlinkOn && xl.nLinks > 0;
    SBX_TRACE("sbx.dense.step");
    TracePhases tr;

    SBX_LAUNCH(ctx, k_dense_set_counts, 1, 1, d_step, t, mot.counts, nM, nSeg, sc->seed, mini.bbCounts, nBb,
               sc->seedBb, f.counts, xlOn ? xl.counts : nullptr);
    // (i) binding
    tr.next("sbx.dense.binding");
    CHK(sbx_motor_publish_head(ctx, nM, b.coord, b.uVec, b.segLength, mot.head, mot.uVec, mot.rodUVec));
    CHK(sbx_filament_publish(ctx, nSeg, fb.coord, fb.segLength, g.cap, g.center, g.boundingRadius, g.ownerStore,
                             g.ownerSlot, g.viewParams, f.filState));
    CHK(sbx_motor_publish(ctx, nM, mot.head, mot.reach, g.cap, g.center, g.boundingRadius, g.ownerStore, g.ownerSlot,
                          mot.publishParams));
    if (bt)
        CHK(sbx_grid_body_cell_batched(ctx, g.cap, g.center, g.gridCounts, g.bodyCell, nSeg, bt->segKey, bt->motKey,
                                       bt->gridParams, bt->gridDims));
    else
        CHK(sbx_grid_body_cell(ctx, g.cap, g.center, g.gridParams, g.gridDims, g.gridCounts, g.bodyCell));
    CHK(sbx_grid_build(ctx, g.cap, g.bodyCell, g.gridCounts, g.totalCells, g.cellCount, g.chunkSum,
                       g.gridCellOffsets, g.gridCellContents, g.cap));
    // the reach walk reads the segment endpoints in cell order (one float4 pair per grid entry)
    float* cellE1 = dense_cell_endpoints(ctx, sc);
    float* cellE2 = cellE1 + 4 * (size_t)std::max(g.cap, 0);
    CHK(sbx_grid_cell_endpoints(ctx, g.cap, g.totalCells, g.gridCellOffsets, g.gridCellContents, g.ownerStore,
                                g.ownerSlot, nSeg, fb.end1, fb.end2, cellE1, cellE2));
    if (bt) {
        CHK(sbx_fusion_grid_reachable_batched(ctx, mot.head, mot.uVec, mot.rodUVec, g.gridCellOffsets, cellE1,
                                              cellE2, g.reachSeg, g.reachCount, mot.kinParams, nM, bt->motKey,
                                              bt->gridParams, bt->gridDims));
        CHK(sbx_nucleotide_release_batched(ctx, nM, mot.boundSeg, mot.forceDotFil, mot.forceMag, mot.cooldown,
                                           mot.stats, mot.capStats, mot.kinParams, mot.counts, bt->motKey,
                                           bt->seeds));
    } else {
        // (the per-head walk: the staged-tile variant, sbx_fusion_grid_reachable_staged, measured
        // 3.2x slower at 2e6 rods on this sparse grid and is not used here)
        CHK(sbx_fusion_grid_reachable(ctx, mot.head, mot.uVec, mot.rodUVec, g.gridParams, g.gridDims,
                                      g.gridCellOffsets, cellE1, cellE2, g.reachSeg, g.reachCount, mot.kinParams,
                                      nM));
        CHK(sbx_nucleotide_release(ctx, nM, mot.boundSeg, mot.forceDotFil, mot.forceMag, mot.cooldown, mot.stats,
                                   mot.capStats, mot.kinParams, mot.counts));
    }
    CHK(sbx_binding_bind_nearest(ctx, mot.head, mot.uVec, mot.rodUVec, nSeg, fb.end1, fb.end2, g.reachSeg,
                                 g.reachCount, mot.boundSeg, mot.bindArc, mot.kinParams, nM));
    if (bt)
        CHK(sbx_nucleotide_cycle_batched(ctx, nM, mot.nucleotideState, mot.boundSeg, mot.forceDotHist, mot.nucParams,
                                         mot.counts, bt->motKey, bt->seeds));
    else
        CHK(sbx_nucleotide_cycle(ctx, nM, mot.nucleotideState, mot.boundSeg, mot.forceDotHist, mot.nucParams,
                                 mot.counts));
    // (iii)-(v) filaments, the part that needs nothing from the minifilament structure below:
    tr.next("sbx.dense.filament_forces");
    // draws, crosslinker kernels and the crosslinker CSR builds. With a side stream it runs
    // concurrently with (ii); the streams join before the motor CSR, which reads the
    // cross-bridge payload. The row-ordered payload copies live in the main scratch.
    float* payA = dense_row_payload(ctx, sc);
    float* payB = payA + 6 * (size_t)std::max(xl.nLinks, 0);
    float* payM = payB + 6 * (size_t)std::max(xl.nLinks, 0);
    {
        SideScope onSide(ctx, side);
        if (side) CHK(onSide.status);
        if (bt) {
            CHK(sbx_zero_accumulators(ctx, nSeg, fb.forceSum, fb.torqueSum));
            CHK(sbx_brownian_force_batched(ctx, nSeg, 1, fb.randForce, fb.randTorque, fb.bTransGam, fb.bRotGam,
                                           fb.brownTransScale, fb.brownRotScale, f.params, f.counts, bt->segKey,
                                           bt->seeds, 2));
        } else {
            CHK(force_build(ctx, nSeg, fb.forceSum, fb.torqueSum, fb.randForce, fb.randTorque, fb.bTransGam,
                            fb.bRotGam, fb.brownTransScale, fb.brownRotScale, f.params, f.counts,
                            noise ? noise->store(noise->nz.fil) : StoreNoise{}));
        }
        // The crosslinker kernels and the CSR builds read no filament accumulator, so they run
        // before the chain forces; chain and the three gathers then share one pass
        // (sbx_fusion_chain_gathers), each gather reading its row-ordered payload copy made by
        // the CSR build. The accumulators get the bits of chain, segGatherA, segGatherB, segGather.
        if (xlOn) {
            if (sc->xlUnbind && bt)
                CHK(sbx_xlink_unbind_batched(ctx, nSeg, fb.uVec, fb.end1, xl.nLinks, xl.linkFilA, xl.linkFilB,
                                             xl.loc1, xl.loc2, xl.linkState, xl.strainHist, xl.strainPlace,
                                             xl.offParams, xl.counts, bt->linkKey, bt->seeds));
            else if (sc->xlUnbind)
                CHK(sbx_xlink_unbind(ctx, nSeg, fb.uVec, fb.end1, xl.nLinks, xl.linkFilA, xl.linkFilB, xl.loc1,
                                     xl.loc2, xl.linkState, xl.strainHist, xl.strainPlace, xl.offParams,
                                     xl.counts));
            CHK(sbx_xlink_count_active(ctx, xl.nLinks, xl.linkState, xl.linkFilA, xl.linkFilB, nSeg,
                                       xl.activeLinkCount));
            CHK(sbx_xlink_forces(ctx, nSeg, fb.coord, fb.uVec, fb.end1, fb.bTransGam, xl.nLinks, xl.linkFilA,
                                 xl.linkFilB, xl.loc1, xl.loc2, xl.activeLinkCount, xl.xlinkData, xl.xlParams));
            CHK(sbx_xlink_torsion(ctx, nSeg, fb.uVec, xl.nLinks, xl.linkFilA, xl.linkFilB, xl.linkState,
                                  xl.linkOrientSame, xl.torqueMagHist, xl.torqueMagPlace, xl.xlinkData,
                                  xl.torsionParams));
            CHK(sbx_csr_build_payload(ctx, xl.linkFilA, xl.nLinks, nSeg, xl.segCountA, xl.segOffsetsA,
                                      xl.segIdxA, xl.xlinkData, XL_STRIDE, 0, xl.linkState, payA));
            CHK(sbx_csr_build_payload(ctx, xl.linkFilB, xl.nLinks, nSeg, xl.segCountB, xl.segOffsetsB,
                                      xl.segIdxB, xl.xlinkData, XL_STRIDE, 6, xl.linkState, payB));
        }
    }
    // (ii) minifilament structure. A single network zeroes and draws in one pass per store
    tr.next("sbx.dense.myosin");
    // (MechanicsFusion.forceBuild, the same values as the zero + Brownian pair)
    if (!bt) {
        CHK(force_build(ctx, nB, b.forceSum, b.torqueSum, b.randForce, b.randTorque, b.bTransGam, b.bRotGam,
                        b.brownTransScale, b.brownRotScale, mot.bodyParams, mot.counts,
                        noise ? noise->store(noise->nz.mot) : StoreNoise{}));
        CHK(force_build(ctx, nBb, bb.forceSum, bb.torqueSum, bb.randForce, bb.randTorque, bb.bTransGam,
                        bb.bRotGam, bb.brownTransScale, bb.brownRotScale, mini.bbBodyParams, mini.bbCounts,
                        noise ? noise->store(noise->nz.bb) : StoreNoise{}));
    } else {
        CHK(sbx_zero_accumulators(ctx, nB, b.forceSum, b.torqueSum));
        CHK(sbx_zero_accumulators(ctx, nBb, bb.forceSum, bb.torqueSum));
    }
    if (bt) {
        CHK(sbx_brownian_force_batched(ctx, nB, 3, b.randForce, b.randTorque, b.bTransGam, b.bRotGam,
                                       b.brownTransScale, b.brownRotScale, mot.bodyParams, mot.counts, bt->motKey,
                                       bt->seeds, 0));
        CHK(sbx_brownian_force_batched(ctx, nBb, 1, bb.randForce, bb.randTorque, bb.bTransGam, bb.bRotGam,
                                       bb.brownTransScale, bb.brownRotScale, mini.bbBodyParams, mini.bbCounts,
                                       bt->bbKey, bt->seeds, 1));
    }
    CHK(sbx_motor_joints(ctx, nB, b.coord, b.uVec, b.segLength, b.bTransGam, b.bRotGam, b.forceSum, b.torqueSum,
                         mot.nucleotideState, mot.jointParams));
    CHK(sbx_dimer_couple(ctx, nB, b.coord, b.uVec, b.segLength, b.bTransGam, b.bRotGam, b.forceSum, b.torqueSum, nD,
                         dim.motorA, dim.motorB, dim.parallel, dim.dimerParams, mot.boundSeg));
    CHK(sbx_mini_tether(ctx, nB, b.coord, b.uVec, b.segLength, b.bTransGam, b.bRotGam, b.forceSum, b.torqueSum, nBb,
                        bb.coord, bb.uVec, mini.bbInvDragY, mini.nDimers, mini.headBackboneSlot, mini.motorA,
                        mini.attachAxial, mini.miniData, mini.miniParams));
    CHK(sbx_csr_build(ctx, mini.headBackboneSlot, mini.nDimers, nBb, mini.bbDimerCount, mini.bbDimerOffsets,
                      mini.bbDimerList));
    CHK(sbx_mini_backbone_gather(ctx, nBb, mini.bbDimerOffsets, mini.bbDimerList, mini.miniData, bb.forceSum,
                                 bb.torqueSum));
    CHK(sbx_xbridge_bond_forces(ctx, nB, b.coord, b.uVec, b.yVec, b.bRotGam, nSeg, fb.coord, fb.uVec, fb.yVec,
                                fb.bRotGam, fb.segLength, mot.boundSeg, mot.bindArc, mot.nucleotideState, sc->bondData,
                                sc->xbParams));
    tr.next("sbx.dense.integrate");
    // the motor-side tail (head forces, motor and backbone integration, force-dot registry)
    // reads no filament state and the filament tail below reads none of it: with a side stream
    // they run concurrently, joined at the end of the step
    if (side) CHK(side_join(ctx, side));
    {
        SideScope onSide(ctx, side, true);
        if (side) CHK(onSide.status);
        CHK(sbx_xbridge_apply_head_force(ctx, nB, sc->bondData, b.forceSum, b.torqueSum));
        if (bt) {
            CHK(sbx_integrate(ctx, nB, b.coord, b.coord64, b.uVec, b.yVec, b.forceSum, b.torqueSum, b.randForce,
                              b.randTorque, b.bTransGam, b.bRotGam, mot.bodyParams));
            CHK(sbx_confine_batched(ctx, nBb, bb.coord, bb.uVec, bb.segLength, bb.bTransGam, bb.forceSum,
                                    bb.torqueSum, bt->boxParams, mini.bbCounts, bt->bbKey));
            CHK(sbx_integrate(ctx, nBb, bb.coord, bb.coord64, bb.uVec, bb.yVec, bb.forceSum, bb.torqueSum,
                              bb.randForce, bb.randTorque, bb.bTransGam, bb.bRotGam, mini.bbBodyParams));
            CHK(sbx_derive(ctx, nB, b.coord, b.uVec, b.yVec, b.zVec, b.end1, b.end2, b.segLength));
            CHK(sbx_derive(ctx, nBb, bb.coord, bb.uVec, bb.yVec, bb.zVec, bb.end1, bb.end2, bb.segLength));
        } else {
            // MechanicsFusion.integDerive / integDeriveConfined: confine, integrate and derive in
            // one pass per store, in that order (the same values as the separate kernels)
            CHK(sbx_fusion_integ_derive(ctx, nB, b.coord, b.coord64, b.uVec, b.yVec, b.zVec, b.segLength, b.end1,
                                        b.end2, b.forceSum, b.torqueSum, b.randForce, b.randTorque, b.bTransGam,
                                        b.bRotGam, mot.bodyParams));
            CHK(sbx_fusion_integ_derive_confined(ctx, nBb, bb.coord, bb.coord64, bb.uVec, bb.yVec, bb.zVec,
                                                 bb.segLength, bb.end1, bb.end2, bb.forceSum, bb.torqueSum,
                                                 bb.randForce, bb.randTorque, bb.bTransGam, bb.bRotGam,
                                                 sc->boxParams, mini.bbCounts));
        }
        CHK(sbx_xbridge_register_force_dot(ctx, nM, sc->bondData, mot.boundSeg, mot.forceDotFil, mot.forceMag,
                                           mot.forceDotHist, mot.forceDotPlace));
    }
    CHK(sbx_csr_build_payload(ctx, mot.boundSeg, nM, nSeg, sc->segMotorCount, sc->segMotorOffsets, sc->segMotorMyo,
                              sc->bondData, XB_STRIDE, 6, nullptr, payM));
    CHK(sbx_fusion_chain_gathers(ctx, nSeg, fb.coord, fb.uVec, fb.segLength, f.end2NbrSlot, f.end2NbrSide,
                                 f.end1NbrSlot, f.end1NbrSide, fb.bTransGam, fb.bRotGam, fb.forceSum, fb.torqueSum,
                                 f.chainParams, xlOn ? xl.segOffsetsA : nullptr, payA,
                                 xlOn ? xl.segOffsetsB : nullptr, payB, sc->segMotorOffsets, payM));
    if (bt) {
        CHK(sbx_confine_batched(ctx, nSeg, fb.coord, fb.uVec, fb.segLength, fb.bTransGam, fb.forceSum, fb.torqueSum,
                                bt->boxParams, f.counts, bt->segKey));
        CHK(sbx_integrate(ctx, nSeg, fb.coord, fb.coord64, fb.uVec, fb.yVec, fb.forceSum, fb.torqueSum, fb.randForce,
                          fb.randTorque, fb.bTransGam, fb.bRotGam, f.params));
        CHK(sbx_derive(ctx, nSeg, fb.coord, fb.uVec, fb.yVec, fb.zVec, fb.end1, fb.end2, fb.segLength));
    } else {
        CHK(sbx_fusion_integ_derive_confined(ctx, nSeg, fb.coord, fb.coord64, fb.uVec, fb.yVec, fb.zVec, fb.segLength,
                                             fb.end1, fb.end2, fb.forceSum, fb.torqueSum, fb.randForce,
                                             fb.randTorque, fb.bTransGam, fb.bRotGam, sc->boxParams, f.counts));
    }
    if (side) CHK(side_join(ctx, side, true));
    return SBX_OK;
}

size_t dense_scratch_bytes(const sbx_dense_scene* sc) {
    return dense_cell_endpoints_offset(sc) + 2 * sizeof(float4) * (size_t)std::max(sc->grid.cap, 0);
}

}  // namespace

struct sbx_dense_plan {
    sbx_ctx* ctx = nullptr;
    sbx_dense_scene scene;
    int* d_step = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int kernels_per_step = 0;
    // fused persistent path
    bool fused_ok = false;
    bool fused_prepared = false;  // its scratch exists (the topology may still be refused)
    bool fused_dirty = true;     // scratch must be (re)initialised before the next fused run
    std::string fused_why;
    FusedArgs fa{};
    int fused_grid = 0;
    std::vector<void*> allocs;
    // packed networks (graph and per-system paths only)
    bool batched = false;
    sbx_batch batch{};
    // the step's scratch (sort temporaries, row-ordered payloads), owned by the plan: the
    // captured graph holds its address, so it must not move when another plan on the same
    // context needs a larger context scratch
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    // the side stream of the step's filament-side work, with its own sort scratch
    SideStream side{};
    bool sideOk = false;
    // supplied-noise mode (sbx_dense_plan_set_noise)
    bool noiseOn = false;
    sbx_dense_noise noise{};
    int* noiseErr = nullptr;        // device word: a step outside the supplied range ran
    // capacity-fallback counters of the fused path (SBX_FUSED_STATS, device)
    unsigned long long* stats = nullptr;
};

namespace {

// Points the context's scratch at the plan's for the duration of a scope (the graph capture
// and the per-system path); the plan's buffer covers every request of the step, so nothing
// inside reallocates it.
struct PlanScratch {
    sbx_ctx* ctx;
    void* saved;
    size_t savedBytes;
    PlanScratch(sbx_dense_plan* p) : ctx(p->ctx), saved(p->ctx->scratch), savedBytes(p->ctx->scratch_bytes) {
        ctx->scratch = p->scratch;
        ctx->scratch_bytes = p->scratch_bytes;
    }
    ~PlanScratch() {
        ctx->scratch = saved;
        ctx->scratch_bytes = savedBytes;
    }
};

void release_side(sbx_dense_plan* p) {
    if (p->side.scratch) cudaFree(p->side.scratch);
    if (p->side.join) cudaEventDestroy(p->side.join);
    if (p->side.join2) cudaEventDestroy(p->side.join2);
    if (p->side.fork2) cudaEventDestroy(p->side.fork2);
    if (p->side.fork) cudaEventDestroy(p->side.fork);
    if (p->side.stream) cudaStreamDestroy(p->side.stream);
    p->side = SideStream{};
}

}  // namespace

namespace {

template <class T>
std::vector<T> d2h(const T* d, size_t n, cudaStream_t s) {
    std::vector<T> h(n);
    if (n) cudaMemcpyAsync(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return h;
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// Checks that the scene has the harness's structure the fused kernel relies on and fills
// the kernel arguments; on failure records why (the graph path remains available).
// The fused kernel's view of the chain topology, read from the device (the plan's stream
// is synchronised): rod groups (FUSED_MAX_ROD slots at most, a multiple of 4), whether every
// chain neighbour lies in its own group (else the rod phase reads cross-group neighbours from
// the step's start view), whether each joint can be computed once. FREE filament slots of
// turnover are allowed: the body view leaves them out of the grid's segments. Called at plan
// creation and by sbx_dense_plan_refresh after a topology change.
bool fused_topology(sbx_dense_plan* p) {
    const sbx_dense_scene& sc = p->scene;
    cudaStream_t st = p->ctx->stream;
    FusedArgs& a = p->fa;
    auto why = [&](const char* w) { p->fused_why = w; return false; };
    auto e1 = d2h(sc.fil.end1NbrSlot, a.nSeg, st), e2 = d2h(sc.fil.end2NbrSlot, a.nSeg, st);
    auto d1 = d2h(sc.fil.end1NbrSide, a.nSeg, st), d2 = d2h(sc.fil.end2NbrSide, a.nSeg, st);
    std::vector<int> lo(a.nSeg), hi(a.nSeg);
    for (int i = 0; i < a.nSeg; i++) {
        lo[i] = i; hi[i] = i;
        int nb[2] = {e1[i], e2[i]};
        for (int j : nb) {
            if (j < -1 || j >= a.nSeg) return why("neighbour slot out of range");
            if (j >= 0) { lo[i] = std::min(lo[i], j); hi[i] = std::max(hi[i], j); }
        }
    }
    // filaments as contiguous slot ranges: a rod group is a run of whole filaments, the
    // smallest group size whose groups fit one wave of CTAs, else the largest valid one
    const int wave = p->fused_grid - FUSED_MIN_HELPERS;
    a.G = 0;
    int largest = 0;
    for (int G = 4; G <= FUSED_MAX_ROD; G += 4) {
        bool ok = true;
        for (int i = 0; i < a.nSeg && ok; i++) ok = (lo[i] / G == i / G) && (hi[i] / G == i / G);
        if (!ok) continue;
        largest = G;
        if (!a.G && (a.nSeg + G - 1) / G <= wave) a.G = G;
    }
    if (!a.G) a.G = largest;
    a.nbrGlobal = 0;
    if (!a.G) {
        // neighbours across every grouping (births into free slots): groups of consecutive
        // slots sized to one wave, cross-group neighbours read from the step's start view
        a.nbrGlobal = 1;
        int G = 4;
        while (G < FUSED_MAX_ROD && (a.nSeg + G - 1) / G > wave) G += 4;
        a.G = G;
    }
    // joint sharing needs every neighbour link to point back: rod i's side s (0 = end2) to
    // slot j at nside means j's side 1 - nside points to i at nside 1 - s
    a.jointShare = 1;
    for (int i = 0; i < a.nSeg && a.jointShare; i++)
        for (int side = 0; side < 2; side++) {
            int j = side == 0 ? e2[i] : e1[i], ns = side == 0 ? d2[i] : d1[i];
            if (j < 0) continue;
            if (j == i || (ns != 0 && ns != 1)) { a.jointShare = 0; break; }
            int back = ns == 0 ? e1[j] : e2[j], backSide = ns == 0 ? d1[j] : d2[j];
            if (back != i || backSide != 1 - side) { a.jointShare = 0; break; }
        }
    a.nRodUnits = (a.nSeg + a.G - 1) / a.G;
    // helper CTAs of the rod phase: those without a rod unit, at least FUSED_MIN_HELPERS
    a.kHelp0 = std::max(0, std::min(a.nRodUnits, p->fused_grid - FUSED_MIN_HELPERS));
    const sbx_rigid_body& fb = sc.fil.body;
    a.useTma = (a.nSeg % 4 == 0) && (a.G % 4 == 0) && aligned16(fb.coord) && aligned16(fb.uVec) &&
               aligned16(fb.segLength) && aligned16(fb.bTransGam) && aligned16(fb.bRotGam);
    return true;
}

bool fused_prepare(sbx_dense_plan* p) {
    const sbx_dense_scene& sc = p->scene;
    cudaStream_t st = p->ctx->stream;
    FusedArgs& a = p->fa;
    a.sc = sc;
    a.nSeg = sc.fil.body.n; a.nM = sc.mot.nMotors; a.nB = sc.mot.body.n; a.nBb = sc.mini.backbone.n;
    a.nD = sc.dim.nDimers; a.nL = sc.xl.nLinks; a.cap = sc.grid.cap; a.C = sc.grid.totalCells;
    a.xlOn = (sc.xlinkOn && sc.xl.nLinks > 0) ? 1 : 0;
    a.xlUnbind = sc.xlUnbind ? 1 : 0;
    auto why = [&](const char* w) { p->fused_why = w; return false; };
    if (a.nSeg <= 0 || a.nM <= 0 || a.nBb <= 0) return why("empty stores");
    if (a.nB != 3 * a.nM || a.nM != 2 * a.nD || sc.mini.nDimers != a.nD) return why("motor/dimer counts");
    if (a.nD % a.nBb) return why("dimers per backbone not uniform");
    a.dpm = a.nD / a.nBb;
    if (6 * a.dpm > FUSED_MAX_SUB || 2 * a.dpm > 32) return why("too many dimers per backbone");
    auto mA = d2h(sc.dim.motorA, a.nD, st), mB = d2h(sc.dim.motorB, a.nD, st);
    auto hbs = d2h(sc.mini.headBackboneSlot, a.nD, st), mmA = d2h(sc.mini.motorA, a.nD, st);
    for (int d = 0; d < a.nD; d++)
        if (mA[d] != 2 * d || mB[d] != 2 * d + 1 || hbs[d] != d / a.dpm || mmA[d] != 2 * d)
            return why("dimer/minifilament topology is not the harness layout");
    auto pub = d2h(sc.mot.publishParams, 1, st);
    if (pub[0] != a.nSeg || a.cap < a.nSeg + a.nM) return why("body-view layout");
    auto gc = d2h(sc.grid.gridCounts, 4, st);
    a.S = gc[1];
    if (a.S < 0 || a.S > a.cap) return why("grid counts");
    auto gd = d2h(sc.grid.gridDims, 4, st);
    a.nX = gd[0]; a.nY = gd[1]; a.nZ = gd[2];
    if (gd[3] != a.C || (long long)a.nX * a.nY * a.nZ != a.C) return why("grid dims");
    int dev = 0, sms = 0, coop = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    int per = fused_max_blocks_per_sm();
    if (!coop || per <= 0) return why("cooperative launch unavailable");
    p->fused_grid = sms * per;
    if (!fused_topology(p)) return false;
    a.tilesC = (a.C + SCAN_CHUNK - 1) / SCAN_CHUNK;
    a.tilesS = (a.nSeg + SCAN_CHUNK - 1) / SCAN_CHUNK;
    auto fc = d2h(sc.fil.counts, 4, st);
    a.filSeed = fc[2];
    // plan-owned scratch
    auto alloc = [&](size_t bytes) -> void* {
        void* q = nullptr;
        if (cudaMalloc(&q, bytes ? bytes : 4) != cudaSuccess) return nullptr;
        p->allocs.push_back(q);
        return q;
    };
    size_t nS = a.nSeg;
    a.cntCell = (int*)alloc(4 * (size_t)a.C);
    a.cntSeg = (int*)alloc(4 * (size_t)a.C);
    a.segCellOff = (int*)alloc(4 * ((size_t)a.C + 1));
    a.cntAct = (int*)alloc(4 * nS); a.cntA = (int*)alloc(4 * nS); a.cntB = (int*)alloc(4 * nS);
    a.cntM = (int*)alloc(4 * nS);
    a.tileSum = (int*)alloc(4 * (size_t)(2 * a.tilesC + 2 * a.tilesS + 1));
    a.mTileSum = (int*)alloc(4 * (size_t)(a.tilesS + 1));
    a.cellSlot = (int*)alloc(4 * (size_t)a.C * FUSED_CELL_SLOTS);
    a.slotA = (int*)alloc(4 * nS * FUSED_ROW_SLOTS); a.slotB = (int*)alloc(4 * nS * FUSED_ROW_SLOTS);
    a.slotM = (int*)alloc(4 * nS * FUSED_MOTOR_SLOTS);
    a.cellHead = (int*)alloc(4 * (size_t)a.C); a.cellNext = (int*)alloc(4 * (size_t)a.cap);
    size_t nLk = (size_t)std::max(a.nL, 1);
    a.headA = (int*)alloc(4 * nS); a.nextA = (int*)alloc(4 * nLk);
    a.headB = (int*)alloc(4 * nS); a.nextB = (int*)alloc(4 * nLk);
    a.headM = (int*)alloc(4 * nS); a.nextM = (int*)alloc(4 * (size_t)a.nM);
    a.segE1 = (float4*)alloc(16 * nS); a.segE2 = (float4*)alloc(16 * nS);
    a.joints = alloc(2 * nS * FUSED_JOINT_BYTES);
    a.terms = alloc((2 * (size_t)a.nM + 4 * (size_t)a.nD) * FUSED_TERM_BYTES);
    a.uSnap = (float*)alloc(12 * nS);
    a.bar = (unsigned long long*)alloc(32);
    a.err = (int*)alloc(16);
    a.d_step = p->d_step;
    a.stats = p->stats;
    a.entCap = FUSED_ENT_CAP;
    a.mCap = FUSED_MCAP;
    a.mIds = FUSED_MIDS;
    a.cellUse = FUSED_CELL_SLOTS;
    a.rowUse = FUSED_ROW_SLOTS;
    a.mRowUse = FUSED_MOTOR_SLOTS;
    for (void* q : p->allocs)
        if (!q) return why("scratch allocation failed");
    // the error word and barrier counters are read by the plan status before any fused run
    cudaMemsetAsync(a.err, 0, 16, st);
    cudaMemsetAsync(a.bar, 0, 32, st);
    p->fused_prepared = true;
    return true;
}

}  // namespace

extern "C" sbx_status sbx_dense_step_unfused(sbx_ctx* ctx, const sbx_dense_scene* sc, int32_t t) {
    if (!ctx || !sc) return SBX_EINVAL;
    CHK(ensure_scratch(ctx, dense_scratch_bytes(sc)));
    return dense_sequence(ctx, sc, nullptr, t);
}

// Captures one step (the sequence, then the step-counter advance) into the plan's graph,
// replacing a previous capture; the supplied noise, when on, is part of the capture.
static sbx_status capture_step(sbx_dense_plan* p) {
    SBX_TRACE("sbx.dense.capture");
    sbx_ctx* ctx = p->ctx;
    cudaStreamSynchronize(ctx->stream);
    int64_t l0 = ctx->launches;
    if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return fail(ctx, SBX_ECUDA, "dense plan: begin capture");
    sbx_status st;
    StepNoise sn{p->noise, p->noiseErr};
    {
        PlanScratch use(p);
        st = dense_sequence(ctx, &p->scene, p->d_step, 0, p->batched ? &p->batch : nullptr, &p->side,
                            p->noiseOn ? &sn : nullptr);
    }
    if (st == SBX_OK) SBX_LAUNCH(ctx, k_step_advance, 1, 1, p->d_step);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
    if (st != SBX_OK || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        ctx->launches = l0;
        cudaGetLastError();
        return st != SBX_OK ? st : fail(ctx, SBX_ECUDA, std::string("end capture: ") + cudaGetErrorString(ce));
    }
    cudaGraphExec_t ex = nullptr;
    if (cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) {
        cudaGraphDestroy(g);
        ctx->launches = l0;
        cudaGetLastError();
        return fail(ctx, SBX_ECUDA, "dense plan: graph instantiate");
    }
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    p->graph = g;
    p->exec = ex;
    p->kernels_per_step = (int)(ctx->launches - l0);
    ctx->launches = l0;
    return SBX_OK;
}

static sbx_status plan_create(sbx_ctx* ctx, const sbx_dense_scene* sc, const sbx_batch* bt, sbx_dense_plan** out) {
    if (!ctx || !sc || !out) return SBX_EINVAL;
    *out = nullptr;
    sbx_dense_plan* p = new sbx_dense_plan();
    p->ctx = ctx;
    p->scene = *sc;
    if (bt) {
        p->batched = true;
        p->batch = *bt;
    }
    p->scratch_bytes = dense_scratch_bytes(sc);
    if (cudaMalloc(&p->scratch, p->scratch_bytes) != cudaSuccess) {
        delete p;
        return fail(ctx, SBX_ENOMEM, "sbx_dense_plan_create: step scratch");
    }
    if (cudaMalloc(&p->d_step, sizeof(int)) != cudaSuccess) {
        cudaFree(p->scratch);
        delete p;
        return fail(ctx, SBX_ENOMEM, "sbx_dense_plan_create: step word");
    }
    p->side.scratchBytes = dense_sort_bytes(sc);
    p->sideOk = cudaStreamCreateWithFlags(&p->side.stream, cudaStreamNonBlocking) == cudaSuccess &&
                cudaEventCreateWithFlags(&p->side.fork, cudaEventDisableTiming) == cudaSuccess &&
                cudaEventCreateWithFlags(&p->side.join, cudaEventDisableTiming) == cudaSuccess &&
                cudaEventCreateWithFlags(&p->side.fork2, cudaEventDisableTiming) == cudaSuccess &&
                cudaEventCreateWithFlags(&p->side.join2, cudaEventDisableTiming) == cudaSuccess &&
                cudaMalloc(&p->side.scratch, p->side.scratchBytes) == cudaSuccess;
    if (!p->sideOk) {
        release_side(p);
        cudaFree(p->d_step);
        cudaFree(p->scratch);
        delete p;
        cudaGetLastError();
        return fail(ctx, SBX_ENOMEM, "sbx_dense_plan_create: side stream");
    }
    if (cudaMalloc(&p->stats, sizeof(unsigned long long) * SBX_FUSED_STATS) != cudaSuccess ||
        cudaMemsetAsync(p->stats, 0, sizeof(unsigned long long) * SBX_FUSED_STATS, ctx->stream) != cudaSuccess) {
        if (p->stats) cudaFree(p->stats);
        cudaFree(p->d_step);
        cudaFree(p->scratch);
        release_side(p);
        delete p;
        cudaGetLastError();
        return fail(ctx, SBX_ENOMEM, "sbx_dense_plan_create: counters");
    }
    // capture one step into a graph
    sbx_status st = capture_step(p);
    if (st != SBX_OK) {
        cudaFree(p->stats);
        cudaFree(p->d_step);
        cudaFree(p->scratch);
        release_side(p);
        delete p;
        return st;
    }
    if (p->batched) {
        p->fused_ok = false;
        p->fused_why = "packed networks run on the graph or per-system path";
    } else {
        p->fused_ok = fused_prepare(p);
    }
    cudaGetLastError();
    *out = p;
    return SBX_OK;
}

extern "C" sbx_status sbx_dense_plan_create(sbx_ctx* ctx, const sbx_dense_scene* sc, sbx_dense_plan** out) {
    return plan_create(ctx, sc, nullptr, out);
}

extern "C" sbx_status sbx_dense_plan_create_batched(sbx_ctx* ctx, const sbx_dense_scene* sc, const sbx_batch* batch,
                                                    sbx_dense_plan** out) {
    if (!batch || batch->nNet < 1 || !batch->segKey || !batch->motKey || !batch->bbKey || !batch->seeds ||
        !batch->gridParams || !batch->gridDims || !batch->boxParams || (sc && sc->xl.nLinks > 0 && !batch->linkKey))
        return ctx ? fail(ctx, SBX_EINVAL, "sbx_dense_plan_create_batched: incomplete batch") : SBX_EINVAL;
    return plan_create(ctx, sc, batch, out);
}

extern "C" sbx_status sbx_dense_plan_run(sbx_dense_plan* p, int32_t t0, int32_t nsteps, int32_t mode) {
    if (!p || nsteps < 0 || mode < 0 || mode > 3) return SBX_EINVAL;
    sbx_ctx* ctx = p->ctx;
    if (nsteps == 0) return SBX_OK;
    if (p->noiseOn && ((int64_t)t0 < p->noise.t0 || (int64_t)t0 + nsteps > (int64_t)p->noise.t0 + p->noise.nsteps))
        return fail(ctx, SBX_EINVAL, "sbx_dense_plan_run: steps outside the supplied-noise range");
    if (mode == 3) mode = (p->fused_ok && p->scene.fil.body.n <= SBX_DENSE_AUTO_MAX_FUSED_RODS) ? 2 : 1;
    if (mode == 2) {
        if (!p->fused_ok) return fail(ctx, SBX_ESTATE, "fused path unavailable: " + p->fused_why);
        // the kernel leaves its histograms zeroed and its barrier words consistent at the
        // end of every completed run; they are reset here only after a failed run
        if (p->fused_dirty) {
            FusedArgs& a = p->fa;
            cudaMemsetAsync(a.cntCell, 0, 4 * (size_t)a.C, ctx->stream);
            cudaMemsetAsync(a.cntSeg, 0, 4 * (size_t)a.C, ctx->stream);
            for (int* q : {a.cntAct, a.cntA, a.cntB, a.cntM}) cudaMemsetAsync(q, 0, 4 * (size_t)a.nSeg, ctx->stream);
            cudaMemsetAsync(a.cellHead, 0xff, 4 * (size_t)a.C, ctx->stream);
            for (int* q : {a.headA, a.headB, a.headM}) cudaMemsetAsync(q, 0xff, 4 * (size_t)a.nSeg, ctx->stream);
            cudaMemsetAsync(a.bar, 0, 32, ctx->stream);
            cudaMemsetAsync(a.err, 0, 16, ctx->stream);
            p->fused_dirty = false;
        }
        SBX_TRACE("sbx.dense.fused_launch");
        return fused_launch(ctx, p->fa, p->fused_grid, t0, nsteps);
    }
    if (mode == 1) {
        SBX_TRACE("sbx.dense.graph_replay");
        SBX_LAUNCH(ctx, k_step_set, 1, 1, p->d_step, t0);
        for (int k = 0; k < nsteps; k++) {
            if (cudaGraphLaunch(p->exec, ctx->stream) != cudaSuccess)
                return fail(ctx, SBX_ECUDA, "sbx_dense_plan_run: graph launch");
            ctx->launches += p->kernels_per_step;
        }
        return check_launch(ctx, "sbx_dense_plan_run");
    }
    SBX_TRACE("sbx.dense.unfused");
    PlanScratch use(p);
    StepNoise sn{p->noise, p->noiseErr};
    for (int k = 0; k < nsteps; k++)
        CHK(dense_sequence(ctx, &p->scene, nullptr, t0 + k, p->batched ? &p->batch : nullptr, &p->side,
                           p->noiseOn ? &sn : nullptr));
    return SBX_OK;
}

extern "C" int32_t sbx_dense_plan_kernels_per_step(sbx_dense_plan* p) { return p ? p->kernels_per_step : -1; }

extern "C" sbx_status sbx_dense_plan_status(sbx_dense_plan* p, int32_t* flags) {
    if (!p || !flags) return SBX_EINVAL;
    *flags = 0;
    if (p->noiseErr) {
        int ne = 0;
        cudaMemcpyAsync(&ne, p->noiseErr, sizeof(int), cudaMemcpyDeviceToHost, p->ctx->stream);
        CHK(sbx_ctx_sync(p->ctx));
        if (ne) {
            cudaMemsetAsync(p->noiseErr, 0, sizeof(int), p->ctx->stream);
            return fail(p->ctx, SBX_EINVAL, "dense step: a step ran outside the supplied-noise range");
        }
    }
    if (!p->fused_ok) return SBX_OK;
    int h = 0;
    cudaMemcpyAsync(&h, p->fa.err, sizeof(int), cudaMemcpyDeviceToHost, p->ctx->stream);
    CHK(sbx_ctx_sync(p->ctx));
    *flags = h;
    if (h) p->fused_dirty = true;
    if (h & 1) return fail(p->ctx, SBX_ETIMEOUT, "fused step: grid barrier wait ran out");
    if (h & 4) return fail(p->ctx, SBX_ETIMEOUT, "fused step: bulk-copy wait ran out");
    if (h & 8) return fail(p->ctx, SBX_ESTATE, "fused step: a linked-list walk ran past its bound");
    if (h & 2) return fail(p->ctx, SBX_EOVERFLOW, "fused step: a reach list exceeded SBX_MAX_CAND");
    return SBX_OK;
}

extern "C" int32_t sbx_dense_plan_fused_available(sbx_dense_plan* p) { return p && p->fused_ok ? 1 : 0; }

extern "C" sbx_status sbx_dense_plan_refresh(sbx_dense_plan* p) {
    if (!p) return SBX_EINVAL;
    if (p->batched || !p->fused_prepared) return SBX_OK;
    p->fused_ok = fused_topology(p);
    return SBX_OK;
}

extern "C" int32_t sbx_dense_plan_fused_grid(sbx_dense_plan* p) { return p ? p->fused_grid : 0; }

extern "C" sbx_status sbx_dense_plan_phase_times(sbx_dense_plan* p, int64_t* dev_times) {
    if (!p) return SBX_EINVAL;
    p->fa.phaseTimes = (long long*)dev_times;
    return SBX_OK;
}

extern "C" sbx_status sbx_dense_plan_test_barrier_extra(sbx_dense_plan* p, int32_t extra) {
    if (!p || extra < 0) return SBX_EINVAL;
    p->fa.barrierExtra = extra;
    p->fused_dirty = true;
    return SBX_OK;
}

extern "C" sbx_status sbx_dense_plan_set_noise(sbx_dense_plan* p, const sbx_dense_noise* nz) {
    if (!p) return SBX_EINVAL;
    sbx_ctx* ctx = p->ctx;
    if (p->batched) return fail(ctx, SBX_EINVAL, "sbx_dense_plan_set_noise: not available for packed plans");
    const sbx_dense_scene& sc = p->scene;
    if (nz) {
        const int64_t nf = sc.fil.body.n, nm = sc.mot.body.n, nb = sc.mini.backbone.n;
        if (nz->nsteps < 1 || (nf > 0 && !nz->fil) || (nm > 0 && !nz->mot) || (nb > 0 && !nz->bb))
            return fail(ctx, SBX_EINVAL, "sbx_dense_plan_set_noise: missing array or empty range");
        const float* arr[3] = {nz->fil, nz->mot, nz->bb};
        const int64_t len[3] = {nf, nm, nb};
        for (int k = 0; k < 3; k++) {
            if (len[k] == 0) continue;
            bool bad = false;
            CHK(any_nonfinite(ctx, arr[k], 6 * len[k] * nz->nsteps, &bad));
            if (bad) return fail(ctx, SBX_ENONFINITE, "sbx_dense_plan_set_noise: noise holds NaN/Inf");
        }
        if (!p->noiseErr) {
            if (cudaMalloc(&p->noiseErr, sizeof(int)) != cudaSuccess)
                return fail(ctx, SBX_ENOMEM, "sbx_dense_plan_set_noise: flag");
            cudaMemsetAsync(p->noiseErr, 0, sizeof(int), ctx->stream);
        }
    }
    bool wasOn = p->noiseOn;
    sbx_dense_noise was = p->noise;
    p->noiseOn = nz != nullptr;
    p->noise = nz ? *nz : sbx_dense_noise{};
    sbx_status st = capture_step(p);
    if (st != SBX_OK) {
        p->noiseOn = wasOn;
        p->noise = was;
        return st;
    }
    FusedArgs& a = p->fa;
    a.nzFil = p->noiseOn ? p->noise.fil : nullptr;
    a.nzMot = p->noiseOn ? p->noise.mot : nullptr;
    a.nzBb = p->noiseOn ? p->noise.bb : nullptr;
    a.nzT0 = p->noise.t0;
    a.nzN = p->noise.nsteps;
    return SBX_OK;
}

extern "C" sbx_status sbx_dense_plan_fused_stats(sbx_dense_plan* p, int64_t* out, int32_t reset) {
    if (!p || !out) return SBX_EINVAL;
    unsigned long long h[SBX_FUSED_STATS];
    cudaMemcpyAsync(h, p->stats, sizeof(h), cudaMemcpyDeviceToHost, p->ctx->stream);
    if (reset) cudaMemsetAsync(p->stats, 0, sizeof(h), p->ctx->stream);
    CHK(sbx_ctx_sync(p->ctx));
    for (int k = 0; k < SBX_FUSED_STATS; k++) out[k] = (int64_t)h[k];
    return SBX_OK;
}

extern "C" sbx_status sbx_dense_plan_test_caps(sbx_dense_plan* p, int32_t entCap, int32_t motorCap, int32_t motorIds,
                                               int32_t rowSlots, int32_t cellSlots) {
    if (!p) return SBX_EINVAL;
    auto clampCap = [](int v, int cap) { return v < 0 ? cap : (v > cap ? cap : v); };
    p->fa.entCap = clampCap(entCap, FUSED_ENT_CAP);
    p->fa.mCap = clampCap(motorCap, FUSED_MCAP);
    p->fa.mIds = clampCap(motorIds, FUSED_MIDS);
    p->fa.rowUse = clampCap(rowSlots, FUSED_ROW_SLOTS);
    p->fa.mRowUse = clampCap(rowSlots, FUSED_MOTOR_SLOTS);
    p->fa.cellUse = clampCap(cellSlots, FUSED_CELL_SLOTS);
    return SBX_OK;
}

extern "C" sbx_status sbx_dense_plan_destroy(sbx_dense_plan* p) {
    if (!p) return SBX_EINVAL;
    // the plan may outlive its context (language runtimes finalise objects in any order at
    // exit), so it touches no context state here: a device-wide wait before the frees
    cudaDeviceSynchronize();
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->d_step) cudaFree(p->d_step);
    if (p->scratch) cudaFree(p->scratch);
    if (p->noiseErr) cudaFree(p->noiseErr);
    if (p->stats) cudaFree(p->stats);
    release_side(p);
    for (void* q : p->allocs) cudaFree(q);
    delete p;
    return SBX_OK;
}
