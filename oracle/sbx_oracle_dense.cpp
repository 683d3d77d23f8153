// sbx_oracle_dense.cpp — CPU ORACLE (test infrastructure): the step sequences of the
// reference harnesses, driven over host arrays described by the public scene structs.
//   orc_dense_step : DenseContractileHarness.cpuStep (DenseContractileHarness.java:350-429)
//   orc_fdt_step   : DiffusionHarness.cpuStepFdt     (DiffusionHarness.java:161-169)
//   orc_chain_step : DiffusionHarness.cpuStepChain   (DiffusionHarness.java:185-196)
// The grid and CSR builds use the serial reference forms (gridHistogram/gridScatter,
// csrHistogram/csrScan/csrScatter); the chunked forms the harness wires produce the
// same arrays (the reference's own parallel==serial gate, tested separately).
#include <cstdint>
#include "../include/softbox_b200.h"

typedef int32_t i32;
#define EXPORT extern "C"

EXPORT void orc_zero_accumulators(int N, float* F, float* T);
EXPORT void orc_brownian_force(int N, float* rF, float* rT, const float* bTG, const float* bRG,
                               const float* tSc, const float* rSc, const float* params, const i32* counts);
EXPORT void orc_integrate(int N, float* coord, double* coord64, float* uVec, float* yVec, const float* F,
                          const float* T, const float* rF, const float* rT, const float* bTG,
                          const float* bRG, const float* params);
EXPORT void orc_derive(int N, const float* coord, const float* uVec, float* yVec, float* zVec,
                       float* end1, float* end2, const float* segLength);
EXPORT void orc_confine(int N, const float* coord, const float* uVec, const float* segLength,
                        const float* bTG, float* F, float* T, const float* boxParams, const i32* counts);
EXPORT void orc_chain_forces(int N, const float* coord, const float* uVec, const float* segLength,
                             const i32* e2s, const i32* e2d, const i32* e1s, const i32* e1d,
                             const float* bTG, const float* bRG, float* F, float* T, const float* chainParams);
EXPORT void orc_fil_publish(int n, const float* coord, const float* segLength, int cap, float* center,
                            float* boundingRadius, i32* ownerStore, i32* ownerSlot, const float* viewParams,
                            const i32* filState);
EXPORT void orc_mot_publish_head(int nM, const float* bodyCoord, const float* bodyUVec,
                                 const float* bodySegLength, float* head, float* uVec, float* rodUVec);
EXPORT void orc_mot_publish(int nM, const float* head, const float* reach, int cap, float* center,
                            float* boundingRadius, i32* ownerStore, i32* ownerSlot, i32 base);
EXPORT void orc_body_cell(int cap, const float* center, const float* gridParams, const i32* gridDims,
                          i32 S, i32* bodyCell);
EXPORT void orc_grid_zero(i32 totalCells, i32* cellCount);
EXPORT void orc_grid_histogram(const i32* bodyCell, i32 S, i32* cellCount);
EXPORT void orc_grid_scan_local(i32 totalCells, const i32* cellCount, i32* offsets, i32* chunkSum);
EXPORT void orc_grid_scan_chunks(i32 totalCells, i32* chunkSum);
EXPORT void orc_grid_scan_add(i32 totalCells, i32* offsets, i32 contentsCap, i32* cellCount, const i32* chunkSum);
EXPORT void orc_grid_scatter(const i32* bodyCell, i32 S, const i32* offsets, i32* contents, i32 contentsCap,
                             i32* cellCount);
EXPORT void orc_grid_reachable(i32 nM, const float* head, const float* uVec, const float* rodUVec, i32 nSeg,
                               const float* segEnd1, const float* segEnd2, const float* gridParams,
                               const i32* gridDims, const i32* offsets, const i32* contents,
                               const i32* ownerStore, const i32* ownerSlot, i32* reachSeg, i32* reachCount,
                               const float* kinParams);
EXPORT void orc_catch_slip_release(i32 nM, i32* boundSeg, const float* forceDotFil, const float* forceMag,
                                   i32* cooldown, i32* stats, i32* capStats, const float* kinParams,
                                   const i32* counts);
EXPORT void orc_bind_nearest(i32 nM, const float* head, const float* uVec, const float* rodUVec, i32 nSeg,
                             const float* segEnd1, const float* segEnd2, const i32* candSeg,
                             const i32* candCount, i32* boundSeg, float* bindArc, const float* kinParams);
EXPORT void orc_cycle(i32 nM, i32* nucleotideState, const i32* boundSeg, const float* forceDotHist,
                      const float* nucParams, const i32* counts);
EXPORT void orc_joints(i32 nB, const float* coord, const float* uVec, const float* segLength, const float* bTG,
                       const float* bRG, float* F, float* T, const i32* nucleotideState, const float* jointParams);
EXPORT void orc_dimer_couple(i32 nB, const float* coord, const float* uVec, const float* segLength,
                             const float* bTG, const float* bRG, float* F, float* T, i32 nD, const i32* motorA,
                             const i32* motorB, const i32* parallel, const float* dimerParams,
                             const i32* boundSeg);
EXPORT void orc_mini_tether(i32 nMB, const float* mC, const float* mU, const float* mLen, const float* mBTG,
                            const float* mBRG, float* mF, float* mT, i32 nBb, const float* bbC, const float* bbU,
                            const float* bbInvDragY, i32 nD, const i32* headBackboneSlot, const i32* motorA,
                            const float* attachAxial, float* miniData, const float* miniParams);
EXPORT void orc_csr_histogram(const i32* keys, i32 nItems, i32 nRows, i32* rowCount);
EXPORT void orc_csr_scan(i32 nRows, i32* rowCount, i32* rowOffsets);
EXPORT void orc_csr_scatter(const i32* keys, i32 nItems, const i32* rowOffsets, i32* rowCount, i32* rowList);
EXPORT void orc_backbone_gather(i32 nBb, const i32* offsets, const i32* list, const float* miniData,
                                float* F, float* T);
EXPORT void orc_bond_forces(i32 nB, const float* mC, const float* mU, const float* mY, const float* mBRG,
                            i32 nSeg, const float* fC, const float* fU, const float* fY, const float* fBRG,
                            const float* fLen, const i32* boundSeg, const float* bindArc,
                            const i32* nucleotideState, float* bondData, const float* xbParams);
EXPORT void orc_apply_head_force(i32 nB, const float* bondData, float* F, float* T);
EXPORT void orc_register_force_dot(i32 nM, const float* bondData, const i32* boundSeg, float* forceDotFil,
                                   float* forceMag, float* forceDotHist, i32* forceDotPlace);
EXPORT void orc_xl_unbind(i32 nSeg, const float* fU, const float* fE1, i32 nLinks, const i32* linkFilA,
                          const i32* linkFilB, const float* loc1, const float* loc2, i32* linkState,
                          float* strainHist, i32* strainPlace, const float* offParams, const i32* counts);
EXPORT void orc_count_active_links(i32 nLinks, const i32* linkState, const i32* linkFilA, const i32* linkFilB,
                                   i32 nSeg, i32* activeLinkCount);
EXPORT void orc_link_forces(i32 nSeg, const float* fC, const float* fU, const float* fE1, const float* fBTG,
                            i32 nLinks, const i32* linkFilA, const i32* linkFilB, const float* loc1,
                            const float* loc2, const i32* filLinkCt, float* xlinkData, const float* xlParams);
EXPORT void orc_link_torsion(i32 nSeg, const float* fU, i32 nLinks, const i32* linkFilA, const i32* linkFilB,
                             const i32* linkState, const i32* linkOrientSame, float* torqueMagHist,
                             i32* torqueMagPlace, float* xlinkData, const float* torsionParams);
EXPORT void orc_seg_gather_a(i32 nSeg, const i32* offsets, const i32* list, const float* xlinkData,
                             const i32* linkState, float* F, float* T);
EXPORT void orc_seg_gather_b(i32 nSeg, const i32* offsets, const i32* list, const float* xlinkData,
                             const i32* linkState, float* F, float* T);
EXPORT void orc_seg_gather(i32 nSeg, const i32* offsets, const i32* list, const float* bondData, float* F, float* T);

static void grid_build_serial(const sbx_grid_state& g) {
    i32 S = g.gridCounts[1];
    orc_grid_zero(g.totalCells, g.cellCount);
    orc_grid_histogram(g.bodyCell, S, g.cellCount);
    orc_grid_scan_local(g.totalCells, g.cellCount, g.gridCellOffsets, g.chunkSum);
    orc_grid_scan_chunks(g.totalCells, g.chunkSum);
    orc_grid_scan_add(g.totalCells, g.gridCellOffsets, g.cap, g.cellCount, g.chunkSum);
    orc_grid_scatter(g.bodyCell, S, g.gridCellOffsets, g.gridCellContents, g.cap, g.cellCount);
}

static void csr_build_serial(const i32* keys, i32 nItems, i32 nRows, i32* cnt, i32* off, i32* list) {
    orc_csr_histogram(keys, nItems, nRows, cnt);
    orc_csr_scan(nRows, cnt, off);
    orc_csr_scatter(keys, nItems, off, cnt, list);
}

EXPORT void orc_brownian_force_supplied(int N, float* rF, float* rT, const float* bTG, const float* bRG,
                                        const float* tSc, const float* rSc, const float* params,
                                        const float* noise);

// Supplied-noise mode of the step: the step's six Gaussians per body come from planar
// arrays [6][n] (filament rods, motor sub-bodies, backbones) instead of the Wang-hash
// Box-Muller draws of BrownianForceSystem.brownianForce (BrownianForceSystem.java:44-106);
// the rest of the step is unchanged.
struct DenseNoise {
    const float* fil;
    const float* mot;
    const float* bb;
};

static void dense_step(const sbx_dense_scene* sc, i32 t, const DenseNoise* nz) {
    const sbx_filament_store& f = sc->fil;
    const sbx_motor_store& mot = sc->mot;
    const sbx_dimer_store& dim = sc->dim;
    const sbx_minifilament_store& mini = sc->mini;
    const sbx_crosslinker_store& xl = sc->xl;
    const sbx_grid_state& g = sc->grid;
    const sbx_rigid_body& b = mot.body;
    const sbx_rigid_body& bb = mini.backbone;
    const sbx_rigid_body& fb = f.body;
    const i32 nSeg = fb.n, nM = mot.nMotors, nB = b.n, nBb = bb.n, nD = dim.nDimers;

    // mot.setCounts(t, SEED, f.n); mini.setBackboneCounts(t, SEED_BB); f.counts.set(1, t)
    mot.counts[0] = nM; mot.counts[1] = t; mot.counts[2] = sc->seed; mot.counts[3] = nSeg;
    mini.bbCounts[0] = nBb; mini.bbCounts[1] = t; mini.bbCounts[2] = sc->seedBb; mini.bbCounts[3] = nBb;
    f.counts[1] = t;

    // ---- (i) binding ----
    orc_mot_publish_head(nM, b.coord, b.uVec, b.segLength, mot.head, mot.uVec, mot.rodUVec);
    orc_fil_publish(nSeg, fb.coord, fb.segLength, g.cap, g.center, g.boundingRadius, g.ownerStore,
                    g.ownerSlot, g.viewParams, f.filState);
    orc_mot_publish(nM, mot.head, mot.reach, g.cap, g.center, g.boundingRadius, g.ownerStore, g.ownerSlot,
                    mot.publishParams[0]);
    orc_body_cell(g.cap, g.center, g.gridParams, g.gridDims, g.gridCounts[1], g.bodyCell);
    grid_build_serial(g);
    orc_grid_reachable(nM, mot.head, mot.uVec, mot.rodUVec, nSeg, fb.end1, fb.end2, g.gridParams, g.gridDims,
                       g.gridCellOffsets, g.gridCellContents, g.ownerStore, g.ownerSlot, g.reachSeg,
                       g.reachCount, mot.kinParams);
    orc_catch_slip_release(nM, mot.boundSeg, mot.forceDotFil, mot.forceMag, mot.cooldown, mot.stats,
                           mot.capStats, mot.kinParams, mot.counts);
    orc_bind_nearest(nM, mot.head, mot.uVec, mot.rodUVec, nSeg, fb.end1, fb.end2, g.reachSeg, g.reachCount,
                     mot.boundSeg, mot.bindArc, mot.kinParams);
    orc_cycle(nM, mot.nucleotideState, mot.boundSeg, mot.forceDotHist, mot.nucParams, mot.counts);

    // ---- (ii) minifilament structure ----
    orc_zero_accumulators(nB, b.forceSum, b.torqueSum);
    orc_zero_accumulators(nBb, bb.forceSum, bb.torqueSum);
    if (nz) {
        orc_brownian_force_supplied(nB, b.randForce, b.randTorque, b.bTransGam, b.bRotGam, b.brownTransScale,
                                    b.brownRotScale, mot.bodyParams, nz->mot);
        orc_brownian_force_supplied(nBb, bb.randForce, bb.randTorque, bb.bTransGam, bb.bRotGam,
                                    bb.brownTransScale, bb.brownRotScale, mini.bbBodyParams, nz->bb);
    } else {
        orc_brownian_force(nB, b.randForce, b.randTorque, b.bTransGam, b.bRotGam, b.brownTransScale,
                           b.brownRotScale, mot.bodyParams, mot.counts);
        orc_brownian_force(nBb, bb.randForce, bb.randTorque, bb.bTransGam, bb.bRotGam, bb.brownTransScale,
                           bb.brownRotScale, mini.bbBodyParams, mini.bbCounts);
    }
    orc_joints(nB, b.coord, b.uVec, b.segLength, b.bTransGam, b.bRotGam, b.forceSum, b.torqueSum,
               mot.nucleotideState, mot.jointParams);
    orc_dimer_couple(nB, b.coord, b.uVec, b.segLength, b.bTransGam, b.bRotGam, b.forceSum, b.torqueSum, nD,
                     dim.motorA, dim.motorB, dim.parallel, dim.dimerParams, mot.boundSeg);
    orc_mini_tether(nB, b.coord, b.uVec, b.segLength, b.bTransGam, b.bRotGam, b.forceSum, b.torqueSum, nBb,
                    bb.coord, bb.uVec, mini.bbInvDragY, mini.nDimers, mini.headBackboneSlot, mini.motorA,
                    mini.attachAxial, mini.miniData, mini.miniParams);
    csr_build_serial(mini.headBackboneSlot, mini.nDimers, nBb, mini.bbDimerCount, mini.bbDimerOffsets,
                     mini.bbDimerList);
    orc_backbone_gather(nBb, mini.bbDimerOffsets, mini.bbDimerList, mini.miniData, bb.forceSum, bb.torqueSum);
    orc_bond_forces(nB, b.coord, b.uVec, b.yVec, b.bRotGam, nSeg, fb.coord, fb.uVec, fb.yVec, fb.bRotGam,
                    fb.segLength, mot.boundSeg, mot.bindArc, mot.nucleotideState, sc->bondData, sc->xbParams);
    orc_apply_head_force(nB, sc->bondData, b.forceSum, b.torqueSum);
    orc_integrate(nB, b.coord, b.coord64, b.uVec, b.yVec, b.forceSum, b.torqueSum, b.randForce, b.randTorque,
                  b.bTransGam, b.bRotGam, mot.bodyParams);
    orc_confine(nBb, bb.coord, bb.uVec, bb.segLength, bb.bTransGam, bb.forceSum, bb.torqueSum, sc->boxParams,
                mini.bbCounts);
    orc_integrate(nBb, bb.coord, bb.coord64, bb.uVec, bb.yVec, bb.forceSum, bb.torqueSum, bb.randForce,
                  bb.randTorque, bb.bTransGam, bb.bRotGam, mini.bbBodyParams);
    orc_derive(nB, b.coord, b.uVec, b.yVec, b.zVec, b.end1, b.end2, b.segLength);
    orc_derive(nBb, bb.coord, bb.uVec, bb.yVec, bb.zVec, bb.end1, bb.end2, bb.segLength);
    orc_register_force_dot(nM, sc->bondData, mot.boundSeg, mot.forceDotFil, mot.forceMag, mot.forceDotHist,
                           mot.forceDotPlace);

    // ---- (iii)-(v) filaments ----
    orc_zero_accumulators(nSeg, fb.forceSum, fb.torqueSum);
    if (nz)
        orc_brownian_force_supplied(nSeg, fb.randForce, fb.randTorque, fb.bTransGam, fb.bRotGam,
                                    fb.brownTransScale, fb.brownRotScale, f.params, nz->fil);
    else
        orc_brownian_force(nSeg, fb.randForce, fb.randTorque, fb.bTransGam, fb.bRotGam, fb.brownTransScale,
                           fb.brownRotScale, f.params, f.counts);
    orc_chain_forces(nSeg, fb.coord, fb.uVec, fb.segLength, f.end2NbrSlot, f.end2NbrSide, f.end1NbrSlot,
                     f.end1NbrSide, fb.bTransGam, fb.bRotGam, fb.forceSum, fb.torqueSum, f.chainParams);
    if (sc->xlinkOn && xl.nLinks > 0) {
        xl.counts[1] = t; xl.counts[2] = sc->seed;
        if (sc->xlUnbind)
            orc_xl_unbind(nSeg, fb.uVec, fb.end1, xl.nLinks, xl.linkFilA, xl.linkFilB, xl.loc1, xl.loc2,
                          xl.linkState, xl.strainHist, xl.strainPlace, xl.offParams, xl.counts);
        orc_count_active_links(xl.nLinks, xl.linkState, xl.linkFilA, xl.linkFilB, nSeg, xl.activeLinkCount);
        orc_link_forces(nSeg, fb.coord, fb.uVec, fb.end1, fb.bTransGam, xl.nLinks, xl.linkFilA, xl.linkFilB,
                        xl.loc1, xl.loc2, xl.activeLinkCount, xl.xlinkData, xl.xlParams);
        orc_link_torsion(nSeg, fb.uVec, xl.nLinks, xl.linkFilA, xl.linkFilB, xl.linkState, xl.linkOrientSame,
                         xl.torqueMagHist, xl.torqueMagPlace, xl.xlinkData, xl.torsionParams);
        csr_build_serial(xl.linkFilA, xl.nLinks, nSeg, xl.segCountA, xl.segOffsetsA, xl.segIdxA);
        orc_seg_gather_a(nSeg, xl.segOffsetsA, xl.segIdxA, xl.xlinkData, xl.linkState, fb.forceSum, fb.torqueSum);
        csr_build_serial(xl.linkFilB, xl.nLinks, nSeg, xl.segCountB, xl.segOffsetsB, xl.segIdxB);
        orc_seg_gather_b(nSeg, xl.segOffsetsB, xl.segIdxB, xl.xlinkData, xl.linkState, fb.forceSum, fb.torqueSum);
    }
    csr_build_serial(mot.boundSeg, nM, nSeg, sc->segMotorCount, sc->segMotorOffsets, sc->segMotorMyo);
    orc_seg_gather(nSeg, sc->segMotorOffsets, sc->segMotorMyo, sc->bondData, fb.forceSum, fb.torqueSum);
    orc_confine(nSeg, fb.coord, fb.uVec, fb.segLength, fb.bTransGam, fb.forceSum, fb.torqueSum, sc->boxParams,
                f.counts);
    orc_integrate(nSeg, fb.coord, fb.coord64, fb.uVec, fb.yVec, fb.forceSum, fb.torqueSum, fb.randForce,
                  fb.randTorque, fb.bTransGam, fb.bRotGam, f.params);
    orc_derive(nSeg, fb.coord, fb.uVec, fb.yVec, fb.zVec, fb.end1, fb.end2, fb.segLength);
}

EXPORT void orc_dense_step(const sbx_dense_scene* sc, i32 t) { dense_step(sc, t, nullptr); }

EXPORT void orc_dense_run(const sbx_dense_scene* sc, i32 t0, i32 nsteps) {
    for (i32 k = 0; k < nsteps; k++) dense_step(sc, t0 + k, nullptr);
}

// Steps t0..t0+nsteps-1 in supplied-noise mode: step t0+k reads noiseFil[k][6][nRods],
// noiseMot[k][6][3 nMotors] and noiseBb[k][6][nBackbones].
EXPORT void orc_dense_run_supplied(const sbx_dense_scene* sc, i32 t0, i32 nsteps, const float* noiseFil,
                                   const float* noiseMot, const float* noiseBb) {
    const int64_t nf = 6 * (int64_t)sc->fil.body.n, nm = 6 * (int64_t)sc->mot.body.n,
                  nb = 6 * (int64_t)sc->mini.backbone.n;
    for (i32 k = 0; k < nsteps; k++) {
        DenseNoise nz{noiseFil + k * nf, noiseMot + k * nm, noiseBb + k * nb};
        dense_step(sc, t0 + k, &nz);
    }
}

// DiffusionHarness.cpuStepFdt: brownian -> integrate -> derive, with counts[1] = step
EXPORT void orc_fdt_run(const sbx_filament_store* f, i32 t0, i32 nsteps) {
    const sbx_rigid_body& b = f->body;
    for (i32 k = 0; k < nsteps; k++) {
        f->counts[1] = t0 + k;
        orc_brownian_force(b.n, b.randForce, b.randTorque, b.bTransGam, b.bRotGam, b.brownTransScale,
                           b.brownRotScale, f->params, f->counts);
        orc_integrate(b.n, b.coord, b.coord64, b.uVec, b.yVec, b.forceSum, b.torqueSum, b.randForce,
                      b.randTorque, b.bTransGam, b.bRotGam, f->params);
        orc_derive(b.n, b.coord, b.uVec, b.yVec, b.zVec, b.end1, b.end2, b.segLength);
    }
}

// DiffusionHarness.cpuStepChain: zero -> brownian -> chain -> integrate -> derive
EXPORT void orc_chain_run(const sbx_filament_store* f, i32 t0, i32 nsteps) {
    const sbx_rigid_body& b = f->body;
    for (i32 k = 0; k < nsteps; k++) {
        f->counts[1] = t0 + k;
        orc_zero_accumulators(b.n, b.forceSum, b.torqueSum);
        orc_brownian_force(b.n, b.randForce, b.randTorque, b.bTransGam, b.bRotGam, b.brownTransScale,
                           b.brownRotScale, f->params, f->counts);
        orc_chain_forces(b.n, b.coord, b.uVec, b.segLength, f->end2NbrSlot, f->end2NbrSide, f->end1NbrSlot,
                         f->end1NbrSide, b.bTransGam, b.bRotGam, b.forceSum, b.torqueSum, f->chainParams);
        orc_integrate(b.n, b.coord, b.coord64, b.uVec, b.yVec, b.forceSum, b.torqueSum, b.randForce,
                      b.randTorque, b.bTransGam, b.bRotGam, f->params);
        orc_derive(b.n, b.coord, b.uVec, b.yVec, b.zVec, b.end1, b.end2, b.segLength);
    }
}
