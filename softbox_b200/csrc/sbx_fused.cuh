// sbx_fused.cuh — arguments of the fused persistent dense-step kernel (sbx_fused.cu).
#pragma once
#include "../../include/softbox_b200.h"
#include "sbx_internal.cuh"

constexpr int FUSED_THREADS = 128;
constexpr int FUSED_MAX_SUB = 120;    // sub-bodies per minifilament CTA (6 per dimer)
constexpr int FUSED_MAX_ROD = 128;    // segments per rod CTA
constexpr int FUSED_MAX_DPM = 16;     // dimers per minifilament (32 heads: one warp)
constexpr int FUSED_ENT_CAP = 256;    // CSR payload entries a rod CTA stages in shared memory

struct FusedArgs {
    sbx_dense_scene sc;
    int nSeg, nM, nB, nBb, nD, nL, cap, S, C;
    int nX, nY, nZ;
    int dpm;                 // dimers per minifilament
    int G, nRodUnits;        // segments per rod unit (whole filaments), units
    int tilesC, tilesS;
    int xlOn, xlUnbind, useTma, filSeed;
    int jointShare;          // chain neighbours are symmetric: each joint computed once
    // private scratch (plan-owned)
    int *cntCell, *cntSeg, *cntAct, *cntA, *cntB, *cntM;   // cntSeg: segments per cell
    int* segCellOff;         // segment-only exclusive prefix over cells (C + 1)
    int* tileSum;
    int *tmpCell, *tmpA, *tmpB, *tmpM;
    float4 *segE1, *segE2;   // segment endpoints in cell order: {end1, slot}, {end2, 0}
    unsigned* bar;           // [0] arrivals, [1] generation
    int* err;                // bit0 barrier timeout, bit1 reach overflow, bit2 TMA wait timeout
    int* d_step;
    int barrierExtra;        // test hook: arrivals the barrier waits for beyond gridDim.x
    long long* phaseTimes;   // optional: %globaltimer after each phase barrier, [nsteps][FUSED_PHASES]
};

constexpr int FUSED_PHASES = 11;

sbx_status fused_launch(sbx_ctx* ctx, FusedArgs& a, int grid, int t0, int nsteps);
int fused_max_blocks_per_sm();
