// sbx_fused.cuh — arguments of the fused persistent dense-step kernel (sbx_fused.cu).
#pragma once
#include "../../include/softbox_b200.h"
#include "sbx_internal.cuh"

constexpr int FUSED_THREADS = 128;
constexpr int FUSED_MAX_SUB = 120;    // sub-bodies per minifilament CTA (6 per dimer)
constexpr int FUSED_MAX_ROD = 64;     // segments per rod CTA (whole filaments)
constexpr int FUSED_MAX_DPM = 16;     // dimers per minifilament (32 heads: one warp)
constexpr int FUSED_ENT_CAP = 256;    // CSR payload entries a rod CTA stages in shared memory
constexpr int FUSED_MCAP = 16;        // motor reactions per segment a rod CTA stages in shared memory
constexpr int FUSED_MIDS = 16;        // motor slots per segment a rod CTA sorts (more: repeated-minimum walk)
constexpr int FUSED_CELL_SLOTS = 4;   // fixed slots per grid cell
constexpr int FUSED_JOINT_BYTES = 64; // one chain joint (ChainJoint, padded)
constexpr int FUSED_TERM_BYTES = 80;  // one position-only myosin term (MotorJoint, CoupleTerm, LeverTerm, TetherTerm)
constexpr int FUSED_ROW_SLOTS = 4;    // fixed slots per segment row of link A ends, of link B ends
constexpr int FUSED_MOTOR_SLOTS = 16; // fixed slots per segment row of bound motors
constexpr int FUSED_MIN_HELPERS = 16; // CTAs kept free of rod units in the rod phase

struct FusedArgs {
    sbx_dense_scene sc;
    int nSeg, nM, nB, nBb, nD, nL, cap, S, C;
    int nX, nY, nZ;
    int dpm;                 // dimers per minifilament
    int G, nRodUnits;        // segments per rod unit (whole filaments), units
    int tilesC, tilesS;
    int xlOn, xlUnbind, useTma, filSeed;
    int jointShare;          // chain neighbours are symmetric: each joint computed once
    int nbrGlobal;           // some chain neighbour lies outside its rod group (turnover topologies)
    float* uSnap;            // with nbrGlobal: this step's start orientations (3 planes of nSeg), from phase A
    int kHelp0;              // first CTA of the rod phase's helpers (motor CSR build, resets)
    // private scratch (plan-owned)
    int *cntCell, *cntSeg, *cntAct, *cntA, *cntB, *cntM;   // cntSeg: segments per cell
    int* segCellOff;         // segment-only exclusive prefix over cells (C + 1)
    void* joints;            // chain joints at (owner rod, owner side): 2 * nSeg slots of FUSED_JOINT_BYTES
    // the position-only myosin terms of the step, 2 nM + 4 nD slots of FUSED_TERM_BYTES:
    // motor joints [which][motor], coupling end variants [dimer][variant], lever torsion
    // [dimer], tethers [dimer]
    void* terms;
    int* tileSum;            // tile sums of the step's scans (cells, segments, link A, link B)
    int* mTileSum;           // tile sums of the motor CSR scan
    // rows of the step's inverse maps (cells -> bodies, segments -> link A/B ends,
    // segments -> bound motors): the first arrivals of a row sit in its fixed slots, the
    // rest in a singly linked overflow list (head per row, next per item; -1 ends)
    int *cellSlot, *slotA, *slotB, *slotM;
    int *cellHead, *cellNext, *headA, *nextA, *headB, *nextB, *headM, *nextM;
    float4 *segE1, *segE2;   // segment endpoints in cell order: {end1, slot}, {end2, 0}
    unsigned long long* bar; // arrival counters (monotonic): [0] grid barrier, [1] rod-phase helpers
    int* err;                // bit0 barrier timeout, bit1 reach overflow, bit2 TMA wait timeout, bit3 list walk
    int* d_step;
    int barrierExtra;        // test hook: arrivals the barrier waits for beyond gridDim.x
    long long* phaseTimes;   // optional: %globaltimer after each phase barrier, [nsteps][FUSED_PHASES]
    // supplied-noise mode (sbx_dense_plan_set_noise): planar [nzN][6][n] per store, or null
    const float *nzFil, *nzMot, *nzBb;
    int nzT0, nzN;
    unsigned long long* stats;   // capacity-fallback counters (SBX_FUSED_STATS)
    int entCap, mCap, mIds;      // staging capacities in use (<= the compiled ones; lowered by a test hook)
    int cellUse, rowUse, mRowUse;   // fixed row slots in use per cell / per link row / per motor row (<= the compiled ones)
};

// counters of sbx_dense_plan_fused_stats
enum FusedStat { ST_CELL_LIST = 0, ST_LINK_LIST, ST_MOTOR_LIST, ST_ENT_GLOBAL, ST_MPAY_GLOBAL, ST_MIDS_WALK,
                 ST_REACH_OVER };

constexpr int FUSED_PHASES = SBX_FUSED_PHASES;

sbx_status fused_launch(sbx_ctx* ctx, FusedArgs& a, int grid, int t0, int nsteps);
int fused_max_blocks_per_sm();
