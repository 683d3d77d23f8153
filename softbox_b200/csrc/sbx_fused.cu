// sbx_fused.cu — the dense contractile step as ONE persistent cooperative kernel.
//
// A launch advances nsteps steps. Within a step, seven phases are separated by a grid-wide
// barrier (bounded spin: a barrier that does not complete within the limit raises
// error bit 0 and every CTA returns, so a fault cannot hang the device):
//
//   A  publish the body view (FilamentStore/MotorStore.publish*), bin bodies
//      (SpatialGrid.bodyCell): cell histogram (+ row slots), segments-per-cell
//      histogram; link-key histograms (+ row slots)
//   B  tile sums of the four histograms; the warps without a tile run the crosslinker
//      Bell unbind and count the active links
//   C  exclusive scans -> gridCellOffsets (+ chunkSum, cellCount), the segment-only cell
//      prefix, segOffsetsA / segOffsetsB (+ counts); the warps without a tile draw the
//      Brownian forces of the motor sub-bodies and backbones
//   E  stable placement by list rank -> gridCellContents, segIdxA, segIdxB and the
//      segment endpoints in cell order (float4) for the reach walk
//   B0 binding of every head, 8 lanes per head: release, the reach walk fused with the
//      nearest-segment choice (the group's lanes test 8 candidates at a time, appended in
//      order), nucleotide cycle; bound heads join their segment's motor list
//   F  one CTA per minifilament: every position-only myosin term, then the ordered sums,
//      the cross-bridge bonds and integrate + derive of its 96 sub-bodies and backbone,
//      all force sums in shared memory; other CTAs compute crosslinker forces + torsion,
//      the chain joints and the filament Brownian draws
//   K  one CTA per group of whole filaments, poses staged in shared memory with TMA
//      bulk copies: chain forces (each joint once), crosslinker A/B gathers, motor
//      gather from the segment's motor list in ascending slot order (FP64 sums),
//      containment, integrate + derive; helper CTAs build the motor CSR arrays and reset
//      the step's histograms and lists
//
// Every slot is computed by the same device functions as the per-system kernels, in the
// reference's accumulation order, so the result is bit-identical to
// DenseContractileHarness.cpuStep (DenseContractileHarness.java:350-429).
#define SBX_SHARE_CALLS 1
#include <cuda_runtime.h>

#include "../../include/softbox_b200.h"
#include "sbx_fused.cuh"
#include "sbx_internal.cuh"
#include "sbx_physics.cuh"

using namespace sbx;

namespace {

constexpr unsigned long long WAIT_NS = 1000000000ULL;   // barrier and bulk-copy waits give up after one second
constexpr int ERR_BARRIER = 1, ERR_REACH_OVERFLOW = 2, ERR_TMA = 4, ERR_LIST = 8;

// shared memory of one CTA, reused by the phases
struct RodSmem {
    float st[10 * FUSED_MAX_ROD];                 // staged rod geometry planes (TMA destination)
    int off[3][FUSED_MAX_ROD + 1];                // the group's CSR row offsets: links A, links B, motors
    float ent[FUSED_ENT_CAP][6];                  // the group's link CSR payloads, in CSR order
    int entOk[FUSED_ENT_CAP];                     // guard passed (active link)
    int mCnt[FUSED_MAX_ROD];                      // motors bound to each rod
    int mLen[FUSED_MAX_ROD];                      // each rod's motor row length (histogram)
    int mRaw[FUSED_MAX_ROD][FUSED_MOTOR_SLOTS];   // a short row's slots in arrival order
    int mIds[FUSED_MAX_ROD][FUSED_MIDS];          // their slots, ascending (the first FUSED_MIDS)
    float mPay[FUSED_MAX_ROD][FUSED_MCAP][6];     // the first FUSED_MCAP bond reactions
};
struct MiniSmem {
    float sF[3 * FUSED_MAX_SUB], sT[3 * FUSED_MAX_SUB];
};
static_assert(sizeof(ChainJoint) <= FUSED_JOINT_BYTES, "joint slot size");
static_assert(sizeof(MotorJoint) <= FUSED_TERM_BYTES && sizeof(CoupleTerm) <= FUSED_TERM_BYTES &&
                  sizeof(LeverTerm) <= FUSED_TERM_BYTES && sizeof(TetherTerm) <= FUSED_TERM_BYTES,
              "myosin term slot size");

// slots of the step's myosin terms (FusedArgs::terms)
__device__ __forceinline__ MotorJoint& term_joint(const FusedArgs& a, int m, int which) {
    return *reinterpret_cast<MotorJoint*>((char*)a.terms + ((size_t)which * a.nM + m) * FUSED_TERM_BYTES);
}
__device__ __forceinline__ CoupleTerm& term_couple(const FusedArgs& a, int d, int variant) {
    return *reinterpret_cast<CoupleTerm*>((char*)a.terms + (2 * (size_t)a.nM + 2 * d + variant) * FUSED_TERM_BYTES);
}
__device__ __forceinline__ LeverTerm& term_lever(const FusedArgs& a, int d) {
    return *reinterpret_cast<LeverTerm*>((char*)a.terms + (2 * (size_t)a.nM + 2 * (size_t)a.nD + d) * FUSED_TERM_BYTES);
}
__device__ __forceinline__ TetherTerm& term_tether(const FusedArgs& a, int d) {
    return *reinterpret_cast<TetherTerm*>((char*)a.terms + (2 * (size_t)a.nM + 3 * (size_t)a.nD + d) * FUSED_TERM_BYTES);
}

union FusedSmem {
    RodSmem rod;
    MiniSmem mini;
};

__device__ __forceinline__ int vload(const int* p) { return *(const volatile int*)p; }

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long ns;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(ns));
    return ns;
}
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add(unsigned long long* p, unsigned long long v) {
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}

// Barrier over `n` CTAs on a monotonic 64-bit arrival counter: after the block barrier,
// thread 0 adds one arrival with release semantics and polls with acquire loads until
// the counter reaches this barrier's target (the previous target + n). A wait longer
// than WAIT_NS, or an error raised elsewhere, sets/sees ERR_BARRIER and returns false.
__device__ bool counter_sync(unsigned long long* ctr, unsigned long long& target, unsigned n, int* err) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        target += n;
        red_release_add(ctr, 1ULL);
        unsigned long long t0 = 0;
        unsigned it = 0;
        bool ok = true;
        while (ld_acquire(ctr) < target) {
            if ((++it & 63u) == 0) {
                if (vload(err) & (ERR_BARRIER | ERR_TMA)) { ok = false; break; }
                unsigned long long now = gtimer();
                if (t0 == 0) t0 = now;
                else if (now - t0 > WAIT_NS) { atomicOr(err, ERR_BARRIER); ok = false; break; }
            }
        }
        s_ok = ok && (vload(err) & (ERR_BARRIER | ERR_TMA)) == 0;
    }
    __syncthreads();
    return s_ok;
}

// the counter value at which this launch's barriers start: every completed barrier adds
// exactly n arrivals, and no barrier completes before every CTA has read the counter
__device__ __forceinline__ unsigned long long counter_base(const unsigned long long* ctr, unsigned n) {
    unsigned long long c = ld_acquire(ctr);
    return c - c % n;
}

__device__ __forceinline__ int gtid() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int gthreads() { return gridDim.x * blockDim.x; }

// BrownianForceSystem.brownianForce (BrownianForceSystem.java:44-106), component j (0..2) of
// one slot: the slot's j-th Box-Muller pair gives its random force and torque components j
// (randF = ((tS * mag) * sqrt(gamma)) * g, :94-104). In supplied-noise mode the Gaussians come
// from noise[t - t0][6][n] (a step outside the supplied range, which the host rejects before
// the launch, draws zeros).
__device__ __forceinline__ void brownian_component(const FusedArgs& a, const sbx_rigid_body& b, int s, int j, int t,
                                                   int seed, float mag, const float* noise) {
    const int n = b.n;
    float gf, gt;
    if (noise) {
        int k = t - a.nzT0;
        bool in = k >= 0 && k < a.nzN;
        const float* q = noise + (int64_t)(in ? k : 0) * 6 * n + s;
        gf = in ? q[(int64_t)j * n] : 0.f;
        gt = in ? q[(int64_t)(3 + j) * n] : 0.f;
    } else {
        gauss_pair_wang(s, t, seed, j, &gf, &gt);
    }
    const float tS = b.brownTransScale[s], rS = b.brownRotScale[s];
    b.randForce[j * n + s] = tS * mag * fsqrt(b.bTransGam[j * n + s]) * gf;
    b.randTorque[j * n + s] = rS * mag * fsqrt(b.bRotGam[j * n + s]) * gt;
}

// ---------------------------------------------------------------- rows: slots + overflow lists
// Rank of `self` in a row = the number of the row's items with a smaller index, counted
// along the row's list: the position the reference's serial scatter gives it (items are
// scattered in ascending index). A walk longer than `bound` marks the list corrupt.
__device__ __forceinline__ int list_rank(const FusedArgs& a, int head, const int* next, int self, int bound) {
    int r = 0, it = 0;
    for (int j = head; j >= 0; j = next[j]) {
        if (!SBX_IDX_OK(j, bound, CK_LIST_ENTRY)) break;
        r += j < self;
        if (++it > bound) {
            atomicOr(a.err, ERR_LIST);
            break;
        }
    }
    return r;
}

// Appends `item` to row r: the histogram's old count is its arrival index; the first `use`
// (<= S, the slot stride) arrivals take the row's fixed slots, later ones join the row's
// overflow list (returns 1).
__device__ __forceinline__ int row_insert(int* cnt, int* slot, int S, int use, int* head, int* next, int r,
                                          int item) {
    int j = atomicAdd(&cnt[r], 1);
    if (j < use) {
        slot[(size_t)r * S + j] = item;
        return 0;
    }
    next[item] = atomicExch(&head[r], item);
    return 1;
}

// adds a thread's count of a capacity fallback to the plan's counters
__device__ __forceinline__ void stat_add(const FusedArgs& a, int which, int v) {
    if (v) atomicAdd(&a.stats[which], (unsigned long long)v);
}

// rank of `item` in row r: the row's members with a smaller index (slots, then the list)
template <int S>
__device__ __forceinline__ int row_rank(const FusedArgs& a, const int* cnt, const int* slot, int use,
                                        const int* head, const int* next, int r, int item, int bound) {
    int n = cnt[r];
    int rank = 0;
#pragma unroll
    for (int j = 0; j < S; j++)
        if (j < n && j < use) rank += slot[(size_t)r * S + j] < item;
    if (n > use) rank += list_rank(a, head[r], next, item, bound);
    return rank;
}

// ---------------------------------------------------------------- phase A
__device__ void phase_publish_bin(const FusedArgs& a, int t) {
    const sbx_dense_scene& sc = a.sc;
    const sbx_grid_state& g = sc.grid;
    const sbx_rigid_body& fb = sc.fil.body;
    const sbx_rigid_body& mb = sc.mot.body;
    const sbx_crosslinker_store& xl = sc.xl;
    const int nSeg = a.nSeg, nM = a.nM, nB = a.nB, cap = a.cap;
    const float* gp = g.gridParams;
    const int nX = a.nX, nY = a.nY, nZ = a.nZ;
    const int nLk = a.xlOn ? a.nL : 0;
    const int total = cap + nLk + nSeg;
    const int* fb_state = sc.fil.filState;      // FREE (< 0) slots of turnover, or none
    int overCell = 0, overLink = 0;
    for (int i = gtid(); i < total; i += gthreads()) {
        if (i >= cap + nLk) {
            // the motor lists and counts of the previous step were last read by its rod phase
            int s = i - (cap + nLk);
            a.headM[s] = -1;
            a.cntM[s] = 0;
            continue;
        }
        if (i < nSeg) {
            float c[3] = {fb.coord[i], fb.coord[nSeg + i], fb.coord[2 * nSeg + i]};
            g.center[i] = c[0]; g.center[cap + i] = c[1]; g.center[2 * cap + i] = c[2];
            g.boundingRadius[i] = 0.5f * fb.segLength[i] + g.viewParams[0];
            g.ownerStore[i] = (fb_state && fb_state[i] < 0) ? STORE_NONE : STORE_FILAMENT;
            if (a.nbrGlobal)
                for (int k = 0; k < 3; k++) a.uSnap[k * nSeg + i] = fb.uVec[k * nSeg + i];
            g.ownerSlot[i] = i;
            if (i < a.S) {
                int cell = cell_coord(c[0], gp[0], gp[4], nX) + cell_coord(c[1], gp[1], gp[4], nY) * nX +
                           cell_coord(c[2], gp[2], gp[4], nZ) * (nX * nY);
                g.bodyCell[i] = cell;
                atomicAdd(&a.cntSeg[cell], 1);
                overCell += row_insert(a.cntCell, a.cellSlot, FUSED_CELL_SLOTS, a.cellUse, a.cellHead, a.cellNext, cell, i);
            } else {
                g.bodyCell[i] = -1;
            }
        } else if (i < nSeg + nM) {
            int m = i - nSeg, h = 3 * m + 2, r = 3 * m;
            float hl = mb.segLength[h];
            float hd[3];
            for (int k = 0; k < 3; k++) {
                hd[k] = mb.coord[k * nB + h] + 0.5f * hl * mb.uVec[k * nB + h];
                sc.mot.head[k * nM + m] = hd[k];
                sc.mot.uVec[k * nM + m] = mb.uVec[k * nB + h];
                sc.mot.rodUVec[k * nM + m] = mb.uVec[k * nB + r];
            }
            int b = i;   // base slot == nSeg (checked at plan creation)
            g.center[b] = hd[0]; g.center[cap + b] = hd[1]; g.center[2 * cap + b] = hd[2];
            g.boundingRadius[b] = sc.mot.reach[m];
            g.ownerStore[b] = STORE_MOTOR;
            g.ownerSlot[b] = m;
            if (b < a.S) {
                int cell = cell_coord(hd[0], gp[0], gp[4], nX) + cell_coord(hd[1], gp[1], gp[4], nY) * nX +
                           cell_coord(hd[2], gp[2], gp[4], nZ) * (nX * nY);
                g.bodyCell[b] = cell;
                overCell += row_insert(a.cntCell, a.cellSlot, FUSED_CELL_SLOTS, a.cellUse, a.cellHead, a.cellNext, cell, b);
            } else {
                g.bodyCell[b] = -1;
            }
        } else if (i < cap) {
            g.bodyCell[i] = -1;
        } else {
            int k = i - cap;
            int la = xl.linkFilA[k], lb = xl.linkFilB[k];
            if (la >= 0 && SBX_IDX_OK(la, nSeg, CK_LINK_END))
                overLink += row_insert(a.cntA, a.slotA, FUSED_ROW_SLOTS, a.rowUse, a.headA, a.nextA, la, k);
            if (lb >= 0 && SBX_IDX_OK(lb, nSeg, CK_LINK_END))
                overLink += row_insert(a.cntB, a.slotB, FUSED_ROW_SLOTS, a.rowUse, a.headB, a.nextB, lb, k);
        }
    }
    stat_add(a, ST_CELL_LIST, overCell);
    stat_add(a, ST_LINK_LIST, overLink);
}

// CrosslinkerSystem.unbind (Bell law over the strain window, CrosslinkerSystem.java:
// 727-756) and countActiveLinks (:694-708), on the warps from `firstWarp` on (all warps
// when there are none). The link CSR keys (linkFilA/B) do not depend on the state.
__device__ void link_unbind(const FusedArgs& a, int t, int firstWarp) {
    const sbx_dense_scene& sc = a.sc;
    const sbx_crosslinker_store& xl = sc.xl;
    const sbx_rigid_body& fb = sc.fil.body;
    int w = gtid() >> 5, nw = gthreads() >> 5;
    if (firstWarp >= nw) firstWarp = 0;
    if (w < firstWarp) return;
    for (int k = (w - firstWarp) * 32 + (threadIdx.x & 31); k < a.nL; k += (nw - firstWarp) * 32) {
        int la = xl.linkFilA[k], lb = xl.linkFilB[k];
        int state = xl.linkState[k];
        if (!SBX_IDX_OK_OR_NONE(la, a.nSeg, CK_LINK_END) || !SBX_IDX_OK_OR_NONE(lb, a.nSeg, CK_LINK_END)) continue;
        if (a.xlUnbind && state >= 0 &&
            unbind_one(k, a.nSeg, fb.uVec, fb.end1, la, lb, xl.loc1[k], xl.loc2[k], xl.strainHist, xl.strainPlace,
                       xl.offParams, t, sc.seed)) {
            state = LINK_FREE;
            xl.linkState[k] = state;
        }
        if (state >= 0) {
            atomicAdd(&a.cntAct[la], 1);
            atomicAdd(&a.cntAct[lb], 1);
        }
    }
}

// BrownianForceSystem for the motor sub-bodies, then the backbones, on the warps from
// `firstWarp` on (all warps when there are none): one thread per (component, slot)
__device__ void motor_brownian(const FusedArgs& a, int t, int firstWarp) {
    const sbx_dense_scene& sc = a.sc;
    int w = gtid() >> 5, nw = gthreads() >> 5;
    if (firstWarp >= nw) firstWarp = 0;
    if (w < firstWarp) return;
    const int nB = a.nB, n = nB + a.nBb;
    for (int q = (w - firstWarp) * 32 + (threadIdx.x & 31); q < 3 * n; q += (nw - firstWarp) * 32) {
        const int c = q / n, j = q - c * n;
        if (j < nB) brownian_component(a, sc.mot.body, j, c, t, sc.seed, sc.mot.bodyParams[1], a.nzMot);
        else brownian_component(a, sc.mini.backbone, j - nB, c, t, sc.seedBb, sc.mini.bbBodyParams[1], a.nzBb);
    }
}

// The position-only terms of the myosin mechanics, none of which depends on this step's
// binding or forces (MotorJointSystem.java:72-123 joint geometry, DimerCouplingSystem.java:
// 99-182 end variants and lever torsion, MiniFilamentSystem tethers with their backbone
// reaction rows), one item per term on the warps from `firstWarp` on (all warps when
// there are none); the minifilament phase accumulates them in the reference's order.
__device__ void myosin_terms(const FusedArgs& a, int firstWarp) {
    const sbx_dense_scene& sc = a.sc;
    const sbx_motor_store& mot = sc.mot;
    const sbx_rigid_body& mb = mot.body;
    const sbx_minifilament_store& mini = sc.mini;
    const sbx_rigid_body& bb = mini.backbone;
    int w = gtid() >> 5, nw = gthreads() >> 5;
    if (firstWarp >= nw) firstWarp = 0;
    if (w < firstWarp) return;
    const int nM = a.nM, nD = a.nD, nB = a.nB;
    const int total = 2 * nM + 4 * nD;
    for (int k = (w - firstWarp) * 32 + (threadIdx.x & 31); k < total; k += (nw - firstWarp) * 32) {
        if (k < 2 * nM) {
            const int which = k >= nM, m = k - which * nM;
            term_joint(a, m, which) = motor_joint(m, which, nB, mb.coord, mb.uVec, mb.segLength, mb.bTransGam,
                                                  mb.bRotGam, mot.jointParams);
        } else if (k < 2 * nM + 2 * nD) {
            const int q = k - 2 * nM, d = q >> 1;
            term_couple(a, d, q & 1) = couple_variant(nB, mb.coord, mb.uVec, mb.segLength, mb.bTransGam, mb.bRotGam,
                                                      2 * d, 2 * d + 1, sc.dim.parallel[d] != 0, sc.dim.dimerParams,
                                                      q & 1);
        } else if (k < 2 * nM + 3 * nD) {
            const int d = k - 2 * nM - 2 * nD;
            term_lever(a, d) = couple_lever(nB, mb.uVec, mb.bRotGam, 2 * d, 2 * d + 1, sc.dim.dimerParams);
        } else {
            const int d = k - 2 * nM - 3 * nD, u = d / a.dpm;
            TetherTerm T = tether_terms(nB, mb.coord, mb.uVec, mb.segLength, mb.bTransGam, mb.bRotGam, a.nBb, bb.coord,
                                        bb.uVec, mini.bbInvDragY, u, 2 * d, mini.attachAxial[d], mini.miniParams);
            term_tether(a, d) = T;
            float* o = mini.miniData + (int64_t)MINI_STRIDE * d;
            for (int j = 0; j < 6; j++) o[j] = T.row[j];
            // backbone CSR of the reference (rows = backbones, items = dimers in index order)
            mini.bbDimerList[d] = d;
        }
    }
}

// ---------------------------------------------------------------- scans (B, C, G, H)
struct ScanArr {
    const int* cnt;   // histogram
    int n;            // rows
    int tile0;        // first tile index in the shared tile-sum array
};

__device__ __forceinline__ int warp_sum(int v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ void tile_sums(const ScanArr* arrs, int narr, int* tileSum, int warp, int nwarps) {
    int lane = threadIdx.x & 31;
    int total = arrs[narr - 1].tile0 + (arrs[narr - 1].n + SCAN_CHUNK - 1) / SCAN_CHUNK;
    for (int tl = warp; tl < total; tl += nwarps) {
        int ai = 0;
        while (ai + 1 < narr && tl >= arrs[ai + 1].tile0) ai++;
        const ScanArr& s = arrs[ai];
        int base = (tl - s.tile0) * SCAN_CHUNK;
        int v = 0;
        for (int j = lane; j < SCAN_CHUNK; j += 32) v += (base + j < s.n) ? s.cnt[base + j] : 0;
        v = warp_sum(v);
        if (lane == 0) tileSum[tl] = v;
    }
}

// exclusive scan of each array into out[ai][0..n] (terminator = min(total, clamp[ai]));
// copy[ai] (optional) receives the counts — the row lengths the reference's serial
// scatter leaves in its write cursors; chunkOut (optional, array 0) gets the tile-prefix
// layout of SpatialGrid.gridScanChunks.
__device__ void tile_scan(const ScanArr* arrs, int narr, const int* tileSum, int* const* out, int* const* copy,
                          const int* clampTotal, int* chunkOut, int warp, int nwarps) {
    int lane = threadIdx.x & 31;
    int total = arrs[narr - 1].tile0 + (arrs[narr - 1].n + SCAN_CHUNK - 1) / SCAN_CHUNK;
    for (int tl = warp; tl < total; tl += nwarps) {
        int ai = 0;
        while (ai + 1 < narr && tl >= arrs[ai + 1].tile0) ai++;
        const ScanArr& s = arrs[ai];
        int ntiles = (s.n + SCAN_CHUNK - 1) / SCAN_CHUNK;
        int local = tl - s.tile0;
        // the preceding tiles' sums: 16 predicated loads per lane in flight together
        int b = 0;
#pragma unroll
        for (int q = 0; q < 16; q++) {
            int j = lane + 32 * q;
            b += (j < local) ? tileSum[s.tile0 + j] : 0;
        }
        for (int j = lane + 512; j < local; j += 32) b += tileSum[s.tile0 + j];
        b = warp_sum(b);
        int base = local * SCAN_CHUNK;
        constexpr int PER = SCAN_CHUNK / 32;
        // coalesced: row j of the tile is elements base + 32 j + lane
        int vals[PER];
#pragma unroll
        for (int j = 0; j < PER; j++) {
            int r = base + 32 * j + lane;
            vals[j] = r < s.n ? s.cnt[r] : 0;
        }
        int run = b;
#pragma unroll
        for (int j = 0; j < PER; j++) {
            int v = vals[j], x = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            int r = base + 32 * j + lane;
            if (r < s.n) {
                out[ai][r] = run + x - v;
                if (copy[ai]) copy[ai][r] = v;
            }
            run += __shfl_sync(0xffffffffu, x, 31);
        }
        if (lane == 0 && ai == 0 && chunkOut) chunkOut[local] = b;
        if (local == ntiles - 1) {
            int tot = run;
            if (lane == 0) {
                out[ai][s.n] = tot < clampTotal[ai] ? tot : clampTotal[ai];
                if (ai == 0 && chunkOut) chunkOut[ntiles] = tot;
            }
        }
    }
}

// ---------------------------------------------------------------- E: stable placement
__device__ void phase_place(const FusedArgs& a) {
    const sbx_dense_scene& sc = a.sc;
    const sbx_grid_state& g = sc.grid;
    const sbx_crosslinker_store& xl = sc.xl;
    const sbx_rigid_body& fb = sc.fil.body;
    const int nSeg = a.nSeg;
    int total = a.cap + (a.xlOn ? a.nL : 0);
    for (int i = gtid(); i < total; i += gthreads()) {
        if (i < a.cap) {
            int c = g.bodyCell[i];
            if (c < 0 || !SBX_IDX_OK(c, a.C, CK_CELL)) continue;
            int rank = row_rank<FUSED_CELL_SLOTS>(a, a.cntCell, a.cellSlot, a.cellUse, a.cellHead, a.cellNext, c, i, a.cap);
            if (!SBX_IDX_OK(g.gridCellOffsets[c] + rank, a.cap, CK_CSR_POS)) continue;
            g.gridCellContents[g.gridCellOffsets[c] + rank] = i;
            // segment endpoints in cell order for the reach walk: within a cell the segments
            // (slots below nSeg) precede the motor heads, so a segment's rank among the
            // segments of its cell equals its rank in the cell
            if (i < nSeg && SBX_IDX_OK(a.segCellOff[c] + rank, nSeg, CK_CSR_POS)) {
                int q = a.segCellOff[c] + rank;
                if (g.ownerStore[i] == STORE_FILAMENT) {
                    a.segE1[q] = make_float4(fb.end1[i], fb.end1[nSeg + i], fb.end1[2 * nSeg + i], __int_as_float(i));
                    a.segE2[q] = make_float4(fb.end2[i], fb.end2[nSeg + i], fb.end2[2 * nSeg + i], 0.f);
                } else {
                    a.segE1[q] = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
                    a.segE2[q] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
            }
        } else {
            int k = i - a.cap;
            int la = xl.linkFilA[k], lb = xl.linkFilB[k];
            if (!SBX_IDX_OK_OR_NONE(la, nSeg, CK_LINK_END) || !SBX_IDX_OK_OR_NONE(lb, nSeg, CK_LINK_END)) continue;
            if (la >= 0)
                xl.segIdxA[xl.segOffsetsA[la] +
                           row_rank<FUSED_ROW_SLOTS>(a, a.cntA, a.slotA, a.rowUse, a.headA, a.nextA, la, k, a.nL)] = k;
            if (lb >= 0)
                xl.segIdxB[xl.segOffsetsB[lb] +
                           row_rank<FUSED_ROW_SLOTS>(a, a.cntB, a.slotB, a.rowUse, a.headB, a.nextB, lb, k, a.nL)] = k;
        }
    }
}

// ---------------------------------------------------------------- F: minifilaments + links
// BindingDetectionSystem.gridReachable (BindingDetectionSystem.java:161-227) over the
// segment-only cell-ordered endpoints, fused with bindNearest's selection
// (BindingDetectionSystem.java:366-388): the same 27 cells in the same order (nine rows of
// three consecutive x-cells), the same predicate, and the first nearest among the first
// MAX_CAND candidates. A group of W lanes (8 or 16) walks one head (the 32 / W groups of a
// warp walk as many heads side by side; every lane of a group calls it with its group's
// head, `valid` false for a group without one): lane r of the group reads stencil row r's
// range (with 8 lanes, lane 0 also row 8), then the entries are tested W at a time, lane k
// of the group taking entry k0 + k. Passing entries are appended in entry order (ballot,
// and the popcount of the group's lower lanes' passes), so the list is the serial walk's
// list; the nearest of the first MAX_CAND (strict <, the first in list order wins) is the
// serial choice: a chunk's minimum with ties to its lowest lane replaces the running best
// only when strictly smaller. Every group runs the same number of chunks (the longest
// walk's), so every shuffle has the whole warp. Returns the reach count; best and arc are
// the same on every lane of the group.
template <int W>
__device__ int group_reach_bind(const FusedArgs& a, int lane, bool valid, float mx, float my, float mz, float mux,
                                float muy, float muz, float rux, float ruy, float ruz, int* out, float tol,
                                float align, int* bestSeg, float* bestArc) {
    static_assert(W == 8 || W == 16, "a group of 8 or 16 lanes walks one head");
    const float* gp = a.sc.grid.gridParams;
    const int* off = a.segCellOff;
    const int hl = lane & (W - 1), grp = lane / W;
    const int nX = a.nX, nY = a.nY, nZ = a.nZ, nXY = nX * nY;
    const int cx = cell_coord(mx, gp[0], gp[4], nX), cy = cell_coord(my, gp[1], gp[4], nY),
              cz = cell_coord(mz, gp[2], gp[4], nZ);
    const int x0 = max(cx - 1, 0), x1 = min(cx + 1, nX - 1);
    // lane hl reads stencil row hl; with 8 lanes, lane 0 also reads row 8
    int rs = 0, len = 0, rs8 = 0, len8 = 0;
    auto row = [&](int r, int& s, int& l) {
        int zz = cz - 1 + r / 3, yy = cy - 1 + r % 3;
        if (zz >= 0 && zz < nZ && yy >= 0 && yy < nY) {
            int c0 = x0 + yy * nX + zz * nXY;
            s = off[c0];
            l = off[c0 + (x1 - x0) + 1] - s;
        }
    };
    if (valid && hl < 9) row(hl, rs, len);
    if (W == 8 && valid && hl == 0) row(8, rs8, len8);
    int inc = len;
#pragma unroll
    for (int o = 1; o < W; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, inc, o, W);
        if (hl >= o) inc += y;
    }
    const int lanesTotal = __shfl_sync(0xffffffffu, inc, W - 1, W);     // rows 0 .. min(8, W - 1)
    const int total = lanesTotal + (W == 8 ? __shfl_sync(0xffffffffu, len8, 0, W) : 0);
    int totalMax = total;
#pragma unroll
    for (int o = W; o < 32; o <<= 1) totalMax = max(totalMax, __shfl_xor_sync(0xffffffffu, totalMax, o));
    // every lane holds its group's nine (start of row in the sequence, start of row in memory) pairs
    int preR[9], rsR[9];
#pragma unroll
    for (int r = 0; r < 9; r++) {
        if (r < W) {
            preR[r] = __shfl_sync(0xffffffffu, inc - len, r, W);
            rsR[r] = __shfl_sync(0xffffffffu, rs, r, W);
        } else {
            preR[r] = lanesTotal;
            rsR[r] = __shfl_sync(0xffffffffu, rs8, 0, W);
        }
    }
    const unsigned lower = (1u << hl) - 1u;
    int cnt = 0, best = -1;
    float bestD = 1.0e30f, arc = 0.f;
    for (int k0 = 0; k0 < totalMax; k0 += W) {
        const int k = k0 + hl;
        bool pass = false;
        float d = 0.f;
        float4 e1 = make_float4(0.f, 0.f, 0.f, 0.f), e2 = e1;
        if (k < total) {
            int idx = rsR[0] + k;
#pragma unroll
            for (int r = 1; r < 9; r++)
                if (k >= preR[r]) idx = rsR[r] + (k - preR[r]);
            if (SBX_IDX_OK(idx, a.nSeg, CK_REACH_ENTRY)) {
                e1 = a.segE1[idx];
                e2 = a.segE2[idx];
                d = reach_test_dist_sq(mx, my, mz, mux, muy, muz, rux, ruy, ruz, e1.x, e1.y, e1.z, e2.x, e2.y, e2.z,
                                       tol, align);
                pass = d >= 0.f && __float_as_int(e1.w) >= 0;
            }
        }
        const unsigned mask = (__ballot_sync(0xffffffffu, pass) >> (W * grp)) & ((1u << W) - 1u);
        const int pos = cnt + __popc(mask & lower);
        const int sg = __float_as_int(e1.w);
        const bool elig = pass && pos < MAX_CAND;
        if (elig) out[pos] = sg;
        float v = elig ? d : 3.0e38f;
        int who = hl;
#pragma unroll
        for (int o = W / 2; o > 0; o >>= 1) {
            float ov = __shfl_xor_sync(0xffffffffu, v, o);
            int ow = __shfl_xor_sync(0xffffffffu, who, o);
            if (ov < v || (ov == v && ow < who)) { v = ov; who = ow; }
        }
        float myArc = 0.f;
        if (v < bestD && hl == who) myArc = bind_arc(mx, my, mz, e1.x, e1.y, e1.z, e2.x, e2.y, e2.z);
        const int bw = __shfl_sync(0xffffffffu, sg, who, W);
        const float ba = __shfl_sync(0xffffffffu, myArc, who, W);
        if (v < bestD) {
            bestD = v;
            best = bw;
            arc = ba;
        }
        cnt += __popc(mask);
    }
    *bestSeg = best;
    *bestArc = arc;
    return cnt;
}

// BindingDetectionSystem / NucleotideCycleSystem for every head: the
// catch-slip release (NucleotideCycleSystem.java:77-134), the reach walk fused with
// bindNearest's choice (BindingDetectionSystem.java:161-227, :366-388), the nucleotide cycle
// (NucleotideCycleSystem.java:33-69) and the bound head's entry in its segment's motor row.
// Warp w takes heads w, w + N, w + 2N, ... (N warps in the grid) in rounds of 32: lane j
// releases and cycles the round's head j; the four 8-lane groups walk heads j .. j + 3 side
// by side. With 2,368 warps and 6,400 heads every warp walks its heads in one pass (16-lane
// groups needed two passes in 70 % of the warps: 1 us more per step).
constexpr int BIND_W = 8;     // lanes per walked head
__device__ void phase_bind(const FusedArgs& a, int t) {
    const sbx_dense_scene& sc = a.sc;
    const sbx_motor_store& mot = sc.mot;
    const float* kp = mot.kinParams;
    const int lane = threadIdx.x & 31, gw = gtid() >> 5, nw = gthreads() >> 5;
    const int nM = a.nM;
    int listed = 0;
    for (int base = gw; base < nM; base += 32 * nw) {
        const int myM = base + lane * nw;
        const bool mine = myM < nM;
        int bs = 0, cd = 0, sb = 0, sr = 0, cs = 0;
        if (mine) {
            bs = mot.boundSeg[myM]; cd = mot.cooldown[myM]; sb = mot.stats[2 * myM]; sr = mot.stats[2 * myM + 1];
            cs = mot.capStats[myM];
            release_one(myM, bs, cd, sb, sr, cs, mot.forceDotFil[myM], mot.forceMag[myM], kp, t, sc.seed);
        }
        for (int j = 0; j < 32; j += 32 / BIND_W) {
            if (base + j * nw >= nM) break;
            // group q walks head j + q (owned by lane j + q)
            const int jh = j + lane / BIND_W, m = base + jh * nw;
            const bool valid = m < nM;
            const int mm = valid ? m : base;
            float mx = mot.head[mm], my = mot.head[nM + mm], mz = mot.head[2 * nM + mm];
            float mux = mot.uVec[mm], muy = mot.uVec[nM + mm], muz = mot.uVec[2 * nM + mm];
            float rux = mot.rodUVec[mm], ruy = mot.rodUVec[nM + mm], ruz = mot.rodUVec[2 * nM + mm];
            int best;
            float arc;
            int rc = group_reach_bind<BIND_W>(a, lane, valid, mx, my, mz, mux, muy, muz, rux, ruy, ruz,
                                     sc.grid.reachSeg + (int64_t)mm * MAX_CAND, kp[7], kp[8], &best, &arc);
            if ((lane & (BIND_W - 1)) == 0 && valid) {
                sc.grid.reachCount[m] = rc;
                if (rc > MAX_CAND) {
                    atomicOr(a.err, ERR_REACH_OVERFLOW);
                    stat_add(a, ST_REACH_OVER, 1);
                }
            }
            // the owner lanes j .. j + 32 / BIND_W - 1 take their group's choice
            const bool owner = lane >= j && lane < j + 32 / BIND_W;
            const int src = owner ? (lane - j) * BIND_W : 0;
            const int bb = __shfl_sync(0xffffffffu, best, src);
            const float ab = __shfl_sync(0xffffffffu, arc, src);
            if (owner && bs == FREE_BINDABLE && bb >= 0) {
                bs = bb;
                mot.bindArc[myM] = ab;
            }
        }
        if (mine) {
            mot.boundSeg[myM] = bs; mot.cooldown[myM] = cd; mot.stats[2 * myM] = sb; mot.stats[2 * myM + 1] = sr;
            mot.capStats[myM] = cs;
            mot.nucleotideState[myM] = cycle_one(myM, mot.nucleotideState[myM], bs >= 0, mot.forceDotHist + 10 * myM,
                                                 mot.nucParams, t, sc.seed);
            if (bs >= 0 && SBX_IDX_OK(bs, a.nSeg, CK_BOUND_SEG))
                listed += row_insert(a.cntM, a.slotM, FUSED_MOTOR_SLOTS, a.mRowUse, a.headM, a.nextM, bs, myM);
        }
    }
    stat_add(a, ST_MOTOR_LIST, listed);
}

// One minifilament per CTA (its heads' binding and its position-only terms ran in earlier
// phases). Stage 2: each sub-body accumulates its terms in the order of the reference's
// System sequence (joints, coupling, tether; the head's bond after its joint). Stage 3:
// integrate.
__device__ void mini_unit(const FusedArgs& a, MiniSmem& ms, int u, int t) {
    const sbx_dense_scene& sc = a.sc;
    const sbx_motor_store& mot = sc.mot;
    const sbx_rigid_body& mb = mot.body;
    const sbx_minifilament_store& mini = sc.mini;
    const sbx_rigid_body& bb = mini.backbone;
    const sbx_rigid_body& fb = sc.fil.body;
    const int nB = a.nB, nSeg = a.nSeg, nBb = a.nBb;
    const int dpm = a.dpm, mpm = 2 * dpm, spm = 6 * dpm;
    const int m0 = u * mpm, s0 = u * spm, d0 = u * dpm;
    const int tid = threadIdx.x;
    float* sF = ms.sF;
    float* sT = ms.sT;
    LocalAcc acc{sF, sT, s0, spm};

    // ---- stage 2
    if (tid < 32) {
        if (tid < mpm) {
            // CrossBridgeSystem.bondForces, then the head's sums: joint 1, then the bond
            int m = m0 + tid;
            float out[XB_STRIDE];
            int bs = mot.boundSeg[m];
            if (!SBX_IDX_OK_OR_NONE(bs, nSeg, CK_BOUND_SEG)) bs = -1;
            bond_one(m, nB, mb.coord, mb.uVec, mb.yVec, mb.bRotGam, nSeg, fb.coord, fb.uVec, fb.yVec, fb.bRotGam,
                     fb.segLength, bs, mot.bindArc[m], mot.nucleotideState[m], sc.xbParams, out);
            for (int k = 0; k < XB_STRIDE; k++) sc.bondData[m * XB_STRIDE + k] = out[k];
            int hl = 3 * tid + 2;
            double f[3] = {0.0, 0.0, 0.0}, tq[3] = {0.0, 0.0, 0.0};
            motor_joint_apply(term_joint(a, m, 1), 1, true, mot.nucleotideState[m], s0 + hl, nB, mb.uVec,
                              mb.segLength, mot.jointParams, f, tq);
            for (int k = 0; k < 3; k++) {
                float F = (float)(0.0 + f[k]), T = (float)(0.0 + tq[k]);
                sF[k * spm + hl] = F + out[k];
                sT[k * spm + hl] = T + out[3 + k];
            }
        }
    } else {
        int w = tid - 32;
        if (w < 2 * mpm) {
            // rods (role 0) and levers (role 1): joints, then dimer coupling, then the tether
            int ml = w >> 1, role = w & 1;
            int m = m0 + ml, sl = 3 * ml + role, s = s0 + sl;
            int nuc = mot.nucleotideState[m];
            double f[3] = {0.0, 0.0, 0.0}, tq[3] = {0.0, 0.0, 0.0};
            if (role == 0) {
                motor_joint_apply(term_joint(a, m, 0), 0, false, nuc, s, nB, mb.uVec, mb.segLength, mot.jointParams, f,
                                  tq);
            } else {
                motor_joint_apply(term_joint(a, m, 0), 0, true, nuc, s, nB, mb.uVec, mb.segLength, mot.jointParams, f,
                                  tq);
                motor_joint_apply(term_joint(a, m, 1), 1, false, nuc, s, nB, mb.uVec, mb.segLength, mot.jointParams, f,
                                  tq);
            }
            for (int k = 0; k < 3; k++) {
                sF[k * spm + sl] = (float)(0.0 + f[k]);
                sT[k * spm + sl] = (float)(0.0 + tq[k]);
            }
            int dl = ml >> 1, d = d0 + dl;
            bool isA = (ml & 1) == 0;            // motorA = 2d, motorB = 2d + 1
            if (role == 0) {
                couple_apply_rod(acc, s, isA, term_couple(a, d, 0));
                couple_apply_rod(acc, s, isA, term_couple(a, d, 1));
                if (isA) tether_apply(acc, s, term_tether(a, d));
            } else {
                bool bothBound = mot.boundSeg[2 * d] >= 0 && mot.boundSeg[2 * d + 1] >= 0;
                if (sc.dim.parallel[d] != 0 && !bothBound) couple_apply_lever(acc, s, isA, term_lever(a, d));
            }
        } else if (w == 2 * mpm) {
            // the backbone: gather its dimers' reactions, confine, integrate, derive
            mini.bbDimerCount[u] = dpm;
            mini.bbDimerOffsets[u] = d0;
            if (u == nBb - 1) mini.bbDimerOffsets[nBb] = d0 + dpm;
            // MiniFilamentSystem.backboneGather over this backbone's CSR row (its dimers, ascending)
            double f[3] = {0, 0, 0}, tq[3] = {0, 0, 0};
            for (int d = d0; d < d0 + dpm; d++) {
                const float* p = mini.miniData + (int64_t)d * MINI_STRIDE;
                f[0] += p[0]; f[1] += p[1]; f[2] += p[2];
                tq[0] += p[3]; tq[1] += p[4]; tq[2] += p[5];
            }
            float F[3], T[3];
            for (int k = 0; k < 3; k++) { F[k] = (float)(0.0f + f[k]); T[k] = (float)(0.0f + tq[k]); }
            BoxParams bx = box_params(sc.boxParams, t);
            float c[3] = {bb.coord[u], bb.coord[nBb + u], bb.coord[2 * nBb + u]};
            float uu[3] = {bb.uVec[u], bb.uVec[nBb + u], bb.uVec[2 * nBb + u]};
            if (bx.active) confine_one(bx, c, uu, bb.segLength[u], bb.bTransGam[u], F, T);
            integrate_derive_store(bb, u, F, T, mini.bbBodyParams[0]);
        }
    }
    __syncthreads();
    // ---- stage 3: integrate + derive the sub-bodies; force-dot registry
    if (tid < spm) {
        int s = s0 + tid;
        float F[3] = {sF[tid], sF[spm + tid], sF[2 * spm + tid]};
        float T[3] = {sT[tid], sT[spm + tid], sT[2 * spm + tid]};
        integrate_derive_store(mb, s, F, T, mot.bodyParams[0]);
    }
    if (tid < mpm) {
        int m = m0 + tid;
        register_force_dot_one(m, sc.bondData, mot.boundSeg[m] >= 0, mot.forceDotFil, mot.forceMag,
                               mot.forceDotHist, mot.forceDotPlace);
    }
    __syncthreads();
}

__device__ void link_item(const FusedArgs& a, int k) {
    const sbx_dense_scene& sc = a.sc;
    const sbx_crosslinker_store& xl = sc.xl;
    const sbx_rigid_body& fb = sc.fil.body;
    float out[XL_STRIDE];
    int la = xl.linkFilA[k], lb = xl.linkFilB[k];
    if (!SBX_IDX_OK_OR_NONE(la, a.nSeg, CK_LINK_END) || !SBX_IDX_OK_OR_NONE(lb, a.nSeg, CK_LINK_END)) return;
    link_forces_one(k, a.nSeg, fb.coord, fb.uVec, fb.end1, fb.bTransGam, la, lb, xl.loc1[k], xl.loc2[k], a.cntAct,
                    xl.xlParams, out);
    for (int j = 0; j < XL_STRIDE; j++) xl.xlinkData[k * XL_STRIDE + j] = out[j];
    if (xl.torsionParams[1] >= 0.5f)
        link_torsion_one(k, a.nSeg, fb.uVec, la, lb, xl.linkState[k], xl.linkOrientSame[k], xl.torqueMagHist,
                         xl.torqueMagPlace, xl.xlinkData, xl.torsionParams[0]);
}

__device__ void phase_motors_links(const FusedArgs& a, FusedSmem& sm, int t) {
    int linkChunks = a.xlOn ? (a.nL + blockDim.x - 1) / blockDim.x : 0;
    int units = a.nBb + linkChunks;
    for (int w = blockIdx.x; w < units; w += gridDim.x) {
        if (w < a.nBb) {
            mini_unit(a, sm.mini, w, t);
        } else {
            int k = (w - a.nBb) * blockDim.x + threadIdx.x;
            if (k < a.nL) link_item(a, k);
        }
    }
    // on the CTAs without a unit (all CTAs when there are none): the chain joints of the
    // filaments (ChainBendingForceSystem's costly part, from this step's start poses; each
    // joint once, by its lower-slot rod: item i computes rod i's first joint with a
    // higher-slot neighbour, then its second one if it has two) and the filament Brownian
    // forcing (one item per component and rod)
    const sbx_filament_store& fs = a.sc.fil;
    const sbx_rigid_body& fb = fs.body;
    int helpers = (int)gridDim.x - units, h0 = units;
    if (helpers <= 0) { helpers = gridDim.x; h0 = 0; }
    if ((int)blockIdx.x >= h0) {
        ChainJoint* J = reinterpret_cast<ChainJoint*>(a.joints);
        const int n = a.nSeg;
        const int nJ = a.jointShare ? n : 0, total = nJ + 3 * n;
        const int g = ((int)blockIdx.x - h0) * blockDim.x + threadIdx.x, H = helpers * blockDim.x;
        // a thread with a joint item takes no Brownian component when the other threads can
        // share them at three or fewer each (the joint is the longer item; 0.9 us off the warm
        // step at 2e4 rods); otherwise every thread strides over all items
        const bool split = nJ > 0 && H - nJ >= n;
        const int qEnd = split && g < nJ ? g + 1 : total;
        const int qStep = split ? (g < nJ ? 1 : H - nJ) : H;
        for (int q = g; q < qEnd; q += qStep) {
            if (q < nJ) {
                const int i = q;
                int s2 = fs.end2NbrSlot[i], s1 = fs.end1NbrSlot[i];
                const int d2 = fs.end2NbrSide[i], d1 = fs.end1NbrSide[i];
                if (!SBX_IDX_OK_OR_NONE(s2, n, CK_NEIGHBOUR)) s2 = -1;
                if (!SBX_IDX_OK_OR_NONE(s1, n, CK_NEIGHBOUR)) s1 = -1;
                if (s2 > i || s1 > i) {
                    ChainParams cp = chain_params(fs.chainParams);
                    const RodGeom me = load_rod(n, i, fb.coord, fb.uVec, fb.segLength, fb.bTransGam, fb.bRotGam);
                    const int side = s2 > i ? 0 : 1, nb = side == 0 ? s2 : s1;
                    J[2 * i + side] = chain_joint(cp, i, side, nb, side == 0 ? d2 : d1, me,
                                                  load_rod(n, nb, fb.coord, fb.uVec, fb.segLength, fb.bTransGam,
                                                           fb.bRotGam));
                    if (side == 0 && s1 > i)
                        J[2 * i + 1] = chain_joint(cp, i, 1, s1, d1, me,
                                                   load_rod(n, s1, fb.coord, fb.uVec, fb.segLength, fb.bTransGam,
                                                            fb.bRotGam));
                }
            } else {
                const int r = q - nJ, c = r / n, i = r - c * n;
                brownian_component(a, fb, i, c, t, a.filSeed, fs.params[1], a.nzFil);
            }
        }
    }
    // the reference's activeLinkCount array holds this step's counts
    if (a.xlOn)
        for (int s = gtid(); s < a.nSeg; s += gthreads()) a.sc.xl.activeLinkCount[s] = a.cntAct[s];
}

// ---------------------------------------------------------------- K: rods
// TMA bulk copy global -> shared, completion on an mbarrier (no multicast)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* mbar) {
    unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    unsigned b = (unsigned)__cvta_generic_to_shared(mbar);
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 :: "r"(d), "l"(src), "r"(bytes), "r"(b) : "memory");
}

// FP64 row sum of CSR c for local rod l, from the fetched entries (global past the cap);
// the arithmetic of csr_gather_row
__device__ __forceinline__ void gather_staged(const RodSmem& rs, int c, int l, int eBase, int entCap, const int* list,
                                              int nItems, const float* payload, int stride, int poff,
                                              const int* guard, double f[3], double t[3]) {
    f[0] = f[1] = f[2] = 0.0;
    t[0] = t[1] = t[2] = 0.0;
    int k0 = rs.off[c][0];
    for (int k = rs.off[c][l]; k < rs.off[c][l + 1]; k++) {
        int e = eBase + (k - k0);
        const float* p;
        if (e < entCap) {
            if (!rs.entOk[e]) continue;
            p = rs.ent[e];
        } else {
            int li = list[k];
            if (!SBX_IDX_OK(li, nItems, CK_LIST_ENTRY)) continue;
            if (guard && guard[li] < 0) continue;
            p = payload + (int64_t)li * stride + poff;
        }
        f[0] += p[0]; f[1] += p[1]; f[2] += p[2];
        t[0] += p[3]; t[1] += p[4]; t[2] += p[5];
    }
}

// Bounded wait of the calling thread on the bulk-copy barrier's phase `phase` (one second by
// %globaltimer); returns whether the phase completed.
__device__ __forceinline__ bool bulk_wait(uint64_t* mbar, unsigned phase) {
    unsigned mb = (unsigned)__cvta_generic_to_shared(mbar);
    unsigned done = 0, it = 0;
    unsigned long long t0 = 0;
    while (!done) {
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(done) : "r"(mb), "r"(phase) : "memory");
        if (!done && (++it & 15u) == 0) {
            unsigned long long now = gtimer();
            if (t0 == 0) t0 = now;
            else if (now - t0 > WAIT_NS) break;
        }
    }
    return done != 0;
}

// One rod group; returns false when its bulk copies did not complete in time (ERR_TMA set;
// the CTA then leaves the launch).
__device__ bool rod_unit(const FusedArgs& a, RodSmem& rs, int u, int t, uint64_t* mbar, unsigned& phase) {
    const sbx_dense_scene& sc = a.sc;
    const sbx_filament_store& f = sc.fil;
    const sbx_rigid_body& fb = f.body;
    const sbx_crosslinker_store& xl = sc.xl;
    const int n = a.nSeg, G = a.G;
    const int g0 = u * G;
    const int cnt = min(G, n - g0);
    const int tid = threadIdx.x;
    // staged rod geometry: coord xyz, uVec xyz, segLength, bTransGam x y, bRotGam y
    float* sc_[10];
    for (int k = 0; k < 10; k++) sc_[k] = rs.st + k * FUSED_MAX_ROD;
    const float* src[10] = {fb.coord + g0, fb.coord + n + g0, fb.coord + 2 * n + g0, fb.uVec + g0, fb.uVec + n + g0,
                            fb.uVec + 2 * n + g0, fb.segLength + g0, fb.bTransGam + g0, fb.bTransGam + n + g0,
                            fb.bRotGam + n + g0};
    __syncthreads();
    bool tma = a.useTma && (cnt % 4 == 0);
    if (tma) {
        // order earlier generic-proxy accesses of the staging buffer before the async writes
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        unsigned bytes = (unsigned)cnt * 4u;
        if (tid == 0) {
            unsigned mb = (unsigned)__cvta_generic_to_shared(mbar);
            asm volatile("mbarrier.arrive.expect_tx.shared.b64 _, [%0], %1;\n" :: "r"(mb), "r"(bytes * 10u) : "memory");
            for (int k = 0; k < 10; k++) bulk_g2s(sc_[k], src[k], bytes, mbar);
        }
    }
    // the group's link CSR row offsets, while the bulk copies run
    if (a.xlOn) {
        const int* offSrc[2] = {xl.segOffsetsA, xl.segOffsetsB};
        for (int j = tid; j < 2 * (cnt + 1); j += blockDim.x) {
            int c = j / (cnt + 1), r = j - c * (cnt + 1);
            rs.off[c][r] = offSrc[c][g0 + r];
        }
    }
    // the group's motor row lengths
    for (int l = tid; l < cnt; l += blockDim.x) rs.mLen[l] = a.cntM[g0 + l];
    int i = g0 + tid;
    int s2 = -1, n2 = 0, s1 = -1, n1 = 0;
    if (tid < cnt) {
        s2 = f.end2NbrSlot[i]; n2 = f.end2NbrSide[i];
        s1 = f.end1NbrSlot[i]; n1 = f.end1NbrSide[i];
        // a rod group holds whole filaments (both neighbours staged rows of the group) unless
        // the topology has neighbours across groups
        if (a.nbrGlobal) {
            if (!SBX_IDX_OK_OR_NONE(s2, n, CK_NEIGHBOUR)) s2 = -1;
            if (!SBX_IDX_OK_OR_NONE(s1, n, CK_NEIGHBOUR)) s1 = -1;
        } else {
            if (s2 >= 0 && !SBX_IDX_OK(s2 - g0, cnt, CK_NEIGHBOUR)) s2 = -1;
            if (s1 >= 0 && !SBX_IDX_OK(s1 - g0, cnt, CK_NEIGHBOUR)) s1 = -1;
        }
    }
    if (tma) {
        // bounded wait on the transaction barrier, one verdict per CTA: the phase completed
        // if any thread saw it complete. Otherwise the copies may still be landing in the
        // staging buffer, so nothing else is written there: the CTA flags the failure,
        // gives its copies one more bounded wait and leaves the launch (the other CTAs see
        // the flag at their next grid barrier and return too).
        bool ok = __syncthreads_or(bulk_wait(mbar, phase)) != 0;
        if (!ok) {
            if (tid == 0) {
                atomicOr(a.err, ERR_TMA);
                bulk_wait(mbar, phase);
            }
            __syncthreads();
            return false;
        }
        phase ^= 1u;
    } else {
        for (int k = 0; k < 10; k++)
            for (int j = tid; j < cnt; j += blockDim.x) sc_[k][j] = src[k][j];
    }
    __syncthreads();
    ChainParams cp = chain_params(f.chainParams);
    // a rod of the group from the staging; a neighbour outside the group (turnover
    // topologies) from the step's start view (phase A's centres and orientation snapshot:
    // its own group may already have integrated it), the same values
    auto rod = [&](int j) {
        int l = j - g0;
        RodGeom r;
        if (l >= 0 && l < cnt) {
            r.cx = sc_[0][l]; r.cy = sc_[1][l]; r.cz = sc_[2][l];
            r.ux = sc_[3][l]; r.uy = sc_[4][l]; r.uz = sc_[5][l];
            r.len = sc_[6][l];
            r.bTGx = sc_[7][l]; r.bTGy = sc_[8][l]; r.bRGy = sc_[9][l];
        } else {
            const float* c = sc.grid.center;
            const int cp_ = a.cap;
            r.cx = c[j]; r.cy = c[cp_ + j]; r.cz = c[2 * cp_ + j];
            r.ux = a.uSnap[j]; r.uy = a.uSnap[n + j]; r.uz = a.uSnap[2 * n + j];
            r.len = fb.segLength[j];
            r.bTGx = fb.bTransGam[j]; r.bTGy = fb.bTransGam[n + j]; r.bRGy = fb.bRotGam[n + j];
        }
        return r;
    };
    // this rod's two joints (computed in the minifilament phase), loaded ahead of use
    const ChainJoint* Jg = reinterpret_cast<const ChainJoint*>(a.joints);
    ChainJoint j2, j1;
    if (a.jointShare && tid < cnt) {
        if (s2 >= 0) j2 = Jg[s2 > i ? 2 * i : 2 * s2 + (1 - n2)];
        if (s1 >= 0) j1 = Jg[s1 > i ? 2 * i + 1 : 2 * s1 + (1 - n1)];
    }
    // the link CSR payloads of the group's rows (link A, link B), one entry per thread
    const int eA = a.xlOn ? rs.off[0][cnt] - rs.off[0][0] : 0;
    const int eB = a.xlOn ? rs.off[1][cnt] - rs.off[1][0] : 0;
    const int eLim = min(eA + eB, a.entCap);
    if (tid == 0) stat_add(a, ST_ENT_GLOBAL, eA + eB - eLim);
    const int first = tid;
    for (int e = first; e < eLim; e += blockDim.x) {
        const float* p;
        bool ok;
        if (e < eA) {
            int li = xl.segIdxA[rs.off[0][0] + e];
            const bool inb = SBX_IDX_OK(li, a.nL, CK_LIST_ENTRY);
            if (!inb) li = 0;                     // (index-check build) stage zeros for it
            ok = inb && xl.linkState[li] >= 0;
            p = xl.xlinkData + (int64_t)li * XL_STRIDE;
        } else {
            int li = xl.segIdxB[rs.off[1][0] + (e - eA)];
            const bool inb = SBX_IDX_OK(li, a.nL, CK_LIST_ENTRY);
            if (!inb) li = 0;
            ok = inb && xl.linkState[li] >= 0;
            p = xl.xlinkData + (int64_t)li * XL_STRIDE + 6;
        }
        float v[6];
        for (int k = 0; k < 6; k++) v[k] = p[k];
        for (int k = 0; k < 6; k++) rs.ent[e][k] = ok ? v[k] : 0.f;
        rs.entOk[e] = ok;
    }
    // each rod's bound motors in ascending slot order (the motor CSR row order). A row held
    // in its fixed slots (the common case): one thread per (row, slot) reads the slot, then,
    // after the block barrier, puts it at its rank among the row's slots and stages its bond
    // reaction. A longer row: one thread walks the row's slots and overflow list.
    auto shortRow = [&](int nm) { return nm <= a.mRowUse && nm <= a.mIds; };
    const int pairs = cnt * FUSED_MOTOR_SLOTS;
    for (int k = tid; k < pairs; k += blockDim.x) {
        const int l = k / FUSED_MOTOR_SLOTS, j = k - l * FUSED_MOTOR_SLOTS;
        const int nm = rs.mLen[l];
        if (j < nm && shortRow(nm)) {
            const int m = a.slotM[(size_t)(g0 + l) * FUSED_MOTOR_SLOTS + j];
            rs.mRaw[l][j] = SBX_IDX_OK(m, a.nM, CK_MOTOR_SLOT) ? m : 0;
        }
    }
    for (int l = first; l < cnt; l += blockDim.x) {
        int* ids = rs.mIds[l];
        const int r = g0 + l;
        const int nm = rs.mLen[l];
        if (shortRow(nm)) {
            rs.mCnt[l] = nm;
            stat_add(a, ST_MPAY_GLOBAL, nm - min(nm, a.mCap));
            continue;
        }
        int got = 0;
        auto put = [&](int m) {
            if (!SBX_IDX_OK(m, a.nM, CK_MOTOR_SLOT)) m = 0;
            if (got < a.mIds) {
                int q = got;
                while (q > 0 && ids[q - 1] > m) { ids[q] = ids[q - 1]; q--; }
                ids[q] = m;
            }
            got++;
        };
        int sl[FUSED_MOTOR_SLOTS];
#pragma unroll
        for (int j = 0; j < FUSED_MOTOR_SLOTS; j++)
            sl[j] = (j < nm && j < a.mRowUse) ? a.slotM[(size_t)r * FUSED_MOTOR_SLOTS + j] : 0;
#pragma unroll
        for (int j = 0; j < FUSED_MOTOR_SLOTS; j++)
            if (j < nm && j < a.mRowUse) put(sl[j]);
        if (nm > a.mRowUse) {
            int it = 0;
            for (int m = a.headM[r]; m >= 0; m = a.nextM[m]) {
                if (!SBX_IDX_OK(m, a.nM, CK_MOTOR_SLOT)) break;
                put(m);
                if (++it > a.nM) { atomicOr(a.err, ERR_LIST); break; }
            }
        }
        rs.mCnt[l] = got == nm ? nm : 0;
        // reactions staged only for rows whose sorted slots are complete (nm <= mIds)
        int np = nm < a.mCap ? nm : a.mCap;
        if (got != nm || nm > a.mIds) np = 0;
        if (got == nm) stat_add(a, nm > a.mIds ? ST_MIDS_WALK : ST_MPAY_GLOBAL, nm > a.mIds ? 1 : nm - np);
        for (int q = 0; q < np; q++) {
            const float* p = sc.bondData + (int64_t)ids[q] * XB_STRIDE + 6;
            for (int k = 0; k < 6; k++) rs.mPay[l][q][k] = p[k];
        }
    }
    __syncthreads();
    for (int k = tid; k < pairs; k += blockDim.x) {
        const int l = k / FUSED_MOTOR_SLOTS, j = k - l * FUSED_MOTOR_SLOTS;
        const int nm = rs.mLen[l];
        if (j >= nm || !shortRow(nm)) continue;
        const int m = rs.mRaw[l][j];
        int rank = 0;
        for (int q = 0; q < nm; q++) rank += rs.mRaw[l][q] < m;
        rs.mIds[l][rank] = m;
        if (rank < a.mCap) {
            const float* p = sc.bondData + (int64_t)m * XB_STRIDE + 6;
            float v[6];
            for (int c = 0; c < 6; c++) v[c] = p[c];
            for (int c = 0; c < 6; c++) rs.mPay[l][rank][c] = v[c];
        }
    }
    __syncthreads();
    if (tid < cnt) {
        RodGeom me = rod(i);
        double fd[3] = {0, 0, 0}, td[3] = {0, 0, 0};
        if (a.jointShare) {
            if (s2 >= 0) chain_apply(cp, i, 0, s2, n2, me, rod(s2), j2, fd, td);
            if (s1 >= 0) chain_apply(cp, i, 1, s1, n1, me, rod(s1), j1, fd, td);
        } else {
            if (s2 >= 0) chain_side(cp, i, 0, s2, n2, me, rod(s2), fd, td);
            if (s1 >= 0) chain_side(cp, i, 1, s1, n1, me, rod(s1), fd, td);
        }
        float F[3], T[3];
        for (int k = 0; k < 3; k++) { F[k] = (float)(0.0f + fd[k]); T[k] = (float)(0.0f + td[k]); }
        double gf[3], gt[3];
        if (a.xlOn) {
            gather_staged(rs, 0, tid, 0, a.entCap, xl.segIdxA, a.nL, xl.xlinkData, XL_STRIDE, 0, xl.linkState, gf,
                          gt);
            for (int k = 0; k < 3; k++) { F[k] = (float)(F[k] + gf[k]); T[k] = (float)(T[k] + gt[k]); }
            gather_staged(rs, 1, tid, eA, a.entCap, xl.segIdxB, a.nL, xl.xlinkData, XL_STRIDE, 6, xl.linkState, gf,
                          gt);
            for (int k = 0; k < 3; k++) { F[k] = (float)(F[k] + gf[k]); T[k] = (float)(T[k] + gt[k]); }
        }
        // CrossBridgeSystem.segGather: FP64 sums of the bound motors' reactions, ascending slot
        gf[0] = gf[1] = gf[2] = 0.0;
        gt[0] = gt[1] = gt[2] = 0.0;
        int nm = rs.mCnt[tid];
        if (nm <= a.mIds) {
            for (int q = 0; q < nm; q++) {
                const float* p = q < a.mCap ? rs.mPay[tid][q]
                                                : sc.bondData + (int64_t)rs.mIds[tid][q] * XB_STRIDE + 6;
                gf[0] += p[0]; gf[1] += p[1]; gf[2] += p[2];
                gt[0] += p[3]; gt[1] += p[4]; gt[2] += p[5];
            }
        } else {
            // a long row: take its members in ascending order by repeated minimum
            int last = -1;
            for (int q = 0; q < nm; q++) {
                int next = 0x7fffffff, it = 0;
                for (int j = 0; j < FUSED_MOTOR_SLOTS; j++) {
                    if (j >= nm || j >= a.mRowUse) break;
                    int m = a.slotM[(size_t)i * FUSED_MOTOR_SLOTS + j];
                    if (!SBX_IDX_OK(m, a.nM, CK_MOTOR_SLOT)) continue;
                    if (m > last && m < next) next = m;
                }
                for (int m = a.headM[i]; m >= 0 && it <= a.nM; m = a.nextM[m], it++) {
                    if (!SBX_IDX_OK(m, a.nM, CK_MOTOR_SLOT)) break;
                    if (m > last && m < next) next = m;
                }
                if (next == 0x7fffffff) {
                    atomicOr(a.err, ERR_LIST);
                    break;
                }
                const float* p = sc.bondData + (int64_t)next * XB_STRIDE + 6;
                gf[0] += p[0]; gf[1] += p[1]; gf[2] += p[2];
                gt[0] += p[3]; gt[1] += p[4]; gt[2] += p[5];
                last = next;
            }
        }
        for (int k = 0; k < 3; k++) { F[k] = (float)(F[k] + gf[k]); T[k] = (float)(T[k] + gt[k]); }
        BoxParams bx = box_params(sc.boxParams, t);
        float c[3] = {sc_[0][tid], sc_[1][tid], sc_[2][tid]};
        float uu[3] = {sc_[3][tid], sc_[4][tid], sc_[5][tid]};
        if (bx.active) confine_one(bx, c, uu, sc_[6][tid], sc_[7][tid], F, T);
        integrate_derive_store(fb, i, F, T, f.params[0]);
    }
    return true;
}

// The motor CSR of the reference's cpuStep (CrossBridgeSystem.csrHistogram/csrScan/
// csrScatter, CrossBridgeSystem.java:190-217) built by the helper CTAs while the rod units
// gather from the lists: tile sums, scan (segMotorOffsets, segMotorCount = row lengths),
// then each bound motor placed at its rank in its segment's list.
__device__ void motor_csr(const FusedArgs& a, int h, int nH, unsigned long long& hTarget) {
    const sbx_dense_scene& sc = a.sc;
    int wpc = blockDim.x >> 5;
    int hw = h * wpc + (threadIdx.x >> 5), nhw = nH * wpc;
    ScanArr arr[1] = {{a.cntM, a.nSeg, 0}};
    tile_sums(arr, 1, a.mTileSum, hw, nhw);
    if (!counter_sync(a.bar + 1, hTarget, nH, a.err)) return;
    int* out[1] = {sc.segMotorOffsets};
    int* copy[1] = {sc.segMotorCount};
    int clamp[1] = {a.nM};
    tile_scan(arr, 1, a.mTileSum, out, copy, clamp, nullptr, hw, nhw);
    if (!counter_sync(a.bar + 1, hTarget, nH, a.err)) return;
    for (int m = h * blockDim.x + threadIdx.x; m < a.nM; m += nH * blockDim.x) {
        int bs = sc.mot.boundSeg[m];
        if (bs < 0 || !SBX_IDX_OK(bs, a.nSeg, CK_BOUND_SEG)) continue;
        int pos = sc.segMotorOffsets[bs] +
                  row_rank<FUSED_MOTOR_SLOTS>(a, a.cntM, a.slotM, a.mRowUse, a.headM, a.nextM, bs, m, a.nM);
        if (pos < a.nM) sc.segMotorMyo[pos] = m;
    }
}

__device__ bool phase_rods(const FusedArgs& a, FusedSmem& sm, int t, uint64_t* mbar, unsigned& phase,
                           unsigned long long& hTarget) {
    for (int u = blockIdx.x; u < a.nRodUnits; u += gridDim.x)
        if (!rod_unit(a, sm.rod, u, t, mbar, phase)) return false;
    if ((int)blockIdx.x >= a.kHelp0) motor_csr(a, blockIdx.x - a.kHelp0, gridDim.x - a.kHelp0, hTarget);
    // reset the histograms and lists of this step's grid and link CSRs for the next step
    for (int i = gtid(); i < a.C; i += gthreads()) { a.cntCell[i] = 0; a.cntSeg[i] = 0; a.cellHead[i] = -1; }
    for (int i = gtid(); i < a.nSeg; i += gthreads()) {
        a.cntAct[i] = 0; a.cntA[i] = 0; a.cntB[i] = 0; a.headA[i] = -1; a.headB[i] = -1;
    }
    return true;
}

__global__ void __launch_bounds__(FUSED_THREADS, 4) k_dense_fused(const __grid_constant__ FusedArgs a, int t0, int nsteps) {
    __shared__ __align__(8) uint64_t mbar;
    extern __shared__ __align__(16) unsigned char fused_dsm[];
    FusedSmem& sm = *reinterpret_cast<FusedSmem*>(fused_dsm);
    unsigned phase = 0;
    // a run after an unreported failure (barrier, bulk-copy or list fault) does nothing
    // until the plan status has been read, which re-initialises the scratch
    if (vload(a.err) & (ERR_BARRIER | ERR_TMA | ERR_LIST)) return;
    const unsigned nGrid = gridDim.x + (unsigned)a.barrierExtra;
    const unsigned nHelp = gridDim.x - (unsigned)a.kHelp0;
    unsigned long long gTarget = 0, hTarget = 0;
    if (threadIdx.x == 0) {
        gTarget = counter_base(a.bar, nGrid);
        hTarget = counter_base(a.bar + 1, nHelp);
    }
    if (threadIdx.x == 0) {
        unsigned mb = (unsigned)__cvta_generic_to_shared(&mbar);
        asm volatile("mbarrier.init.shared.b64 [%0], 1;\n" :: "r"(mb) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    const sbx_dense_scene& sc = a.sc;
    ScanArr first[4] = {{a.cntCell, a.C, 0}, {a.cntSeg, a.C, a.tilesC}, {a.cntA, a.nSeg, 2 * a.tilesC},
                        {a.cntB, a.nSeg, 2 * a.tilesC + a.tilesS}};
    int narr1 = a.xlOn ? 4 : 2;
    const int nTiles1 = first[narr1 - 1].tile0 + (first[narr1 - 1].n + SCAN_CHUNK - 1) / SCAN_CHUNK;
    int* out1[4] = {sc.grid.gridCellOffsets, a.segCellOff, sc.xl.segOffsetsA, sc.xl.segOffsetsB};
    int* copy1[4] = {sc.grid.cellCount, nullptr, sc.xl.segCountA, sc.xl.segCountB};
    int clamp1[4] = {a.cap, a.nSeg, a.nL, a.nL};
    const int gw = gtid() >> 5, nw = gthreads() >> 5;
    int ph = 0;
    auto stamp = [&](int s_) {
        if (a.phaseTimes && gtid() == 0) {
            long long ns;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(ns));
            a.phaseTimes[(long long)s_ * FUSED_PHASES + ph] = ns;
        }
        ph++;
    };
    for (int s = 0; s < nsteps; s++) {
        int t = t0 + s;
        ph = 0;
        if (gtid() == 0) {
            // MotorStore.setCounts, MiniFilamentStore.setBackboneCounts, counts.set(1, t), xl.setCounts
            int* mc = sc.mot.counts; mc[0] = a.nM; mc[1] = t; mc[2] = sc.seed; mc[3] = a.nSeg;
            int* bc = sc.mini.bbCounts; bc[0] = a.nBb; bc[1] = t; bc[2] = sc.seedBb; bc[3] = a.nBb;
            sc.fil.counts[1] = t;
            if (a.xlOn) { sc.xl.counts[1] = t; sc.xl.counts[2] = sc.seed; }
        }
        // A: body view, bins, histograms and lists, crosslinker unbind
        phase_publish_bin(a, t);
        if (!counter_sync(a.bar, gTarget, nGrid, a.err)) return;
        stamp(s);
        // B, C: scans of the cell, segment-per-cell and link-key histograms (+ motor Brownian)
        tile_sums(first, narr1, a.tileSum, gw, nw);
        if (a.xlOn) link_unbind(a, t, nTiles1);
        myosin_terms(a, nTiles1 + (a.xlOn ? (a.nL + 31) / 32 : 0));
        if (!counter_sync(a.bar, gTarget, nGrid, a.err)) return;
        stamp(s);
        tile_scan(first, narr1, a.tileSum, out1, copy1, clamp1, sc.grid.chunkSum, gw, nw);
        motor_brownian(a, t, nTiles1);
        if (!counter_sync(a.bar, gTarget, nGrid, a.err)) return;
        stamp(s);
        // E: stable placement (grid contents, segment endpoints, link CSR lists)
        phase_place(a);
        if (!counter_sync(a.bar, gTarget, nGrid, a.err)) return;
        stamp(s);
        // B0: binding of every head (8 lanes per head)
        phase_bind(a, t);
        if (!counter_sync(a.bar, gTarget, nGrid, a.err)) return;
        stamp(s);
        // F: minifilament mechanics, crosslinker forces, chain joints, filament Brownian
        phase_motors_links(a, sm, t);
        if (!counter_sync(a.bar, gTarget, nGrid, a.err)) return;
        stamp(s);
        // K: rods; helpers build the motor CSR and reset the step's histograms and lists
        if (!phase_rods(a, sm, t, &mbar, phase, hTarget)) return;
        if (!counter_sync(a.bar, gTarget, nGrid, a.err)) return;
        stamp(s);
    }
    if (gtid() == 0 && a.d_step) *a.d_step = t0 + nsteps;
}

}  // namespace

sbx_status fused_launch(sbx_ctx* ctx, FusedArgs& a, int grid, int t0, int nsteps) {
    void* args[] = {&a, &t0, &nsteps};
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_dense_fused, grid, FUSED_THREADS, args,
                                                sizeof(FusedSmem), ctx->stream);
    ctx->launches++;
    if (e != cudaSuccess) return fail(ctx, SBX_ECUDA, std::string("fused launch: ") + cudaGetErrorString(e));
    return SBX_OK;
}

int fused_max_blocks_per_sm() {
    int nb = 0;
    if (cudaFuncSetAttribute(k_dense_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(FusedSmem)) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_dense_fused, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess)
        return 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_dense_fused, FUSED_THREADS, sizeof(FusedSmem));
    return nb;
}

const void* fused_kernel_ptr() { return (const void*)k_dense_fused; }

SBX_CHECK_EXPORT(fused)
