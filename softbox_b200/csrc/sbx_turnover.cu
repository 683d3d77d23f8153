// sbx_turnover.cu — actin turnover entry points of the C ABI: barbed-end growth with the
// split at 2 stdSegLength (GrowthSystem.java:73-229), pointed-end depolymerisation and
// death (DepolySystem.java:70-189), cofilin severing (SeveringSystem.java:37-99), filament
// birth into free slots (FilamentBirthSystem.java:61-87), nucleotide aging
// (AgingSystem.java:40-125) and filament identity by pointer doubling (FilIDSystem.java:38-59).
// `C` is the filament slot capacity. growCounts/depolyCounts carry [1] step, [2] seed,
// [3] fires; severCounts/agingCounts carry [1] fires. Integer parameters travel as floats and
// are read with a C cast, which on the device (cvt.rzi) clamps and maps NaN to 0 as Java's
// (int) does. Every kernel is one thread per slot (or per request) writing its own slot, except the
// split rewire and the death link-break, whose neighbour writes go to distinct slots.
#include <cuda_runtime.h>

#include "../../include/softbox_b200.h"
#include "sbx_internal.cuh"
#include "sbx_physics.cuh"

using namespace sbx;

namespace {

constexpr int FIL_FREE_STATE = -1, FIL_ACTIVE_STATE = 0;   // FilamentStore.java:112-113

// the accepted-rank -> slot mapping of the allocator companions; -1 when not formed
__device__ __forceinline__ int formed_slot(int r, const int* rankOffsets, const int* freeList, int nFree) {
    int rank = rankOffsets[r];
    if (!(rankOffsets[r + 1] > rank) || rank >= nFree) return -1;
    return freeList[rank];
}

// GrowthSystem.grow (:73-104)
__global__ void k_grow(int C, const int* seedNode, int* monomerCount, float* coord, const float* uVec, int* grewFlag,
                       const float* gp, const int* gc) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= C) return;
    int fires = gc[3], step = gc[1], seed = gc[2];
    float P = gp[0], halfmono = gp[1];
    int maxMon = (int)gp[2];
    grewFlag[s] = 0;
    if (fires == 0 || seedNode[s] < 0 || monomerCount[s] >= maxMon) return;
    float u = unit_salted(s, step, seed, 0x47524F57u);
    if (u >= P) return;
    monomerCount[s] = monomerCount[s] + 1;
    float ux = uVec[s], uy = uVec[C + s], uz = uVec[2 * C + s];
    coord[s] = coord[s] - 0.5f * halfmono * ux;
    coord[C + s] = coord[C + s] - 0.5f * halfmono * uy;
    coord[2 * C + s] = coord[2 * C + s] - 0.5f * halfmono * uz;
    grewFlag[s] = 1;
}

// GrowthSystem.markSplits (:113-136)
__global__ void k_mark_splits(int C, const int* seedNode, const int* monomerCount, const float* coord,
                              const float* uVec, const float* yVec, int* acceptFlag, float* reqCoord, float* reqUVec,
                              float* reqYVec, int RC, const float* sp, const int* gc) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= C) return;
    acceptFlag[s] = 0;
    if (gc[3] == 0 || seedNode[s] < 0) return;
    double halfmono = sp[0];
    int splitThresh = (int)sp[1], childMon = (int)sp[2];
    int M = monomerCount[s];
    if (M < splitThresh) return;
    int parentNewMon = M - childMon;
    double Lold = (M + 1) * halfmono, Lpar = (parentNewMon + 1) * halfmono, Lchild = (childMon + 1) * halfmono;
    double ux = uVec[s], uy = uVec[C + s], uz = uVec[2 * C + s];
    double shift = 0.5 * Lold - Lpar - 0.5 * Lchild + halfmono;
    reqCoord[s] = (float)(coord[s] + shift * ux);
    reqCoord[RC + s] = (float)(coord[C + s] + shift * uy);
    reqCoord[2 * RC + s] = (float)(coord[2 * C + s] + shift * uz);
    reqUVec[s] = (float)ux; reqUVec[RC + s] = (float)uy; reqUVec[2 * RC + s] = (float)uz;
    reqYVec[s] = yVec[s]; reqYVec[RC + s] = yVec[C + s]; reqYVec[2 * RC + s] = yVec[2 * C + s];
    acceptFlag[s] = 1;
}

// GrowthSystem.splitWire (:147-190): distinct growing tips own distinct {parent, child,
// outward neighbour} triples
__global__ void k_split_wire(int K, int C, const int* rankOffsets, const int* freeList, const int* freeOffsets,
                             int* monomerCount, float* coord, const float* uVec, int* e1s, int* e1d, int* e2s,
                             int* e2d, int* seedNode, const float* sp) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= K) return;
    int Cs = formed_slot(r, rankOffsets, freeList, freeOffsets[C]);
    if (Cs < 0) return;
    double halfmono = sp[0];
    int childMon = (int)sp[2];
    int Gs = r;
    int M = monomerCount[Gs];
    int parentNewMon = M - childMon;
    int Mold = e1s[Gs], MoldSide = e1d[Gs];
    double Lold = (M + 1) * halfmono, Lpar = (parentNewMon + 1) * halfmono;
    double ux = uVec[Gs], uy = uVec[C + Gs], uz = uVec[2 * C + Gs];
    double shift = 0.5 * Lold - 0.5 * Lpar;
    coord[Gs] = (float)(coord[Gs] + shift * ux);
    coord[C + Gs] = (float)(coord[C + Gs] + shift * uy);
    coord[2 * C + Gs] = (float)(coord[2 * C + Gs] + shift * uz);
    monomerCount[Gs] = parentNewMon;
    monomerCount[Cs] = childMon;
    seedNode[Cs] = -1;
    e1s[Gs] = Cs; e1d[Gs] = 1;
    e2s[Cs] = Gs; e2d[Cs] = 0;
    e1s[Cs] = Mold;
    e1d[Cs] = Mold >= 0 ? MoldSide : -1;
    if (Mold >= 0) {
        if (MoldSide == 0) e1s[Mold] = Cs;
        else e2s[Mold] = Cs;
    }
}

// GrowthSystem.recomputeDrag (:200-228)
__global__ void k_recompute_drag(int C, const int* monomerCount, float* segLength, const int* e1s, const int* e2s,
                                 float* bTG, float* bRG, float* bTD, float* bRD, const float* dp, const int* gc) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C || gc[3] == 0) return;
    double halfmono = dp[0], aeta = dp[1], radius = dp[2], kT = dp[3];
    double aPar = dp[4], aOrth = dp[5], aTurn = dp[6];
    int stdSeg = (int)dp[7], minMon = (int)dp[8];
    int mc = monomerCount[i];
    double length = (mc + 1) * halfmono;
    segLength[i] = (float)length;
    bool atEnd = (e1s[i] < 0) || (e2s[i] < 0);
    double minLength = (atEnd ? stdSeg : minMon) * halfmono;
    double asIf = length < minLength ? minLength : length;
    double LM = 1.0e-6 * asIf, RM = radius * 1.0e-6;
    double logT = sbxm::log(LM / (2.0 * RM));
    double bTGx = (2.0 * PI_D * aeta * LM) / (logT + aPar);
    double bTGy = (4.0 * PI_D * aeta * LM) / (logT + aOrth);
    double bRGx = 4.0 * PI_D * aeta * RM * RM * LM;
    double bRGy = (PI_D * aeta * (LM * LM * LM)) / (3.0 * (logT + aTurn));
    int iy = C + i, iz = 2 * C + i;
    bTG[i] = (float)bTGx; bTG[iy] = (float)bTGy; bTG[iz] = (float)bTGy;
    bRG[i] = (float)bRGx; bRG[iy] = (float)bRGy; bRG[iz] = (float)bRGy;
    bTD[i] = (float)(kT / bTGx); bTD[iy] = (float)(kT / bTGy); bTD[iz] = (float)(kT / bTGy);
    bRD[i] = (float)(kT / bRGx); bRD[iy] = (float)(kT / bRGy); bRD[iz] = (float)(kT / bRGy);
}

// DepolySystem.depoly (:70-101) / depolyProxy (:113-145, rate from the ADP fraction)
__global__ void k_depoly(int C, const int* filState, int* monomerCount, float* coord, const float* uVec,
                         const int* e1s, const float* nucFrac, int* returnedMon, int* deathFlag, const float* dp,
                         const float* rp, const int* dc) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= C) return;
    returnedMon[s] = 0;
    deathFlag[s] = 0;
    if (dc[3] == 0 || filState[s] < 0 || e1s[s] >= 0) return;
    float halfmono = dp[1];
    int floorM = (int)dp[2];
    int M = monomerCount[s];
    float P;
    if (rp) {
        float adp = nucFrac[2 * C + s];
        P = rp[0] * (1.0f - adp) + rp[1] * adp;
    } else {
        P = dp[0];
    }
    if (M >= floorM) {
        float u = unit_salted(s, dc[1], dc[2], 0x4445504Fu);
        if (u >= P) return;
        monomerCount[s] = M - 1;
        float ux = uVec[s], uy = uVec[C + s], uz = uVec[2 * C + s];
        coord[s] = coord[s] + 0.5f * halfmono * ux;
        coord[C + s] = coord[C + s] + 0.5f * halfmono * uy;
        coord[2 * C + s] = coord[2 * C + s] + 0.5f * halfmono * uz;
        returnedMon[s] = 1;
    } else {
        deathFlag[s] = 1;
        returnedMon[s] = M;
    }
}

// DepolySystem.applyDeath (:155-188). A dying slot clears its own links and the back-pointer
// of each neighbour that is not dying itself (a dying neighbour clears its own): the same
// final links as the serial pass, with no slot's fields written by two threads or read while
// another thread writes them.
__global__ void k_apply_death(int C, int* filState, int* monomerCount, int* seedNode, int* e1s, int* e1d, int* e2s,
                              int* e2d, float* bTS, float* bRS, const int* deathFlag) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= C || deathFlag[s] == 0) return;
    filState[s] = FIL_FREE_STATE;
    bTS[s] = 0.f;
    bRS[s] = 0.f;
    monomerCount[s] = 0;
    int n2 = e2s[s], n2side = e2d[s], n1 = e1s[s], n1side = e1d[s];
    if (n2 >= 0) {
        if (deathFlag[n2] == 0) {
            if (n2side == 0) { e1s[n2] = -1; e1d[n2] = -1; }
            else { e2s[n2] = -1; e2d[n2] = -1; }
        }
        e2s[s] = -1; e2d[s] = -1;
    }
    if (n1 >= 0) {
        if (deathFlag[n1] == 0) {
            if (n1side == 0) { e1s[n1] = -1; e1d[n1] = -1; }
            else { e2s[n1] = -1; e2d[n1] = -1; }
        }
        e1s[s] = -1; e1d[s] = -1;
    }
    if (seedNode[s] >= 0) seedNode[s] = -1;
}

// SeveringSystem.cofilinAccumulate (:37-49) / cofilinDissolve (:58-74)
__global__ void k_cofilin(int C, const int* filState, const float* nucFrac, float* cofFrac, const int* monomerCount,
                          int* severDeathFlag, int* severReturnedMon, const float* cp, const int* sc, int dissolve) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= C) return;
    if (dissolve) {
        severDeathFlag[s] = 0;
        severReturnedMon[s] = 0;
        if (sc[1] == 0 || filState[s] < 0) return;
        if (cofFrac[s] > cp[1]) {
            severDeathFlag[s] = 1;
            severReturnedMon[s] = monomerCount[s];
        }
    } else {
        if (sc[1] == 0 || filState[s] < 0) return;
        float fADP = nucFrac[2 * C + s], fCof = cofFrac[s];
        cofFrac[s] = fCof + (fADP - fCof) * cp[0];
    }
}

// per formed request: 0 cofilin fresh, 1 ATP fresh, 2 split inherit (child <- parent r)
__global__ void k_formed_init(int K, int C, const int* rankOffsets, const int* freeList, const int* freeOffsets,
                              float* a, int what) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= K) return;
    int slot = formed_slot(r, rankOffsets, freeList, freeOffsets[C]);
    if (slot < 0) return;
    if (what == 0) {
        a[slot] = 0.f;
    } else if (what == 1) {
        a[slot] = 1.0f; a[C + slot] = 0.f; a[2 * C + slot] = 0.f;
    } else {
        a[slot] = a[r]; a[C + slot] = a[C + r]; a[2 * C + slot] = a[2 * C + r];
    }
}

// FilamentBirthSystem.allocate (:61-87)
__global__ void k_birth_allocate(int K, int C, int RC, const float* reqCoord, const float* reqUVec,
                                 const float* reqYVec, const int* rankOffsets, const int* freeList,
                                 const int* freeOffsets, float* coord, float* uVec, float* yVec, float* bTS, float* bRS,
                                 int* filState, const float* bp) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= K) return;
    int slot = formed_slot(r, rankOffsets, freeList, freeOffsets[C]);
    if (slot < 0) return;
    for (int k = 0; k < 3; k++) {
        coord[k * C + slot] = reqCoord[k * RC + r];
        uVec[k * C + slot] = reqUVec[k * RC + r];
        yVec[k * C + slot] = reqYVec[k * RC + r];
    }
    bTS[slot] = bp[0];
    bRS[slot] = bp[1];
    filState[slot] = FIL_ACTIVE_STATE;
}

// AgingSystem.age (:40-57) and growthAtp (:65-77)
__global__ void k_age(int C, const int* filState, float* nucFrac, const float* ap, const int* ac) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= C || ac[1] == 0 || filState[s] < 0) return;
    float pH = ap[0], pD = ap[1];
    float fATP = nucFrac[s], fADPPi = nucFrac[C + s];
    float nATP = fATP * (1.0f - pH);
    float nADPPi = fADPPi * (1.0f - pD) + fATP * pH;
    float nADP = 1.0f - nATP - nADPPi;
    nucFrac[s] = nATP; nucFrac[C + s] = nADPPi; nucFrac[2 * C + s] = nADP;
}

__global__ void k_growth_atp(int C, const int* grewFlag, const int* monomerCount, float* nucFrac) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= C || grewFlag[s] == 0) return;
    int M = monomerCount[s];
    if (M <= 0) return;
    float w = (float)(M - 1) / (float)M;
    float inv = 1.0f / (float)M;
    nucFrac[s] = nucFrac[s] * w + inv;
    nucFrac[C + s] = nucFrac[C + s] * w;
    nucFrac[2 * C + s] = nucFrac[2 * C + s] * w;
}

// FilIDSystem.init (:38-47) / jump (:51-58)
__global__ void k_filid_init(int n, const int* filState, const int* e2s, int* ptr) {
    int seg = blockIdx.x * blockDim.x + threadIdx.x;
    if (seg >= n) return;
    if (filState[seg] < 0) { ptr[seg] = -seg - 2; return; }
    int nx = e2s[seg];
    ptr[seg] = (nx >= 0 && nx != seg && filState[nx] >= 0) ? nx : seg;
}

__global__ void k_filid_jump(int n, const int* ptrIn, int* ptrOut, const int* filState) {
    int seg = blockIdx.x * blockDim.x + threadIdx.x;
    if (seg >= n) return;
    ptrOut[seg] = filState[seg] < 0 ? ptrIn[seg] : ptrIn[ptrIn[seg]];
}

// links and bound heads on FREE segments let go (the network-turnover rule of this library)
__global__ void k_release_dead(const int* filState, int nLinks, const int* linkFilA, const int* linkFilB,
                               int* linkState, int nMotors, int* boundSeg) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nLinks && linkState[i] >= 0) {
        int a = linkFilA[i], b = linkFilB[i];
        if ((a >= 0 && filState[a] < 0) || (b >= 0 && filState[b] < 0)) linkState[i] = -1;
    }
    if (i < nMotors) {
        int sg = boundSeg[i];
        if (sg >= 0 && filState[sg] < 0) boundSeg[i] = -1;
    }
}

// birth requests that restore the polymer mass: deficit = returned - taken (ledger since the
// pool was made) in whole seeds; request r < K gets a uniform position in the box and a
// uniform in-plane axis. bp: [0..2] box half-widths, [3] monomers per seed
__global__ void k_birth_emit(int reqCap, const sbx_actin_pool* pool, const float* bp, int step, int seed,
                             int* accept, float* reqCoord, float* reqUVec, float* reqYVec) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= reqCap) return;
    long long deficit = pool->totalReturned - pool->totalTaken;
    int seedMon = (int)bp[3];
    long long K = (deficit > 0 && seedMon > 0) ? deficit / seedMon : 0;
    if (r >= K) { accept[r] = 0; return; }
    accept[r] = 1;
    float ux = unit_salted(r, step, seed, 0x42495231u), uy = unit_salted(r, step, seed, 0x42495232u);
    float uz = unit_salted(r, step, seed, 0x42495233u), ua = unit_salted(r, step, seed, 0x42495234u);
    reqCoord[r] = (float)((2.0 * ux - 1.0) * bp[0]);
    reqCoord[reqCap + r] = (float)((2.0 * uy - 1.0) * bp[1]);
    reqCoord[2 * reqCap + r] = (float)((2.0 * uz - 1.0) * bp[2]);
    double th = 2.0 * PI_D * ua, c = sbxm::cos(th), sn = sbxm::sin(th);
    reqUVec[r] = (float)c; reqUVec[reqCap + r] = (float)sn; reqUVec[2 * reqCap + r] = 0.f;
    reqYVec[r] = (float)(-sn); reqYVec[reqCap + r] = (float)c; reqYVec[2 * reqCap + r] = 0.f;
}

// NodeNucleationSystem.initNewborn (NodeNucleationSystem.java:228-244) and tagSeeds (:95-106)
__global__ void k_newborn(int K, int C, const int* rankOffsets, const int* freeList, const int* freeOffsets,
                          int* monomerCount, float* segLength, int* seedNode, const float* sp) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= K) return;
    int slot = formed_slot(r, rankOffsets, freeList, freeOffsets[C]);
    if (slot < 0) return;
    if (monomerCount) { monomerCount[slot] = (int)sp[0]; segLength[slot] = sp[1]; }
    if (seedNode) seedNode[slot] = r;
}

// the births' monomers leave the pool: min(accepted, nFree) seeds (FullSystemDemoHarness.java:689-691)
__global__ void k_pool_births(sbx_actin_pool* pool, const int* rankOffsets, int K, const int* freeOffsets, int C,
                              int seedMon) {
    int nb = min(rankOffsets[K], freeOffsets[C]);
    if (nb <= 0) return;
    int m = nb * seedMon;
    double c = pool->conc - m * pool->uMPerMonomer;
    pool->conc = c < 0.0 ? 0.0 : c;
    pool->totalTaken += m;
}

// ActinPool.put (ActinPool.java:53-56) / take (:42-46) of a scan total, one thread
__global__ void k_pool(sbx_actin_pool* pool, const int* offsets, int n, int take) {
    int m = offsets[n];
    if (take) {
        if (m <= 0) return;                     // GrowthStore.depletePoolForGrows takes only when nGrew > 0
        double c = pool->conc - m * pool->uMPerMonomer;
        pool->conc = c < 0.0 ? 0.0 : c;
        pool->totalTaken += m;
    } else {
        pool->conc = pool->conc + m * pool->uMPerMonomer;
        pool->totalReturned += m;
    }
}

// the per-step counters and the pool-dependent growth probability, one thread
__global__ void k_turnover_begin(int step, int seed, int fires, double onRate, double bdt,
                                 const sbx_actin_pool* pool, float* growParams, int* gc, int* dc, int* ac, int* sc) {
    if (gc) { gc[1] = step; gc[2] = seed; gc[3] = fires; }
    if (dc) { dc[1] = step; dc[2] = seed; dc[3] = fires; }
    if (ac) ac[1] = fires;
    if (sc) sc[1] = fires;
    if (growParams) {
        double P = fires ? onRate * pool->conc * bdt : 0.0;
        growParams[0] = (float)P;
    }
}

}  // namespace

#define SBX_DONE(name) return check_launch(ctx, name)

extern "C" sbx_status sbx_growth_grow(sbx_ctx* ctx, int32_t C, const int32_t* seedNode, int32_t* monomerCount,
                                      float* coord, const float* uVec, int32_t* grewFlag, const float* growParams,
                                      const int32_t* growCounts) {
    SBX_REQUIRE(ctx && C >= 0 && (C == 0 || (seedNode && monomerCount && coord && uVec && grewFlag && growParams &&
                                             growCounts)));
    if (C == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_grow, blocks(C), 256, C, seedNode, monomerCount, coord, uVec, grewFlag, growParams, growCounts);
    SBX_DONE("sbx_growth_grow");
}

extern "C" sbx_status sbx_growth_mark_splits(sbx_ctx* ctx, int32_t C, const int32_t* seedNode,
                                             const int32_t* monomerCount, const float* coord, const float* uVec,
                                             const float* yVec, int32_t* acceptFlag, float* reqCoord, float* reqUVec,
                                             float* reqYVec, int32_t reqCap, const float* splitParams,
                                             const int32_t* growCounts) {
    SBX_REQUIRE(ctx && C >= 0 && reqCap >= C && (C == 0 || (seedNode && monomerCount && coord && uVec && yVec &&
                                                             acceptFlag && reqCoord && reqUVec && reqYVec &&
                                                             splitParams && growCounts)));
    if (C == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_mark_splits, blocks(C), 256, C, seedNode, monomerCount, coord, uVec, yVec, acceptFlag, reqCoord,
               reqUVec, reqYVec, reqCap, splitParams, growCounts);
    SBX_DONE("sbx_growth_mark_splits");
}

extern "C" sbx_status sbx_growth_split_wire(sbx_ctx* ctx, int32_t K, int32_t C, const int32_t* rankOffsets,
                                            const int32_t* freeList, const int32_t* freeOffsets,
                                            int32_t* monomerCount, float* coord, const float* uVec,
                                            int32_t* end1NbrSlot, int32_t* end1NbrSide, int32_t* end2NbrSlot,
                                            int32_t* end2NbrSide, int32_t* seedNode, const float* splitParams) {
    SBX_REQUIRE(ctx && K >= 0 && C >= 0 && K <= C && rankOffsets && freeOffsets &&
                (K == 0 || (freeList && monomerCount && coord && uVec && end1NbrSlot && end1NbrSide && end2NbrSlot &&
                            end2NbrSide && seedNode && splitParams)));
    if (K == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_split_wire, blocks(K), 256, K, C, rankOffsets, freeList, freeOffsets, monomerCount, coord, uVec,
               end1NbrSlot, end1NbrSide, end2NbrSlot, end2NbrSide, seedNode, splitParams);
    SBX_DONE("sbx_growth_split_wire");
}

extern "C" sbx_status sbx_growth_recompute_drag(sbx_ctx* ctx, int32_t C, const int32_t* monomerCount,
                                                float* segLength, const int32_t* end1NbrSlot,
                                                const int32_t* end2NbrSlot, float* bTransGam, float* bRotGam,
                                                float* bTransDiff, float* bRotDiff, const float* dragParams,
                                                const int32_t* growCounts) {
    SBX_REQUIRE(ctx && C >= 0 && (C == 0 || (monomerCount && segLength && end1NbrSlot && end2NbrSlot && bTransGam &&
                                             bRotGam && bTransDiff && bRotDiff && dragParams && growCounts)));
    if (C == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_recompute_drag, blocks(C), 256, C, monomerCount, segLength, end1NbrSlot, end2NbrSlot, bTransGam,
               bRotGam, bTransDiff, bRotDiff, dragParams, growCounts);
    SBX_DONE("sbx_growth_recompute_drag");
}

extern "C" sbx_status sbx_depoly(sbx_ctx* ctx, int32_t C, const int32_t* filState, int32_t* monomerCount,
                                 float* coord, const float* uVec, const int32_t* end1NbrSlot, int32_t* returnedMon,
                                 int32_t* deathFlag, const float* depolyParams, const int32_t* depolyCounts) {
    SBX_REQUIRE(ctx && C >= 0 && (C == 0 || (filState && monomerCount && coord && uVec && end1NbrSlot &&
                                             returnedMon && deathFlag && depolyParams && depolyCounts)));
    if (C == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_depoly, blocks(C), 256, C, filState, monomerCount, coord, uVec, end1NbrSlot, nullptr, returnedMon,
               deathFlag, depolyParams, nullptr, depolyCounts);
    SBX_DONE("sbx_depoly");
}

extern "C" sbx_status sbx_depoly_proxy(sbx_ctx* ctx, int32_t C, const int32_t* filState, int32_t* monomerCount,
                                       float* coord, const float* uVec, const int32_t* end1NbrSlot,
                                       const float* nucFrac, int32_t* returnedMon, int32_t* deathFlag,
                                       const float* depolyParams, const float* depolyRateParams,
                                       const int32_t* depolyCounts) {
    SBX_REQUIRE(ctx && C >= 0 && (C == 0 || (filState && monomerCount && coord && uVec && end1NbrSlot && nucFrac &&
                                             returnedMon && deathFlag && depolyParams && depolyRateParams &&
                                             depolyCounts)));
    if (C == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_depoly, blocks(C), 256, C, filState, monomerCount, coord, uVec, end1NbrSlot, nucFrac, returnedMon,
               deathFlag, depolyParams, depolyRateParams, depolyCounts);
    SBX_DONE("sbx_depoly_proxy");
}

extern "C" sbx_status sbx_depoly_apply_death(sbx_ctx* ctx, int32_t C, int32_t* filState, int32_t* monomerCount,
                                             int32_t* seedNode, int32_t* end1NbrSlot, int32_t* end1NbrSide,
                                             int32_t* end2NbrSlot, int32_t* end2NbrSide, float* brownTransScale,
                                             float* brownRotScale, const int32_t* deathFlag) {
    SBX_REQUIRE(ctx && C >= 0 && (C == 0 || (filState && monomerCount && seedNode && end1NbrSlot && end1NbrSide &&
                                             end2NbrSlot && end2NbrSide && brownTransScale && brownRotScale &&
                                             deathFlag)));
    if (C == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_apply_death, blocks(C), 256, C, filState, monomerCount, seedNode, end1NbrSlot, end1NbrSide,
               end2NbrSlot, end2NbrSide, brownTransScale, brownRotScale, deathFlag);
    SBX_DONE("sbx_depoly_apply_death");
}

extern "C" sbx_status sbx_sever_cofilin_accumulate(sbx_ctx* ctx, int32_t C, const int32_t* filState,
                                                   const float* nucFrac, float* cofFrac, const float* cofilinParams,
                                                   const int32_t* severCounts) {
    SBX_REQUIRE(ctx && C >= 0 && (C == 0 || (filState && nucFrac && cofFrac && cofilinParams && severCounts)));
    if (C == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_cofilin, blocks(C), 256, C, filState, nucFrac, cofFrac, nullptr, nullptr, nullptr,
               cofilinParams, severCounts, 0);
    SBX_DONE("sbx_sever_cofilin_accumulate");
}

extern "C" sbx_status sbx_sever_cofilin_dissolve(sbx_ctx* ctx, int32_t C, const int32_t* filState,
                                                 const int32_t* monomerCount, const float* cofFrac,
                                                 int32_t* severDeathFlag, int32_t* severReturnedMon,
                                                 const float* cofilinParams, const int32_t* severCounts) {
    SBX_REQUIRE(ctx && C >= 0 && (C == 0 || (filState && monomerCount && cofFrac && severDeathFlag &&
                                             severReturnedMon && cofilinParams && severCounts)));
    if (C == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_cofilin, blocks(C), 256, C, filState, nullptr, const_cast<float*>(cofFrac), monomerCount,
               severDeathFlag, severReturnedMon, cofilinParams, severCounts, 1);
    SBX_DONE("sbx_sever_cofilin_dissolve");
}

static sbx_status formed_init(sbx_ctx* ctx, int32_t K, int32_t C, const int32_t* rankOffsets, const int32_t* freeList,
                              const int32_t* freeOffsets, float* a, int what, const char* name) {
    SBX_REQUIRE(ctx && K >= 0 && C >= 0 && rankOffsets && freeOffsets && (K == 0 || (freeList && a)));
    if (K == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_formed_init, blocks(K), 256, K, C, rankOffsets, freeList, freeOffsets, a, what);
    SBX_DONE(name);
}

extern "C" sbx_status sbx_sever_nucleate_fresh_cofilin(sbx_ctx* ctx, int32_t K, int32_t C, const int32_t* rankOffsets,
                                                       const int32_t* freeList, const int32_t* freeOffsets,
                                                       float* cofFrac) {
    return formed_init(ctx, K, C, rankOffsets, freeList, freeOffsets, cofFrac, 0, "sbx_sever_nucleate_fresh_cofilin");
}

extern "C" sbx_status sbx_aging_nucleate_fresh_atp(sbx_ctx* ctx, int32_t K, int32_t C, const int32_t* rankOffsets,
                                                   const int32_t* freeList, const int32_t* freeOffsets,
                                                   float* nucFrac) {
    return formed_init(ctx, K, C, rankOffsets, freeList, freeOffsets, nucFrac, 1, "sbx_aging_nucleate_fresh_atp");
}

extern "C" sbx_status sbx_aging_split_inherit_nuc(sbx_ctx* ctx, int32_t K, int32_t C, const int32_t* rankOffsets,
                                                  const int32_t* freeList, const int32_t* freeOffsets,
                                                  float* nucFrac) {
    return formed_init(ctx, K, C, rankOffsets, freeList, freeOffsets, nucFrac, 2, "sbx_aging_split_inherit_nuc");
}

extern "C" sbx_status sbx_birth_allocate(sbx_ctx* ctx, int32_t K, int32_t C, int32_t reqCap, const float* reqCoord,
                                         const float* reqUVec, const float* reqYVec, const int32_t* rankOffsets,
                                         const int32_t* freeList, const int32_t* freeOffsets, float* coord,
                                         float* uVec, float* yVec, float* brownTransScale, float* brownRotScale,
                                         int32_t* filState, const float* birthParams) {
    SBX_REQUIRE(ctx && K >= 0 && C >= 0 && reqCap >= K && rankOffsets && freeOffsets &&
                (K == 0 || (reqCoord && reqUVec && reqYVec && freeList && coord && uVec && yVec && brownTransScale &&
                            brownRotScale && filState && birthParams)));
    if (K == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_birth_allocate, blocks(K), 256, K, C, reqCap, reqCoord, reqUVec, reqYVec, rankOffsets, freeList,
               freeOffsets, coord, uVec, yVec, brownTransScale, brownRotScale, filState, birthParams);
    SBX_DONE("sbx_birth_allocate");
}

extern "C" sbx_status sbx_aging_age(sbx_ctx* ctx, int32_t C, const int32_t* filState, float* nucFrac,
                                    const float* agingParams, const int32_t* agingCounts) {
    SBX_REQUIRE(ctx && C >= 0 && (C == 0 || (filState && nucFrac && agingParams && agingCounts)));
    if (C == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_age, blocks(C), 256, C, filState, nucFrac, agingParams, agingCounts);
    SBX_DONE("sbx_aging_age");
}

extern "C" sbx_status sbx_aging_growth_atp(sbx_ctx* ctx, int32_t C, const int32_t* grewFlag,
                                           const int32_t* monomerCount, float* nucFrac) {
    SBX_REQUIRE(ctx && C >= 0 && (C == 0 || (grewFlag && monomerCount && nucFrac)));
    if (C == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_growth_atp, blocks(C), 256, C, grewFlag, monomerCount, nucFrac);
    SBX_DONE("sbx_aging_growth_atp");
}

extern "C" sbx_status sbx_filid_init(sbx_ctx* ctx, int32_t n, const int32_t* filState, const int32_t* end2NbrSlot,
                                     int32_t* ptr) {
    SBX_REQUIRE(ctx && n >= 0 && (n == 0 || (filState && end2NbrSlot && ptr)));
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_filid_init, blocks(n), 256, n, filState, end2NbrSlot, ptr);
    SBX_DONE("sbx_filid_init");
}

extern "C" sbx_status sbx_filid_jump(sbx_ctx* ctx, int32_t n, const int32_t* ptrIn, int32_t* ptrOut,
                                     const int32_t* filState) {
    SBX_REQUIRE(ctx && n >= 0 && ptrIn != ptrOut && (n == 0 || (ptrIn && ptrOut && filState)));
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_filid_jump, blocks(n), 256, n, ptrIn, ptrOut, filState);
    SBX_DONE("sbx_filid_jump");
}

extern "C" sbx_status sbx_actin_pool_put_total(sbx_ctx* ctx, sbx_actin_pool* pool, const int32_t* offsets, int32_t n) {
    SBX_REQUIRE(ctx && pool && offsets && n >= 0);
    SBX_LAUNCH(ctx, k_pool, 1, 1, pool, offsets, n, 0);
    SBX_DONE("sbx_actin_pool_put_total");
}

extern "C" sbx_status sbx_actin_pool_take_total(sbx_ctx* ctx, sbx_actin_pool* pool, const int32_t* offsets,
                                                int32_t n) {
    SBX_REQUIRE(ctx && pool && offsets && n >= 0);
    SBX_LAUNCH(ctx, k_pool, 1, 1, pool, offsets, n, 1);
    SBX_DONE("sbx_actin_pool_take_total");
}

extern "C" sbx_status sbx_turnover_begin(sbx_ctx* ctx, int32_t step, int32_t seed, int32_t fires, double onRate,
                                         double biochemDeltaT, const sbx_actin_pool* pool, float* growParams,
                                         int32_t* growCounts, int32_t* depolyCounts, int32_t* agingCounts,
                                         int32_t* severCounts) {
    SBX_REQUIRE(ctx && (fires == 0 || fires == 1) && (growParams == nullptr || pool != nullptr));
    SBX_LAUNCH(ctx, k_turnover_begin, 1, 1, step, seed, fires, onRate, biochemDeltaT, pool, growParams, growCounts,
               depolyCounts, agingCounts, severCounts);
    SBX_DONE("sbx_turnover_begin");
}

extern "C" sbx_status sbx_turnover_release_dead(sbx_ctx* ctx, const int32_t* filState, int32_t nLinks,
                                                const int32_t* linkFilA, const int32_t* linkFilB, int32_t* linkState,
                                                int32_t nMotors, int32_t* boundSeg) {
    SBX_REQUIRE(ctx && filState && nLinks >= 0 && nMotors >= 0 && (nLinks == 0 || (linkFilA && linkFilB && linkState)) &&
                (nMotors == 0 || boundSeg));
    int n = nLinks > nMotors ? nLinks : nMotors;
    if (n == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_release_dead, blocks(n), 256, filState, nLinks, linkFilA, linkFilB, linkState, nMotors, boundSeg);
    SBX_DONE("sbx_turnover_release_dead");
}

extern "C" sbx_status sbx_birth_emit_constant_actin(sbx_ctx* ctx, int32_t reqCap, const sbx_actin_pool* pool,
                                                    const float* birthBox, int32_t step, int32_t seed,
                                                    int32_t* acceptFlag, float* reqCoord, float* reqUVec,
                                                    float* reqYVec) {
    SBX_REQUIRE(ctx && reqCap >= 0 && (reqCap == 0 || (pool && birthBox && acceptFlag && reqCoord && reqUVec && reqYVec)));
    if (reqCap == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_birth_emit, blocks(reqCap), 256, reqCap, pool, birthBox, step, seed, acceptFlag, reqCoord,
               reqUVec, reqYVec);
    SBX_DONE("sbx_birth_emit_constant_actin");
}

extern "C" sbx_status sbx_birth_init_newborn(sbx_ctx* ctx, int32_t K, int32_t C, const int32_t* rankOffsets,
                                             const int32_t* freeList, const int32_t* freeOffsets,
                                             int32_t* monomerCount, float* segLength, const float* seedParams) {
    SBX_REQUIRE(ctx && K >= 0 && C >= 0 && rankOffsets && freeOffsets &&
                (K == 0 || (freeList && monomerCount && segLength && seedParams)));
    if (K == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_newborn, blocks(K), 256, K, C, rankOffsets, freeList, freeOffsets, monomerCount, segLength,
               nullptr, seedParams);
    SBX_DONE("sbx_birth_init_newborn");
}

extern "C" sbx_status sbx_birth_tag_seeds(sbx_ctx* ctx, int32_t K, int32_t C, const int32_t* rankOffsets,
                                          const int32_t* freeList, const int32_t* freeOffsets, int32_t* seedNode) {
    SBX_REQUIRE(ctx && K >= 0 && C >= 0 && rankOffsets && freeOffsets && (K == 0 || (freeList && seedNode)));
    if (K == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_newborn, blocks(K), 256, K, C, rankOffsets, freeList, freeOffsets, nullptr, nullptr, seedNode,
               nullptr);
    SBX_DONE("sbx_birth_tag_seeds");
}

extern "C" sbx_status sbx_actin_pool_take_births(sbx_ctx* ctx, sbx_actin_pool* pool, const int32_t* rankOffsets,
                                                 int32_t K, const int32_t* freeOffsets, int32_t C,
                                                 int32_t monomersPerBirth) {
    SBX_REQUIRE(ctx && pool && rankOffsets && freeOffsets && K >= 0 && C >= 0 && monomersPerBirth >= 0);
    SBX_LAUNCH(ctx, k_pool_births, 1, 1, pool, rankOffsets, K, freeOffsets, C, monomersPerBirth);
    SBX_DONE("sbx_actin_pool_take_births");
}
