// sbx_turnover_batch.cu — actin turnover of packed networks (each network's filament slots
// a contiguous range, as the packed dense step lays them out).
//
// The per-slot kernels are sbx_turnover.cu's with the network looked up per slot: the draws
// are keyed by the slot's local index and its network's seed, the rates come from the
// network's row of the parameter tables, and each network has its own actin pool. The
// allocator is segmented without new passes: the free list and the request ranks are the
// global exclusive scans, and a network's slice of each is found at its base index, so
// request r of network k claims freeList[freeOffsets[slotBase_k] + (rank_r - rank at the
// network's first request)] when that local rank is below the network's free count. Every
// network therefore gets the slots, ranks and draws of its run alone, bit for bit; the
// kernels that use no rate, draw or allocation (death, release, splits' requests, drag,
// filament ids, the scans) run unchanged over the packed arrays.
#include <cuda_runtime.h>

#include "../../include/softbox_b200.h"
#include "sbx_internal.cuh"
#include "sbx_physics.cuh"

using namespace sbx;

namespace {

constexpr int FIL_ACTIVE_STATE = 0;

struct TB {
    int nNet;
    const int* slotKey;
    const int* slotBase;
    const int* seeds;
    float* growParams;
    const float* depolyParams;
    const float* depolyRateParams;
    const float* agingParams;
    const float* cofilinParams;
    const float* birthBox;
    const double* onRate;
    sbx_actin_pool* pools;
    const int* birthNet;
    const int* birthBase;
};

TB to_tb(const sbx_turnover_batch* t) {
    return TB{t->nNet, t->slotKey, t->slotBase, t->seeds, t->growParams, t->depolyParams, t->depolyRateParams,
              t->agingParams, t->cofilinParams, t->birthBox, t->onRate, t->pools, t->birthNet, t->birthBase};
}

// request r of a request space (0: the slots themselves, 1: birth requests) -> (network, first request)
__device__ __forceinline__ void req_net(const TB& tb, int space, int r, int& k, int& rb) {
    if (space == 0) {
        k = tb.slotKey[2 * r];
        rb = tb.slotBase[k];
    } else {
        k = tb.birthNet[r];
        rb = tb.birthBase[k];
    }
}

// the claimed global slot of request r, or -1
__device__ __forceinline__ int formed_slot_b(const TB& tb, int space, int r, const int* rankOffsets,
                                             const int* freeList, const int* freeOffsets) {
    int rank = rankOffsets[r];
    if (!(rankOffsets[r + 1] > rank)) return -1;
    int k, rb;
    req_net(tb, space, r, k, rb);
    int local = rank - rankOffsets[rb];
    int f0 = freeOffsets[tb.slotBase[k]], nFree = freeOffsets[tb.slotBase[k + 1]] - f0;
    if (local >= nFree) return -1;
    return freeList[f0 + local];
}

__global__ void k_tb_begin(TB tb, int fires, double bdt) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= tb.nNet) return;
    double P = fires ? tb.onRate[k] * tb.pools[k].conc * bdt : 0.0;
    tb.growParams[3 * k] = (float)P;
}

__global__ void k_tb_grow(TB tb, int C, const int* seedNode, int* monomerCount, float* coord, const float* uVec,
                          int* grewFlag, const int* gc) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= C) return;
    grewFlag[s] = 0;
    int k = tb.slotKey[2 * s], ls = tb.slotKey[2 * s + 1];
    const float* gp = tb.growParams + 3 * k;
    float P = gp[0], halfmono = gp[1];
    int maxMon = (int)gp[2];
    if (gc[3] == 0 || seedNode[s] < 0 || monomerCount[s] >= maxMon) return;
    float u = unit_salted(ls, gc[1], tb.seeds[k], 0x47524F57u);
    if (u >= P) return;
    monomerCount[s] = monomerCount[s] + 1;
    float ux = uVec[s], uy = uVec[C + s], uz = uVec[2 * C + s];
    coord[s] = coord[s] - 0.5f * halfmono * ux;
    coord[C + s] = coord[C + s] - 0.5f * halfmono * uy;
    coord[2 * C + s] = coord[2 * C + s] - 0.5f * halfmono * uz;
    grewFlag[s] = 1;
}

__global__ void k_tb_depoly_proxy(TB tb, int C, const int* filState, int* monomerCount, float* coord,
                                  const float* uVec, const int* e1s, const float* nucFrac, int* returnedMon,
                                  int* deathFlag, const int* dc) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= C) return;
    returnedMon[s] = 0;
    deathFlag[s] = 0;
    if (dc[3] == 0 || filState[s] < 0 || e1s[s] >= 0) return;
    int k = tb.slotKey[2 * s], ls = tb.slotKey[2 * s + 1];
    const float* dp = tb.depolyParams + 3 * k;
    const float* rp = tb.depolyRateParams + 2 * k;
    float halfmono = dp[1];
    int floorM = (int)dp[2];
    int M = monomerCount[s];
    float adp = nucFrac[2 * C + s];
    float P = rp[0] * (1.0f - adp) + rp[1] * adp;
    if (M >= floorM) {
        float u = unit_salted(ls, dc[1], tb.seeds[k], 0x4445504Fu);
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

__global__ void k_tb_age(TB tb, int C, const int* filState, float* nucFrac, const int* ac) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= C || ac[1] == 0 || filState[s] < 0) return;
    const float* ap = tb.agingParams + 2 * tb.slotKey[2 * s];
    float pH = ap[0], pD = ap[1];
    float fATP = nucFrac[s], fADPPi = nucFrac[C + s];
    float nATP = fATP * (1.0f - pH);
    float nADPPi = fADPPi * (1.0f - pD) + fATP * pH;
    float nADP = 1.0f - nATP - nADPPi;
    nucFrac[s] = nATP; nucFrac[C + s] = nADPPi; nucFrac[2 * C + s] = nADP;
}

__global__ void k_tb_cofilin(TB tb, int C, const int* filState, const float* nucFrac, float* cofFrac,
                             const int* monomerCount, int* severDeathFlag, int* severReturnedMon, const int* sc,
                             int dissolve) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= C) return;
    const float* cp = tb.cofilinParams + 2 * tb.slotKey[2 * s];
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

// per network: put (take = 0) or take (1) the network's slice total of a slot scan
__global__ void k_tb_pool(TB tb, const int* offsets, int take) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= tb.nNet) return;
    sbx_actin_pool* pool = tb.pools + k;
    int m = offsets[tb.slotBase[k + 1]] - offsets[tb.slotBase[k]];
    if (take) {
        if (m <= 0) return;
        double c = pool->conc - m * pool->uMPerMonomer;
        pool->conc = c < 0.0 ? 0.0 : c;
        pool->totalTaken += m;
    } else {
        pool->conc = pool->conc + m * pool->uMPerMonomer;
        pool->totalReturned += m;
    }
}

__global__ void k_tb_split_wire(TB tb, int C, const int* rankOffsets, const int* freeList, const int* freeOffsets,
                                int* monomerCount, float* coord, const float* uVec, int* e1s, int* e1d, int* e2s,
                                int* e2d, int* seedNode, const float* sp) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= C) return;
    int Cs = formed_slot_b(tb, 0, r, rankOffsets, freeList, freeOffsets);
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

// 0 cofilin fresh, 1 ATP fresh, 2 split inherit (child <- parent r, slot space only)
__global__ void k_tb_formed_init(TB tb, int space, int K, int C, const int* rankOffsets, const int* freeList,
                                 const int* freeOffsets, float* a, int what) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= K) return;
    int slot = formed_slot_b(tb, space, r, rankOffsets, freeList, freeOffsets);
    if (slot < 0) return;
    if (what == 0) {
        a[slot] = 0.f;
    } else if (what == 1) {
        a[slot] = 1.0f; a[C + slot] = 0.f; a[2 * C + slot] = 0.f;
    } else {
        a[slot] = a[r]; a[C + slot] = a[C + r]; a[2 * C + slot] = a[2 * C + r];
    }
}

__global__ void k_tb_birth_allocate(TB tb, int space, int K, int C, int RC, const float* reqCoord,
                                    const float* reqUVec, const float* reqYVec, const int* rankOffsets,
                                    const int* freeList, const int* freeOffsets, float* coord, float* uVec,
                                    float* yVec, float* bTS, float* bRS, int* filState, const float* bp) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= K) return;
    int slot = formed_slot_b(tb, space, r, rankOffsets, freeList, freeOffsets);
    if (slot < 0) return;
    for (int c = 0; c < 3; c++) {
        coord[c * C + slot] = reqCoord[c * RC + r];
        uVec[c * C + slot] = reqUVec[c * RC + r];
        yVec[c * C + slot] = reqYVec[c * RC + r];
    }
    bTS[slot] = bp[0];
    bRS[slot] = bp[1];
    filState[slot] = FIL_ACTIVE_STATE;
}

__global__ void k_tb_birth_emit(TB tb, int R, int step, int* accept, float* reqCoord, float* reqUVec,
                                float* reqYVec) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    int k = tb.birthNet[r], lr = r - tb.birthBase[k];
    const sbx_actin_pool* pool = tb.pools + k;
    const float* bp = tb.birthBox + 4 * k;
    long long deficit = pool->totalReturned - pool->totalTaken;
    int seedMon = (int)bp[3];
    long long Kb = (deficit > 0 && seedMon > 0) ? deficit / seedMon : 0;
    if (lr >= Kb) { accept[r] = 0; return; }
    accept[r] = 1;
    int seed = tb.seeds[k];
    float ux = unit_salted(lr, step, seed, 0x42495231u), uy = unit_salted(lr, step, seed, 0x42495232u);
    float uz = unit_salted(lr, step, seed, 0x42495233u), ua = unit_salted(lr, step, seed, 0x42495234u);
    reqCoord[r] = (float)((2.0 * ux - 1.0) * bp[0]);
    reqCoord[R + r] = (float)((2.0 * uy - 1.0) * bp[1]);
    reqCoord[2 * R + r] = (float)((2.0 * uz - 1.0) * bp[2]);
    double th = 2.0 * PI_D * ua, c = sbxm::cos(th), sn = sbxm::sin(th);
    reqUVec[r] = (float)c; reqUVec[R + r] = (float)sn; reqUVec[2 * R + r] = 0.f;
    reqYVec[r] = (float)(-sn); reqYVec[R + r] = (float)c; reqYVec[2 * R + r] = 0.f;
}

// initNewborn + tagSeeds for birth requests (tag = the request's local index)
__global__ void k_tb_newborn(TB tb, int R, const int* rankOffsets, const int* freeList, const int* freeOffsets,
                             int* monomerCount, float* segLength, int* seedNode, const float* sp) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    int slot = formed_slot_b(tb, 1, r, rankOffsets, freeList, freeOffsets);
    if (slot < 0) return;
    monomerCount[slot] = (int)sp[0];
    segLength[slot] = sp[1];
    seedNode[slot] = r - tb.birthBase[tb.birthNet[r]];
}

__global__ void k_tb_pool_births(TB tb, const int* rankOffsets, const int* freeOffsets, int seedMon) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= tb.nNet) return;
    int acc = rankOffsets[tb.birthBase[k + 1]] - rankOffsets[tb.birthBase[k]];
    int nFree = freeOffsets[tb.slotBase[k + 1]] - freeOffsets[tb.slotBase[k]];
    int nb = min(acc, nFree);
    if (nb <= 0) return;
    sbx_actin_pool* pool = tb.pools + k;
    int m = nb * seedMon;
    double c = pool->conc - m * pool->uMPerMonomer;
    pool->conc = c < 0.0 ? 0.0 : c;
    pool->totalTaken += m;
}

bool tb_ok(const sbx_turnover_batch* t) {
    return t && t->nNet >= 1 && t->slotKey && t->slotBase && t->seeds && t->growParams && t->depolyParams &&
           t->depolyRateParams && t->agingParams && t->cofilinParams && t->onRate && t->pools;
}

}  // namespace

#define SBX_DONE(name) return check_launch(ctx, name)

extern "C" sbx_status sbx_tb_begin(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t fires, double biochemDeltaT) {
    SBX_REQUIRE(ctx && tb_ok(tb) && (fires == 0 || fires == 1));
    SBX_LAUNCH(ctx, k_tb_begin, blocks(tb->nNet), 256, to_tb(tb), fires, biochemDeltaT);
    SBX_DONE("sbx_tb_begin");
}

extern "C" sbx_status sbx_tb_grow(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t C, const int32_t* seedNode,
                                  int32_t* monomerCount, float* coord, const float* uVec, int32_t* grewFlag,
                                  const int32_t* growCounts) {
    SBX_REQUIRE(ctx && tb_ok(tb) && C >= 0 && (C == 0 || (seedNode && monomerCount && coord && uVec && grewFlag &&
                                                          growCounts)));
    if (C == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_tb_grow, blocks(C), 256, to_tb(tb), C, seedNode, monomerCount, coord, uVec, grewFlag,
               growCounts);
    SBX_DONE("sbx_tb_grow");
}

extern "C" sbx_status sbx_tb_depoly_proxy(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t C,
                                          const int32_t* filState, int32_t* monomerCount, float* coord,
                                          const float* uVec, const int32_t* end1NbrSlot, const float* nucFrac,
                                          int32_t* returnedMon, int32_t* deathFlag, const int32_t* depolyCounts) {
    SBX_REQUIRE(ctx && tb_ok(tb) && C >= 0 && (C == 0 || (filState && monomerCount && coord && uVec && end1NbrSlot &&
                                                          nucFrac && returnedMon && deathFlag && depolyCounts)));
    if (C == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_tb_depoly_proxy, blocks(C), 256, to_tb(tb), C, filState, monomerCount, coord, uVec,
               end1NbrSlot, nucFrac, returnedMon, deathFlag, depolyCounts);
    SBX_DONE("sbx_tb_depoly_proxy");
}

extern "C" sbx_status sbx_tb_age(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t C, const int32_t* filState,
                                 float* nucFrac, const int32_t* agingCounts) {
    SBX_REQUIRE(ctx && tb_ok(tb) && C >= 0 && (C == 0 || (filState && nucFrac && agingCounts)));
    if (C == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_tb_age, blocks(C), 256, to_tb(tb), C, filState, nucFrac, agingCounts);
    SBX_DONE("sbx_tb_age");
}

extern "C" sbx_status sbx_tb_cofilin(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t C, int32_t dissolve,
                                     const int32_t* filState, const float* nucFrac, float* cofFrac,
                                     const int32_t* monomerCount, int32_t* severDeathFlag, int32_t* severReturnedMon,
                                     const int32_t* severCounts) {
    SBX_REQUIRE(ctx && tb_ok(tb) && C >= 0 && (dissolve == 0 || dissolve == 1) &&
                (C == 0 || (filState && cofFrac && severCounts &&
                            (dissolve ? (monomerCount && severDeathFlag && severReturnedMon) : nucFrac != nullptr))));
    if (C == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_tb_cofilin, blocks(C), 256, to_tb(tb), C, filState, nucFrac, cofFrac, monomerCount,
               severDeathFlag, severReturnedMon, severCounts, dissolve);
    SBX_DONE("sbx_tb_cofilin");
}

extern "C" sbx_status sbx_tb_pool(sbx_ctx* ctx, const sbx_turnover_batch* tb, const int32_t* offsets, int32_t take) {
    SBX_REQUIRE(ctx && tb_ok(tb) && offsets && (take == 0 || take == 1));
    SBX_LAUNCH(ctx, k_tb_pool, blocks(tb->nNet), 256, to_tb(tb), offsets, take);
    SBX_DONE("sbx_tb_pool");
}

extern "C" sbx_status sbx_tb_split_wire(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t C,
                                        const int32_t* rankOffsets, const int32_t* freeList,
                                        const int32_t* freeOffsets, int32_t* monomerCount, float* coord,
                                        const float* uVec, int32_t* end1NbrSlot, int32_t* end1NbrSide,
                                        int32_t* end2NbrSlot, int32_t* end2NbrSide, int32_t* seedNode,
                                        const float* splitParams) {
    SBX_REQUIRE(ctx && tb_ok(tb) && C >= 0 && rankOffsets && freeOffsets &&
                (C == 0 || (freeList && monomerCount && coord && uVec && end1NbrSlot && end1NbrSide && end2NbrSlot &&
                            end2NbrSide && seedNode && splitParams)));
    if (C == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_tb_split_wire, blocks(C), 256, to_tb(tb), C, rankOffsets, freeList, freeOffsets, monomerCount,
               coord, uVec, end1NbrSlot, end1NbrSide, end2NbrSlot, end2NbrSide, seedNode, splitParams);
    SBX_DONE("sbx_tb_split_wire");
}

extern "C" sbx_status sbx_tb_formed_init(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t space, int32_t K,
                                         int32_t C, const int32_t* rankOffsets, const int32_t* freeList,
                                         const int32_t* freeOffsets, float* a, int32_t what) {
    SBX_REQUIRE(ctx && tb_ok(tb) && (space == 0 || (space == 1 && tb->birthNet && tb->birthBase)) && K >= 0 &&
                C >= 0 && (what >= 0 && what <= 2) && (what != 2 || space == 0) && rankOffsets && freeOffsets &&
                (K == 0 || (freeList && a)));
    if (K == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_tb_formed_init, blocks(K), 256, to_tb(tb), space, K, C, rankOffsets, freeList, freeOffsets, a,
               what);
    SBX_DONE("sbx_tb_formed_init");
}

extern "C" sbx_status sbx_tb_birth_allocate(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t space, int32_t K,
                                            int32_t C, int32_t reqCap, const float* reqCoord, const float* reqUVec,
                                            const float* reqYVec, const int32_t* rankOffsets, const int32_t* freeList,
                                            const int32_t* freeOffsets, float* coord, float* uVec, float* yVec,
                                            float* brownTransScale, float* brownRotScale, int32_t* filState,
                                            const float* birthParams) {
    SBX_REQUIRE(ctx && tb_ok(tb) && (space == 0 || (space == 1 && tb->birthNet && tb->birthBase)) && K >= 0 &&
                C >= 0 && reqCap >= K && rankOffsets && freeOffsets &&
                (K == 0 || (reqCoord && reqUVec && reqYVec && freeList && coord && uVec && yVec && brownTransScale &&
                            brownRotScale && filState && birthParams)));
    if (K == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_tb_birth_allocate, blocks(K), 256, to_tb(tb), space, K, C, reqCap, reqCoord, reqUVec, reqYVec,
               rankOffsets, freeList, freeOffsets, coord, uVec, yVec, brownTransScale, brownRotScale, filState,
               birthParams);
    SBX_DONE("sbx_tb_birth_allocate");
}

extern "C" sbx_status sbx_tb_birth_emit(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t R, int32_t step,
                                        int32_t* acceptFlag, float* reqCoord, float* reqUVec, float* reqYVec) {
    SBX_REQUIRE(ctx && tb_ok(tb) && tb->birthNet && tb->birthBase && tb->birthBox && R >= 0 &&
                (R == 0 || (acceptFlag && reqCoord && reqUVec && reqYVec)));
    if (R == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_tb_birth_emit, blocks(R), 256, to_tb(tb), R, step, acceptFlag, reqCoord, reqUVec, reqYVec);
    SBX_DONE("sbx_tb_birth_emit");
}

extern "C" sbx_status sbx_tb_newborn(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t R,
                                     const int32_t* rankOffsets, const int32_t* freeList, const int32_t* freeOffsets,
                                     int32_t* monomerCount, float* segLength, int32_t* seedNode,
                                     const float* seedParams) {
    SBX_REQUIRE(ctx && tb_ok(tb) && tb->birthNet && tb->birthBase && R >= 0 && rankOffsets && freeOffsets &&
                (R == 0 || (freeList && monomerCount && segLength && seedNode && seedParams)));
    if (R == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_tb_newborn, blocks(R), 256, to_tb(tb), R, rankOffsets, freeList, freeOffsets, monomerCount,
               segLength, seedNode, seedParams);
    SBX_DONE("sbx_tb_newborn");
}

extern "C" sbx_status sbx_tb_pool_births(sbx_ctx* ctx, const sbx_turnover_batch* tb, const int32_t* rankOffsets,
                                         const int32_t* freeOffsets, int32_t monomersPerBirth) {
    SBX_REQUIRE(ctx && tb_ok(tb) && tb->birthBase && rankOffsets && freeOffsets && monomersPerBirth >= 0);
    SBX_LAUNCH(ctx, k_tb_pool_births, blocks(tb->nNet), 256, to_tb(tb), rankOffsets, freeOffsets, monomersPerBirth);
    SBX_DONE("sbx_tb_pool_births");
}
