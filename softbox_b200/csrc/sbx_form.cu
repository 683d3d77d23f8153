// sbx_form.cu — crosslinker formation and the scan-rank free-list allocator of the C ABI.
//
// CrosslinkerSystem formation (CrosslinkerSystem.java:405-756): candidate segment pairs
// (all-pairs or over a dedicated formation grid, FormationGrid.java), per-candidate
// gates, one-new-link-per-segment admission against start-of-step state, then the
// allocator (:297-345): free list of FREE slots in index order, dense ranks of the
// accepted candidates, rank r claims freeList[r]. Every output is a pure function of
// the inputs: candidate order is lexicographic, the per-segment minimum is an integer
// min, ranks come from prefix sums — so the arrays equal the serial reference bit for bit.
#include <cuda_runtime.h>

#include <climits>
#include <string>

#include "../../include/softbox_b200.h"
#include "sbx_internal.cuh"
#include "sbx_physics.cuh"

using namespace sbx;

namespace {

constexpr int FORM_MAXC = 256;          // CrosslinkerSystem.java:457
constexpr int LINK_ACTIVE_STATE = 0;    // CrosslinkerStore.java:57

// the coarse capsule bound of filFilCandidates / gridFormCount (CrosslinkerSystem.java:414-420)
__device__ __forceinline__ bool form_pair_ok(int nSeg, const float* coord, const float* segLength, const int* filID,
                                             int fi, int j, double cix, double ciy, double ciz, double hi,
                                             double grab) {
    if (filID[j] == fi) return false;
    double dx = cix - coord[j], dy = ciy - coord[nSeg + j], dz = ciz - coord[2 * nSeg + j];
    double cd = sqrt(dx * dx + dy * dy + dz * dz);
    double bound = hi + 0.5 * segLength[j] + grab;
    return !(cd > bound);
}

// ---------------------------------------------------------------- all-pairs candidates
__global__ void k_ff_count(int nSeg, const float* coord, const float* segLength, const int* filID, const float* fp,
                           int* cnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nSeg) return;
    double grab = fp[6];
    double cix = coord[i], ciy = coord[nSeg + i], ciz = coord[2 * nSeg + i];
    double hi = 0.5 * segLength[i];
    int fi = filID[i], c = 0;
    for (int j = i + 1; j < nSeg; j++) c += form_pair_ok(nSeg, coord, segLength, filID, fi, j, cix, ciy, ciz, hi, grab);
    cnt[i] = c;
}

__global__ void k_ff_emit(int nSeg, const float* coord, const float* segLength, const int* filID, const float* fp,
                          const int* base, int reqCap, int* reqFilA, int* reqFilB) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nSeg) return;
    double grab = fp[6];
    int p = base[i];
    if (p >= reqCap) return;
    double cix = coord[i], ciy = coord[nSeg + i], ciz = coord[2 * nSeg + i];
    double hi = 0.5 * segLength[i];
    int fi = filID[i];
    for (int j = i + 1; j < nSeg && p < reqCap; j++) {
        if (!form_pair_ok(nSeg, coord, segLength, filID, fi, j, cix, ciy, ciz, hi, grab)) continue;
        reqFilA[p] = i;
        reqFilB[p] = j;
        p++;
    }
}

// formCounts[0] = min(total, reqCap); the unused tail keyed -1
__global__ void k_form_tail(const int* totalPtr, int reqCap, int* reqFilA, int* reqFilB, int* formCounts) {
    int total = *totalPtr;
    if (total > reqCap) total = reqCap;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k == 0) formCounts[0] = total;
    for (; k < reqCap; k += gridDim.x * blockDim.x)
        if (k >= total) {
            reqFilA[k] = -1;
            reqFilB[k] = -1;
        }
}

// ---------------------------------------------------------------- grid candidates
__device__ __forceinline__ void form_cells(double cix, double ciy, double ciz, const float* gp, const int* gd, int lo[3],
                                           int up[3]) {
    int n[3] = {gd[0], gd[1], gd[2]};
    int c[3] = {cell_coord((float)cix, gp[0], gp[4], n[0]), cell_coord((float)ciy, gp[1], gp[4], n[1]),
                cell_coord((float)ciz, gp[2], gp[4], n[2])};
    for (int k = 0; k < 3; k++) {
        lo[k] = max(c[k] - 1, 0);
        up[k] = min(c[k] + 1, n[k] - 1);
    }
}

// CrosslinkerSystem.gridFormCount (CrosslinkerSystem.java:461-512)
__global__ void k_grid_form_count(int nSeg, const float* coord, const float* segLength, const int* filID,
                                  const float* gp, const int* gd, const int* offsets, const int* contents,
                                  int* candCountSeg, const float* fp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nSeg) return;
    double grab = fp[6];
    double cix = coord[i], ciy = coord[nSeg + i], ciz = coord[2 * nSeg + i];
    double hi = 0.5 * segLength[i];
    int fi = filID[i];
    int lo[3], up[3];
    form_cells(cix, ciy, ciz, gp, gd, lo, up);
    int nX = gd[0], nXY = gd[0] * gd[1];
    int cnt = 0;
    for (int zz = lo[2]; zz <= up[2]; zz++)
        for (int yy = lo[1]; yy <= up[1]; yy++) {
            int c0 = lo[0] + yy * nX + zz * nXY;
            for (int idx = offsets[c0]; idx < offsets[c0 + (up[0] - lo[0]) + 1]; idx++) {
                int j = contents[idx];
                if (j <= i) continue;
                cnt += form_pair_ok(nSeg, coord, segLength, filID, fi, j, cix, ciy, ciz, hi, grab);
            }
        }
    candCountSeg[i] = cnt < FORM_MAXC ? cnt : FORM_MAXC;
}

// CrosslinkerSystem.gridFormEmit (CrosslinkerSystem.java:535-602): partners ascending in
// the segment's owned region; a full region keeps the smallest FORM_MAXC
__global__ void k_grid_form_emit(int nSeg, const float* coord, const float* segLength, const int* filID,
                                 const float* gp, const int* gd, const int* offsets, const int* contents,
                                 const int* candBaseSeg, const int* candCountSeg, int reqCap, int* reqFilA,
                                 int* reqFilB, const float* fp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nSeg) return;
    double grab = fp[6];
    int base = candBaseSeg[i];
    int cap = candCountSeg[i];
    if (base >= reqCap) cap = 0;
    else if (base + cap > reqCap) cap = reqCap - base;
    if (cap <= 0) return;
    double cix = coord[i], ciy = coord[nSeg + i], ciz = coord[2 * nSeg + i];
    double hi = 0.5 * segLength[i];
    int fi = filID[i];
    int lo[3], up[3];
    form_cells(cix, ciy, ciz, gp, gd, lo, up);
    int nX = gd[0], nXY = gd[0] * gd[1];
    int cnt = 0;
    for (int zz = lo[2]; zz <= up[2]; zz++)
        for (int yy = lo[1]; yy <= up[1]; yy++) {
            int c0 = lo[0] + yy * nX + zz * nXY;
            for (int idx = offsets[c0]; idx < offsets[c0 + (up[0] - lo[0]) + 1]; idx++) {
                int j = contents[idx];
                if (j <= i) continue;
                if (!form_pair_ok(nSeg, coord, segLength, filID, fi, j, cix, ciy, ciz, hi, grab)) continue;
                if (cnt < cap) {
                    int p = base + cnt;
                    while (p > base && reqFilB[p - 1] > j) { reqFilB[p] = reqFilB[p - 1]; p--; }
                    reqFilB[p] = j;
                    cnt++;
                } else if (j < reqFilB[base + cap - 1]) {
                    int p = base + cap - 1;
                    while (p > base && reqFilB[p - 1] > j) { reqFilB[p] = reqFilB[p - 1]; p--; }
                    reqFilB[p] = j;
                }
            }
        }
    for (int k = 0; k < cap; k++) reqFilA[base + k] = i;
}

// ---------------------------------------------------------------- gates
// CrosslinkerSystem.formGates (CrosslinkerSystem.java:607-675)
__global__ void k_form_gates(int nSeg, const float* fU, const float* fE1, const float* fE2, const float* segLength,
                             int reqCap, const int* reqFilA, const int* reqFilB, float* reqLoc1, float* reqLoc2,
                             int* reqOrient, int* gatePass, const float* fp, const int* fc) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= reqCap) return;
    int step = fc[1], seed = fc[2], mode = fc[3];
    double maxAngle = fp[0], grabSq = fp[1], pForm = fp[4], jit = fp[5];
    gatePass[c] = 0;
    reqOrient[c] = 0;
    int a = reqFilA[c], b = reqFilB[c];
    if (a < 0 || b < 0) return;
    double uax = fU[a], uay = fU[nSeg + a], uaz = fU[2 * nSeg + a];
    double ubx = fU[b], uby = fU[nSeg + b], ubz = fU[2 * nSeg + b];
    double dot = uax * ubx + uay * uby + uaz * ubz;
    double angT = fast_acos(dot), angTR = fast_acos(-dot);
    bool alignOk;
    if (mode == 1) alignOk = angT <= maxAngle;
    else if (mode == -1) alignOk = angTR <= maxAngle;
    else alignOk = (angT <= maxAngle) || (angTR <= maxAngle);
    if (!alignOk) return;
    reqOrient[c] = dot >= 0.0 ? 1 : 0;
    double e1ax = fE1[a], e1ay = fE1[nSeg + a], e1az = fE1[2 * nSeg + a];
    double e2ax = fE2[a], e2ay = fE2[nSeg + a], e2az = fE2[2 * nSeg + a];
    double e1bx = fE1[b], e1by = fE1[nSeg + b], e1bz = fE1[2 * nSeg + b];
    double e2bx = fE2[b], e2by = fE2[nSeg + b], e2bz = fE2[2 * nSeg + b];
    double r1x = e2ax - e1ax, r1y = e2ay - e1ay, r1z = e2az - e1az;
    double r2x = e2bx - e1bx, r2y = e2by - e1by, r2z = e2bz - e1bz;
    double r3x = e1bx - e1ax, r3y = e1by - e1ay, r3z = e1bz - e1az;
    double r4x = r1y * r2z - r1z * r2y, r4y = r1z * r2x - r1x * r2z, r4z = r1x * r2y - r1y * r2x;
    double smallNum = 1e-20;
    if (r4x < smallNum && r4y < smallNum && r4z < smallNum) return;
    double denom = r4x * r4x + r4y * r4y + r4z * r4z;
    double c32x = r3y * r2z - r3z * r2y, c32y = r3z * r2x - r3x * r2z, c32z = r3x * r2y - r3y * r2x;
    double alpha = (r4x * c32x + r4y * c32y + r4z * c32z) / denom;
    if (alpha < 0.0 || alpha > 1.0) return;
    double c31x = r3y * r1z - r3z * r1y, c31y = r3z * r1x - r3x * r1z, c31z = r3x * r1y - r3y * r1x;
    double beta = (r4x * c31x + r4y * c31y + r4z * c31z) / denom;
    if (beta < 0.0 || beta > 1.0) return;
    double p1x = e1ax + alpha * r1x, p1y = e1ay + alpha * r1y, p1z = e1az + alpha * r1z;
    double p2x = e1bx + beta * r2x, p2y = e1by + beta * r2y, p2z = e1bz + beta * r2z;
    double ddx = p1x - p2x, ddy = p1y - p2y, ddz = p1z - p2z;
    double conDistSq = ddx * ddx + ddy * ddy + ddz * ddz;
    if (conDistSq >= grabSq) return;
    uint32_t base = sbxm::rng_base(c, step, seed);
    double da = sqrt((p1x - e1ax) * (p1x - e1ax) + (p1y - e1ay) * (p1y - e1ay) + (p1z - e1az) * (p1z - e1az));
    double db = sqrt((p2x - e1bx) * (p2x - e1bx) + (p2y - e1by) * (p2y - e1by) + (p2z - e1bz) * (p2z - e1bz));
    float uj1 = sbxm::unit_from_hash(sbxm::wang_hash(base ^ 0x584C4A31u));
    float uj2 = sbxm::unit_from_hash(sbxm::wang_hash(base ^ 0x584C4A32u));
    double loc1 = da + (2.0 * uj1 - 1.0) * jit;
    double loc2 = db + (2.0 * uj2 - 1.0) * jit;
    double lenA = segLength[a], lenB = segLength[b];
    if (loc1 > lenA) loc1 = lenA;
    if (loc1 < 0.0) loc1 = 0.0;
    if (loc2 > lenB) loc2 = lenB;
    if (loc2 < 0.0) loc2 = 0.0;
    reqLoc1[c] = (float)loc1;
    reqLoc2[c] = (float)loc2;
    float up = sbxm::unit_from_hash(sbxm::wang_hash(base ^ 0x584C4650u));
    if (up < pForm) gatePass[c] = 1;
}

// ---------------------------------------------------------------- admission
__global__ void k_fill(int* a, int n, int v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = v;
}

// CrosslinkerSystem.formAdmitReduce (CrosslinkerSystem.java:680-691): an integer minimum,
// whatever the order of the updates
__global__ void k_admit_reduce(int reqCap, const int* reqFilA, const int* reqFilB, const int* gatePass, int* minCand) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= reqCap || gatePass[c] == 0) return;
    atomicMin(&minCand[reqFilA[c]], c);
    atomicMin(&minCand[reqFilB[c]], c);
}

// CrosslinkerSystem.formAdmit (CrosslinkerSystem.java:713-738): the spacing test is an OR
// over the existing ACTIVE links, so it may stop at the first violation
__global__ void k_admit(int reqCap, const int* reqFilA, const int* reqFilB, const float* reqLoc1, const float* reqLoc2,
                        const int* gatePass, const int* minCand, const int* activeLinkCount, int nLinks,
                        const int* linkState, const int* linkFilA, const int* linkFilB, const float* loc1,
                        const float* loc2, int* acceptFlag, const float* fp) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= reqCap) return;
    acceptFlag[c] = 0;
    if (gatePass[c] == 0) return;
    double minSep = fp[0 + 2];
    int maxLinks = (int)fp[3];
    int segA = reqFilA[c], segB = reqFilB[c];
    if (minCand[segA] != c || minCand[segB] != c) return;
    if (activeLinkCount[segA] >= maxLinks || activeLinkCount[segB] >= maxLinks) return;
    double la = reqLoc1[c], lb = reqLoc2[c];
    for (int L = 0; L < nLinks; L++) {
        if (linkState[L] < 0) continue;
        int fa = linkFilA[L], fb = linkFilB[L];
        if (fa == segA && fabs(la - (double)loc1[L]) < minSep) return;
        if (fb == segA && fabs(la - (double)loc2[L]) < minSep) return;
        if (fa == segB && fabs(lb - (double)loc1[L]) < minSep) return;
        if (fb == segB && fabs(lb - (double)loc2[L]) < minSep) return;
    }
    acceptFlag[c] = 1;
}

// ---------------------------------------------------------------- allocator
__global__ void k_free_flags(int C, const int* linkState, int* freeCount) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < C) freeCount[s] = linkState[s] < 0 ? 1 : 0;
}

__global__ void k_free_scatter(int C, const int* linkState, const int* freeOffsets, int* freeList) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < C && linkState[s] < 0) freeList[freeOffsets[s]] = s;
}

// CrosslinkerSystem.allocate (CrosslinkerSystem.java:323-345)
__global__ void k_allocate(int K, const int* reqFilA, const int* reqFilB, const float* reqLoc1, const float* reqLoc2,
                           const int* rankOffsets, const int* freeList, const int* freeOffsets, int C, int* linkFilA,
                           int* linkFilB, float* loc1, float* loc2, int* linkState, float* strainHist,
                           int* strainPlace) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= K) return;
    int nFree = freeOffsets[C];
    int rank = rankOffsets[r];
    if (rankOffsets[r + 1] <= rank || rank >= nFree) return;
    int slot = freeList[rank];
    linkFilA[slot] = reqFilA[r];
    linkFilB[slot] = reqFilB[r];
    loc1[slot] = reqLoc1[r];
    loc2[slot] = reqLoc2[r];
    for (int j = 0; j < STRAIN_WIN; j++) strainHist[slot * STRAIN_WIN + j] = 0.f;
    strainPlace[slot] = 0;
    linkState[slot] = LINK_ACTIVE_STATE;
}

// CrosslinkerSystem.placeOrient (CrosslinkerSystem.java:742-756)
__global__ void k_place_orient(int K, const int* reqOrient, const int* rankOffsets, const int* freeList,
                               const int* freeOffsets, int C, int* linkOrientSame, float* torqueMagHist,
                               int* torqueMagPlace) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= K) return;
    int nFree = freeOffsets[C];
    int rank = rankOffsets[r];
    if (rankOffsets[r + 1] <= rank || rank >= nFree) return;
    int slot = freeList[rank];
    linkOrientSame[slot] = reqOrient[r];
    torqueMagPlace[slot] = 0;
    for (int j = 0; j < TORQUE_WIN; j++) torqueMagHist[slot * TORQUE_WIN + j] = 0.f;
}

size_t chunk_ints(int n) { return (size_t)(n + SCAN_CHUNK - 1) / SCAN_CHUNK + 1; }

}  // namespace

extern "C" sbx_status sbx_csr_scan(sbx_ctx* ctx, int32_t n, int32_t* counts, int32_t* offsets) {
    SBX_REQUIRE(ctx && n >= 0 && offsets && (n == 0 || counts));
    sbx_status st = ensure_scratch(ctx, sizeof(int) * chunk_ints(n));
    if (st) return st;
    return exclusive_scan(ctx, counts, n, offsets, true, (int*)ctx->scratch, "sbx_csr_scan");
}

extern "C" sbx_status sbx_xlink_fil_fil_candidates(sbx_ctx* ctx, int32_t nSeg, const float* coord,
                                                   const float* segLength, const int32_t* filID, int32_t reqCap,
                                                   int32_t* reqFilA, int32_t* reqFilB, const float* formParams,
                                                   int32_t* formCounts) {
    SBX_REQUIRE(ctx && nSeg >= 0 && reqCap > 0 && reqFilA && reqFilB && formParams && formCounts &&
                (nSeg == 0 || (coord && segLength && filID)));
    size_t nc = chunk_ints(nSeg);
    sbx_status st = ensure_scratch(ctx, sizeof(int) * (nc + 2 * (size_t)nSeg + 1));
    if (st) return st;
    int* chunk = (int*)ctx->scratch;
    int* cnt = chunk + nc;
    int* base = cnt + nSeg;
    if (nSeg > 0) SBX_LAUNCH(ctx, k_ff_count, blocks(nSeg, 128), 128, nSeg, coord, segLength, filID, formParams, cnt);
    st = exclusive_scan(ctx, cnt, nSeg, base, false, chunk, "sbx_xlink_fil_fil_candidates");
    if (st) return st;
    if (nSeg > 0)
        SBX_LAUNCH(ctx, k_ff_emit, blocks(nSeg, 128), 128, nSeg, coord, segLength, filID, formParams, base, reqCap,
                   reqFilA, reqFilB);
    SBX_LAUNCH(ctx, k_form_tail, blocks(reqCap), 256, base + nSeg, reqCap, reqFilA, reqFilB, formCounts);
    return check_launch(ctx, "sbx_xlink_fil_fil_candidates");
}

extern "C" sbx_status sbx_xlink_grid_form_count(sbx_ctx* ctx, int32_t nSeg, const float* coord, const float* segLength,
                                                const int32_t* filID, const float* gridParams,
                                                const int32_t* gridDims, const int32_t* offsets,
                                                const int32_t* contents, int32_t* candCountSeg,
                                                const float* formParams) {
    SBX_REQUIRE(ctx && nSeg >= 0 && (nSeg == 0 || (coord && segLength && filID && gridParams && gridDims && offsets &&
                                                   contents && candCountSeg && formParams)));
    if (nSeg == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_grid_form_count, blocks(nSeg, 128), 128, nSeg, coord, segLength, filID, gridParams, gridDims,
               offsets, contents, candCountSeg, formParams);
    return check_launch(ctx, "sbx_xlink_grid_form_count");
}

extern "C" sbx_status sbx_xlink_grid_form_scan(sbx_ctx* ctx, int32_t nSeg, const int32_t* candCountSeg,
                                               int32_t* candBaseSeg, int32_t reqCap, int32_t* reqFilA,
                                               int32_t* reqFilB, int32_t* formCounts) {
    SBX_REQUIRE(ctx && nSeg >= 0 && reqCap > 0 && candBaseSeg && reqFilA && reqFilB && formCounts &&
                (nSeg == 0 || candCountSeg));
    sbx_status st = ensure_scratch(ctx, sizeof(int) * chunk_ints(nSeg));
    if (st) return st;
    st = exclusive_scan(ctx, const_cast<int*>(candCountSeg), nSeg, candBaseSeg, false, (int*)ctx->scratch,
                        "sbx_xlink_grid_form_scan");
    if (st) return st;
    SBX_LAUNCH(ctx, k_form_tail, blocks(reqCap), 256, candBaseSeg + nSeg, reqCap, reqFilA, reqFilB, formCounts);
    return check_launch(ctx, "sbx_xlink_grid_form_scan");
}

extern "C" sbx_status sbx_xlink_grid_form_emit(sbx_ctx* ctx, int32_t nSeg, const float* coord, const float* segLength,
                                               const int32_t* filID, const float* gridParams, const int32_t* gridDims,
                                               const int32_t* offsets, const int32_t* contents,
                                               const int32_t* candBaseSeg, const int32_t* candCountSeg,
                                               int32_t reqCap, int32_t* reqFilA, int32_t* reqFilB,
                                               const float* formParams) {
    SBX_REQUIRE(ctx && nSeg >= 0 && reqCap > 0 && reqFilA && reqFilB &&
                (nSeg == 0 || (coord && segLength && filID && gridParams && gridDims && offsets && contents &&
                               candBaseSeg && candCountSeg && formParams)));
    if (nSeg == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_grid_form_emit, blocks(nSeg, 128), 128, nSeg, coord, segLength, filID, gridParams, gridDims,
               offsets, contents, candBaseSeg, candCountSeg, reqCap, reqFilA, reqFilB, formParams);
    return check_launch(ctx, "sbx_xlink_grid_form_emit");
}

extern "C" sbx_status sbx_xlink_form_gates(sbx_ctx* ctx, int32_t nSeg, const float* uVec, const float* end1,
                                           const float* end2, const float* segLength, int32_t reqCap,
                                           const int32_t* reqFilA, const int32_t* reqFilB, float* reqLoc1,
                                           float* reqLoc2, int32_t* reqOrient, int32_t* gatePass,
                                           const float* formParams, const int32_t* formCounts) {
    SBX_REQUIRE(ctx && nSeg >= 0 && reqCap > 0 && uVec && end1 && end2 && segLength && reqFilA && reqFilB &&
                reqLoc1 && reqLoc2 && reqOrient && gatePass && formParams && formCounts);
    SBX_LAUNCH(ctx, k_form_gates, blocks(reqCap, 128), 128, nSeg, uVec, end1, end2, segLength, reqCap, reqFilA,
               reqFilB, reqLoc1, reqLoc2, reqOrient, gatePass, formParams, formCounts);
    return check_launch(ctx, "sbx_xlink_form_gates");
}

extern "C" sbx_status sbx_xlink_form_admit_reduce(sbx_ctx* ctx, int32_t reqCap, const int32_t* reqFilA,
                                                  const int32_t* reqFilB, const int32_t* gatePass, int32_t nSeg,
                                                  int32_t* minCand) {
    SBX_REQUIRE(ctx && reqCap > 0 && nSeg >= 0 && reqFilA && reqFilB && gatePass && (nSeg == 0 || minCand));
    if (nSeg > 0) SBX_LAUNCH(ctx, k_fill, blocks(nSeg), 256, minCand, nSeg, reqCap);
    SBX_LAUNCH(ctx, k_admit_reduce, blocks(reqCap), 256, reqCap, reqFilA, reqFilB, gatePass, minCand);
    return check_launch(ctx, "sbx_xlink_form_admit_reduce");
}

extern "C" sbx_status sbx_xlink_form_admit(sbx_ctx* ctx, int32_t reqCap, const int32_t* reqFilA,
                                           const int32_t* reqFilB, const float* reqLoc1, const float* reqLoc2,
                                           const int32_t* gatePass, const int32_t* minCand,
                                           const int32_t* activeLinkCount, int32_t nLinks, const int32_t* linkState,
                                           const int32_t* linkFilA, const int32_t* linkFilB, const float* loc1,
                                           const float* loc2, int32_t* acceptFlag, const float* formParams) {
    SBX_REQUIRE(ctx && reqCap > 0 && nLinks >= 0 && reqFilA && reqFilB && reqLoc1 && reqLoc2 && gatePass &&
                minCand && activeLinkCount && acceptFlag && formParams &&
                (nLinks == 0 || (linkState && linkFilA && linkFilB && loc1 && loc2)));
    SBX_LAUNCH(ctx, k_admit, blocks(reqCap, 128), 128, reqCap, reqFilA, reqFilB, reqLoc1, reqLoc2, gatePass, minCand,
               activeLinkCount, nLinks, linkState, linkFilA, linkFilB, loc1, loc2, acceptFlag, formParams);
    return check_launch(ctx, "sbx_xlink_form_admit");
}

extern "C" sbx_status sbx_xlink_free_flags(sbx_ctx* ctx, int32_t C, const int32_t* linkState, int32_t* freeCount) {
    SBX_REQUIRE(ctx && C >= 0 && (C == 0 || (linkState && freeCount)));
    if (C == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_free_flags, blocks(C), 256, C, linkState, freeCount);
    return check_launch(ctx, "sbx_xlink_free_flags");
}

extern "C" sbx_status sbx_xlink_free_scatter(sbx_ctx* ctx, int32_t C, const int32_t* linkState,
                                             const int32_t* freeOffsets, int32_t* freeList) {
    SBX_REQUIRE(ctx && C >= 0 && (C == 0 || (linkState && freeOffsets && freeList)));
    if (C == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_free_scatter, blocks(C), 256, C, linkState, freeOffsets, freeList);
    return check_launch(ctx, "sbx_xlink_free_scatter");
}

extern "C" sbx_status sbx_xlink_allocate(sbx_ctx* ctx, int32_t K, const int32_t* reqFilA, const int32_t* reqFilB,
                                         const float* reqLoc1, const float* reqLoc2, const int32_t* rankOffsets,
                                         const int32_t* freeList, const int32_t* freeOffsets, int32_t C,
                                         int32_t* linkFilA, int32_t* linkFilB, float* loc1, float* loc2,
                                         int32_t* linkState, float* strainHist, int32_t* strainPlace) {
    SBX_REQUIRE(ctx && K >= 0 && C >= 0 && rankOffsets && freeOffsets &&
                (K == 0 || (reqFilA && reqFilB && reqLoc1 && reqLoc2)) &&
                (C == 0 || (freeList && linkFilA && linkFilB && loc1 && loc2 && linkState && strainHist && strainPlace)));
    if (K == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_allocate, blocks(K), 256, K, reqFilA, reqFilB, reqLoc1, reqLoc2, rankOffsets, freeList,
               freeOffsets, C, linkFilA, linkFilB, loc1, loc2, linkState, strainHist, strainPlace);
    return check_launch(ctx, "sbx_xlink_allocate");
}

extern "C" sbx_status sbx_xlink_place_orient(sbx_ctx* ctx, int32_t K, const int32_t* reqOrient,
                                             const int32_t* rankOffsets, const int32_t* freeList,
                                             const int32_t* freeOffsets, int32_t C, int32_t* linkOrientSame,
                                             float* torqueMagHist, int32_t* torqueMagPlace) {
    SBX_REQUIRE(ctx && K >= 0 && C >= 0 && rankOffsets && freeOffsets && (K == 0 || reqOrient) &&
                (C == 0 || (freeList && linkOrientSame && torqueMagHist && torqueMagPlace)));
    if (K == 0) return SBX_OK;
    SBX_LAUNCH(ctx, k_place_orient, blocks(K), 256, K, reqOrient, rankOffsets, freeList, freeOffsets, C,
               linkOrientSame, torqueMagHist, torqueMagPlace);
    return check_launch(ctx, "sbx_xlink_place_orient");
}
