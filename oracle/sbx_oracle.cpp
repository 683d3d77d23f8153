// sbx_oracle.cpp — CPU ORACLE (test infrastructure, not the product).
//
// A serial, bit-faithful C++ restatement of the reference's per-step rigid-rod
// mechanics (notaboxllc/SoftBox, package softbox/). Only tests/, the smoke check
// and bench.py's CPU-baseline leg may load this library; nothing in the product
// path links or calls it.
//
// Every function follows one Java static method, line for line, with Java's
// arithmetic rules restated for C++:
//   * float/double expressions evaluate left to right with no FMA contraction
//     (built with -ffp-contract=off, SSE2, no fast-math);
//   * Java int wraparound -> uint32_t arithmetic, >>> -> logical shift;
//   * (int) of a float/double truncates toward zero, NaN -> 0, saturating;
//   * (float)Math.sqrt((double)f) == correctly rounded sqrtf;
//   * Math.log/sin/cos/exp: libm by default (the reference's platform math), or,
//     when built with -DSBX_ORACLE_DEVMATH, the portable double-precision
//     functions of softbox_b200/csrc/sbx_math.h that the CUDA kernels use, so
//     that GPU-vs-oracle comparisons are bit-exact.
// Loops marked PAR are per-slot independent in the reference (each iteration
// writes only its own slot) and may run under OpenMP without changing results.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../softbox_b200/csrc/sbx_math.h"

#ifdef SBX_ORACLE_DEVMATH
#define JLOG(x) sbxm::log(x)
#define JEXP(x) sbxm::exp(x)
#define JSIN(x) sbxm::sin(x)
#define JCOS(x) sbxm::cos(x)
#else
#define JLOG(x) std::log(x)
#define JEXP(x) std::exp(x)
#define JSIN(x) std::sin(x)
#define JCOS(x) std::cos(x)
#endif

#define PAR _Pragma("omp parallel for schedule(static)")
#define EXPORT extern "C"

typedef int32_t i32;

namespace {

// Constants.java:25-67
const double KT = 1.380662e-23 * 298.15;
const double PI_D = 3.141592653589793;
const double ACTIN_MONO_RADIUS = 0.0054 / 2.0;
const double ACTIN_RADIUS = 0.007 / 2.0;
const int STD_SEG_LENGTH = 32;
const double A_PARALLEL = -0.20, A_ORTHOG = 0.84, A_TURNING = -0.662;

// MotorStore.java:45-46, MiniFilamentStore.java:34
const double ROD_LEN = 0.080, LEVER_LEN = 0.008, HEAD_LEN = 0.020;
const double ROD_R = 0.003, LEVER_R = 0.002, HEAD_R = 0.010;
const double BACKBONE_R = 0.005;

const int STORE_FILAMENT = 0, STORE_MOTOR = 1, STORE_NONE = -1;
const int MAX_CAND = 256;          // SpatialGrid.java:48
const int GRID_SCAN_CHUNK = 512;   // SpatialGrid.java:46
const int NUC_NONE = 0, NUC_ATP = 1, NUC_ADPPI = 2, NUC_ADP = 3;   // MotorStore.java:117
const int FREE_BINDABLE = -1, FREE_COOLDOWN = -2;                   // MotorStore.java:111-112
const int XB_STRIDE = 13;          // CrossBridgeSystem.java:36
const int XL_STRIDE = 12;          // CrosslinkerStore.java:33
const int STRAIN_WIN = 10, TORQUE_WIN = 5;   // CrosslinkerStore.java:64,118
const int MINI_STRIDE = 6;         // MiniFilamentStore.java:51
const int LINK_FREE = -1, LINK_ACTIVE = 0;   // CrosslinkerStore.java:58-59

// Java (int) cast of a float / double
inline i32 jf2i(float f) {
    if (f != f) return 0;
    if (f >= 2147483648.0f) return INT32_MAX;
    if (f <= -2147483648.0f) return INT32_MIN;
    return (i32)f;
}
inline i32 jd2i(double d) {
    if (d != d) return 0;
    if (d >= 2147483648.0) return INT32_MAX;
    if (d <= -2147483649.0) return INT32_MIN;
    return (i32)d;
}
inline float jsqrtf(float x) { return (float)std::sqrt((double)x); }

// ChainBendingForceSystem.java:48-72 (identical copies in CrossBridgeSystem.java:38-55,
// MotorJointSystem.java:37-57, DimerCouplingSystem.java:36-56, MiniFilamentSystem.java:36-56,
// CrosslinkerSystem.java:382-399)
double accurate_acos(double x) {
    if (x > 1.0) x = 1.0;
    if (x < -1.0) x = -1.0;
    double y;
    if (x > 0.95) {
        double t = 1.0 - x;
        if (t < 0.0) t = 0.0;
        y = std::sqrt(2.0 * t);
    } else if (x < -0.95) {
        double t = 1.0 + x;
        if (t < 0.0) t = 0.0;
        y = 3.141592653589793 - std::sqrt(2.0 * t);
    } else {
        double ax = (x < 0.0) ? -x : x;
        double p = (-0.0187293 * ax + 0.0742610) * ax - 0.2121144;
        p = (p * ax + 1.5707963);
        p = p * std::sqrt(1.0 - ax);
        y = (x < 0.0) ? (3.141592653589793 - p) : p;
    }
    double s = JSIN(y);
    if (s > 1.0e-12 || s < -1.0e-12) { y = y + (JCOS(y) - x) / s; }
    s = JSIN(y);
    if (s > 1.0e-12 || s < -1.0e-12) { y = y + (JCOS(y) - x) / s; }
    return y;
}

// ChainBendingForceSystem.java:76-84
double accurate_asin(double s) {
    double s2 = s * s;
    double y = s * (1.0 + s2 * (0.16666666666666666 + s2 * (0.075 + s2 * 0.044642857142857)));
    double cy = JCOS(y);
    if (cy > 1.0e-12) y = y + (s - JSIN(y)) / cy;
    cy = JCOS(y);
    if (cy > 1.0e-12) y = y + (s - JSIN(y)) / cy;
    return y;
}

// ChainBendingForceSystem.java:95-103
double angle_from_sin_cos(double sin2, double cos) {
    double s = std::sqrt(sin2);
    double ac = (cos < 0.0) ? -cos : cos;
    if (s <= ac) {
        double base = accurate_asin(s);
        return (cos >= 0.0) ? base : (PI_D - base);
    }
    return accurate_acos(cos);
}

// CrosslinkerSystem.java:372-376
double fast_acos(double dot) {
    if (dot > 0.95) { double t = 1.0 - dot; if (t < 0) t = 0; return std::sqrt(2.0 * t); }
    if (dot < -0.95) { double t = 1.0 + dot; if (t < 0) t = 0; return PI_D - std::sqrt(2.0 * t); }
    return accurate_acos(dot);
}

// MotorJointSystem.java:61-70 (== DimerCouplingSystem.java:61-70)
double move_c(double ux, double uy, double uz, double lx, double ly, double lz,
              double bTGx, double bTGy, double bRGy, double lenUm) {
    double cosB = ux * lx + uy * ly + uz * lz;
    if (cosB > 1.0) cosB = 1.0;
    if (cosB < -1.0) cosB = -1.0;
    double cosB2 = cosB * cosB;
    double cosA2 = 1.0 - cosB2;
    double lSq = 1.0e-12 * lenUm * lenUm;
    return cosB2 / bTGx + cosA2 / bTGy + lSq * cosA2 / (4.0 * bRGy);
}

// ContainmentSystem.java:130-136 (== MechanicsFusion.java:341-347)
double wall_push(double d, double halfDim) {
    double s = (d > 0.0) ? 1.0 : ((d < 0.0) ? -1.0 : 0.0);
    double push = s * halfDim - d;
    double ps = (push > 0.0) ? 1.0 : ((push < 0.0) ? -1.0 : 0.0);
    if (ps == s) return 0.0;
    return push;
}

// Box-Muller from six uniforms: BrownianForceSystem.java:78-92
inline void box_muller6(float u1, float u2, float u3, float u4, float u5, float u6, float g[6]) {
    const float TWO_PI_F = 2.0f * 3.14159265f;
    float r1 = jsqrtf(-2.0f * (float)JLOG((double)u1));
    float th1 = TWO_PI_F * u2;
    g[0] = r1 * (float)JCOS((double)th1);
    g[3] = r1 * (float)JSIN((double)th1);
    float r2 = jsqrtf(-2.0f * (float)JLOG((double)u3));
    float th2 = TWO_PI_F * u4;
    g[1] = r2 * (float)JCOS((double)th2);
    g[4] = r2 * (float)JSIN((double)th2);
    float r3 = jsqrtf(-2.0f * (float)JLOG((double)u5));
    float th3 = TWO_PI_F * u6;
    g[2] = r3 * (float)JCOS((double)th3);
    g[5] = r3 * (float)JSIN((double)th3);
}

// Wang-hash keyed draws of BrownianForceSystem.java:63-92 -> g = {gfx,gfy,gfz,gtx,gty,gtz}
inline void gauss6_wang(i32 i, i32 step, i32 seed, float g[6]) {
    uint32_t base = sbxm::rng_base(i, step, seed);
    uint32_t h1 = sbxm::wang_hash(base);
    uint32_t h2 = sbxm::wang_hash(base ^ 0x9e3779b9u);
    uint32_t h3 = sbxm::wang_hash(base ^ 0x85ebca6bu);
    uint32_t h4 = sbxm::wang_hash(base ^ 0xc2b2ae35u);
    uint32_t h5 = sbxm::wang_hash(base ^ 0x517cc1b7u);
    uint32_t h6 = sbxm::wang_hash(base ^ 0x1f0a7ed5u);
    float u1 = std::max((float)1.0e-7f, sbxm::unit_from_hash(h1));
    float u2 = sbxm::unit_from_hash(h2);
    float u3 = std::max((float)1.0e-7f, sbxm::unit_from_hash(h3));
    float u4 = sbxm::unit_from_hash(h4);
    float u5 = std::max((float)1.0e-7f, sbxm::unit_from_hash(h5));
    float u6 = sbxm::unit_from_hash(h6);
    box_muller6(u1, u2, u3, u4, u5, u6, g);
}

// Philox4x32-10 keyed (seed, step, slot): two blocks -> six uniforms, same transform
inline void gauss6_philox(i32 i, i32 step, uint64_t seed, float g[6]) {
    uint32_t c0[4] = {(uint32_t)i, (uint32_t)step, 0u, 0x53425830u};
    uint32_t c1[4] = {(uint32_t)i, (uint32_t)step, 1u, 0x53425830u};
    sbxm::philox4x32_10(c0, (uint32_t)seed, (uint32_t)(seed >> 32));
    sbxm::philox4x32_10(c1, (uint32_t)seed, (uint32_t)(seed >> 32));
    float u1 = std::max((float)1.0e-7f, sbxm::unit_from_hash(c0[0]));
    float u2 = sbxm::unit_from_hash(c0[1]);
    float u3 = std::max((float)1.0e-7f, sbxm::unit_from_hash(c0[2]));
    float u4 = sbxm::unit_from_hash(c0[3]);
    float u5 = std::max((float)1.0e-7f, sbxm::unit_from_hash(c1[0]));
    float u6 = sbxm::unit_from_hash(c1[1]);
    box_muller6(u1, u2, u3, u4, u5, u6, g);
}

}  // namespace

// ============================================================================
// threads
// ============================================================================
EXPORT void orc_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : 1);
#else
    (void)n;
#endif
}
EXPORT int orc_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// scalar helpers exported for tests
EXPORT double orc_accurate_acos(double x) { return accurate_acos(x); }
EXPORT double orc_angle_from_sin_cos(double s2, double c) { return angle_from_sin_cos(s2, c); }
EXPORT double orc_kT() { return KT; }

// ============================================================================
// DragTensorSystem.java:33-122, MiniFilamentStore.java:121-134
// ============================================================================
EXPORT void orc_rod_drag_si(double lengthUm, double radiusUm, double aeta, double* g) {
    double LM = 1.0e-6 * lengthUm;
    double RM = radiusUm * 1.0e-6;
    double logT = JLOG(LM / (2 * RM));
    g[0] = (2 * PI_D * aeta * LM) / (logT + A_PARALLEL);
    g[1] = (4 * PI_D * aeta * LM) / (logT + A_ORTHOG);
    g[2] = g[1];
    g[3] = 4 * PI_D * aeta * RM * RM * LM;
    g[4] = (PI_D * aeta * (LM * LM * LM)) / (3 * (logT + A_TURNING));
    g[5] = g[4];
}

EXPORT void orc_sphere_drag_si(double radiusUm, double aeta, double* g) {
    double RM = radiusUm * 1.0e-6;
    double bTG = 6 * PI_D * aeta * RM;
    double bRG = 8 * PI_D * aeta * (RM * RM * RM);
    g[0] = g[1] = g[2] = bTG;
    g[3] = g[4] = g[5] = bRG;
}

static void store_drag(int n, int i, const double* g, float* bTG, float* bRG, float* bTD, float* bRD) {
    bTG[i] = (float)g[0]; bTG[n + i] = (float)g[1]; bTG[2 * n + i] = (float)g[2];
    bRG[i] = (float)g[3]; bRG[n + i] = (float)g[4]; bRG[2 * n + i] = (float)g[5];
    bTD[i] = (float)(KT / g[0]); bTD[n + i] = (float)(KT / g[1]); bTD[2 * n + i] = (float)(KT / g[2]);
    bRD[i] = (float)(KT / g[3]); bRD[n + i] = (float)(KT / g[4]); bRD[2 * n + i] = (float)(KT / g[5]);
}

EXPORT void orc_drag_run_filament(int n, const i32* monomerCount, const i32* end1NbrSlot,
                                  const i32* end2NbrSlot, double aeta, float* segLength,
                                  float* bTG, float* bRG, float* bTD, float* bRD) {
    const double halfmono = ACTIN_MONO_RADIUS;
    const int minMonomerCt = 30;
    for (int i = 0; i < n; i++) {
        int monomerCt = monomerCount[i];
        double length = (monomerCt + 1) * ACTIN_MONO_RADIUS;
        segLength[i] = (float)length;
        double minLength;
        if (end1NbrSlot[i] == -1 || end2NbrSlot[i] == -1) minLength = STD_SEG_LENGTH * halfmono;
        else minLength = minMonomerCt * halfmono;
        double asIfLength = length;
        if (asIfLength < minLength) asIfLength = minLength;
        double g[6];
        orc_rod_drag_si(asIfLength, ACTIN_RADIUS, aeta, g);
        store_drag(n, i, g, bTG, bRG, bTD, bRD);
    }
}

EXPORT void orc_drag_run_motor(int nMotors, double aeta, float* segLength,
                               float* bTG, float* bRG, float* bTD, float* bRD) {
    int n = 3 * nMotors;
    double gr[6], gl[6], gh[6];
    orc_rod_drag_si(ROD_LEN, ROD_R, aeta, gr);
    orc_rod_drag_si(LEVER_LEN, LEVER_R, aeta, gl);
    orc_sphere_drag_si(HEAD_R, aeta, gh);
    for (int m = 0; m < nMotors; m++) {
        int rod = 3 * m, lever = 3 * m + 1, head = 3 * m + 2;
        segLength[rod] = (float)ROD_LEN;
        segLength[lever] = (float)LEVER_LEN;
        segLength[head] = (float)HEAD_LEN;
        store_drag(n, rod, gr, bTG, bRG, bTD, bRD);
        store_drag(n, lever, gl, bTG, bRG, bTD, bRD);
        store_drag(n, head, gh, bTG, bRG, bTD, bRD);
    }
}

EXPORT void orc_backbone_drag(int nBb, double bbLen, double aeta, float* segLength,
                              float* bTG, float* bRG, float* bTD, float* bRD, float* bbInvDragY) {
    double g[6];
    orc_rod_drag_si(bbLen, BACKBONE_R, aeta, g);
    for (int bb = 0; bb < nBb; bb++) {
        segLength[bb] = (float)bbLen;
        store_drag(nBb, bb, g, bTG, bRG, bTD, bRD);
        bbInvDragY[bb] = (float)(1.0 / g[1]);
        bbInvDragY[nBb + bb] = (float)(1.0 / g[4]);
    }
}

// ============================================================================
// BrownianForceSystem.java:44-106 (wang), plus the Philox and supplied-noise modes
// ============================================================================
static inline void brownian_store(int N, int i, const float g[6], float* rF, float* rT,
                                  const float* bTG, const float* bRG, const float* tSc,
                                  const float* rSc, float mag) {
    int iy = N + i, iz = 2 * N + i;
    float tS = tSc[i], rS = rSc[i];
    rF[i] = tS * mag * jsqrtf(bTG[i]) * g[0];
    rF[iy] = tS * mag * jsqrtf(bTG[iy]) * g[1];
    rF[iz] = tS * mag * jsqrtf(bTG[iz]) * g[2];
    rT[i] = rS * mag * jsqrtf(bRG[i]) * g[3];
    rT[iy] = rS * mag * jsqrtf(bRG[iy]) * g[4];
    rT[iz] = rS * mag * jsqrtf(bRG[iz]) * g[5];
}

EXPORT void orc_brownian_force(int N, float* rF, float* rT, const float* bTG, const float* bRG,
                               const float* tSc, const float* rSc, const float* params,
                               const i32* counts) {
    i32 step = counts[1], seed = counts[2];
    float mag = params[1];
    PAR for (int i = 0; i < N; i++) {
        float g[6];
        gauss6_wang(i, step, seed, g);
        brownian_store(N, i, g, rF, rT, bTG, bRG, tSc, rSc, mag);
    }
}

EXPORT void orc_brownian_force_philox(int N, float* rF, float* rT, const float* bTG, const float* bRG,
                                      const float* tSc, const float* rSc, const float* params,
                                      const i32* counts, uint64_t seed) {
    i32 step = counts[1];
    float mag = params[1];
    PAR for (int i = 0; i < N; i++) {
        float g[6];
        gauss6_philox(i, step, seed, g);
        brownian_store(N, i, g, rF, rT, bTG, bRG, tSc, rSc, mag);
    }
}

// noise: planar [6][N] = gfx | gfy | gfz | gtx | gty | gtz
EXPORT void orc_brownian_force_supplied(int N, float* rF, float* rT, const float* bTG, const float* bRG,
                                        const float* tSc, const float* rSc, const float* params,
                                        const float* noise) {
    float mag = params[1];
    PAR for (int i = 0; i < N; i++) {
        float g[6];
        for (int k = 0; k < 6; k++) g[k] = noise[(int64_t)k * N + i];
        brownian_store(N, i, g, rF, rT, bTG, bRG, tSc, rSc, mag);
    }
}

// raw wang-mode gaussians (for tests of the noise generator itself): out planar [6][N]
EXPORT void orc_gauss6_wang(int N, i32 step, i32 seed, float* out) {
    PAR for (int i = 0; i < N; i++) {
        float g[6]; gauss6_wang(i, step, seed, g);
        for (int k = 0; k < 6; k++) out[(int64_t)k * N + i] = g[k];
    }
}
EXPORT void orc_gauss6_philox(int N, i32 step, uint64_t seed, float* out) {
    PAR for (int i = 0; i < N; i++) {
        float g[6]; gauss6_philox(i, step, seed, g);
        for (int k = 0; k < 6; k++) out[(int64_t)k * N + i] = g[k];
    }
}

// ChainBendingForceSystem.java:38-45
EXPORT void orc_zero_accumulators(int N, float* F, float* T) {
    PAR for (int i = 0; i < N; i++) {
        F[i] = 0.f; F[N + i] = 0.f; F[2 * N + i] = 0.f;
        T[i] = 0.f; T[N + i] = 0.f; T[2 * N + i] = 0.f;
    }
}

// ============================================================================
// RigidRodLangevinIntegrationSystem.java:33-112 and DerivedGeometrySystem.java:27-73
// coord64 (optional, may be null): FP64 accumulation of the centre; the FP32 coord
// is then the rounded projection. The per-step increment dt*v is the reference's.
// ============================================================================
static inline void integrate_one(int N, int i, float* coord, double* coord64, float* uVec, float* yVec,
                                 const float* F, const float* T, const float* rF, const float* rT,
                                 const float* bTG, const float* bRG, float dt) {
    int iy = N + i, iz = 2 * N + i;
    float ux = uVec[i], uyc = uVec[iy], uzc = uVec[iz];
    float yx = yVec[i], yyc = yVec[iy], yzc = yVec[iz];
    float zx = uyc * yzc - uzc * yyc;
    float zy = uzc * yx - ux * yzc;
    float zz = ux * yyc - uyc * yx;
    float zlen = 1.0f / jsqrtf(zx * zx + zy * zy + zz * zz);
    zx *= zlen; zy *= zlen; zz *= zlen;
    float fx = F[i], fy = F[iy], fz = F[iz];
    float tx = T[i], ty = T[iy], tz = T[iz];
    float bfx = ux * fx + uyc * fy + uzc * fz + rF[i];
    float bfy = yx * fx + yyc * fy + yzc * fz + rF[iy];
    float bfz = zx * fx + zy * fy + zz * fz + rF[iz];
    float btx = ux * tx + uyc * ty + uzc * tz + rT[i];
    float bty = yx * tx + yyc * ty + yzc * tz + rT[iy];
    float btz = zx * tx + zy * ty + zz * tz + rT[iz];
    float bvx = 1.0e6f * bfx / bTG[i];
    float bvy = 1.0e6f * bfy / bTG[iy];
    float bvz = 1.0e6f * bfz / bTG[iz];
    float bwx = btx / bRG[i];
    float bwy = bty / bRG[iy];
    float bwz = btz / bRG[iz];
    float vx = ux * bvx + yx * bvy + zx * bvz;
    float vy = uyc * bvx + yyc * bvy + zy * bvz;
    float vz = uzc * bvx + yzc * bvy + zz * bvz;
    if (coord64) {
        double cx = coord64[i] + (double)(dt * vx);
        double cy = coord64[iy] + (double)(dt * vy);
        double cz = coord64[iz] + (double)(dt * vz);
        coord64[i] = cx; coord64[iy] = cy; coord64[iz] = cz;
        coord[i] = (float)cx; coord[iy] = (float)cy; coord[iz] = (float)cz;
    } else {
        coord[i] = coord[i] + dt * vx;
        coord[iy] = coord[iy] + dt * vy;
        coord[iz] = coord[iz] + dt * vz;
    }
    float uTransInZ = -bwy * dt;
    float uTransInY = bwz * dt;
    float nuX = ux + yx * uTransInY + zx * uTransInZ;
    float nuY = uyc + yyc * uTransInY + zy * uTransInZ;
    float nuZ = uzc + yzc * uTransInY + zz * uTransInZ;
    float nuInv = 1.0f / jsqrtf(nuX * nuX + nuY * nuY + nuZ * nuZ);
    uVec[i] = nuX * nuInv; uVec[iy] = nuY * nuInv; uVec[iz] = nuZ * nuInv;
    float yTransInX = -uTransInY;
    float yTransInZ = bwx * dt;
    float nyX = ux * yTransInX + yx + zx * yTransInZ;
    float nyY = uyc * yTransInX + yyc + zy * yTransInZ;
    float nyZ = uzc * yTransInX + yzc + zz * yTransInZ;
    float nyInv = 1.0f / jsqrtf(nyX * nyX + nyY * nyY + nyZ * nyZ);
    yVec[i] = nyX * nyInv; yVec[iy] = nyY * nyInv; yVec[iz] = nyZ * nyInv;
}

static inline void derive_one(int N, int i, const float* coord, const float* uVec, float* yVec,
                              float* zVec, float* end1, float* end2, const float* segLength) {
    int iy = N + i, iz = 2 * N + i;
    float ux = uVec[i], uyc = uVec[iy], uzc = uVec[iz];
    float yx = yVec[i], yyc = yVec[iy], yzc = yVec[iz];
    float zx = uyc * yzc - uzc * yyc;
    float zy = uzc * yx - ux * yzc;
    float zz = ux * yyc - uyc * yx;
    float zmag2 = zx * zx + zy * zy + zz * zz;
    if (zmag2 > 0.f) {
        float inv = 1.0f / jsqrtf(zmag2);
        zx *= inv; zy *= inv; zz *= inv;
    }
    zVec[i] = zx; zVec[iy] = zy; zVec[iz] = zz;
    float nyx = zy * uzc - zz * uyc;
    float nyy = zz * ux - zx * uzc;
    float nyz = zx * uyc - zy * ux;
    yVec[i] = nyx; yVec[iy] = nyy; yVec[iz] = nyz;
    float cx = coord[i], cy = coord[iy], cz = coord[iz];
    float halfLen = segLength[i] * 0.5f;
    end1[i] = cx - halfLen * ux; end1[iy] = cy - halfLen * uyc; end1[iz] = cz - halfLen * uzc;
    end2[i] = cx + halfLen * ux; end2[iy] = cy + halfLen * uyc; end2[iz] = cz + halfLen * uzc;
}

EXPORT void orc_integrate(int N, float* coord, double* coord64, float* uVec, float* yVec,
                          const float* F, const float* T, const float* rF, const float* rT,
                          const float* bTG, const float* bRG, const float* params) {
    float dt = params[0];
    PAR for (int i = 0; i < N; i++)
        integrate_one(N, i, coord, coord64, uVec, yVec, F, T, rF, rT, bTG, bRG, dt);
}

EXPORT void orc_derive(int N, const float* coord, const float* uVec, float* yVec, float* zVec,
                       float* end1, float* end2, const float* segLength) {
    PAR for (int i = 0; i < N; i++) derive_one(N, i, coord, uVec, yVec, zVec, end1, end2, segLength);
}

// ============================================================================
// ContainmentSystem.java:58-126
// boxParams: [0]=tau [1..3]=box dims [4]=R inset [5]=coeff [6]=checkInt
// ============================================================================
static inline void confine_one(int N, int i, const float* coord, const float* uVec, const float* segLength,
                               const float* bTG, float* F, float* T, double tau, double halfX,
                               double halfY, double halfZ, double coeff) {
    int iy = N + i, iz = 2 * N + i;
    double cx = coord[i], cy = coord[iy], cz = coord[iz];
    double ux = uVec[i], uy = uVec[iy], uz = uVec[iz];
    double half = 0.5 * (double)segLength[i];
    double bTGx = bTG[i];
    double fx = 0.0, fy = 0.0, fz = 0.0, tx = 0.0, ty = 0.0, tz = 0.0;
    bool touched = false;
    for (int e = 0; e < 2; e++) {
        double sgn = (e == 0) ? -1.0 : 1.0;
        double dx = cx + sgn * half * ux;
        double dy = cy + sgn * half * uy;
        double dz = cz + sgn * half * uz;
        double fux = wall_push(dx, halfX);
        double fuy = wall_push(dy, halfY);
        double fuz = wall_push(dz, halfZ);
        double delta2 = fux * fux + fuy * fuy + fuz * fuz;
        if (delta2 > 0.0) {
            double delta = std::sqrt(delta2);
            double inv = 1.0 / delta;
            double lux = fux * inv, luy = fuy * inv, luz = fuz * inv;
            double mag = coeff * 1.0e-6 * delta * bTGx / tau;
            double Fx = mag * lux, Fy = mag * luy, Fz = mag * luz;
            double rx = sgn * half * ux * 1.0e-6;
            double ry = sgn * half * uy * 1.0e-6;
            double rz = sgn * half * uz * 1.0e-6;
            fx += Fx; fy += Fy; fz += Fz;
            tx += ry * Fz - rz * Fy;
            ty += rz * Fx - rx * Fz;
            tz += rx * Fy - ry * Fx;
            touched = true;
        }
    }
    if (touched) {
        F[i] = (float)((double)F[i] + fx);
        F[iy] = (float)((double)F[iy] + fy);
        F[iz] = (float)((double)F[iz] + fz);
        T[i] = (float)((double)T[i] + tx);
        T[iy] = (float)((double)T[iy] + ty);
        T[iz] = (float)((double)T[iz] + tz);
    }
}

static inline bool confine_cadence(const float* boxParams, i32 step) {
    i32 checkInt = jf2i(boxParams[6]);
    return !(checkInt > 1 && (step % checkInt) != 0);
}

EXPORT void orc_confine(int N, const float* coord, const float* uVec, const float* segLength,
                        const float* bTG, float* F, float* T, const float* boxParams, const i32* counts) {
    if (!confine_cadence(boxParams, counts[1])) return;
    double tau = boxParams[0];
    double halfX = 0.5 * boxParams[1] - boxParams[4];
    double halfY = 0.5 * boxParams[2] - boxParams[4];
    double halfZ = 0.5 * boxParams[3] - boxParams[4];
    double coeff = boxParams[5];
    PAR for (int i = 0; i < N; i++)
        confine_one(N, i, coord, uVec, segLength, bTG, F, T, tau, halfX, halfY, halfZ, coeff);
}

// ============================================================================
// MechanicsFusion.java:52-338 — exact concatenations (bit-identical to the parts)
// ============================================================================
EXPORT void orc_force_build(int N, float* F, float* T, float* rF, float* rT, const float* bTG,
                            const float* bRG, const float* tSc, const float* rSc,
                            const float* params, const i32* counts) {
    orc_zero_accumulators(N, F, T);
    orc_brownian_force(N, rF, rT, bTG, bRG, tSc, rSc, params, counts);
}

EXPORT void orc_integ_derive(int N, float* coord, double* coord64, float* uVec, float* yVec,
                             float* zVec, const float* segLength, float* end1, float* end2,
                             const float* F, const float* T, const float* rF, const float* rT,
                             const float* bTG, const float* bRG, const float* params) {
    float dt = params[0];
    PAR for (int i = 0; i < N; i++) {
        integrate_one(N, i, coord, coord64, uVec, yVec, F, T, rF, rT, bTG, bRG, dt);
        derive_one(N, i, coord, uVec, yVec, zVec, end1, end2, segLength);
    }
}

// boxParams [7] = dt (MechanicsFusion.java:30-31)
EXPORT void orc_integ_derive_confined(int N, float* coord, double* coord64, float* uVec, float* yVec,
                                      float* zVec, const float* segLength, float* end1, float* end2,
                                      float* F, float* T, const float* rF, const float* rT,
                                      const float* bTG, const float* bRG, const float* boxParams,
                                      const i32* counts) {
    bool doConfine = confine_cadence(boxParams, counts[1]);
    double tau = boxParams[0];
    double halfX = 0.5 * boxParams[1] - boxParams[4];
    double halfY = 0.5 * boxParams[2] - boxParams[4];
    double halfZ = 0.5 * boxParams[3] - boxParams[4];
    double coeff = boxParams[5];
    float dt = boxParams[7];
    PAR for (int i = 0; i < N; i++) {
        if (doConfine) confine_one(N, i, coord, uVec, segLength, bTG, F, T, tau, halfX, halfY, halfZ, coeff);
        integrate_one(N, i, coord, coord64, uVec, yVec, F, T, rF, rT, bTG, bRG, dt);
        derive_one(N, i, coord, uVec, yVec, zVec, end1, end2, segLength);
    }
}

// ============================================================================
// ChainBendingForceSystem.java:105-331
// chainParams: [0]=dt [1]=fracMove [2]=fracR [3]=fracMoveTorq [4]=springActive [5]=spring [6]=monoR
// ============================================================================
EXPORT void orc_chain_forces(int N, const float* coord, const float* uVec, const float* segLength,
                             const i32* end2NbrSlot, const i32* end2NbrSide, const i32* end1NbrSlot,
                             const i32* end1NbrSide, const float* bTG, const float* bRG,
                             float* F, float* T, const float* chainParams) {
    double dt = (double)chainParams[0];
    double fracMove = (double)chainParams[1];
    double fracR = (double)chainParams[2];
    double fracMoveTorq = (double)chainParams[3];
    double filTorqSpringActive = (double)chainParams[4];
    double filTorqSpring = (double)chainParams[5];
    double actinMonoRadius = (double)chainParams[6];
    double DEG2RAD = PI_D / 180.0;
    double RAD2DEG = 180.0 / PI_D;

    PAR for (int i = 0; i < N; i++) {
        int iy = N + i, iz = 2 * N + i;
        double cx = coord[i], cy = coord[iy], cz = coord[iz];
        double ux = uVec[i], uy = uVec[iy], uz = uVec[iz];
        double len = segLength[i];
        double halfLen_um = 0.5 * len;
        double lSqSelf = 1.0e-12 * len * len;
        double rBTGx = bTG[i];
        double rBTGy = bTG[iy];
        double rBRGy = bRG[iy];
        double fx = 0.0, fy = 0.0, fz = 0.0, tx = 0.0, ty = 0.0, tz = 0.0;
        int e2Slot = end2NbrSlot[i];
        int e1Slot = end1NbrSlot[i];
        for (int side = 0; side < 2; side++) {
            // side 0 = end2 block (:152-235), side 1 = end1 block (:237-321)
            int slot = (side == 0) ? e2Slot : e1Slot;
            if (slot < 0) continue;
            int nside = (side == 0) ? end2NbrSide[i] : end1NbrSide[i];
            int jx = slot, jy = N + slot, jz = 2 * N + slot;
            double ncx = coord[jx], ncy = coord[jy], ncz = coord[jz];
            double nux = uVec[jx], nuy = uVec[jy], nuz = uVec[jz];
            double nlen = segLength[slot];
            double nHalfLen_um = 0.5 * nlen;
            double lSqN = 1.0e-12 * nlen * nlen;
            double nBTGx = bTG[jx];
            double nBTGy = bTG[jy];
            double nBRGy = bRG[jy];
            double ex, ey, ez, selfLpx, selfLpy, selfLpz;
            if (side == 0) {
                ex = cx + halfLen_um * ux; ey = cy + halfLen_um * uy; ez = cz + halfLen_um * uz;
                selfLpx = ex - actinMonoRadius * ux;
                selfLpy = ey - actinMonoRadius * uy;
                selfLpz = ez - actinMonoRadius * uz;
            } else {
                ex = cx - halfLen_um * ux; ey = cy - halfLen_um * uy; ez = cz - halfLen_um * uz;
                selfLpx = ex + actinMonoRadius * ux;
                selfLpy = ey + actinMonoRadius * uy;
                selfLpz = ez + actinMonoRadius * uz;
            }
            double nbrTipx, nbrTipy, nbrTipz;
            if (nside == 0) {
                nbrTipx = ncx - nHalfLen_um * nux; nbrTipy = ncy - nHalfLen_um * nuy; nbrTipz = ncz - nHalfLen_um * nuz;
            } else {
                nbrTipx = ncx + nHalfLen_um * nux; nbrTipy = ncy + nHalfLen_um * nuy; nbrTipz = ncz + nHalfLen_um * nuz;
            }
            double nbrLpx, nbrLpy, nbrLpz;
            if (nside == 0) {
                nbrLpx = nbrTipx + actinMonoRadius * nux; nbrLpy = nbrTipy + actinMonoRadius * nuy; nbrLpz = nbrTipz + actinMonoRadius * nuz;
            } else {
                nbrLpx = nbrTipx - actinMonoRadius * nux; nbrLpy = nbrTipy - actinMonoRadius * nuy; nbrLpz = nbrTipz - actinMonoRadius * nuz;
            }
            double linkPtX, linkPtY, linkPtZ, ptAtEndX, ptAtEndY, ptAtEndZ;
            if (i < slot) {
                linkPtX = selfLpx; linkPtY = selfLpy; linkPtZ = selfLpz;
                ptAtEndX = nbrTipx; ptAtEndY = nbrTipy; ptAtEndZ = nbrTipz;
            } else {
                linkPtX = nbrLpx; linkPtY = nbrLpy; linkPtZ = nbrLpz;
                ptAtEndX = ex; ptAtEndY = ey; ptAtEndZ = ez;
            }
            double dx = ptAtEndX - linkPtX, dy = ptAtEndY - linkPtY, dz = ptAtEndZ - linkPtZ;
            double strainDist = std::sqrt(dx * dx + dy * dy + dz * dz);
            double invStrain = (strainDist > 0.0) ? (1.0 / strainDist) : 0.0;
            double luX = dx * invStrain, luY = dy * invStrain, luZ = dz * invStrain;

            double cosB1 = ux * luX + uy * luY + uz * luZ;
            if (cosB1 > 1.0) cosB1 = 1.0;
            if (cosB1 < -1.0) cosB1 = -1.0;
            double cosA1 = JSIN(accurate_acos(cosB1));
            double cosA1_2 = cosA1 * cosA1;
            double moveC1 = cosB1 * cosB1 / rBTGx + cosA1_2 / rBTGy + lSqSelf * cosA1_2 / (4.0 * rBRGy);

            double cosB2 = nux * luX + nuy * luY + nuz * luZ;
            if (cosB2 > 1.0) cosB2 = 1.0;
            if (cosB2 < -1.0) cosB2 = -1.0;
            double cosA2 = JSIN(accurate_acos(cosB2));
            double cosA2_2 = cosA2 * cosA2;
            double moveC2 = cosB2 * cosB2 / nBTGx + cosA2_2 / nBTGy + lSqN * cosA2_2 / (4.0 * nBRGy);

            double denom = dt * (moveC1 + moveC2);
            double forceMag = (denom > 0.0) ? (fracMove * 1.0e-6 * strainDist / denom) : 0.0;
            double fSign = (i < slot) ? 1.0 : -1.0;
            double Fx = fSign * forceMag * luX, Fy = fSign * forceMag * luY, Fz = fSign * forceMag * luZ;
            fx += Fx; fy += Fy; fz += Fz;
            double Rscale = (side == 0) ? (0.5e-6 * len * fracR) : (-0.5e-6 * len * fracR);
            double Rx = Rscale * ux, Ry = Rscale * uy, Rz = Rscale * uz;
            tx += Ry * Fz - Rz * Fy; ty += Rz * Fx - Rx * Fz; tz += Rx * Fy - Ry * Fx;

            double nuxE, nuyE, nuzE;
            if (nside == 0) { nuxE = nux; nuyE = nuy; nuzE = nuz; } else { nuxE = -nux; nuyE = -nuy; nuzE = -nuz; }
            double mux, muy, muz;
            if (side == 0) { mux = ux; muy = uy; muz = uz; } else { mux = -ux; muy = -uy; muz = -uz; }
            double tvx = muy * nuzE - muz * nuyE, tvy = muz * nuxE - mux * nuzE, tvz = mux * nuyE - muy * nuxE;
            double tvMag2 = tvx * tvx + tvy * tvy + tvz * tvz;
            if (tvMag2 > 1.0e-30) {
                double invMag = 1.0 / std::sqrt(tvMag2);
                tvx *= invMag; tvy *= invMag; tvz *= invMag;
                double dotV = mux * nuxE + muy * nuyE + muz * nuzE;
                if (dotV > 1.0) dotV = 1.0;
                if (dotV < -1.0) dotV = -1.0;
                double angTween = angle_from_sin_cos(tvMag2, dotV) * RAD2DEG;
                double torsionMag;
                if (filTorqSpringActive > 0.5) {
                    torsionMag = fracMoveTorq * filTorqSpring * angTween;
                } else {
                    double invBRG = 1.0 / rBRGy + 1.0 / nBRGy;
                    torsionMag = fracMoveTorq * DEG2RAD * angTween / (invBRG * dt);
                }
                tx += tvx * torsionMag; ty += tvy * torsionMag; tz += tvz * torsionMag;
            }
        }
        F[i] = (float)(F[i] + fx);
        F[iy] = (float)(F[iy] + fy);
        F[iz] = (float)(F[iz] + fz);
        T[i] = (float)(T[i] + tx);
        T[iy] = (float)(T[iy] + ty);
        T[iz] = (float)(T[iz] + tz);
    }
}

// DeflectionSupport.java:24-58 (test support for the chain-law fixture)
EXPORT void orc_seed_accumulators(int N, float* F, float* T, const float* extForce, const i32* counts) {
    float load = (float)counts[3];
    for (int i = 0; i < N; i++) {
        int iy = N + i, iz = 2 * N + i;
        F[i] = load * extForce[i]; F[iy] = load * extForce[iy]; F[iz] = load * extForce[iz];
        T[i] = 0.f; T[iy] = 0.f; T[iz] = 0.f;
    }
}
EXPORT void orc_pin_endpoints(int N, float* coord, const float* uVec, const float* segLength, int P,
                              const i32* pinSeg, const i32* pinEnd, const float* pinAnchor) {
    for (int p = 0; p < P; p++) {
        int s = pinSeg[p];
        int sx = s, sy = N + s, sz = 2 * N + s;
        float cx = coord[sx], cy = coord[sy], cz = coord[sz];
        float ux = uVec[sx], uy = uVec[sy], uz = uVec[sz];
        float half = 0.5f * segLength[s];
        float ex, ey, ez;
        if (pinEnd[p] == 1) { ex = cx - half * ux; ey = cy - half * uy; ez = cz - half * uz; }
        else { ex = cx + half * ux; ey = cy + half * uy; ez = cz + half * uz; }
        float dx = pinAnchor[3 * p] - ex;
        float dy = pinAnchor[3 * p + 1] - ey;
        float dz = pinAnchor[3 * p + 2] - ez;
        coord[sx] = cx + dx; coord[sy] = cy + dy; coord[sz] = cz + dz;
    }
}

// ============================================================================
// Body-view publishing: FilamentStore.java:275-328, MotorStore.java:300-347
// ============================================================================
EXPORT void orc_fil_publish(int n, const float* coord, const float* segLength, int cap, float* center,
                            float* boundingRadius, i32* ownerStore, i32* ownerSlot,
                            const float* viewParams, const i32* filState) {
    float actinRadius = viewParams[0];
    PAR for (int i = 0; i < n; i++) {
        center[i] = coord[i];
        center[cap + i] = coord[n + i];
        center[2 * cap + i] = coord[2 * n + i];
        boundingRadius[i] = 0.5f * segLength[i] + actinRadius;
        ownerStore[i] = (filState && filState[i] < 0) ? STORE_NONE : STORE_FILAMENT;
        ownerSlot[i] = i;
    }
}

EXPORT void orc_mot_publish_head(int nM, const float* bodyCoord, const float* bodyUVec,
                                 const float* bodySegLength, float* head, float* uVec, float* rodUVec) {
    int nB = 3 * nM;
    PAR for (int m = 0; m < nM; m++) {
        int h = 3 * m + 2, r = 3 * m;
        float hl = bodySegLength[h];
        head[m] = bodyCoord[h] + 0.5f * hl * bodyUVec[h];
        head[nM + m] = bodyCoord[nB + h] + 0.5f * hl * bodyUVec[nB + h];
        head[2 * nM + m] = bodyCoord[2 * nB + h] + 0.5f * hl * bodyUVec[2 * nB + h];
        uVec[m] = bodyUVec[h]; uVec[nM + m] = bodyUVec[nB + h]; uVec[2 * nM + m] = bodyUVec[2 * nB + h];
        rodUVec[m] = bodyUVec[r]; rodUVec[nM + m] = bodyUVec[nB + r]; rodUVec[2 * nM + m] = bodyUVec[2 * nB + r];
    }
}

EXPORT void orc_mot_publish(int nM, const float* head, const float* reach, int cap, float* center,
                            float* boundingRadius, i32* ownerStore, i32* ownerSlot, i32 base) {
    PAR for (int m = 0; m < nM; m++) {
        int b = base + m;
        center[b] = head[m];
        center[cap + b] = head[nM + m];
        center[2 * cap + b] = head[2 * nM + m];
        boundingRadius[b] = reach[m];
        ownerStore[b] = STORE_MOTOR;
        ownerSlot[b] = m;
    }
}

// ============================================================================
// SpatialGrid.java:51-445
// gridParams: [0..2]=min [3]=cell [4]=invCell [5]=cutoff; gridDims: [0..2]=nX,nY,nZ [3]=cells
// ============================================================================
EXPORT void orc_body_cell(int cap, const float* center, const float* gridParams, const i32* gridDims,
                          i32 S, i32* bodyCell) {
    float xMin = gridParams[0], yMin = gridParams[1], zMin = gridParams[2];
    float invCell = gridParams[4];
    int nX = gridDims[0], nY = gridDims[1], nZ = gridDims[2];
    int nXY = nX * nY;
    PAR for (int i = 0; i < cap; i++) {
        if (i >= S) { bodyCell[i] = -1; continue; }
        int ix = jf2i((center[i] - xMin) * invCell);
        int iy = jf2i((center[cap + i] - yMin) * invCell);
        int iz = jf2i((center[2 * cap + i] - zMin) * invCell);
        if (ix < 0) ix = 0; if (ix >= nX) ix = nX - 1;
        if (iy < 0) iy = 0; if (iy >= nY) iy = nY - 1;
        if (iz < 0) iz = 0; if (iz >= nZ) iz = nZ - 1;
        bodyCell[i] = ix + iy * nX + iz * nXY;
    }
}

EXPORT void orc_grid_zero(i32 totalCells, i32* cellCount) {
    for (int c = 0; c < totalCells; c++) cellCount[c] = 0;
}
EXPORT void orc_grid_histogram(const i32* bodyCell, i32 S, i32* cellCount) {
    for (int s = 0; s < S; s++) { int c = bodyCell[s]; if (c >= 0) cellCount[c] = cellCount[c] + 1; }
}
EXPORT void orc_grid_scan_local(i32 totalCells, const i32* cellCount, i32* offsets, i32* chunkSum) {
    int numChunks = (totalCells + GRID_SCAN_CHUNK - 1) / GRID_SCAN_CHUNK;
    for (int ch = 0; ch < numChunks; ch++) {
        int start = ch * GRID_SCAN_CHUNK, end = start + GRID_SCAN_CHUNK;
        if (end > totalCells) end = totalCells;
        int acc = 0;
        for (int c = start; c < end; c++) { offsets[c] = acc; acc += cellCount[c]; }
        chunkSum[ch] = acc;
    }
}
EXPORT void orc_grid_scan_chunks(i32 totalCells, i32* chunkSum) {
    int numChunks = (totalCells + GRID_SCAN_CHUNK - 1) / GRID_SCAN_CHUNK;
    int acc = 0;
    for (int ch = 0; ch < numChunks; ch++) { int t = chunkSum[ch]; chunkSum[ch] = acc; acc += t; }
    chunkSum[numChunks] = acc;
}
EXPORT void orc_grid_scan_add(i32 totalCells, i32* offsets, i32 contentsCap, i32* cellCount, const i32* chunkSum) {
    int numChunks = (totalCells + GRID_SCAN_CHUNK - 1) / GRID_SCAN_CHUNK;
    for (int ch = 0; ch < numChunks; ch++) {
        int start = ch * GRID_SCAN_CHUNK, end = start + GRID_SCAN_CHUNK;
        if (end > totalCells) end = totalCells;
        int base = chunkSum[ch];
        for (int c = start; c < end; c++) { offsets[c] = offsets[c] + base; cellCount[c] = 0; }
        if (ch == 0) {
            int total = chunkSum[numChunks];
            offsets[totalCells] = total < contentsCap ? total : contentsCap;
        }
    }
}
EXPORT void orc_grid_scatter(const i32* bodyCell, i32 S, const i32* offsets, i32* contents,
                             i32 contentsCap, i32* cellCount) {
    for (int s = 0; s < S; s++) {
        int c = bodyCell[s];
        if (c < 0) continue;
        int writePos = offsets[c] + cellCount[c];
        if (writePos < contentsCap) contents[writePos] = s;
        cellCount[c] = cellCount[c] + 1;
    }
}

EXPORT i32 orc_body_chunk_size(i32 bodyCount, i32 totalCells) {
    if (bodyCount <= 0 || totalCells <= 0) return 1;
    int sqrtN = (int)(int64_t)std::floor(std::sqrt((double)bodyCount) + 0.5);
    int64_t memMin = (int64_t)std::ceil((double)bodyCount * (double)totalCells / (double)(64LL << 20));
    int64_t bcs = std::max((int64_t)sqrtN, memMin);
    return (i32)std::max((int64_t)1, bcs);
}

EXPORT void orc_grid_chunk_zero(i32 numChunks, i32 totalCells, i32* m) {
    int64_t total = (int64_t)numChunks * totalCells;
    for (int64_t e = 0; e < total; e++) m[e] = 0;
}
EXPORT void orc_grid_chunk_histogram(const i32* bodyCell, i32 S, i32 chunkSize, i32 numChunks,
                                     i32 totalCells, i32* m) {
    PAR for (int bc = 0; bc < numChunks; bc++) {
        int start = bc * chunkSize, end = start + chunkSize;
        if (end > S) end = S;
        int64_t rowBase = (int64_t)bc * totalCells;
        for (int s = start; s < end; s++) { int c = bodyCell[s]; if (c >= 0) m[rowBase + c] += 1; }
    }
}
EXPORT void orc_grid_chunk_reduce(i32 totalCells, i32 numChunks, i32* m, i32* cellCount) {
    PAR for (int c = 0; c < totalCells; c++) {
        int acc = 0;
        for (int bc = 0; bc < numChunks; bc++) {
            int64_t idx = (int64_t)bc * totalCells + c;
            int v = m[idx]; m[idx] = acc; acc += v;
        }
        cellCount[c] = acc;
    }
}
EXPORT void orc_grid_chunk_scatter(const i32* bodyCell, i32 S, i32 chunkSize, i32 numChunks,
                                   i32 totalCells, const i32* offsets, i32* contents, i32 contentsCap, i32* m) {
    PAR for (int bc = 0; bc < numChunks; bc++) {
        int start = bc * chunkSize, end = start + chunkSize;
        if (end > S) end = S;
        int64_t rowBase = (int64_t)bc * totalCells;
        for (int s = start; s < end; s++) {
            int c = bodyCell[s];
            if (c < 0) continue;
            int64_t idx = rowBase + c;
            int writePos = offsets[c] + m[idx];
            if (writePos < contentsCap) contents[writePos] = s;
            m[idx] += 1;
        }
    }
}

EXPORT void orc_broad_phase(int cap, const float* center, const float* boundingRadius, const i32* bodyCell,
                            const i32* offsets, const i32* contents, const i32* gridDims,
                            const float* gridParams, i32 S, i32* candPartner, i32* candCount) {
    int nX = gridDims[0], nY = gridDims[1], nZ = gridDims[2];
    int nXY = nX * nY;
    float cutoff = gridParams[5];
    PAR for (int i = 0; i < cap; i++) {
        candCount[i] = 0;
        if (i >= S) continue;
        int c = bodyCell[i];
        if (c < 0) continue;
        int cz = c / nXY, rem = c - cz * nXY, cy = rem / nX, cx = rem - cy * nX;
        float icx = center[i], icy = center[cap + i], icz = center[2 * cap + i];
        float ri = boundingRadius[i];
        int x0 = cx - 1; if (x0 < 0) x0 = 0;
        int x1 = cx + 1; if (x1 >= nX) x1 = nX - 1;
        int y0 = cy - 1; if (y0 < 0) y0 = 0;
        int y1 = cy + 1; if (y1 >= nY) y1 = nY - 1;
        int z0 = cz - 1; if (z0 < 0) z0 = 0;
        int z1 = cz + 1; if (z1 >= nZ) z1 = nZ - 1;
        int cnt = 0;
        for (int zz = z0; zz <= z1; zz++) {
            int zOff = zz * nXY;
            for (int yy = y0; yy <= y1; yy++) {
                int yOff = yy * nX;
                for (int xx = x0; xx <= x1; xx++) {
                    int cc = xx + yOff + zOff;
                    int start = offsets[cc], end = offsets[cc + 1];
                    for (int idx = start; idx < end; idx++) {
                        int j = contents[idx];
                        if (j <= i) continue;
                        float dx = icx - center[j];
                        float dy = icy - center[cap + j];
                        float dz = icz - center[2 * cap + j];
                        float distSq = dx * dx + dy * dy + dz * dz;
                        float reach = ri + boundingRadius[j] + cutoff;
                        if (distSq <= reach * reach) {
                            if (cnt < MAX_CAND) candPartner[(int64_t)i * MAX_CAND + cnt] = j;
                            cnt++;
                        }
                    }
                }
            }
        }
        candCount[i] = cnt;
    }
}

EXPORT void orc_brute_force(int cap, const float* center, const float* boundingRadius,
                            const float* gridParams, i32 S, i32* brutePartner, i32* bruteCount) {
    float cutoff = gridParams[5];
    PAR for (int i = 0; i < cap; i++) {
        bruteCount[i] = 0;
        if (i >= S) continue;
        float icx = center[i], icy = center[cap + i], icz = center[2 * cap + i];
        float ri = boundingRadius[i];
        int cnt = 0;
        for (int j = i + 1; j < S; j++) {
            float dx = icx - center[j];
            float dy = icy - center[cap + j];
            float dz = icz - center[2 * cap + j];
            float distSq = dx * dx + dy * dy + dz * dz;
            float reach = ri + boundingRadius[j] + cutoff;
            if (distSq <= reach * reach) {
                if (cnt < MAX_CAND) brutePartner[(int64_t)i * MAX_CAND + cnt] = j;
                cnt++;
            }
        }
        bruteCount[i] = cnt;
    }
}

// ============================================================================
// BindingDetectionSystem.java:59-389
// kinParams: [7]=myoColTol [8]=alignTol (full layout MotorStore.java:84-94)
// ============================================================================
static inline float reach_test_dist_sq(float mx, float my, float mz, float mux, float muy, float muz,
                                       float rux, float ruy, float ruz, float e1x, float e1y, float e1z,
                                       float e2x, float e2y, float e2z, float myoColTol, float alignTol) {
    float r1x = e2x - e1x, r1y = e2y - e1y, r1z = e2z - e1z;
    float denom = r1x * r1x + r1y * r1y + r1z * r1z;
    if (denom <= 0.f) return -1.f;
    float r2x = mx - e1x, r2y = my - e1y, r2z = mz - e1z;
    float numer = r2x * r1x + r2y * r1y + r2z * r1z;
    float alpha = numer / denom;
    if (alpha < 0.f || alpha > 1.f) return -1.f;
    float cpx = e1x + alpha * r1x, cpy = e1y + alpha * r1y, cpz = e1z + alpha * r1z;
    float dx = cpx - mx, dy = cpy - my, dz = cpz - mz;
    float conDistSq = dx * dx + dy * dy + dz * dz;
    if (conDistSq >= myoColTol * myoColTol) return -1.f;
    float inv = 1.0f / jsqrtf(denom);
    float fux = r1x * inv, fuy = r1y * inv, fuz = r1z * inv;
    float motDotFil = mux * fux + muy * fuy + muz * fuz;
    if (motDotFil < alignTol) return -1.f;
    float rodDotFil = rux * fux + ruy * fuy + ruz * fuz;
    if (rodDotFil < 0.f) return -1.f;
    return conDistSq;
}

EXPORT void orc_invert_candidates(const i32* candPartner, const i32* candCount, const i32* ownerStore,
                                  const i32* ownerSlot, i32 S, i32 nM, i32* motorCandSeg, i32* motorCandCount) {
    for (int m = 0; m < nM; m++) motorCandCount[m] = 0;
    for (int i = 0; i < S; i++) {
        int storeI = ownerStore[i];
        int cnt = candCount[i];
        if (cnt > MAX_CAND) cnt = MAX_CAND;
        int64_t base = (int64_t)i * MAX_CAND;
        for (int k = 0; k < cnt; k++) {
            int j = candPartner[base + k];
            int storeJ = ownerStore[j];
            int motor = -1, seg = -1;
            if (storeI == STORE_MOTOR && storeJ == STORE_FILAMENT) { motor = ownerSlot[i]; seg = ownerSlot[j]; }
            else if (storeI == STORE_FILAMENT && storeJ == STORE_MOTOR) { motor = ownerSlot[j]; seg = ownerSlot[i]; }
            if (motor >= 0) {
                int c = motorCandCount[motor];
                if (c < MAX_CAND) motorCandSeg[(int64_t)motor * MAX_CAND + c] = seg;
                motorCandCount[motor] = c + 1;
            }
        }
    }
}

EXPORT void orc_grid_reachable(i32 nM, const float* head, const float* uVec, const float* rodUVec,
                               i32 nSeg, const float* segEnd1, const float* segEnd2,
                               const float* gridParams, const i32* gridDims, const i32* offsets,
                               const i32* contents, const i32* ownerStore, const i32* ownerSlot,
                               i32* reachSeg, i32* reachCount, const float* kinParams) {
    float myoColTol = kinParams[7], alignTol = kinParams[8];
    float xMin = gridParams[0], yMin = gridParams[1], zMin = gridParams[2];
    float invCell = gridParams[4];
    int nX = gridDims[0], nY = gridDims[1], nZ = gridDims[2];
    int nXY = nX * nY;
    PAR for (int m = 0; m < nM; m++) {
        float mx = head[m], my = head[nM + m], mz = head[2 * nM + m];
        float mux = uVec[m], muy = uVec[nM + m], muz = uVec[2 * nM + m];
        float rux = rodUVec[m], ruy = rodUVec[nM + m], ruz = rodUVec[2 * nM + m];
        int cx = jf2i((mx - xMin) * invCell);
        int cy = jf2i((my - yMin) * invCell);
        int cz = jf2i((mz - zMin) * invCell);
        if (cx < 0) cx = 0; if (cx >= nX) cx = nX - 1;
        if (cy < 0) cy = 0; if (cy >= nY) cy = nY - 1;
        if (cz < 0) cz = 0; if (cz >= nZ) cz = nZ - 1;
        int x0 = cx - 1; if (x0 < 0) x0 = 0;
        int x1 = cx + 1; if (x1 >= nX) x1 = nX - 1;
        int y0 = cy - 1; if (y0 < 0) y0 = 0;
        int y1 = cy + 1; if (y1 >= nY) y1 = nY - 1;
        int z0 = cz - 1; if (z0 < 0) z0 = 0;
        int z1 = cz + 1; if (z1 >= nZ) z1 = nZ - 1;
        int out = 0;
        for (int zz = z0; zz <= z1; zz++) {
            int zOff = zz * nXY;
            for (int yy = y0; yy <= y1; yy++) {
                int yOff = yy * nX;
                for (int xx = x0; xx <= x1; xx++) {
                    int cc = xx + yOff + zOff;
                    int start = offsets[cc], end = offsets[cc + 1];
                    for (int idx = start; idx < end; idx++) {
                        int j = contents[idx];
                        if (ownerStore[j] != STORE_FILAMENT) continue;
                        int s = ownerSlot[j];
                        float e1x = segEnd1[s], e1y = segEnd1[nSeg + s], e1z = segEnd1[2 * nSeg + s];
                        float e2x = segEnd2[s], e2y = segEnd2[nSeg + s], e2z = segEnd2[2 * nSeg + s];
                        float d = reach_test_dist_sq(mx, my, mz, mux, muy, muz, rux, ruy, ruz,
                                                     e1x, e1y, e1z, e2x, e2y, e2z, myoColTol, alignTol);
                        if (d >= 0.f) {
                            if (out < MAX_CAND) reachSeg[(int64_t)m * MAX_CAND + out] = s;
                            out++;
                        }
                    }
                }
            }
        }
        reachCount[m] = out;
    }
}

EXPORT void orc_compute_reachable(i32 nM, const float* head, const float* uVec, const float* rodUVec,
                                  i32 nSeg, const float* segEnd1, const float* segEnd2,
                                  const i32* motorCandSeg, const i32* motorCandCount,
                                  i32* reachSeg, i32* reachCount, const float* kinParams) {
    float myoColTol = kinParams[7], alignTol = kinParams[8];
    PAR for (int m = 0; m < nM; m++) {
        float mx = head[m], my = head[nM + m], mz = head[2 * nM + m];
        float mux = uVec[m], muy = uVec[nM + m], muz = uVec[2 * nM + m];
        float rux = rodUVec[m], ruy = rodUVec[nM + m], ruz = rodUVec[2 * nM + m];
        int cnt = motorCandCount[m]; if (cnt > MAX_CAND) cnt = MAX_CAND;
        int out = 0;
        for (int k = 0; k < cnt; k++) {
            int s = motorCandSeg[(int64_t)m * MAX_CAND + k];
            float d = reach_test_dist_sq(mx, my, mz, mux, muy, muz, rux, ruy, ruz,
                                         segEnd1[s], segEnd1[nSeg + s], segEnd1[2 * nSeg + s],
                                         segEnd2[s], segEnd2[nSeg + s], segEnd2[2 * nSeg + s], myoColTol, alignTol);
            if (d >= 0.f) { if (out < MAX_CAND) reachSeg[(int64_t)m * MAX_CAND + out] = s; out++; }
        }
        reachCount[m] = out;
    }
}

EXPORT void orc_brute_reachable(i32 nM, const float* head, const float* uVec, const float* rodUVec,
                                i32 nSeg, const float* segEnd1, const float* segEnd2,
                                i32* reachSeg, i32* reachCount, const float* kinParams) {
    float myoColTol = kinParams[7], alignTol = kinParams[8];
    PAR for (int m = 0; m < nM; m++) {
        float mx = head[m], my = head[nM + m], mz = head[2 * nM + m];
        float mux = uVec[m], muy = uVec[nM + m], muz = uVec[2 * nM + m];
        float rux = rodUVec[m], ruy = rodUVec[nM + m], ruz = rodUVec[2 * nM + m];
        int out = 0;
        for (int s = 0; s < nSeg; s++) {
            float d = reach_test_dist_sq(mx, my, mz, mux, muy, muz, rux, ruy, ruz,
                                         segEnd1[s], segEnd1[nSeg + s], segEnd1[2 * nSeg + s],
                                         segEnd2[s], segEnd2[nSeg + s], segEnd2[2 * nSeg + s], myoColTol, alignTol);
            if (d >= 0.f) { if (out < MAX_CAND) reachSeg[(int64_t)m * MAX_CAND + out] = s; out++; }
        }
        reachCount[m] = out;
    }
}

static inline void bind_nearest_one(int m, i32 nM, const float* head, const float* uVec, const float* rodUVec,
                                    i32 nSeg, const float* segEnd1, const float* segEnd2,
                                    const i32* candSeg, const i32* candCount, i32* boundSeg,
                                    float* bindArc, float myoColTol, float alignTol) {
    float mx = head[m], my = head[nM + m], mz = head[2 * nM + m];
    float mux = uVec[m], muy = uVec[nM + m], muz = uVec[2 * nM + m];
    float rux = rodUVec[m], ruy = rodUVec[nM + m], ruz = rodUVec[2 * nM + m];
    int cnt = candCount[m]; if (cnt > MAX_CAND) cnt = MAX_CAND;
    int bestSeg = -1; float bestD = 1.0e30f; float bestArc = 0.f;
    for (int k = 0; k < cnt; k++) {
        int s = candSeg[(int64_t)m * MAX_CAND + k];
        float e1x = segEnd1[s], e1y = segEnd1[nSeg + s], e1z = segEnd1[2 * nSeg + s];
        float e2x = segEnd2[s], e2y = segEnd2[nSeg + s], e2z = segEnd2[2 * nSeg + s];
        float d = reach_test_dist_sq(mx, my, mz, mux, muy, muz, rux, ruy, ruz,
                                     e1x, e1y, e1z, e2x, e2y, e2z, myoColTol, alignTol);
        if (d >= 0.f && d < bestD) {
            bestD = d; bestSeg = s;
            float r1x = e2x - e1x, r1y = e2y - e1y, r1z = e2z - e1z;
            float denom = r1x * r1x + r1y * r1y + r1z * r1z;
            float numer = (mx - e1x) * r1x + (my - e1y) * r1y + (mz - e1z) * r1z;
            bestArc = numer / jsqrtf(denom);
        }
    }
    if (bestSeg >= 0) { boundSeg[m] = bestSeg; bindArc[m] = bestArc; }
}

EXPORT void orc_bind_nearest(i32 nM, const float* head, const float* uVec, const float* rodUVec,
                             i32 nSeg, const float* segEnd1, const float* segEnd2,
                             const i32* candSeg, const i32* candCount, i32* boundSeg, float* bindArc,
                             const float* kinParams) {
    float myoColTol = kinParams[7], alignTol = kinParams[8];
    PAR for (int m = 0; m < nM; m++) {
        if (boundSeg[m] != FREE_BINDABLE) continue;
        bind_nearest_one(m, nM, head, uVec, rodUVec, nSeg, segEnd1, segEnd2, candSeg, candCount,
                         boundSeg, bindArc, myoColTol, alignTol);
    }
}

// BindingDetectionSystem.java:292-348 (the F=0 kinetics variant)
EXPORT void orc_bind_kinetics(i32 nM, const float* head, const float* uVec, const float* rodUVec,
                              i32 nSeg, const float* segEnd1, const float* segEnd2,
                              const i32* candSeg, const i32* candCount, i32* boundSeg, float* bindArc,
                              i32* stats, const float* kinParams, const i32* counts) {
    i32 step = counts[1], seed = counts[2];
    float kOff = kinParams[0], aCatch = kinParams[1], aSlip = kinParams[2];
    float xCatch = kinParams[3], xSlip = kinParams[4], kT = kinParams[5], dt = kinParams[6];
    float myoColTol = kinParams[7], alignTol = kinParams[8], F = kinParams[9];
    float rate = kOff * (aCatch * (float)JEXP((double)(-F * xCatch / kT)) + aSlip * (float)JEXP((double)(F * xSlip / kT)));
    float pOff = rate * dt;
    PAR for (int m = 0; m < nM; m++) {
        int bs = boundSeg[m];
        if (bs >= 0) {
            stats[2 * m] = stats[2 * m] + 1;
            uint32_t h = sbxm::wang_hash(sbxm::rng_base(m, step, seed) ^ 0x4D54u);
            float u = sbxm::unit_from_hash(h);
            if (u < pOff) { boundSeg[m] = FREE_COOLDOWN; stats[2 * m + 1] = stats[2 * m + 1] + 1; }
        } else if (bs == FREE_COOLDOWN) {
            boundSeg[m] = FREE_BINDABLE;
        } else {
            bind_nearest_one(m, nM, head, uVec, rodUVec, nSeg, segEnd1, segEnd2, candSeg, candCount,
                             boundSeg, bindArc, myoColTol, alignTol);
        }
    }
}

// ============================================================================
// NucleotideCycleSystem.java:33-134
// nucParams: [0]=dt [1]=atpOn [2..7]=on/off rates;  kinParams layout MotorStore.java:84-94
// ============================================================================
EXPORT void orc_cycle(i32 nM, i32* nucleotideState, const i32* boundSeg, const float* forceDotHist,
                      const float* nucParams, const i32* counts) {
    i32 step = counts[1], seed = counts[2];
    float dt = nucParams[0], atpOn = nucParams[1];
    float onATP = nucParams[2], offATP = nucParams[3];
    float onPi = nucParams[4], offPi = nucParams[5];
    float onADP = nucParams[6], offADP = nucParams[7];
    PAR for (int m = 0; m < nM; m++) {
        int state = nucleotideState[m];
        bool bound = boundSeg[m] >= 0;
        uint32_t h = sbxm::wang_hash(sbxm::rng_base(m, step, seed) ^ 0x4E55u);
        float u = sbxm::unit_from_hash(h);
        if (state == NUC_NONE) {
            if (u < atpOn * dt) state = NUC_ATP;
        } else if (state == NUC_ATP) {
            float rate = bound ? onATP : offATP;
            if (u < rate * dt) state = NUC_ADPPI;
        } else if (state == NUC_ADPPI) {
            float rate = bound ? onPi : offPi;
            if (u < rate * dt) state = NUC_ADP;
        } else {
            float avg = 0.f;
            int b = m * 10;
            for (int k = 0; k < 10; k++) avg += forceDotHist[b + k];
            avg *= 0.1f;
            if (avg <= 0.f) {
                float rate = bound ? onADP : offADP;
                if (u < rate * dt) state = NUC_NONE;
            }
        }
        nucleotideState[m] = state;
    }
}

EXPORT void orc_catch_slip_release(i32 nM, i32* boundSeg, const float* forceDotFil, const float* forceMag,
                                   i32* cooldown, i32* stats, i32* capStats, const float* kinParams,
                                   const i32* counts) {
    i32 step = counts[1], seed = counts[2];
    float kOff = kinParams[0], aCatch = kinParams[1], aSlip = kinParams[2];
    float xCatch = kinParams[3], xSlip = kinParams[4], kT = kinParams[5], dt = kinParams[6];
    int refractorySteps = jf2i(kinParams[10]);
    float breakForceN = kinParams[11];
    bool capOn = kinParams[12] > 0.5f;
    float blockProb = kinParams[13];
    PAR for (int m = 0; m < nM; m++) {
        int bs = boundSeg[m];
        if (bs >= 0) {
            stats[2 * m] = stats[2 * m] + 1;
            bool enterRefractory = refractorySteps > 0;
            if (blockProb < 1.0f) {
                uint32_t rh = sbxm::wang_hash(sbxm::rng_base(m, step, seed) ^ 0x52465241u);
                float ru = sbxm::unit_from_hash(rh);
                enterRefractory = enterRefractory && (ru < blockProb);
            }
            if (capOn && forceMag[m] > breakForceN) {
                capStats[m] = capStats[m] + 1;
                if (enterRefractory) { boundSeg[m] = FREE_COOLDOWN; cooldown[m] = refractorySteps; }
                else boundSeg[m] = FREE_BINDABLE;
                continue;
            }
            float F = forceDotFil[m];
            float rate = kOff * (aCatch * (float)JEXP((double)(-F * xCatch / kT)) + aSlip * (float)JEXP((double)(F * xSlip / kT)));
            uint32_t h = sbxm::wang_hash(sbxm::rng_base(m, step, seed) ^ 0x4D54u);
            float u = sbxm::unit_from_hash(h);
            if (u < rate * dt) {
                stats[2 * m + 1] = stats[2 * m + 1] + 1;
                if (enterRefractory) { boundSeg[m] = FREE_COOLDOWN; cooldown[m] = refractorySteps; }
                else boundSeg[m] = FREE_BINDABLE;
            }
        } else if (bs == FREE_COOLDOWN) {
            int c = cooldown[m] - 1;
            if (c <= 0) boundSeg[m] = FREE_BINDABLE;
            else cooldown[m] = c;
        }
    }
}

// ============================================================================
// CrossBridgeSystem.java:58-337
// xbParams: [0]=myoSpring [2]=j1FracMoveTorq [3]=dt [4]=HEAD_LEN [5]=xbias
// ============================================================================
EXPORT void orc_bond_forces(i32 nB, const float* mC, const float* mU, const float* mY, const float* mBRG,
                            i32 nSeg, const float* fC, const float* fU, const float* fY, const float* fBRG,
                            const float* fLen, const i32* boundSeg, const float* bindArc,
                            const i32* nucleotideState, float* bondData, const float* xbParams) {
    double myoSpring = xbParams[0], j1FMT = xbParams[2];
    double dt = xbParams[3], headLen = xbParams[4];
    double xbias = xbParams[5];
    double DEG2RAD = PI_D / 180.0, RAD2DEG = 180.0 / PI_D;
    int nM = nB / 3;
    PAR for (int m = 0; m < nM; m++) {
        int d = m * XB_STRIDE;
        for (int k = 0; k < XB_STRIDE; k++) bondData[d + k] = 0.f;
        int s = boundSeg[m];
        if (s < 0) continue;
        int h = 3 * m + 2;
        double hcx = mC[h], hcy = mC[nB + h], hcz = mC[2 * nB + h];
        double hux = mU[h], huy = mU[nB + h], huz = mU[2 * nB + h];
        double hyx = mY[h], hyy = mY[nB + h], hyz = mY[2 * nB + h];
        double hbRGx = mBRG[h], hbRGy = mBRG[nB + h];
        double htipx = hcx + 0.5 * headLen * hux, htipy = hcy + 0.5 * headLen * huy, htipz = hcz + 0.5 * headLen * huz;
        double scx = fC[s], scy = fC[nSeg + s], scz = fC[2 * nSeg + s];
        double sux = fU[s], suy = fU[nSeg + s], suz = fU[2 * nSeg + s];
        double syx = fY[s], syy = fY[nSeg + s], syz = fY[2 * nSeg + s];
        double sbRGx = fBRG[s], sbRGy = fBRG[nSeg + s];
        double slen = fLen[s];
        double aOff = bindArc[m] - 0.5 * slen;
        double apx = scx + aOff * sux, apy = scy + aOff * suy, apz = scz + aOff * suz;
        double dx = apx - htipx, dy = apy - htipy, dz = apz - htipz;
        double dist = std::sqrt(dx * dx + dy * dy + dz * dz);
        double fmag = myoSpring * dist;
        double Fx = 0, Fy = 0, Fz = 0;
        if (dist > 0.0) { double inv = fmag / dist; Fx = inv * dx; Fy = inv * dy; Fz = inv * dz; }
        double RHx = (htipx - hcx) * 1e-6, RHy = (htipy - hcy) * 1e-6, RHz = (htipz - hcz) * 1e-6;
        double THx = RHy * Fz - RHz * Fy, THy = RHz * Fx - RHx * Fz, THz = RHx * Fy - RHy * Fx;
        double RSx = (apx - scx) * 1e-6, RSy = (apy - scy) * 1e-6, RSz = (apz - scz) * 1e-6;
        double nFx = -Fx, nFy = -Fy, nFz = -Fz;
        double TSx = RSy * nFz - RSz * nFy, TSy = RSz * nFx - RSx * nFz, TSz = RSx * nFy - RSy * nFx;
        double restF9 = (nucleotideState[m] != NUC_ADPPI) ? 120.0 : 90.0;
        double t9x = suy * huz - suz * huy, t9y = suz * hux - sux * huz, t9z = sux * huy - suy * hux;
        double m9 = t9x * t9x + t9y * t9y + t9z * t9z;
        double T9x = 0, T9y = 0, T9z = 0;
        if (m9 > 1.0e-30) {
            double im = 1.0 / std::sqrt(m9); t9x *= im; t9y *= im; t9z *= im;
            double dot = sux * hux + suy * huy + suz * huz; if (dot > 1) dot = 1; if (dot < -1) dot = -1;
            double angD = accurate_acos(dot) * RAD2DEG - restF9;
            double tm = j1FMT * DEG2RAD * angD / ((1.0 / hbRGy + 1.0 / sbRGy) * dt);
            T9x = tm * t9x; T9y = tm * t9y; T9z = tm * t9z;
        }
        double t10x = syy * hyz - syz * hyy, t10y = syz * hyx - syx * hyz, t10z = syx * hyy - syy * hyx;
        double m10 = t10x * t10x + t10y * t10y + t10z * t10z;
        double T10x = 0, T10y = 0, T10z = 0;
        if (m10 > 1.0e-30) {
            double im = 1.0 / std::sqrt(m10); t10x *= im; t10y *= im; t10z *= im;
            double dot = syx * hyx + syy * hyy + syz * hyz; if (dot > 1) dot = 1; if (dot < -1) dot = -1;
            double ang = accurate_acos(dot) * RAD2DEG;
            double tm = j1FMT * DEG2RAD * ang / ((1.0 / hbRGx + 1.0 / sbRGx) * dt);
            T10x = tm * t10x; T10y = tm * t10y; T10z = tm * t10z;
        }
        bondData[d] = (float)Fx; bondData[d + 1] = (float)Fy; bondData[d + 2] = (float)Fz;
        bondData[d + 3] = (float)(THx - T9x - T10x);
        bondData[d + 4] = (float)(THy - T9y - T10y);
        bondData[d + 5] = (float)(THz - T9z - T10z);
        bondData[d + 6] = (float)(nFx - xbias); bondData[d + 7] = (float)nFy; bondData[d + 8] = (float)nFz;
        bondData[d + 9] = (float)(TSx + T9x + T10x);
        bondData[d + 10] = (float)(TSy + T9y + T10y);
        bondData[d + 11] = (float)(TSz + T9z + T10z);
        bondData[d + 12] = (float)(Fx * sux + Fy * suy + Fz * suz);
    }
}

EXPORT void orc_apply_head_force(i32 nB, const float* bondData, float* F, float* T) {
    int nM = nB / 3;
    PAR for (int m = 0; m < nM; m++) {
        int h = 3 * m + 2, d = m * XB_STRIDE;
        F[h] = F[h] + bondData[d];
        F[nB + h] = F[nB + h] + bondData[d + 1];
        F[2 * nB + h] = F[2 * nB + h] + bondData[d + 2];
        T[h] = T[h] + bondData[d + 3];
        T[nB + h] = T[nB + h] + bondData[d + 4];
        T[2 * nB + h] = T[2 * nB + h] + bondData[d + 5];
    }
}

EXPORT void orc_register_force_dot(i32 nM, const float* bondData, const i32* boundSeg, float* forceDotFil,
                                   float* forceMag, float* forceDotHist, i32* forceDotPlace) {
    PAR for (int m = 0; m < nM; m++) {
        if (boundSeg[m] >= 0) {
            int d = m * XB_STRIDE;
            float fd = bondData[d + 12];
            forceDotFil[m] = fd;
            float fx = bondData[d], fy = bondData[d + 1], fz = bondData[d + 2];
            forceMag[m] = jsqrtf(fx * fx + fy * fy + fz * fz);
            int p = forceDotPlace[m];
            forceDotHist[m * 10 + p] = fd;
            forceDotPlace[m] = (p + 1) % 10;
        } else {
            forceDotFil[m] = 0.f;
            forceMag[m] = 0.f;
            forceDotPlace[m] = 0;
            int b = m * 10;
            for (int k = 0; k < 10; k++) forceDotHist[b + k] = 0.f;
        }
    }
}

// serial CSR-inverse: CrossBridgeSystem.java:190-217 (nItems keys -> nRows rows)
EXPORT void orc_csr_histogram(const i32* keys, i32 nItems, i32 nRows, i32* rowCount) {
    for (int s = 0; s < nRows; s++) rowCount[s] = 0;
    for (int m = 0; m < nItems; m++) { int s = keys[m]; if (s >= 0) rowCount[s] = rowCount[s] + 1; }
}
EXPORT void orc_csr_scan(i32 nRows, i32* rowCount, i32* rowOffsets) {
    int acc = 0;
    for (int s = 0; s < nRows; s++) { rowOffsets[s] = acc; acc += rowCount[s]; rowCount[s] = 0; }
    rowOffsets[nRows] = acc;
}
EXPORT void orc_csr_scatter(const i32* keys, i32 nItems, const i32* rowOffsets, i32* rowCount, i32* rowList) {
    for (int m = 0; m < nItems; m++) {
        int s = keys[m]; if (s < 0) continue;
        int pos = rowOffsets[s] + rowCount[s];
        rowList[pos] = m;
        rowCount[s] = rowCount[s] + 1;
    }
}
// parallel chunk variant: CrossBridgeSystem.java:232-298
EXPORT void orc_csr_chunk_zero(i32 numChunks, i32 nRows, i32* mtx) {
    int64_t total = (int64_t)numChunks * nRows;
    for (int64_t e = 0; e < total; e++) mtx[e] = 0;
}
EXPORT void orc_csr_chunk_histogram(const i32* keys, i32 nItems, i32 nRows, i32 chunkSize, i32 numChunks, i32* mtx) {
    PAR for (int mc = 0; mc < numChunks; mc++) {
        int start = mc * chunkSize, end = start + chunkSize;
        if (end > nItems) end = nItems;
        int64_t rowBase = (int64_t)mc * nRows;
        for (int m = start; m < end; m++) { int s = keys[m]; if (s >= 0) mtx[rowBase + s] += 1; }
    }
}
EXPORT void orc_csr_chunk_reduce(i32 nRows, i32 numChunks, i32* mtx, i32* rowCount) {
    PAR for (int s = 0; s < nRows; s++) {
        int acc = 0;
        for (int mc = 0; mc < numChunks; mc++) {
            int64_t idx = (int64_t)mc * nRows + s;
            int v = mtx[idx]; mtx[idx] = acc; acc += v;
        }
        rowCount[s] = acc;
    }
}
EXPORT void orc_csr_chunk_scatter(const i32* keys, i32 nItems, i32 nRows, i32 chunkSize, i32 numChunks,
                                  const i32* rowOffsets, i32* rowList, i32* mtx) {
    PAR for (int mc = 0; mc < numChunks; mc++) {
        int start = mc * chunkSize, end = start + chunkSize;
        if (end > nItems) end = nItems;
        int64_t rowBase = (int64_t)mc * nRows;
        for (int m = start; m < end; m++) {
            int s = keys[m]; if (s < 0) continue;
            int64_t idx = rowBase + s;
            int pos = rowOffsets[s] + mtx[idx];
            rowList[pos] = m;
            mtx[idx] += 1;
        }
    }
}

// CrossBridgeSystem.java:302-337; generic stride/offset gather shared with the
// crosslinker passes (CrosslinkerSystem.java:129-173, stateGuard = linkState) and the
// backbone gather (MiniFilamentSystem.java:137-155).
static void csr_gather(i32 nRows, const i32* offsets, const i32* list, const float* payload, int stride,
                       int off, const i32* stateGuard, float* F, float* T) {
    PAR for (int s = 0; s < nRows; s++) {
        double fx = 0, fy = 0, fz = 0, tx = 0, ty = 0, tz = 0;
        int start = offsets[s], end = offsets[s + 1];
        for (int k = start; k < end; k++) {
            int li = list[k];
            if (stateGuard && stateGuard[li] < 0) continue;
            int d = li * stride + off;
            fx += payload[d]; fy += payload[d + 1]; fz += payload[d + 2];
            tx += payload[d + 3]; ty += payload[d + 4]; tz += payload[d + 5];
        }
        F[s] = (float)(F[s] + fx);
        F[nRows + s] = (float)(F[nRows + s] + fy);
        F[2 * nRows + s] = (float)(F[2 * nRows + s] + fz);
        T[s] = (float)(T[s] + tx);
        T[nRows + s] = (float)(T[nRows + s] + ty);
        T[2 * nRows + s] = (float)(T[2 * nRows + s] + tz);
    }
}

EXPORT void orc_seg_gather(i32 nSeg, const i32* offsets, const i32* list, const float* bondData, float* F, float* T) {
    csr_gather(nSeg, offsets, list, bondData, XB_STRIDE, 6, nullptr, F, T);
}
EXPORT void orc_xb_brute_gather(i32 nSeg, i32 nM, const i32* boundSeg, const float* bondData, float* F, float* T) {
    PAR for (int s = 0; s < nSeg; s++) {
        double fx = 0, fy = 0, fz = 0, tx = 0, ty = 0, tz = 0;
        for (int m = 0; m < nM; m++) {
            if (boundSeg[m] != s) continue;
            int d = m * XB_STRIDE;
            fx += bondData[d + 6]; fy += bondData[d + 7]; fz += bondData[d + 8];
            tx += bondData[d + 9]; ty += bondData[d + 10]; tz += bondData[d + 11];
        }
        F[s] = (float)fx; F[nSeg + s] = (float)fy; F[2 * nSeg + s] = (float)fz;
        T[s] = (float)tx; T[nSeg + s] = (float)ty; T[2 * nSeg + s] = (float)tz;
    }
}

// ============================================================================
// CrosslinkerSystem.java:51-281, 694-808
// xlParams: [0]=restLength [1]=fracMoveBase [2]=dt; offParams: [0]=const [1]=coeff [2]=exp [3]=dt [4]=rest
// torsionParams: [0]=spring [1]=active
// ============================================================================
EXPORT void orc_link_forces(i32 nSeg, const float* fC, const float* fU, const float* fE1, const float* fBTG,
                            i32 nLinks, const i32* linkFilA, const i32* linkFilB, const float* loc1,
                            const float* loc2, const i32* filLinkCt, float* xlinkData, const float* xlParams) {
    double restLength = xlParams[0], fracMoveBase = xlParams[1], dt = xlParams[2];
    PAR for (int k = 0; k < nLinks; k++) {
        int d = k * XL_STRIDE;
        for (int j = 0; j < XL_STRIDE; j++) xlinkData[d + j] = 0.f;
        int a = linkFilA[k], b = linkFilB[k];
        if (a < 0 || b < 0) continue;
        double l1 = loc1[k];
        double uax = fU[a], uay = fU[nSeg + a], uaz = fU[2 * nSeg + a];
        double p1x = fE1[a] + l1 * uax;
        double p1y = fE1[nSeg + a] + l1 * uay;
        double p1z = fE1[2 * nSeg + a] + l1 * uaz;
        double l2 = loc2[k];
        double ubx = fU[b], uby = fU[nSeg + b], ubz = fU[2 * nSeg + b];
        double p2x = fE1[b] + l2 * ubx;
        double p2y = fE1[nSeg + b] + l2 * uby;
        double p2z = fE1[2 * nSeg + b] + l2 * ubz;
        double lvx = p2x - p1x, lvy = p2y - p1y, lvz = p2z - p1z;
        double linkLength = std::sqrt(lvx * lvx + lvy * lvy + lvz * lvz);
        double stretch = linkLength - restLength;
        if (stretch < 0.0) stretch = 0.0;
        int ctA = filLinkCt[a], ctB = filLinkCt[b];
        int maxLinks = ctA > ctB ? ctA : ctB;
        if (maxLinks < 1) maxLinks = 1;
        double fracMove = fracMoveBase / maxLinks;
        double g1 = fBTG[a];
        double g2 = fBTG[b];
        double curForceMag = (fracMove * 1.0e-6 * stretch / dt) / (1.0 / g1 + 1.0 / g2);
        double Fx = curForceMag * lvx, Fy = curForceMag * lvy, Fz = curForceMag * lvz;
        double rax = (p1x - fC[a]) * 1e-6;
        double ray = (p1y - fC[nSeg + a]) * 1e-6;
        double raz = (p1z - fC[2 * nSeg + a]) * 1e-6;
        double TAx = ray * Fz - raz * Fy;
        double TAy = raz * Fx - rax * Fz;
        double TAz = rax * Fy - ray * Fx;
        double nFx = -Fx, nFy = -Fy, nFz = -Fz;
        double rbx = (p2x - fC[b]) * 1e-6;
        double rby = (p2y - fC[nSeg + b]) * 1e-6;
        double rbz = (p2z - fC[2 * nSeg + b]) * 1e-6;
        double TBx = rby * nFz - rbz * nFy;
        double TBy = rbz * nFx - rbx * nFz;
        double TBz = rbx * nFy - rby * nFx;
        xlinkData[d] = (float)Fx; xlinkData[d + 1] = (float)Fy; xlinkData[d + 2] = (float)Fz;
        xlinkData[d + 3] = (float)TAx; xlinkData[d + 4] = (float)TAy; xlinkData[d + 5] = (float)TAz;
        xlinkData[d + 6] = (float)nFx; xlinkData[d + 7] = (float)nFy; xlinkData[d + 8] = (float)nFz;
        xlinkData[d + 9] = (float)TBx; xlinkData[d + 10] = (float)TBy; xlinkData[d + 11] = (float)TBz;
    }
}

EXPORT void orc_seg_gather_a(i32 nSeg, const i32* offsets, const i32* list, const float* xlinkData,
                             const i32* linkState, float* F, float* T) {
    csr_gather(nSeg, offsets, list, xlinkData, XL_STRIDE, 0, linkState, F, T);
}
EXPORT void orc_seg_gather_b(i32 nSeg, const i32* offsets, const i32* list, const float* xlinkData,
                             const i32* linkState, float* F, float* T) {
    csr_gather(nSeg, offsets, list, xlinkData, XL_STRIDE, 6, linkState, F, T);
}
EXPORT void orc_xl_brute_gather(i32 nSeg, i32 nLinks, const i32* linkFilA, const i32* linkFilB,
                                const float* xlinkData, const i32* linkState, float* F, float* T) {
    PAR for (int s = 0; s < nSeg; s++) {
        double fx = 0, fy = 0, fz = 0, tx = 0, ty = 0, tz = 0;
        for (int k = 0; k < nLinks; k++) {
            if (linkState[k] < 0) continue;
            int d = k * XL_STRIDE;
            if (linkFilA[k] == s) {
                fx += xlinkData[d]; fy += xlinkData[d + 1]; fz += xlinkData[d + 2];
                tx += xlinkData[d + 3]; ty += xlinkData[d + 4]; tz += xlinkData[d + 5];
            }
            if (linkFilB[k] == s) {
                fx += xlinkData[d + 6]; fy += xlinkData[d + 7]; fz += xlinkData[d + 8];
                tx += xlinkData[d + 9]; ty += xlinkData[d + 10]; tz += xlinkData[d + 11];
            }
        }
        F[s] = (float)fx; F[nSeg + s] = (float)fy; F[2 * nSeg + s] = (float)fz;
        T[s] = (float)tx; T[nSeg + s] = (float)ty; T[2 * nSeg + s] = (float)tz;
    }
}

EXPORT void orc_xl_unbind(i32 nSeg, const float* fU, const float* fE1, i32 nLinks, const i32* linkFilA,
                          const i32* linkFilB, const float* loc1, const float* loc2, i32* linkState,
                          float* strainHist, i32* strainPlace, const float* offParams, const i32* counts) {
    i32 step = counts[1], seed = counts[2];
    double offConst = offParams[0], offCoeff = offParams[1], offExp = offParams[2];
    double dt = offParams[3], restLength = offParams[4];
    const int W = STRAIN_WIN;
    PAR for (int k = 0; k < nLinks; k++) {
        if (linkState[k] < 0) continue;
        int a = linkFilA[k], b = linkFilB[k];
        double l1 = loc1[k];
        double uax = fU[a], uay = fU[nSeg + a], uaz = fU[2 * nSeg + a];
        double p1x = fE1[a] + l1 * uax;
        double p1y = fE1[nSeg + a] + l1 * uay;
        double p1z = fE1[2 * nSeg + a] + l1 * uaz;
        double l2 = loc2[k];
        double ubx = fU[b], uby = fU[nSeg + b], ubz = fU[2 * nSeg + b];
        double p2x = fE1[b] + l2 * ubx;
        double p2y = fE1[nSeg + b] + l2 * uby;
        double p2z = fE1[2 * nSeg + b] + l2 * ubz;
        double lvx = p2x - p1x, lvy = p2y - p1y, lvz = p2z - p1z;
        double linkLength = std::sqrt(lvx * lvx + lvy * lvy + lvz * lvz);
        double stretch = linkLength - restLength;
        if (stretch < 0.0) stretch = 0.0;
        double strain = stretch / restLength;
        int base = k * W;
        int p = strainPlace[k];
        strainHist[base + p] = (float)strain;
        strainPlace[k] = (p + 1) % W;
        double ave = 0.0;
        for (int j = 0; j < W; j++) ave += strainHist[base + j];
        ave /= W;
        double kOff = offConst + offCoeff * JEXP(ave * offExp);
        double pBreak = kOff * dt;
        uint32_t h = sbxm::wang_hash(sbxm::rng_base(k, step, seed) ^ 0x584C4B42u);
        float u = sbxm::unit_from_hash(h);
        if (u < pBreak) linkState[k] = LINK_FREE;
    }
}

EXPORT void orc_count_active_links(i32 nLinks, const i32* linkState, const i32* linkFilA,
                                   const i32* linkFilB, i32 nSeg, i32* activeLinkCount) {
    for (int s = 0; s < nSeg; s++) activeLinkCount[s] = 0;
    for (int L = 0; L < nLinks; L++) {
        if (linkState[L] < 0) continue;
        int a = linkFilA[L], b = linkFilB[L];
        activeLinkCount[a] = activeLinkCount[a] + 1;
        activeLinkCount[b] = activeLinkCount[b] + 1;
    }
}

EXPORT void orc_link_torsion(i32 nSeg, const float* fU, i32 nLinks, const i32* linkFilA, const i32* linkFilB,
                             const i32* linkState, const i32* linkOrientSame, float* torqueMagHist,
                             i32* torqueMagPlace, float* xlinkData, const float* torsionParams) {
    if (torsionParams[1] < 0.5f) return;
    double spring = torsionParams[0];
    const int W = TORQUE_WIN;
    PAR for (int k = 0; k < nLinks; k++) {
        if (linkState[k] < 0) continue;
        int a = linkFilA[k], b = linkFilB[k];
        if (a < 0 || b < 0) continue;
        double uax = fU[a], uay = fU[nSeg + a], uaz = fU[2 * nSeg + a];
        double ubx = fU[b], uby = fU[nSeg + b], ubz = fU[2 * nSeg + b];
        bool same = linkOrientSame[k] != 0;
        double vbx = same ? ubx : -ubx, vby = same ? uby : -uby, vbz = same ? ubz : -ubz;
        double tx = uay * vbz - uaz * vby, ty = uaz * vbx - uax * vbz, tz = uax * vby - uay * vbx;
        double m2 = tx * tx + ty * ty + tz * tz;
        if (!(m2 > 1.0e-30)) continue;
        double im = 1.0 / std::sqrt(m2); tx *= im; ty *= im; tz *= im;
        double dot = uax * ubx + uay * uby + uaz * ubz;
        if (dot > 1.0) dot = 1.0;
        if (dot < -1.0) dot = -1.0;
        double angT = same ? fast_acos(dot) : std::fabs(fast_acos(dot) - PI_D);
        double curMag = spring * angT;
        int base = k * W;
        int p = torqueMagPlace[k];
        torqueMagHist[base + p] = (float)curMag;
        torqueMagPlace[k] = (p + 1) % W;
        double avg = 0.0;
        for (int j = 0; j < W; j++) avg += torqueMagHist[base + j];
        avg /= W;
        double Tx = avg * tx, Ty = avg * ty, Tz = avg * tz;
        int d = k * XL_STRIDE;
        xlinkData[d + 3] = (float)(xlinkData[d + 3] + Tx);
        xlinkData[d + 4] = (float)(xlinkData[d + 4] + Ty);
        xlinkData[d + 5] = (float)(xlinkData[d + 5] + Tz);
        xlinkData[d + 9] = (float)(xlinkData[d + 9] - Tx);
        xlinkData[d + 10] = (float)(xlinkData[d + 10] - Ty);
        xlinkData[d + 11] = (float)(xlinkData[d + 11] - Tz);
    }
}

// CrosslinkerStore.java:249-257
EXPORT void orc_compute_fil_link_ct(i32 nLinks, const i32* linkState, const i32* linkFilA,
                                    const i32* linkFilB, i32 nSeg, i32* filLinkCt) {
    orc_count_active_links(nLinks, linkState, linkFilA, linkFilB, nSeg, filLinkCt);
}

// ============================================================================
// MotorJointSystem.java:72-197
// jointParams: [0]=dt J1 [1]=fracMove [2]=fracR [3]=fracMoveTorq [4]=rest; J2 [5..8]; [9] anchor; [10] stall pN
// ============================================================================
EXPORT void orc_joints(i32 nB, const float* coord, const float* uVec, const float* segLength,
                       const float* bTG, const float* bRG, float* F, float* T,
                       const i32* nucleotideState, const float* jointParams) {
    double dt = jointParams[0];
    double j1FracMove = jointParams[1], j1FracR = jointParams[2];
    double j1FracMoveTorq = jointParams[3];
    double j2FracMove = jointParams[5], j2FracR = jointParams[6];
    double j2FracMoveTorq = jointParams[7], j2Rest = jointParams[8];
    double stallPN = jointParams[10];
    double DEG2RAD = PI_D / 180.0, RAD2DEG = 180.0 / PI_D;
    PAR for (int s = 0; s < nB; s++) {
        int m = s / 3;
        int role = s - 3 * m;
        double j1Rest = (nucleotideState[m] != NUC_ADPPI) ? 60.0 : 0.0;
        int rod = 3 * m, lever = 3 * m + 1, head = 3 * m + 2;
        double rcx = coord[rod], rcy = coord[nB + rod], rcz = coord[2 * nB + rod];
        double rux = uVec[rod], ruy = uVec[nB + rod], ruz = uVec[2 * nB + rod];
        double rlen = segLength[rod];
        double lcx = coord[lever], lcy = coord[nB + lever], lcz = coord[2 * nB + lever];
        double lux = uVec[lever], luy = uVec[nB + lever], luz = uVec[2 * nB + lever];
        double llen = segLength[lever];
        double hcx = coord[head], hcy = coord[nB + head], hcz = coord[2 * nB + head];
        double hux = uVec[head], huy = uVec[nB + head], huz = uVec[2 * nB + head];
        double hlen = segLength[head];
        double fx = 0, fy = 0, fz = 0, tx = 0, ty = 0, tz = 0;
        if (role == 0 || role == 1) {
            double aEx = rcx + 0.5 * rlen * rux, aEy = rcy + 0.5 * rlen * ruy, aEz = rcz + 0.5 * rlen * ruz;
            double bEx = lcx - 0.5 * llen * lux, bEy = lcy - 0.5 * llen * luy, bEz = lcz - 0.5 * llen * luz;
            double dx = aEx - bEx, dy = aEy - bEy, dz = aEz - bEz;
            double strain = std::sqrt(dx * dx + dy * dy + dz * dz);
            double inv = (strain > 0.0) ? 1.0 / strain : 0.0;
            double lx = dx * inv, ly = dy * inv, lz = dz * inv;
            double mcRod = move_c(rux, ruy, ruz, lx, ly, lz, bTG[rod], bTG[nB + rod], bRG[nB + rod], rlen);
            double mcLever = move_c(lux, luy, luz, lx, ly, lz, bTG[lever], bTG[nB + lever], bRG[nB + lever], llen);
            double denom = dt * (mcRod + mcLever);
            double forceMag = (denom > 0.0) ? (j2FracMove * 1.0e-6 * strain / denom) : 0.0;
            double tvx = ruy * luz - ruz * luy, tvy = ruz * lux - rux * luz, tvz = rux * luy - ruy * lux;
            double tvm2 = tvx * tvx + tvy * tvy + tvz * tvz;
            double torsionMag = 0.0;
            if (tvm2 > 1.0e-30) {
                double im = 1.0 / std::sqrt(tvm2); tvx *= im; tvy *= im; tvz *= im;
                double dotV = rux * lux + ruy * luy + ruz * luz;
                if (dotV > 1.0) dotV = 1.0;
                if (dotV < -1.0) dotV = -1.0;
                double ang = accurate_acos(dotV) * RAD2DEG;
                double invBRG = 1.0 / bRG[nB + rod] + 1.0 / bRG[nB + lever];
                torsionMag = j2FracMoveTorq * DEG2RAD * (ang - j2Rest) / (invBRG * dt);
            }
            if (role == 0) {
                double Fx = -forceMag * lx, Fy = -forceMag * ly, Fz = -forceMag * lz;
                fx += Fx; fy += Fy; fz += Fz;
                double Rs = 0.5e-6 * rlen * j2FracR, Rx = Rs * rux, Ry = Rs * ruy, Rz = Rs * ruz;
                tx += Ry * Fz - Rz * Fy; ty += Rz * Fx - Rx * Fz; tz += Rx * Fy - Ry * Fx;
                tx += tvx * torsionMag; ty += tvy * torsionMag; tz += tvz * torsionMag;
            } else {
                double Fx = forceMag * lx, Fy = forceMag * ly, Fz = forceMag * lz;
                fx += Fx; fy += Fy; fz += Fz;
                double Rs = -0.5e-6 * llen * j2FracR, Rx = Rs * lux, Ry = Rs * luy, Rz = Rs * luz;
                tx += Ry * Fz - Rz * Fy; ty += Rz * Fx - Rx * Fz; tz += Rx * Fy - Ry * Fx;
                tx -= tvx * torsionMag; ty -= tvy * torsionMag; tz -= tvz * torsionMag;
            }
        }
        if (role == 1 || role == 2) {
            double aEx = lcx + 0.5 * llen * lux, aEy = lcy + 0.5 * llen * luy, aEz = lcz + 0.5 * llen * luz;
            double bEx = hcx - 0.5 * hlen * hux, bEy = hcy - 0.5 * hlen * huy, bEz = hcz - 0.5 * hlen * huz;
            double dx = aEx - bEx, dy = aEy - bEy, dz = aEz - bEz;
            double strain = std::sqrt(dx * dx + dy * dy + dz * dz);
            double inv = (strain > 0.0) ? 1.0 / strain : 0.0;
            double lx = dx * inv, ly = dy * inv, lz = dz * inv;
            double mcLever = move_c(lux, luy, luz, lx, ly, lz, bTG[lever], bTG[nB + lever], bRG[nB + lever], llen);
            double mcHead = move_c(hux, huy, huz, lx, ly, lz, bTG[head], bTG[nB + head], bRG[nB + head], hlen);
            double denom = dt * (mcLever + mcHead);
            double forceMag = (denom > 0.0) ? (j1FracMove * 1.0e-6 * strain / denom) : 0.0;
            double tvx = luy * huz - luz * huy, tvy = luz * hux - lux * huz, tvz = lux * huy - luy * hux;
            double tvm2 = tvx * tvx + tvy * tvy + tvz * tvz;
            double torsionMag = 0.0;
            if (tvm2 > 1.0e-30) {
                double im = 1.0 / std::sqrt(tvm2); tvx *= im; tvy *= im; tvz *= im;
                double dotV = lux * hux + luy * huy + luz * huz;
                if (dotV > 1.0) dotV = 1.0;
                if (dotV < -1.0) dotV = -1.0;
                double ang = accurate_acos(dotV) * RAD2DEG;
                double invBRG = 1.0 / bRG[nB + lever] + 1.0 / bRG[nB + head];
                torsionMag = j1FracMoveTorq * DEG2RAD * (ang - j1Rest) / (invBRG * dt);
                double maxMag = stallPN * 0.5 * hlen * 1.0e-18;
                if (torsionMag > maxMag) torsionMag = maxMag;
            }
            if (role == 1) {
                double Fx = -forceMag * lx, Fy = -forceMag * ly, Fz = -forceMag * lz;
                fx += Fx; fy += Fy; fz += Fz;
                double Rs = 0.5e-6 * llen * j1FracR, Rx = Rs * lux, Ry = Rs * luy, Rz = Rs * luz;
                tx += Ry * Fz - Rz * Fy; ty += Rz * Fx - Rx * Fz; tz += Rx * Fy - Ry * Fx;
                tx += tvx * torsionMag; ty += tvy * torsionMag; tz += tvz * torsionMag;
            } else {
                double Fx = forceMag * lx, Fy = forceMag * ly, Fz = forceMag * lz;
                fx += Fx; fy += Fy; fz += Fz;
                double Rs = -0.5e-6 * hlen * j1FracR, Rx = Rs * hux, Ry = Rs * huy, Rz = Rs * huz;
                tx += Ry * Fz - Rz * Fy; ty += Rz * Fx - Rx * Fz; tz += Rx * Fy - Ry * Fx;
                tx -= tvx * torsionMag; ty -= tvy * torsionMag; tz -= tvz * torsionMag;
            }
        }
        F[s] = (float)(F[s] + fx);
        F[nB + s] = (float)(F[nB + s] + fy);
        F[2 * nB + s] = (float)(F[2 * nB + s] + fz);
        T[s] = (float)(T[s] + tx);
        T[nB + s] = (float)(T[nB + s] + ty);
        T[2 * nB + s] = (float)(T[2 * nB + s] + tz);
    }
}

// ============================================================================
// DimerCouplingSystem.java:83-184
// dimerParams: [0]=dt [1]=rodFracMove [2]=leverFracMoveTorq [3]=leverDeg [4]=rodLen
// ============================================================================
EXPORT void orc_dimer_couple(i32 nB, const float* coord, const float* uVec, const float* segLength,
                             const float* bTG, const float* bRG, float* F, float* T, i32 nD,
                             const i32* motorA, const i32* motorB, const i32* parallel,
                             const float* dimerParams, const i32* boundSeg) {
    double dt = dimerParams[0], fracMove = dimerParams[1], leverTorq = dimerParams[2];
    double leverDeg = dimerParams[3], rodLen = dimerParams[4];
    PAR for (int d = 0; d < nD; d++) {
        int mA = motorA[d], mB = motorB[d];
        int rodA = 3 * mA, rodB = 3 * mB;
        bool par = parallel[d] != 0;
        for (int variant = 0; variant < 2; variant++) {
            double endSelA = (variant == 0) ? -1.0 : 1.0;
            double endSelB = par ? endSelA : -endSelA;
            double aCx = coord[rodA], aCy = coord[nB + rodA], aCz = coord[2 * nB + rodA];
            double aUx = uVec[rodA], aUy = uVec[nB + rodA], aUz = uVec[2 * nB + rodA];
            double bCx = coord[rodB], bCy = coord[nB + rodB], bCz = coord[2 * nB + rodB];
            double bUx = uVec[rodB], bUy = uVec[nB + rodB], bUz = uVec[2 * nB + rodB];
            double aLen = segLength[rodA], bLen = segLength[rodB];
            double pAx = aCx + endSelA * 0.5 * aLen * aUx, pAy = aCy + endSelA * 0.5 * aLen * aUy, pAz = aCz + endSelA * 0.5 * aLen * aUz;
            double pBx = bCx + endSelB * 0.5 * bLen * bUx, pBy = bCy + endSelB * 0.5 * bLen * bUy, pBz = bCz + endSelB * 0.5 * bLen * bUz;
            double dx = pBx - pAx, dy = pBy - pAy, dz = pBz - pAz;
            double strain = std::sqrt(dx * dx + dy * dy + dz * dz);
            if (strain > 0.0) {
                double inv = 1.0 / strain;
                double lx = dx * inv, ly = dy * inv, lz = dz * inv;
                double mcA = move_c(aUx, aUy, aUz, lx, ly, lz, bTG[rodA], bTG[nB + rodA], bRG[nB + rodA], aLen);
                double mcB = move_c(bUx, bUy, bUz, lx, ly, lz, bTG[rodB], bTG[nB + rodB], bRG[nB + rodB], bLen);
                double denom = dt * (mcA + mcB);
                double forceMag = (denom > 0.0) ? (fracMove * 1.0e-6 * strain / denom) : 0.0;
                double FAx = forceMag * lx, FAy = forceMag * ly, FAz = forceMag * lz;
                double RsA = 0.5e-6 * rodLen * endSelA;
                double TAx = (RsA * aUy) * FAz - (RsA * aUz) * FAy;
                double TAy = (RsA * aUz) * FAx - (RsA * aUx) * FAz;
                double TAz = (RsA * aUx) * FAy - (RsA * aUy) * FAx;
                F[rodA] = (float)(F[rodA] + FAx);
                F[nB + rodA] = (float)(F[nB + rodA] + FAy);
                F[2 * nB + rodA] = (float)(F[2 * nB + rodA] + FAz);
                T[rodA] = (float)(T[rodA] + TAx);
                T[nB + rodA] = (float)(T[nB + rodA] + TAy);
                T[2 * nB + rodA] = (float)(T[2 * nB + rodA] + TAz);
                double RsB = 0.5e-6 * rodLen * endSelB;
                double TBx = (RsB * bUy) * (-FAz) - (RsB * bUz) * (-FAy);
                double TBy = (RsB * bUz) * (-FAx) - (RsB * bUx) * (-FAz);
                double TBz = (RsB * bUx) * (-FAy) - (RsB * bUy) * (-FAx);
                F[rodB] = (float)(F[rodB] - FAx);
                F[nB + rodB] = (float)(F[nB + rodB] - FAy);
                F[2 * nB + rodB] = (float)(F[2 * nB + rodB] - FAz);
                T[rodB] = (float)(T[rodB] + TBx);
                T[nB + rodB] = (float)(T[nB + rodB] + TBy);
                T[2 * nB + rodB] = (float)(T[2 * nB + rodB] + TBz);
            }
        }
        bool bothBound = boundSeg[mA] >= 0 && boundSeg[mB] >= 0;
        if (par && !bothBound) {
            int leverA = 3 * mA + 1, leverB = 3 * mB + 1;
            double u1x = uVec[leverA], u1y = uVec[nB + leverA], u1z = uVec[2 * nB + leverA];
            double u2x = uVec[leverB], u2y = uVec[nB + leverB], u2z = uVec[2 * nB + leverB];
            double tvx = u1y * u2z - u1z * u2y, tvy = u1z * u2x - u1x * u2z, tvz = u1x * u2y - u1y * u2x;
            double tvm2 = tvx * tvx + tvy * tvy + tvz * tvz;
            if (tvm2 > 1.0e-30) {
                double im = 1.0 / std::sqrt(tvm2); tvx *= im; tvy *= im; tvz *= im;
                double dot = u1x * u2x + u1y * u2y + u1z * u2z;
                if (dot > 1.0) dot = 1.0;
                if (dot < -1.0) dot = -1.0;
                double ang = accurate_acos(dot) * 180.0 / PI_D;
                double invBRG = 1.0 / bRG[nB + leverA] + 1.0 / bRG[nB + leverB];
                double torsionMag = leverTorq * (PI_D / 180.0) * (ang - leverDeg) / (invBRG * dt);
                T[leverA] = (float)(T[leverA] + tvx * torsionMag);
                T[nB + leverA] = (float)(T[nB + leverA] + tvy * torsionMag);
                T[2 * nB + leverA] = (float)(T[2 * nB + leverA] + tvz * torsionMag);
                T[leverB] = (float)(T[leverB] - tvx * torsionMag);
                T[nB + leverB] = (float)(T[nB + leverB] - tvy * torsionMag);
                T[2 * nB + leverB] = (float)(T[2 * nB + leverB] - tvz * torsionMag);
            }
        }
    }
}

// ============================================================================
// MiniFilamentSystem.java:65-172; miniParams: [0]=dt [1]=fracMove [2]=align
// ============================================================================
EXPORT void orc_mini_tether(i32 nMB, const float* mC, const float* mU, const float* mLen, const float* mBTG,
                            const float* mBRG, float* mF, float* mT, i32 nBb, const float* bbC,
                            const float* bbU, const float* bbInvDragY, i32 nD, const i32* headBackboneSlot,
                            const i32* motorA, const float* attachAxial, float* miniData,
                            const float* miniParams) {
    double dt = miniParams[0], fracMove = miniParams[1], align = miniParams[2];
    PAR for (int d = 0; d < nD; d++) {
        int bb = headBackboneSlot[d];
        int rodA = 3 * motorA[d];
        double ax = attachAxial[d];
        double bcx = bbC[bb], bcy = bbC[nBb + bb], bcz = bbC[2 * nBb + bb];
        double bux = bbU[bb], buy = bbU[nBb + bb], buz = bbU[2 * nBb + bb];
        double pax = bcx + ax * bux, pay = bcy + ax * buy, paz = bcz + ax * buz;
        double rcx = mC[rodA], rcy = mC[nMB + rodA], rcz = mC[2 * nMB + rodA];
        double rux = mU[rodA], ruy = mU[nMB + rodA], ruz = mU[2 * nMB + rodA];
        double rlen = mLen[rodA];
        double re1x = rcx - 0.5 * rlen * rux, re1y = rcy - 0.5 * rlen * ruy, re1z = rcz - 0.5 * rlen * ruz;
        double fbx = 0, fby = 0, fbz = 0, tbx = 0, tby = 0, tbz = 0;
        double dx = pax - re1x, dy = pay - re1y, dz = paz - re1z;
        double strain = std::sqrt(dx * dx + dy * dy + dz * dz);
        if (strain > 0.0) {
            double inv = 1.0 / strain;
            double lx = dx * inv, ly = dy * inv, lz = dz * inv;
            double denom = dt * (1.0 / mBTG[nMB + rodA] + bbInvDragY[bb]);
            double forceMag = (denom > 0.0) ? (fracMove * 1.0e-6 * strain / denom) : 0.0;
            double Frx = forceMag * lx, Fry = forceMag * ly, Frz = forceMag * lz;
            mF[rodA] = (float)(mF[rodA] + Frx);
            mF[nMB + rodA] = (float)(mF[nMB + rodA] + Fry);
            mF[2 * nMB + rodA] = (float)(mF[2 * nMB + rodA] + Frz);
            fbx = -Frx; fby = -Fry; fbz = -Frz;
        }
        double alignSign = (ax < 0.0) ? -1.0 : 1.0;
        double tux = alignSign * bux, tuy = alignSign * buy, tuz = alignSign * buz;
        double tvx = ruy * tuz - ruz * tuy, tvy = ruz * tux - rux * tuz, tvz = rux * tuy - ruy * tux;
        double tvm2 = tvx * tvx + tvy * tvy + tvz * tvz;
        if (tvm2 > 1.0e-30) {
            double im = 1.0 / std::sqrt(tvm2); tvx *= im; tvy *= im; tvz *= im;
            double dot = rux * tux + ruy * tuy + ruz * tuz;
            if (dot > 1.0) dot = 1.0;
            if (dot < -1.0) dot = -1.0;
            double angDeg = accurate_acos(dot) * 180.0 / PI_D;
            double denomR = (1.0 / mBRG[nMB + rodA] + bbInvDragY[nBb + bb]) * dt;
            double tmag = align * (PI_D / 180.0) * angDeg / denomR;
            mT[rodA] = (float)(mT[rodA] + tvx * tmag);
            mT[nMB + rodA] = (float)(mT[nMB + rodA] + tvy * tmag);
            mT[2 * nMB + rodA] = (float)(mT[2 * nMB + rodA] + tvz * tmag);
            tbx = -tvx * tmag; tby = -tvy * tmag; tbz = -tvz * tmag;
        }
        int o = MINI_STRIDE * d;
        miniData[o] = (float)fbx; miniData[o + 1] = (float)fby; miniData[o + 2] = (float)fbz;
        miniData[o + 3] = (float)tbx; miniData[o + 4] = (float)tby; miniData[o + 5] = (float)tbz;
    }
}

EXPORT void orc_backbone_gather(i32 nBb, const i32* offsets, const i32* list, const float* miniData,
                                float* F, float* T) {
    csr_gather(nBb, offsets, list, miniData, MINI_STRIDE, 0, nullptr, F, T);
}

EXPORT void orc_mini_brute_gather(i32 nBb, i32 nD, const i32* headBackboneSlot, const float* miniData,
                                  float* F, float* T) {
    PAR for (int s = 0; s < nBb; s++) {
        double fx = 0, fy = 0, fz = 0, tx = 0, ty = 0, tz = 0;
        for (int d = 0; d < nD; d++) {
            if (headBackboneSlot[d] != s) continue;
            int o = d * MINI_STRIDE;
            fx += miniData[o]; fy += miniData[o + 1]; fz += miniData[o + 2];
            tx += miniData[o + 3]; ty += miniData[o + 4]; tz += miniData[o + 5];
        }
        F[s] = (float)fx; F[nBb + s] = (float)fy; F[2 * nBb + s] = (float)fz;
        T[s] = (float)tx; T[nBb + s] = (float)ty; T[2 * nBb + s] = (float)tz;
    }
}

// ThermostatDiag.java:127-145 (diagnostic torsional restore toward +z; Math.acos = libm)
EXPORT void orc_torsional_restore(i32 nMotors, const float* uVec, const float* bRG, float* T,
                                  double coeff, double dt) {
    int nB = 3 * nMotors;
    for (int m = 0; m < nMotors; m++) {
        int rod = 3 * m;
        double ux = uVec[rod], uy = uVec[nB + rod], uz = uVec[2 * nB + rod];
        double axx = uy, axy = -ux, axz = 0.0;
        double am2 = axx * axx + axy * axy + axz * axz;
        if (am2 <= 1.0e-30) continue;
        double im = 1.0 / std::sqrt(am2); axx *= im; axy *= im; axz *= im;
        double dot = uz; if (dot > 1) dot = 1; if (dot < -1) dot = -1;
        double angDeg = std::acos(dot) * 180.0 / PI_D;
        double invBRG = 1.0 / bRG[nB + rod];
        double tmag = coeff * (PI_D / 180.0) * angDeg / (invBRG * dt);
        T[rod] = (float)(T[rod] + axx * tmag);
        T[nB + rod] = (float)(T[nB + rod] + axy * tmag);
        T[2 * nB + rod] = (float)(T[2 * nB + rod] + axz * tmag);
    }
}

// The portable transcendentals of sbx_math.h, exported for the accuracy tests.
EXPORT double orc_m_log(double x) { return sbxm::log(x); }
EXPORT double orc_m_exp(double x) { return sbxm::exp(x); }
EXPORT double orc_m_sin(double x) { return sbxm::sin(x); }
EXPORT double orc_m_cos(double x) { return sbxm::cos(x); }
// which: 0 log, 1 exp, 2 sin, 3 cos, 4 / 5 the sine / cosine of sbxm::sincos
EXPORT void orc_m_eval(int which, int n, const double* x, double* y) {
    PAR for (int i = 0; i < n; i++) {
        double v = x[i];
        if (which >= 4) {
            double sn, cs;
            sbxm::sincos(v, &sn, &cs);
            y[i] = which == 4 ? sn : cs;
            continue;
        }
        y[i] = which == 0 ? sbxm::log(v) : which == 1 ? sbxm::exp(v) : which == 2 ? sbxm::sin(v) : sbxm::cos(v);
    }
}

// ============================================================================
// Crosslinker formation (CrosslinkerSystem.java:405-756) and the scan-rank free-list
// allocator (CrosslinkerSystem.java:297-345); FormationGrid.java:28-109 builds its grid
// with the SpatialGrid functions above.
// formParams: [0] maxXLinkBondAngle (rad) [1] crossLinkGrabDist^2 [2] minSepBetweenXLinks
//             [3] maxXLinksOnSeg [4] P_form [5] loc jitter half-range [6] crossLinkGrabDist
// formCounts: [0] nCand [1] step [2] seed [3] xLinkMode (0 both, 1 parallel, -1 antiparallel)
// ============================================================================
namespace {
const int FORM_MAXC = 256;   // CrosslinkerSystem.java:457

// the coarse capsule bound of filFilCandidates / gridFormCount (CrosslinkerSystem.java:414-420)
inline bool form_pair_ok(i32 nSeg, const float* coord, const float* segLength, const i32* filID, int i, int j,
                         double cix, double ciy, double ciz, double hi, double grab) {
    if (filID[j] == filID[i]) return false;
    double dx = cix - coord[j], dy = ciy - coord[nSeg + j], dz = ciz - coord[2 * nSeg + j];
    double cd = std::sqrt(dx * dx + dy * dy + dz * dz);
    double bound = hi + 0.5 * segLength[j] + grab;
    return !(cd > bound);
}

inline void form_cell_range(double cix, double ciy, double ciz, const float* gp, const i32* gd, int* lo, int* hi) {
    float xMin = gp[0], yMin = gp[1], zMin = gp[2], invCell = gp[4];
    int n[3] = {gd[0], gd[1], gd[2]};
    int c[3] = {jf2i(((float)cix - xMin) * invCell), jf2i(((float)ciy - yMin) * invCell),
                jf2i(((float)ciz - zMin) * invCell)};
    for (int k = 0; k < 3; k++) {
        if (c[k] < 0) c[k] = 0;
        if (c[k] >= n[k]) c[k] = n[k] - 1;
        lo[k] = c[k] - 1; if (lo[k] < 0) lo[k] = 0;
        hi[k] = c[k] + 1; if (hi[k] >= n[k]) hi[k] = n[k] - 1;
    }
}
}  // namespace

// CrosslinkerSystem.filFilCandidates (CrosslinkerSystem.java:405-427): all distinct
// cross-filament pairs i<j within the coarse bound, lexicographic, capped at reqCap
EXPORT void orc_xl_fil_fil_candidates(i32 nSeg, const float* coord, const float* segLength, const i32* filID,
                                      i32 reqCap, i32* reqFilA, i32* reqFilB, const float* formParams,
                                      i32* formCounts) {
    double grab = formParams[6];
    int c = 0;
    for (int i = 0; i < nSeg; i++) {
        double cix = coord[i], ciy = coord[nSeg + i], ciz = coord[2 * nSeg + i];
        double hi = 0.5 * segLength[i];
        for (int j = i + 1; j < nSeg; j++) {
            if (!form_pair_ok(nSeg, coord, segLength, filID, i, j, cix, ciy, ciz, hi, grab)) continue;
            if (c < reqCap) { reqFilA[c] = i; reqFilB[c] = j; c++; }
        }
    }
    formCounts[0] = c;
    for (int k = c; k < reqCap; k++) { reqFilA[k] = -1; reqFilB[k] = -1; }
}

// CrosslinkerSystem.gridFormCount (CrosslinkerSystem.java:461-512)
EXPORT void orc_xl_grid_form_count(i32 nSeg, const float* coord, const float* segLength, const i32* filID,
                                   const float* gridParams, const i32* gridDims, const i32* offsets,
                                   const i32* contents, i32* candCountSeg, const float* formParams) {
    double grab = formParams[6];
    int nX = gridDims[0], nY = gridDims[1], nXY = nX * nY;
    (void)nY;
    PAR for (int i = 0; i < nSeg; i++) {
        double cix = coord[i], ciy = coord[nSeg + i], ciz = coord[2 * nSeg + i];
        double hi = 0.5 * segLength[i];
        int lo[3], up[3];
        form_cell_range(cix, ciy, ciz, gridParams, gridDims, lo, up);
        int cnt = 0;
        for (int zz = lo[2]; zz <= up[2]; zz++)
            for (int yy = lo[1]; yy <= up[1]; yy++)
                for (int xx = lo[0]; xx <= up[0]; xx++) {
                    int cc = xx + yy * nX + zz * nXY;
                    for (int idx = offsets[cc]; idx < offsets[cc + 1]; idx++) {
                        int j = contents[idx];
                        if (j <= i) continue;
                        if (!form_pair_ok(nSeg, coord, segLength, filID, i, j, cix, ciy, ciz, hi, grab)) continue;
                        cnt++;
                    }
                }
        candCountSeg[i] = cnt < FORM_MAXC ? cnt : FORM_MAXC;
    }
}

// CrosslinkerSystem.gridFormScan (CrosslinkerSystem.java:516-528)
EXPORT void orc_xl_grid_form_scan(i32 nSeg, const i32* candCountSeg, i32* candBaseSeg, i32 reqCap, i32* reqFilA,
                                  i32* reqFilB, i32* formCounts) {
    int acc = 0;
    for (int s = 0; s < nSeg; s++) { candBaseSeg[s] = acc; acc += candCountSeg[s]; }
    candBaseSeg[nSeg] = acc;
    int total = acc < reqCap ? acc : reqCap;
    formCounts[0] = total;
    for (int k = total; k < reqCap; k++) { reqFilA[k] = -1; reqFilB[k] = -1; }
}

// CrosslinkerSystem.gridFormEmit (CrosslinkerSystem.java:535-602): partners ascending in
// each segment's owned region; a full region keeps the smallest FORM_MAXC
EXPORT void orc_xl_grid_form_emit(i32 nSeg, const float* coord, const float* segLength, const i32* filID,
                                  const float* gridParams, const i32* gridDims, const i32* offsets,
                                  const i32* contents, const i32* candBaseSeg, const i32* candCountSeg, i32 reqCap,
                                  i32* reqFilA, i32* reqFilB, const float* formParams) {
    double grab = formParams[6];
    int nX = gridDims[0], nXY = nX * gridDims[1];
    PAR for (int i = 0; i < nSeg; i++) {
        int base = candBaseSeg[i];
        int cap = candCountSeg[i];
        if (base >= reqCap) cap = 0;
        else if (base + cap > reqCap) cap = reqCap - base;
        if (cap <= 0) continue;
        double cix = coord[i], ciy = coord[nSeg + i], ciz = coord[2 * nSeg + i];
        double hi = 0.5 * segLength[i];
        int lo[3], up[3];
        form_cell_range(cix, ciy, ciz, gridParams, gridDims, lo, up);
        int cnt = 0;
        for (int zz = lo[2]; zz <= up[2]; zz++)
            for (int yy = lo[1]; yy <= up[1]; yy++)
                for (int xx = lo[0]; xx <= up[0]; xx++) {
                    int cc = xx + yy * nX + zz * nXY;
                    for (int idx = offsets[cc]; idx < offsets[cc + 1]; idx++) {
                        int j = contents[idx];
                        if (j <= i) continue;
                        if (!form_pair_ok(nSeg, coord, segLength, filID, i, j, cix, ciy, ciz, hi, grab)) continue;
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
}

// CrosslinkerSystem.formGates (CrosslinkerSystem.java:607-675)
EXPORT void orc_xl_form_gates(i32 nSeg, const float* fU, const float* fE1, const float* fE2, const float* segLength,
                              i32 reqCap, const i32* reqFilA, const i32* reqFilB, float* reqLoc1, float* reqLoc2,
                              i32* reqOrient, i32* gatePass, const float* formParams, const i32* formCounts) {
    i32 step = formCounts[1], seed = formCounts[2], mode = formCounts[3];
    double maxAngle = formParams[0], grabSq = formParams[1];
    double pForm = formParams[4], jit = formParams[5];
    PAR for (int c = 0; c < reqCap; c++) {
        gatePass[c] = 0; reqOrient[c] = 0;
        int a = reqFilA[c], b = reqFilB[c];
        if (a < 0 || b < 0) continue;
        double uax = fU[a], uay = fU[nSeg + a], uaz = fU[2 * nSeg + a];
        double ubx = fU[b], uby = fU[nSeg + b], ubz = fU[2 * nSeg + b];
        double dot = uax * ubx + uay * uby + uaz * ubz;
        double angT = fast_acos(dot), angTR = fast_acos(-dot);
        bool alignOk;
        if (mode == 1) alignOk = angT <= maxAngle;
        else if (mode == -1) alignOk = angTR <= maxAngle;
        else alignOk = (angT <= maxAngle) || (angTR <= maxAngle);
        if (!alignOk) continue;
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
        if (r4x < smallNum && r4y < smallNum && r4z < smallNum) continue;
        double denom = r4x * r4x + r4y * r4y + r4z * r4z;
        double c32x = r3y * r2z - r3z * r2y, c32y = r3z * r2x - r3x * r2z, c32z = r3x * r2y - r3y * r2x;
        double alpha = (r4x * c32x + r4y * c32y + r4z * c32z) / denom;
        if (alpha < 0.0 || alpha > 1.0) continue;
        double c31x = r3y * r1z - r3z * r1y, c31y = r3z * r1x - r3x * r1z, c31z = r3x * r1y - r3y * r1x;
        double beta = (r4x * c31x + r4y * c31y + r4z * c31z) / denom;
        if (beta < 0.0 || beta > 1.0) continue;
        double p1x = e1ax + alpha * r1x, p1y = e1ay + alpha * r1y, p1z = e1az + alpha * r1z;
        double p2x = e1bx + beta * r2x, p2y = e1by + beta * r2y, p2z = e1bz + beta * r2z;
        double ddx = p1x - p2x, ddy = p1y - p2y, ddz = p1z - p2z;
        double conDistSq = ddx * ddx + ddy * ddy + ddz * ddz;
        if (conDistSq >= grabSq) continue;
        uint32_t base = sbxm::rng_base(c, step, seed);
        double da = std::sqrt((p1x - e1ax) * (p1x - e1ax) + (p1y - e1ay) * (p1y - e1ay) + (p1z - e1az) * (p1z - e1az));
        double db = std::sqrt((p2x - e1bx) * (p2x - e1bx) + (p2y - e1by) * (p2y - e1by) + (p2z - e1bz) * (p2z - e1bz));
        float uj1 = sbxm::unit_from_hash(sbxm::wang_hash(base ^ 0x584C4A31u));
        float uj2 = sbxm::unit_from_hash(sbxm::wang_hash(base ^ 0x584C4A32u));
        double loc1 = da + (2.0 * uj1 - 1.0) * jit;
        double loc2 = db + (2.0 * uj2 - 1.0) * jit;
        double lenA = segLength[a], lenB = segLength[b];
        if (loc1 > lenA) loc1 = lenA;
        if (loc1 < 0.0) loc1 = 0.0;
        if (loc2 > lenB) loc2 = lenB;
        if (loc2 < 0.0) loc2 = 0.0;
        reqLoc1[c] = (float)loc1; reqLoc2[c] = (float)loc2;
        float up = sbxm::unit_from_hash(sbxm::wang_hash(base ^ 0x584C4650u));
        if (up < pForm) gatePass[c] = 1;
    }
}

// CrosslinkerSystem.formAdmitReduce (CrosslinkerSystem.java:680-691)
EXPORT void orc_xl_form_admit_reduce(i32 reqCap, const i32* reqFilA, const i32* reqFilB, const i32* gatePass,
                                     i32 nSeg, i32* minCand) {
    for (int s = 0; s < nSeg; s++) minCand[s] = reqCap;
    for (int c = 0; c < reqCap; c++) {
        if (gatePass[c] == 0) continue;
        int a = reqFilA[c], b = reqFilB[c];
        if (c < minCand[a]) minCand[a] = c;
        if (c < minCand[b]) minCand[b] = c;
    }
}

// CrosslinkerSystem.formAdmit (CrosslinkerSystem.java:713-738)
EXPORT void orc_xl_form_admit(i32 reqCap, const i32* reqFilA, const i32* reqFilB, const float* reqLoc1,
                              const float* reqLoc2, const i32* gatePass, const i32* minCand,
                              const i32* activeLinkCount, i32 nLinks, const i32* linkState, const i32* linkFilA,
                              const i32* linkFilB, const float* loc1, const float* loc2, i32* acceptFlag,
                              const float* formParams) {
    double minSep = formParams[2];
    int maxLinks = jf2i(formParams[3]);
    PAR for (int c = 0; c < reqCap; c++) {
        acceptFlag[c] = 0;
        if (gatePass[c] == 0) continue;
        int segA = reqFilA[c], segB = reqFilB[c];
        if (minCand[segA] != c || minCand[segB] != c) continue;
        if (activeLinkCount[segA] >= maxLinks || activeLinkCount[segB] >= maxLinks) continue;
        double la = reqLoc1[c], lb = reqLoc2[c];
        bool ok = true;
        for (int L = 0; L < nLinks; L++) {
            if (linkState[L] < 0) continue;
            int fa = linkFilA[L], fb = linkFilB[L];
            if (fa == segA && std::fabs(la - loc1[L]) < minSep) ok = false;
            if (fb == segA && std::fabs(la - loc2[L]) < minSep) ok = false;
            if (fa == segB && std::fabs(lb - loc1[L]) < minSep) ok = false;
            if (fb == segB && std::fabs(lb - loc2[L]) < minSep) ok = false;
        }
        if (ok) acceptFlag[c] = 1;
    }
}

// CrosslinkerSystem.freeFlags (:297-302), CrossBridgeSystem.csrScan, freeScatter (:306-314)
EXPORT void orc_xl_free_flags(i32 C, const i32* linkState, i32* freeCount) {
    for (int s = 0; s < C; s++) freeCount[s] = linkState[s] < 0 ? 1 : 0;
}
EXPORT void orc_xl_free_scatter(i32 C, const i32* linkState, const i32* freeOffsets, i32* freeList) {
    for (int s = 0; s < C; s++)
        if (linkState[s] < 0) freeList[freeOffsets[s]] = s;
}

// CrosslinkerSystem.allocate (:322-341) then placeOrient (:740-752)
EXPORT void orc_xl_allocate(i32 K, const i32* reqFilA, const i32* reqFilB, const float* reqLoc1,
                            const float* reqLoc2, const i32* rankOffsets, const i32* freeList,
                            const i32* freeOffsets, i32 C, i32* linkFilA, i32* linkFilB, float* loc1, float* loc2,
                            i32* linkState, float* strainHist, i32* strainPlace) {
    int nFree = freeOffsets[C];
    for (int r = 0; r < K; r++) {
        int rank = rankOffsets[r];
        bool accepted = rankOffsets[r + 1] > rank;
        if (!accepted) continue;
        if (rank >= nFree) continue;
        int slot = freeList[rank];
        linkFilA[slot] = reqFilA[r];
        linkFilB[slot] = reqFilB[r];
        loc1[slot] = reqLoc1[r];
        loc2[slot] = reqLoc2[r];
        int base = slot * STRAIN_WIN;
        for (int j = 0; j < STRAIN_WIN; j++) strainHist[base + j] = 0.f;
        strainPlace[slot] = 0;
        linkState[slot] = LINK_ACTIVE;
    }
}
EXPORT void orc_xl_place_orient(i32 K, const i32* reqOrient, const i32* rankOffsets, const i32* freeList,
                                const i32* freeOffsets, i32 C, i32* linkOrientSame, float* torqueMagHist,
                                i32* torqueMagPlace) {
    int nFree = freeOffsets[C];
    for (int r = 0; r < K; r++) {
        int rank = rankOffsets[r];
        if (rankOffsets[r + 1] <= rank) continue;
        if (rank >= nFree) continue;
        int slot = freeList[rank];
        linkOrientSame[slot] = reqOrient[r];
        torqueMagPlace[slot] = 0;
        int b = slot * TORQUE_WIN;
        for (int j = 0; j < TORQUE_WIN; j++) torqueMagHist[b + j] = 0.f;
    }
}

// ============================================================================
// Actin turnover: GrowthSystem.java:73-229, DepolySystem.java:70-189,
// SeveringSystem.java:37-99, FilamentBirthSystem.java:41-88, AgingSystem.java:40-125,
// FilIDSystem.java:38-59. Per-slot decisions are integer/wang-hash; poses float/double as
// the Java source. `C` = the filament slot capacity; counts[1] = step, [2] = seed, [3] = fires.
// ============================================================================
namespace {
const int FIL_FREE = -1, FIL_ACTIVE = 0;   // FilamentStore.java:112-113
inline float turnover_unit(int s, i32 step, i32 seed, uint32_t salt) {
    return sbxm::unit_from_hash(sbxm::wang_hash(sbxm::rng_base(s, step, seed) ^ salt));
}
}  // namespace

// GrowthSystem.grow (:73-104)
EXPORT void orc_growth_grow(i32 C, const i32* seedNode, i32* monomerCount, float* coord, const float* uVec,
                            i32* grewFlag, const float* growParams, const i32* growCounts) {
    i32 fires = growCounts[3], step = growCounts[1], seed = growCounts[2];
    float P = growParams[0], halfmono = growParams[1];
    int maxMon = jf2i(growParams[2]);
    for (int s = 0; s < C; s++) {
        grewFlag[s] = 0;
        if (fires == 0) continue;
        if (seedNode[s] < 0) continue;
        if (monomerCount[s] >= maxMon) continue;
        float u = turnover_unit(s, step, seed, 0x47524F57u);
        if (u >= P) continue;
        monomerCount[s] = monomerCount[s] + 1;
        float ux = uVec[s], uy = uVec[C + s], uz = uVec[2 * C + s];
        coord[s] = coord[s] - 0.5f * halfmono * ux;
        coord[C + s] = coord[C + s] - 0.5f * halfmono * uy;
        coord[2 * C + s] = coord[2 * C + s] - 0.5f * halfmono * uz;
        grewFlag[s] = 1;
    }
}

// GrowthSystem.markSplits (:113-136); RC = request planar stride
EXPORT void orc_growth_mark_splits(i32 C, const i32* seedNode, const i32* monomerCount, const float* coord,
                                   const float* uVec, const float* yVec, i32* acceptFlag, float* reqCoord,
                                   float* reqUVec, float* reqYVec, i32 RC, const float* splitParams,
                                   const i32* growCounts) {
    i32 fires = growCounts[3];
    double halfmono = splitParams[0];
    int splitThresh = jf2i(splitParams[1]), childMon = jf2i(splitParams[2]);
    for (int s = 0; s < C; s++) {
        acceptFlag[s] = 0;
        if (fires == 0) continue;
        if (seedNode[s] < 0) continue;
        int M = monomerCount[s];
        if (M < splitThresh) continue;
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
}

// GrowthSystem.splitWire (:147-190); K requests (request index == parent slot)
EXPORT void orc_growth_split_wire(i32 K, i32 C, const i32* rankOffsets, const i32* freeList, const i32* freeOffsets,
                                  i32* monomerCount, float* coord, const float* uVec, i32* e1s, i32* e1d, i32* e2s,
                                  i32* e2d, i32* seedNode, const float* splitParams) {
    int nFree = freeOffsets[C];
    double halfmono = splitParams[0];
    int childMon = jf2i(splitParams[2]);
    for (int r = 0; r < K; r++) {
        int rank = rankOffsets[r];
        if (!(rankOffsets[r + 1] > rank)) continue;
        if (rank >= nFree) continue;
        int Gs = r, Cs = freeList[rank];
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
}

// GrowthSystem.recomputeDrag (:200-228); dragParams [halfmono, aeta, radius, kT, aPar, aOrth, aTurn, stdSeg, minMon]
EXPORT void orc_growth_recompute_drag(i32 C, const i32* monomerCount, float* segLength, const i32* e1s,
                                      const i32* e2s, float* bTG, float* bRG, float* bTD, float* bRD,
                                      const float* dragParams, const i32* growCounts) {
    i32 fires = growCounts[3];
    double halfmono = dragParams[0], aeta = dragParams[1], radius = dragParams[2], kT = dragParams[3];
    double aPar = dragParams[4], aOrth = dragParams[5], aTurn = dragParams[6];
    int stdSeg = jf2i(dragParams[7]), minMon = jf2i(dragParams[8]);
    PAR for (int i = 0; i < C; i++) {
        if (fires == 0) continue;
        int mc = monomerCount[i];
        double length = (mc + 1) * halfmono;
        segLength[i] = (float)length;
        bool atEnd = (e1s[i] < 0) || (e2s[i] < 0);
        double minLength = (atEnd ? stdSeg : minMon) * halfmono;
        double asIf = length < minLength ? minLength : length;
        double LM = 1.0e-6 * asIf, RM = radius * 1.0e-6;
        double logT = JLOG(LM / (2.0 * RM));
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
}

// DepolySystem.depoly (:70-101) and depolyProxy (:113-145); rate = NULL for the fixed-rate form
static void depoly_impl(i32 C, const i32* filState, i32* monomerCount, float* coord, const float* uVec,
                        const i32* e1s, const float* nucFrac, i32* returnedMon, i32* deathFlag,
                        const float* depolyParams, const float* rateParams, const i32* depolyCounts) {
    i32 fires = depolyCounts[3], step = depolyCounts[1], seed = depolyCounts[2];
    float halfmono = depolyParams[1];
    int floorM = jf2i(depolyParams[2]);
    for (int s = 0; s < C; s++) {
        returnedMon[s] = 0;
        deathFlag[s] = 0;
        if (fires == 0) continue;
        if (filState[s] < 0) continue;
        if (e1s[s] >= 0) continue;
        int M = monomerCount[s];
        float P;
        if (rateParams) {
            float adp = nucFrac[2 * C + s];
            P = rateParams[0] * (1.0f - adp) + rateParams[1] * adp;
        } else {
            P = depolyParams[0];
        }
        if (M >= floorM) {
            float u = turnover_unit(s, step, seed, 0x4445504Fu);
            if (u >= P) continue;
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
}
EXPORT void orc_depoly(i32 C, const i32* filState, i32* monomerCount, float* coord, const float* uVec, const i32* e1s,
                       i32* returnedMon, i32* deathFlag, const float* depolyParams, const i32* depolyCounts) {
    depoly_impl(C, filState, monomerCount, coord, uVec, e1s, nullptr, returnedMon, deathFlag, depolyParams, nullptr,
                depolyCounts);
}
EXPORT void orc_depoly_proxy(i32 C, const i32* filState, i32* monomerCount, float* coord, const float* uVec,
                             const i32* e1s, const float* nucFrac, i32* returnedMon, i32* deathFlag,
                             const float* depolyParams, const float* rateParams, const i32* depolyCounts) {
    depoly_impl(C, filState, monomerCount, coord, uVec, e1s, nucFrac, returnedMon, deathFlag, depolyParams, rateParams,
                depolyCounts);
}

// DepolySystem.applyDeath (:155-188), serial
EXPORT void orc_apply_death(i32 C, i32* filState, i32* monomerCount, i32* seedNode, i32* e1s, i32* e1d, i32* e2s,
                            i32* e2d, float* bTS, float* bRS, const i32* deathFlag) {
    for (int s = 0; s < C; s++) {
        if (deathFlag[s] == 0) continue;
        filState[s] = FIL_FREE;
        bTS[s] = 0.f;
        bRS[s] = 0.f;
        monomerCount[s] = 0;
        int n2 = e2s[s], n2side = e2d[s];
        if (n2 >= 0) {
            if (n2side == 0) { e1s[n2] = -1; e1d[n2] = -1; }
            else { e2s[n2] = -1; e2d[n2] = -1; }
            e2s[s] = -1; e2d[s] = -1;
        }
        int n1 = e1s[s], n1side = e1d[s];
        if (n1 >= 0) {
            if (n1side == 0) { e1s[n1] = -1; e1d[n1] = -1; }
            else { e2s[n1] = -1; e2d[n1] = -1; }
            e1s[s] = -1; e1d[s] = -1;
        }
        if (seedNode[s] >= 0) seedNode[s] = -1;
    }
}

// SeveringSystem.cofilinAccumulate (:37-49), cofilinDissolve (:58-74), nucleateFreshCofilin (:87-98)
EXPORT void orc_cofilin_accumulate(i32 C, const i32* filState, const float* nucFrac, float* cofFrac,
                                   const float* cofilinParams, const i32* severCounts) {
    i32 fires = severCounts[1];
    float pCof = cofilinParams[0];
    for (int s = 0; s < C; s++) {
        if (fires == 0) continue;
        if (filState[s] < 0) continue;
        float fADP = nucFrac[2 * C + s], fCof = cofFrac[s];
        cofFrac[s] = fCof + (fADP - fCof) * pCof;
    }
}
EXPORT void orc_cofilin_dissolve(i32 C, const i32* filState, const i32* monomerCount, const float* cofFrac,
                                 i32* severDeathFlag, i32* severReturnedMon, const float* cofilinParams,
                                 const i32* severCounts) {
    i32 fires = severCounts[1];
    float ratio = cofilinParams[1];
    for (int s = 0; s < C; s++) {
        severDeathFlag[s] = 0;
        severReturnedMon[s] = 0;
        if (fires == 0) continue;
        if (filState[s] < 0) continue;
        if (cofFrac[s] > ratio) { severDeathFlag[s] = 1; severReturnedMon[s] = monomerCount[s]; }
    }
}
// the accepted-rank -> slot pattern of the allocator companions (rank < nFree)
static inline int alloc_slot(int r, const i32* rankOffsets, const i32* freeList, int nFree) {
    int rank = rankOffsets[r];
    if (!(rankOffsets[r + 1] > rank) || rank >= nFree) return -1;
    return freeList[rank];
}
EXPORT void orc_nucleate_fresh_cofilin(i32 K, i32 C, const i32* rankOffsets, const i32* freeList,
                                       const i32* freeOffsets, float* cofFrac) {
    int nFree = freeOffsets[C];
    for (int r = 0; r < K; r++) {
        int slot = alloc_slot(r, rankOffsets, freeList, nFree);
        if (slot >= 0) cofFrac[slot] = 0.f;
    }
}

// FilamentBirthSystem.allocate (:61-87); freeFlags/freeScatter = orc_xl_free_flags/_scatter on filState
EXPORT void orc_birth_allocate(i32 K, i32 C, i32 RC, const float* reqCoord, const float* reqUVec, const float* reqYVec,
                               const i32* rankOffsets, const i32* freeList, const i32* freeOffsets, float* coord,
                               float* uVec, float* yVec, float* bTS, float* bRS, i32* filState,
                               const float* birthParams) {
    int nFree = freeOffsets[C];
    float bt = birthParams[0], br = birthParams[1];
    for (int r = 0; r < K; r++) {
        int slot = alloc_slot(r, rankOffsets, freeList, nFree);
        if (slot < 0) continue;
        for (int k = 0; k < 3; k++) {
            coord[k * C + slot] = reqCoord[k * RC + r];
            uVec[k * C + slot] = reqUVec[k * RC + r];
            yVec[k * C + slot] = reqYVec[k * RC + r];
        }
        bTS[slot] = bt;
        bRS[slot] = br;
        filState[slot] = FIL_ACTIVE;
    }
}

// AgingSystem.age (:40-57), growthAtp (:65-77), splitInheritNuc (:88-102), nucleateFreshAtp (:114-125)
EXPORT void orc_aging_age(i32 C, const i32* filState, float* nucFrac, const float* agingParams,
                          const i32* agingCounts) {
    i32 fires = agingCounts[1];
    float pH = agingParams[0], pD = agingParams[1];
    for (int s = 0; s < C; s++) {
        if (fires == 0) continue;
        if (filState[s] < 0) continue;
        float fATP = nucFrac[s], fADPPi = nucFrac[C + s];
        float nATP = fATP * (1.0f - pH);
        float nADPPi = fADPPi * (1.0f - pD) + fATP * pH;
        float nADP = 1.0f - nATP - nADPPi;
        nucFrac[s] = nATP; nucFrac[C + s] = nADPPi; nucFrac[2 * C + s] = nADP;
    }
}
EXPORT void orc_aging_growth_atp(i32 C, const i32* grewFlag, const i32* monomerCount, float* nucFrac) {
    for (int s = 0; s < C; s++) {
        if (grewFlag[s] == 0) continue;
        int M = monomerCount[s];
        if (M <= 0) continue;
        float w = (float)(M - 1) / (float)M;
        float inv = 1.0f / (float)M;
        nucFrac[s] = nucFrac[s] * w + inv;
        nucFrac[C + s] = nucFrac[C + s] * w;
        nucFrac[2 * C + s] = nucFrac[2 * C + s] * w;
    }
}
EXPORT void orc_aging_split_inherit_nuc(i32 K, i32 C, const i32* rankOffsets, const i32* freeList,
                                        const i32* freeOffsets, float* nucFrac) {
    int nFree = freeOffsets[C];
    for (int r = 0; r < K; r++) {
        int Cs = alloc_slot(r, rankOffsets, freeList, nFree);
        if (Cs < 0) continue;
        int Gs = r;
        nucFrac[Cs] = nucFrac[Gs]; nucFrac[C + Cs] = nucFrac[C + Gs]; nucFrac[2 * C + Cs] = nucFrac[2 * C + Gs];
    }
}
EXPORT void orc_aging_nucleate_fresh_atp(i32 K, i32 C, const i32* rankOffsets, const i32* freeList,
                                         const i32* freeOffsets, float* nucFrac) {
    int nFree = freeOffsets[C];
    for (int r = 0; r < K; r++) {
        int slot = alloc_slot(r, rankOffsets, freeList, nFree);
        if (slot < 0) continue;
        nucFrac[slot] = 1.0f; nucFrac[C + slot] = 0.f; nucFrac[2 * C + slot] = 0.f;
    }
}

// FilIDSystem.init (:38-47) and one pointer-doubling round, jump (:51-58)
EXPORT void orc_filid_init(i32 n, const i32* filState, const i32* e2s, i32* ptr) {
    for (int seg = 0; seg < n; seg++) {
        if (filState[seg] < 0) { ptr[seg] = -seg - 2; continue; }
        int nx = e2s[seg];
        ptr[seg] = (nx >= 0 && nx != seg && filState[nx] >= 0) ? nx : seg;
    }
}
EXPORT void orc_filid_jump(i32 n, const i32* ptrIn, i32* ptrOut, const i32* filState) {
    for (int seg = 0; seg < n; seg++) {
        if (filState[seg] < 0) { ptrOut[seg] = ptrIn[seg]; continue; }
        ptrOut[seg] = ptrIn[ptrIn[seg]];
    }
}

// ActinPool (ActinPool.java:27-63) as the 32-byte record {conc, uMPerMonomer, totalTaken,
// totalReturned}; put (:49-52) / take (:42-46) of a scan total; GrowthStore.depletePoolForGrows
// (GrowthStore.java:94-99) takes only a positive count.
struct OrcPool { double conc; double uM; int64_t taken; int64_t returned; };
EXPORT void orc_pool_put_total(void* poolp, const i32* offsets, i32 n) {
    OrcPool* p = (OrcPool*)poolp;
    int m = offsets[n];
    p->conc += m * p->uM;
    p->returned += m;
}
EXPORT void orc_pool_take_total(void* poolp, const i32* offsets, i32 n) {
    OrcPool* p = (OrcPool*)poolp;
    int m = offsets[n];
    if (m <= 0) return;
    p->conc -= m * p->uM;
    if (p->conc < 0.0) p->conc = 0.0;
    p->taken += m;
}
// the host prologue of the turnover block (FullSystemDemoHarness.java:648-651): setCounts,
// setFires and GrowthStore.refreshRate (GrowthStore.java:81-91)
EXPORT void orc_turnover_begin(i32 step, i32 seed, i32 fires, double onRate, double bdt, const void* poolp,
                               float* growParams, i32* gc, i32* dc, i32* ac, i32* sc) {
    const OrcPool* p = (const OrcPool*)poolp;
    if (gc) { gc[1] = step; gc[2] = seed; gc[3] = fires; }
    if (dc) { dc[1] = step; dc[2] = seed; dc[3] = fires; }
    if (ac) ac[1] = fires;
    if (sc) sc[1] = fires;
    if (growParams) {
        double P = fires ? onRate * p->conc * bdt : 0.0;
        growParams[0] = (float)P;
    }
}

// network turnover companions (same rules as the library's entry points of these names)
EXPORT void orc_turnover_release_dead(const i32* filState, i32 nLinks, const i32* linkFilA, const i32* linkFilB,
                                      i32* linkState, i32 nMotors, i32* boundSeg) {
    for (int i = 0; i < nLinks; i++) {
        if (linkState[i] < 0) continue;
        int a = linkFilA[i], b = linkFilB[i];
        if ((a >= 0 && filState[a] < 0) || (b >= 0 && filState[b] < 0)) linkState[i] = -1;
    }
    for (int m = 0; m < nMotors; m++) {
        int sg = boundSeg[m];
        if (sg >= 0 && filState[sg] < 0) boundSeg[m] = -1;
    }
}
EXPORT void orc_birth_emit_constant_actin(i32 reqCap, const void* poolp, const float* bp, i32 step, i32 seed,
                                          i32* accept, float* reqCoord, float* reqUVec, float* reqYVec) {
    const OrcPool* p = (const OrcPool*)poolp;
    long long deficit = p->returned - p->taken;
    int seedMon = jf2i(bp[3]);
    long long K = (deficit > 0 && seedMon > 0) ? deficit / seedMon : 0;
    for (int r = 0; r < reqCap; r++) {
        if (r >= K) { accept[r] = 0; continue; }
        accept[r] = 1;
        float ux = turnover_unit(r, step, seed, 0x42495231u), uy = turnover_unit(r, step, seed, 0x42495232u);
        float uz = turnover_unit(r, step, seed, 0x42495233u), ua = turnover_unit(r, step, seed, 0x42495234u);
        reqCoord[r] = (float)((2.0 * ux - 1.0) * bp[0]);
        reqCoord[reqCap + r] = (float)((2.0 * uy - 1.0) * bp[1]);
        reqCoord[2 * reqCap + r] = (float)((2.0 * uz - 1.0) * bp[2]);
        double th = 2.0 * PI_D * ua, c = JCOS(th), sn = JSIN(th);
        reqUVec[r] = (float)c; reqUVec[reqCap + r] = (float)sn; reqUVec[2 * reqCap + r] = 0.f;
        reqYVec[r] = (float)(-sn); reqYVec[reqCap + r] = (float)c; reqYVec[2 * reqCap + r] = 0.f;
    }
}
// NodeNucleationSystem.initNewborn (NodeNucleationSystem.java:228-244), tagSeeds (:95-106)
EXPORT void orc_birth_init_newborn(i32 K, i32 C, const i32* rankOffsets, const i32* freeList, const i32* freeOffsets,
                                   i32* monomerCount, float* segLength, const float* seedParams) {
    int nFree = freeOffsets[C];
    for (int r = 0; r < K; r++) {
        int slot = alloc_slot(r, rankOffsets, freeList, nFree);
        if (slot < 0) continue;
        monomerCount[slot] = jf2i(seedParams[0]);
        segLength[slot] = seedParams[1];
    }
}
EXPORT void orc_birth_tag_seeds(i32 K, i32 C, const i32* rankOffsets, const i32* freeList, const i32* freeOffsets,
                                i32* seedNode) {
    int nFree = freeOffsets[C];
    for (int r = 0; r < K; r++) {
        int slot = alloc_slot(r, rankOffsets, freeList, nFree);
        if (slot >= 0) seedNode[slot] = r;
    }
}
EXPORT void orc_pool_take_births(void* poolp, const i32* rankOffsets, i32 K, const i32* freeOffsets, i32 C,
                                 i32 seedMon) {
    OrcPool* p = (OrcPool*)poolp;
    int nb = std::min(rankOffsets[K], freeOffsets[C]);
    if (nb <= 0) return;
    int m = nb * seedMon;
    p->conc -= m * p->uM;
    if (p->conc < 0.0) p->conc = 0.0;
    p->taken += m;
}

// ============================================================================
// Observables (the library's sbx_obs_* entry points): the same FP64 summation order —
// 256 strided partial sums per network, then the fixed tree — and union-find clusters.
// ============================================================================
namespace {
const int OBS_T = 256;
void obs_tree(double* p) {
    for (int s = OBS_T / 2; s > 0; s >>= 1)
        for (int t = 0; t < s; t++) p[t] += p[t + s];
}
inline double obs_c(const float* c, const double* c64, int n, int i, int k) {
    return c64 ? c64[(int64_t)k * n + i] : (double)c[(int64_t)k * n + i];
}
}  // namespace

EXPORT void orc_obs_extent(i32 nNet, const i32* segBase, i32 n, const float* coord, const double* coord64,
                           const i32* filState, double* out) {
    for (int net = 0; net < nNet; net++) {
        int b0 = segBase[net], b1 = segBase[net + 1];
        double pc[OBS_T], px[OBS_T], py[OBS_T], pz[OBS_T];
        for (int t = 0; t < OBS_T; t++) {
            double cnt = 0, sx = 0, sy = 0, sz = 0;
            for (int i = b0 + t; i < b1; i += OBS_T) {
                if (filState && filState[i] < 0) continue;
                cnt += 1.0;
                sx += obs_c(coord, coord64, n, i, 0);
                sy += obs_c(coord, coord64, n, i, 1);
                sz += obs_c(coord, coord64, n, i, 2);
            }
            pc[t] = cnt; px[t] = sx; py[t] = sy; pz[t] = sz;
        }
        obs_tree(pc); obs_tree(px); obs_tree(py); obs_tree(pz);
        double c = pc[0];
        double mx = c > 0 ? px[0] / c : 0.0, my = c > 0 ? py[0] / c : 0.0, mz = c > 0 ? pz[0] / c : 0.0;
        double p2[OBS_T];
        for (int t = 0; t < OBS_T; t++) {
            double s2 = 0;
            for (int i = b0 + t; i < b1; i += OBS_T) {
                if (filState && filState[i] < 0) continue;
                double dx = obs_c(coord, coord64, n, i, 0) - mx;
                double dy = obs_c(coord, coord64, n, i, 1) - my;
                double dz = obs_c(coord, coord64, n, i, 2) - mz;
                s2 += dx * dx + dy * dy + dz * dz;
            }
            p2[t] = s2;
        }
        obs_tree(p2);
        out[2 * net] = c > 0 ? std::sqrt(p2[0] / c) : 0.0;
        out[2 * net + 1] = c;
    }
}

EXPORT void orc_obs_stress(i32 nNet, i32 nSeg, const float* fC, const float* fU, const float* fE1, const float* fLen,
                           const i32* linkBase, const i32* linkA, const i32* linkB, const i32* linkState,
                           const float* loc1, const float* loc2, const float* xd, i32 nMotors, const i32* motBase,
                           const float* mC, const float* mU, const i32* boundSeg, const float* bindArc,
                           const float* bd, double headLen, const float* volume, double* out) {
    int nB = 3 * nMotors;
    for (int net = 0; net < nNet; net++) {
        double p[OBS_T];
        for (int t = 0; t < OBS_T; t++) {
            double w = 0;
            if (linkBase)
                for (int k = linkBase[net] + t; k < linkBase[net + 1]; k += OBS_T) {
                    if (linkState[k] < 0) continue;
                    int a = linkA[k], b = linkB[k];
                    if (a < 0 || b < 0) continue;
                    double l1 = loc1[k], l2 = loc2[k];
                    double rx = (fE1[a] + l1 * fU[a]) - (fE1[b] + l2 * fU[b]);
                    double ry = (fE1[nSeg + a] + l1 * fU[nSeg + a]) - (fE1[nSeg + b] + l2 * fU[nSeg + b]);
                    w += 1.0e-6 * rx * xd[12 * (int64_t)k] + 1.0e-6 * ry * xd[12 * (int64_t)k + 1];
                }
            if (motBase)
                for (int m = motBase[net] + t; m < motBase[net + 1]; m += OBS_T) {
                    int s = boundSeg[m];
                    if (s < 0) continue;
                    int h = 3 * m + 2;
                    double hx = mC[h] + 0.5 * headLen * mU[h], hy = mC[nB + h] + 0.5 * headLen * mU[nB + h];
                    double off = (double)bindArc[m] - 0.5 * fLen[s];
                    double ax = fC[s] + off * fU[s], ay = fC[nSeg + s] + off * fU[nSeg + s];
                    w += 1.0e-6 * (hx - ax) * bd[13 * (int64_t)m] + 1.0e-6 * (hy - ay) * bd[13 * (int64_t)m + 1];
                }
            p[t] = w;
        }
        obs_tree(p);
        out[net] = -p[0] / (2.0 * volume[net] * 1.0e-18);
    }
}

namespace {
int uf_find(std::vector<int>& par, int x) {
    while (par[x] != x) { par[x] = par[par[x]]; x = par[x]; }
    return x;
}
void uf_union(std::vector<int>& par, int a, int b) {
    int ra = uf_find(par, a), rb = uf_find(par, b);
    if (ra == rb) return;
    if (ra < rb) par[rb] = ra; else par[ra] = rb;
}
}  // namespace

EXPORT void orc_obs_clusters(i32 nNet, const i32* segBase, i32 nSeg, const i32* filState, const i32* e2, i32 nLinks,
                             const i32* linkA, const i32* linkB, const i32* linkState, i32 nMotors,
                             const i32* boundSeg, const i32* motorBackbone, i32 nBackbones, i32* label, i32* size,
                             i32* out) {
    int nNode = nSeg + nBackbones;
    std::vector<int> par(nNode);
    for (int i = 0; i < nNode; i++) par[i] = i;
    auto live = [&](int x) { return x >= 0 && (x >= nSeg || !filState || filState[x] >= 0); };
    for (int s = 0; s < nSeg; s++)
        if (live(s) && e2[s] >= 0 && live(e2[s])) uf_union(par, s, e2[s]);
    for (int k = 0; k < nLinks; k++)
        if (linkState[k] >= 0 && live(linkA[k]) && live(linkB[k])) uf_union(par, linkA[k], linkB[k]);
    for (int m = 0; m < nMotors; m++)
        if (boundSeg[m] >= 0 && motorBackbone[m] >= 0 && live(boundSeg[m]))
            uf_union(par, boundSeg[m], nSeg + motorBackbone[m]);
    for (int i = 0; i < nNode; i++) { label[i] = live(i) ? uf_find(par, i) : -1; size[i] = 0; }
    for (int s = 0; s < nSeg; s++) if (label[s] >= 0) size[label[s]]++;
    for (int net = 0; net < nNet; net++) {
        int best = 0, cnt = 0;
        for (int s = segBase[net]; s < segBase[net + 1]; s++) {
            if (label[s] < 0) continue;
            cnt++;
            best = std::max(best, size[label[s]]);
        }
        out[2 * net] = best;
        out[2 * net + 1] = cnt;
    }
}
