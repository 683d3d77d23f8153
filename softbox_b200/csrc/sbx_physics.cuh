// sbx_physics.cuh — per-element device physics of the rigid-rod mechanics path.
//
// Each function evaluates one slot of one reference System method with the same
// sequence of IEEE operations as the Java source (file:line in each comment), so that a
// kernel built from it — compiled with -fmad=false, -prec-div=true, -prec-sqrt=true —
// produces the reference's bits. The per-system kernels (sbx_systems.cu) and the fused
// step kernels (sbx_dense.cu, sbx_free.cu) both call these functions, which is what
// makes a fused step bit-identical to the per-system sequence.
#pragma once
#include <stdint.h>
#include "sbx_math.h"
#include "../../include/softbox_b200.h"

#define SBX_DEV __device__ __forceinline__
// functions with many call sites in one kernel (SBX_SHARE_CALLS: one out-of-line copy)
#if defined(SBX_SHARE_CALLS)
#define SBX_DEV_CALL static __device__ __noinline__
#else
#define SBX_DEV_CALL SBX_DEV
#endif

namespace sbx {

constexpr int MAX_CAND = 256;
constexpr int XB_STRIDE = 13, XL_STRIDE = 12, MINI_STRIDE = 6;
constexpr int STRAIN_WIN = 10, TORQUE_WIN = 5;
constexpr int STORE_FILAMENT = 0, STORE_MOTOR = 1, STORE_NONE = -1;
constexpr int NUC_NONE = 0, NUC_ATP = 1, NUC_ADPPI = 2, NUC_ADP = 3;
constexpr int FREE_BINDABLE = -1, FREE_COOLDOWN = -2;
constexpr int LINK_FREE = -1;
constexpr double PI_D = 3.141592653589793;

SBX_DEV float fsqrt(float x) { return __fsqrt_rn(x); }

// ---------------------------------------------------------------- Gaussian draws
// Box-Muller of BrownianForceSystem.java:78-92; g = {gfx,gfy,gfz,gtx,gty,gtz}
SBX_DEV void box_muller6(float u1, float u2, float u3, float u4, float u5, float u6, float g[6]) {
    const float TWO_PI_F = 2.0f * 3.14159265f;
    double sn, cs;
    float r1 = fsqrt(-2.0f * (float)sbxm::log((double)u1));
    float th1 = TWO_PI_F * u2;
    sbxm::sincos((double)th1, &sn, &cs);
    g[0] = r1 * (float)cs;
    g[3] = r1 * (float)sn;
    float r2 = fsqrt(-2.0f * (float)sbxm::log((double)u3));
    float th2 = TWO_PI_F * u4;
    sbxm::sincos((double)th2, &sn, &cs);
    g[1] = r2 * (float)cs;
    g[4] = r2 * (float)sn;
    float r3 = fsqrt(-2.0f * (float)sbxm::log((double)u5));
    float th3 = TWO_PI_F * u6;
    sbxm::sincos((double)th3, &sn, &cs);
    g[2] = r3 * (float)cs;
    g[5] = r3 * (float)sn;
}

// BrownianForceSystem.java:63-76: keyed (slot, step, seed)
SBX_DEV void gauss6_wang(int32_t i, int32_t step, int32_t seed, float g[6]) {
    uint32_t base = sbxm::rng_base(i, step, seed);
    float u1 = fmaxf(1.0e-7f, sbxm::unit_from_hash(sbxm::wang_hash(base)));
    float u2 = sbxm::unit_from_hash(sbxm::wang_hash(base ^ 0x9e3779b9u));
    float u3 = fmaxf(1.0e-7f, sbxm::unit_from_hash(sbxm::wang_hash(base ^ 0x85ebca6bu)));
    float u4 = sbxm::unit_from_hash(sbxm::wang_hash(base ^ 0xc2b2ae35u));
    float u5 = fmaxf(1.0e-7f, sbxm::unit_from_hash(sbxm::wang_hash(base ^ 0x517cc1b7u)));
    float u6 = sbxm::unit_from_hash(sbxm::wang_hash(base ^ 0x1f0a7ed5u));
    box_muller6(u1, u2, u3, u4, u5, u6, g);
}

// Pair j (0..2) of gauss6_wang alone: g[j] and g[3 + j] by the same operations (the three
// pairs of a slot are independent, so three threads can draw one slot)
SBX_DEV void gauss_pair_wang(int32_t i, int32_t step, int32_t seed, int j, float* gc, float* gs) {
    const uint32_t base = sbxm::rng_base(i, step, seed);
    const uint32_t ka = j == 0 ? 0u : (j == 1 ? 0x85ebca6bu : 0x517cc1b7u);
    const uint32_t kb = j == 0 ? 0x9e3779b9u : (j == 1 ? 0xc2b2ae35u : 0x1f0a7ed5u);
    float ua = fmaxf(1.0e-7f, sbxm::unit_from_hash(sbxm::wang_hash(base ^ ka)));
    float ub = sbxm::unit_from_hash(sbxm::wang_hash(base ^ kb));
    const float TWO_PI_F = 2.0f * 3.14159265f;
    double sn, cs;
    float r = fsqrt(-2.0f * (float)sbxm::log((double)ua));
    float th = TWO_PI_F * ub;
    sbxm::sincos((double)th, &sn, &cs);
    *gc = r * (float)cs;
    *gs = r * (float)sn;
}

// Counter-based Philox4x32-10 keyed (seed64, step, slot); same uniform/Box-Muller map
SBX_DEV void gauss6_philox(int32_t i, int32_t step, uint64_t seed, float g[6]) {
    uint32_t c0[4] = {(uint32_t)i, (uint32_t)step, 0u, 0x53425830u};
    uint32_t c1[4] = {(uint32_t)i, (uint32_t)step, 1u, 0x53425830u};
    sbxm::philox4x32_10(c0, (uint32_t)seed, (uint32_t)(seed >> 32));
    sbxm::philox4x32_10(c1, (uint32_t)seed, (uint32_t)(seed >> 32));
    float u1 = fmaxf(1.0e-7f, sbxm::unit_from_hash(c0[0]));
    float u2 = sbxm::unit_from_hash(c0[1]);
    float u3 = fmaxf(1.0e-7f, sbxm::unit_from_hash(c0[2]));
    float u4 = sbxm::unit_from_hash(c0[3]);
    float u5 = fmaxf(1.0e-7f, sbxm::unit_from_hash(c1[0]));
    float u6 = sbxm::unit_from_hash(c1[1]);
    box_muller6(u1, u2, u3, u4, u5, u6, g);
}

// BrownianForceSystem.java:94-104: randF = ((tS*mag)*sqrt(gamma))*g
SBX_DEV void brownian_amplitudes(const float g[6], float tS, float rS, float mag, const float gT[3],
                                 const float gR[3], float rf[3], float rt[3]) {
    for (int k = 0; k < 3; k++) rf[k] = tS * mag * fsqrt(gT[k]) * g[k];
    for (int k = 0; k < 3; k++) rt[k] = rS * mag * fsqrt(gR[k]) * g[3 + k];
}

// ---------------------------------------------------------------- Langevin step
struct Pose {
    float c[3], u[3], y[3];
};

// RigidRodLangevinIntegrationSystem.java:53-110 (and MechanicsFusion.java:134-176).
// Returns the new pose; `dc` receives the FP32 increments dt*v for FP64 accumulation.
SBX_DEV void integrate_pose(const Pose& p, const float F[3], const float T[3], const float rF[3],
                            const float rT[3], const float gT[3], const float gR[3], float dt, Pose& q,
                            float dc[3]) {
    float ux = p.u[0], uyc = p.u[1], uzc = p.u[2];
    float yx = p.y[0], yyc = p.y[1], yzc = p.y[2];
    float zx = uyc * yzc - uzc * yyc;
    float zy = uzc * yx - ux * yzc;
    float zz = ux * yyc - uyc * yx;
    float zlen = 1.0f / fsqrt(zx * zx + zy * zy + zz * zz);
    zx *= zlen; zy *= zlen; zz *= zlen;
    float fx = F[0], fy = F[1], fz = F[2];
    float tx = T[0], ty = T[1], tz = T[2];
    float bfx = ux * fx + uyc * fy + uzc * fz + rF[0];
    float bfy = yx * fx + yyc * fy + yzc * fz + rF[1];
    float bfz = zx * fx + zy * fy + zz * fz + rF[2];
    float btx = ux * tx + uyc * ty + uzc * tz + rT[0];
    float bty = yx * tx + yyc * ty + yzc * tz + rT[1];
    float btz = zx * tx + zy * ty + zz * tz + rT[2];
    float bvx = 1.0e6f * bfx / gT[0];
    float bvy = 1.0e6f * bfy / gT[1];
    float bvz = 1.0e6f * bfz / gT[2];
    float bwx = btx / gR[0];
    float bwy = bty / gR[1];
    float bwz = btz / gR[2];
    float vx = ux * bvx + yx * bvy + zx * bvz;
    float vy = uyc * bvx + yyc * bvy + zy * bvz;
    float vz = uzc * bvx + yzc * bvy + zz * bvz;
    dc[0] = dt * vx; dc[1] = dt * vy; dc[2] = dt * vz;
    q.c[0] = p.c[0] + dc[0];
    q.c[1] = p.c[1] + dc[1];
    q.c[2] = p.c[2] + dc[2];
    float uTransInZ = -bwy * dt;
    float uTransInY = bwz * dt;
    float nuX = ux + yx * uTransInY + zx * uTransInZ;
    float nuY = uyc + yyc * uTransInY + zy * uTransInZ;
    float nuZ = uzc + yzc * uTransInY + zz * uTransInZ;
    float nuInv = 1.0f / fsqrt(nuX * nuX + nuY * nuY + nuZ * nuZ);
    q.u[0] = nuX * nuInv; q.u[1] = nuY * nuInv; q.u[2] = nuZ * nuInv;
    float yTransInX = -uTransInY;
    float yTransInZ = bwx * dt;
    float nyX = ux * yTransInX + yx + zx * yTransInZ;
    float nyY = uyc * yTransInX + yyc + zy * yTransInZ;
    float nyZ = uzc * yTransInX + yzc + zz * yTransInZ;
    float nyInv = 1.0f / fsqrt(nyX * nyX + nyY * nyY + nyZ * nyZ);
    q.y[0] = nyX * nyInv; q.y[1] = nyY * nyInv; q.y[2] = nyZ * nyInv;
}

// DerivedGeometrySystem.java:43-71: z = unit(u x y), y' = z x u, ends = c -/+ (L/2) u
SBX_DEV void derive_pose(const float c[3], const float u[3], float y[3], float z[3], float e1[3], float e2[3],
                         float segLength) {
    float ux = u[0], uyc = u[1], uzc = u[2];
    float yx = y[0], yyc = y[1], yzc = y[2];
    float zx = uyc * yzc - uzc * yyc;
    float zy = uzc * yx - ux * yzc;
    float zz = ux * yyc - uyc * yx;
    float zmag2 = zx * zx + zy * zy + zz * zz;
    if (zmag2 > 0.f) {
        float inv = 1.0f / fsqrt(zmag2);
        zx *= inv; zy *= inv; zz *= inv;
    }
    z[0] = zx; z[1] = zy; z[2] = zz;
    y[0] = zy * uzc - zz * uyc;
    y[1] = zz * ux - zx * uzc;
    y[2] = zx * uyc - zy * ux;
    float halfLen = segLength * 0.5f;
    e1[0] = c[0] - halfLen * ux; e1[1] = c[1] - halfLen * uyc; e1[2] = c[2] - halfLen * uzc;
    e2[0] = c[0] + halfLen * ux; e2[1] = c[1] + halfLen * uyc; e2[2] = c[2] + halfLen * uzc;
}

// ---------------------------------------------------------------- containment
SBX_DEV double wall_push(double d, double halfDim) {       // ContainmentSystem.java:130-136
    double s = (d > 0.0) ? 1.0 : ((d < 0.0) ? -1.0 : 0.0);
    double push = s * halfDim - d;
    double ps = (push > 0.0) ? 1.0 : ((push < 0.0) ? -1.0 : 0.0);
    if (ps == s) return 0.0;
    return push;
}

struct BoxParams {
    double tau, halfX, halfY, halfZ, coeff;
    bool active;        // cadence gate of this step
};

// ContainmentSystem.java:64-72 for step `step`
SBX_DEV BoxParams box_params(const float* bp, int32_t step) {
    BoxParams b;
    int32_t checkInt = (int32_t)bp[6];
    b.active = !(checkInt > 1 && (step % checkInt) != 0);
    b.tau = bp[0];
    b.halfX = 0.5 * bp[1] - bp[4];
    b.halfY = 0.5 * bp[2] - bp[4];
    b.halfZ = 0.5 * bp[3] - bp[4];
    b.coeff = bp[5];
    return b;
}

// ContainmentSystem.java:75-125: += into F/T only on penetration
// Returns whether an endpoint touched a wall (F and T are unchanged otherwise).
SBX_DEV bool confine_one(const BoxParams& bx, const float c[3], const float u[3], float segLength, float bTGx,
                         float F[3], float T[3]) {
    double cx = c[0], cy = c[1], cz = c[2];
    double ux = u[0], uy = u[1], uz = u[2];
    double half = 0.5 * (double)segLength;
    double g = bTGx;
    double fx = 0.0, fy = 0.0, fz = 0.0, tx = 0.0, ty = 0.0, tz = 0.0;
    bool touched = false;
    for (int e = 0; e < 2; e++) {
        double sgn = (e == 0) ? -1.0 : 1.0;
        double dx = cx + sgn * half * ux;
        double dy = cy + sgn * half * uy;
        double dz = cz + sgn * half * uz;
        double fux = wall_push(dx, bx.halfX);
        double fuy = wall_push(dy, bx.halfY);
        double fuz = wall_push(dz, bx.halfZ);
        double delta2 = fux * fux + fuy * fuy + fuz * fuz;
        if (delta2 > 0.0) {
            double delta = sqrt(delta2);
            double inv = 1.0 / delta;
            double lux = fux * inv, luy = fuy * inv, luz = fuz * inv;
            double mag = bx.coeff * 1.0e-6 * delta * g / bx.tau;
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
        F[0] = (float)((double)F[0] + fx);
        F[1] = (float)((double)F[1] + fy);
        F[2] = (float)((double)F[2] + fz);
        T[0] = (float)((double)T[0] + tx);
        T[1] = (float)((double)T[1] + ty);
        T[2] = (float)((double)T[2] + tz);
    }
    return touched;
}

// ---------------------------------------------------------------- angles
// ChainBendingForceSystem.java:48-72 (same polynomial + two Newton steps in every System)
SBX_DEV_CALL double accurate_acos(double x) {
    if (x > 1.0) x = 1.0;
    if (x < -1.0) x = -1.0;
    double y;
    if (x > 0.95) {
        double t = 1.0 - x;
        if (t < 0.0) t = 0.0;
        y = sqrt(2.0 * t);
    } else if (x < -0.95) {
        double t = 1.0 + x;
        if (t < 0.0) t = 0.0;
        y = 3.141592653589793 - sqrt(2.0 * t);
    } else {
        double ax = (x < 0.0) ? -x : x;
        double p = (-0.0187293 * ax + 0.0742610) * ax - 0.2121144;
        p = (p * ax + 1.5707963);
        p = p * sqrt(1.0 - ax);
        y = (x < 0.0) ? (3.141592653589793 - p) : p;
    }
    double s, c;
    sbxm::sincos(y, &s, &c);
    if (s > 1.0e-12 || s < -1.0e-12) y = y + (c - x) / s;
    sbxm::sincos(y, &s, &c);
    if (s > 1.0e-12 || s < -1.0e-12) y = y + (c - x) / s;
    return y;
}

SBX_DEV_CALL double accurate_asin(double s) {                    // ChainBendingForceSystem.java:76-84
    double s2 = s * s;
    double y = s * (1.0 + s2 * (0.16666666666666666 + s2 * (0.075 + s2 * 0.044642857142857)));
    double sy, cy;
    sbxm::sincos(y, &sy, &cy);
    if (cy > 1.0e-12) y = y + (s - sy) / cy;
    sbxm::sincos(y, &sy, &cy);
    if (cy > 1.0e-12) y = y + (s - sy) / cy;
    return y;
}

SBX_DEV double angle_from_sin_cos(double sin2, double cosv) {   // ChainBendingForceSystem.java:95-103
    double s = sqrt(sin2);
    double ac = (cosv < 0.0) ? -cosv : cosv;
    if (s <= ac) {
        double base = accurate_asin(s);
        return (cosv >= 0.0) ? base : (PI_D - base);
    }
    return accurate_acos(cosv);
}

SBX_DEV double fast_acos(double dot) {                      // CrosslinkerSystem.java:372-376
    if (dot > 0.95) { double t = 1.0 - dot; if (t < 0) t = 0; return sqrt(2.0 * t); }
    if (dot < -0.95) { double t = 1.0 + dot; if (t < 0) t = 0; return PI_D - sqrt(2.0 * t); }
    return accurate_acos(dot);
}

// MotorJointSystem.java:61-70
SBX_DEV double move_c(double ux, double uy, double uz, double lx, double ly, double lz, double bTGx,
                      double bTGy, double bRGy, double lenUm) {
    double cosB = ux * lx + uy * ly + uz * lz;
    if (cosB > 1.0) cosB = 1.0;
    if (cosB < -1.0) cosB = -1.0;
    double cosB2 = cosB * cosB;
    double cosA2 = 1.0 - cosB2;
    double lSq = 1.0e-12 * lenUm * lenUm;
    return cosB2 / bTGx + cosA2 / bTGy + lSq * cosA2 / (4.0 * bRGy);
}

// ---------------------------------------------------------------- chain (F3 link + F4 bend)
struct ChainParams {
    double dt, fracMove, fracR, fracMoveTorq, springActive, spring, monoR;
};
SBX_DEV ChainParams chain_params(const float* p) {
    ChainParams c;
    c.dt = p[0]; c.fracMove = p[1]; c.fracR = p[2]; c.fracMoveTorq = p[3];
    c.springActive = p[4]; c.spring = p[5]; c.monoR = p[6];
    return c;
}

struct RodGeom {        // the per-rod reads of ChainBendingForceSystem.java:136-144 / :156-163
    double cx, cy, cz, ux, uy, uz, len, bTGx, bTGy, bRGy;
};

// A chain joint seen from rod i's `side` (side 0 = end2 block :152-235, side 1 = end1 block
// :237-321) with neighbour `slot` attached at its `nside` (0 = the neighbour's end1).
// chain_joint holds the costly scalars of the joint; both rods of a joint get the same
// values: seen from the neighbour (side' = 1 - nside, nside' = 1 - side) the strain points,
// the two moveC terms (swapped, and summed commutatively), the torsion axis (negated) and
// the bend angle come out bit-identical.
struct ChainJoint {
    double forceMag, luX, luY, luZ, invMag, torsionMag;
    int tvOK;
};

// The joint's strain geometry: strain vector, its length and unit vector, and the two rods'
// (clamped) direction cosines to it (ChainBendingForceSystem.java:165-190 / :250-276).
struct JointGeom {
    double strainDist, luX, luY, luZ, cosB1, cosB2;
};

SBX_DEV JointGeom chain_joint_geom(const ChainParams& cp, int i, int side, int slot, int nside, const RodGeom& r,
                                   const RodGeom& nb) {
    JointGeom G;
    double halfLen_um = 0.5 * r.len;
    double nHalfLen_um = 0.5 * nb.len;
    double ex, ey, ez, selfLpx, selfLpy, selfLpz;
    if (side == 0) {
        ex = r.cx + halfLen_um * r.ux; ey = r.cy + halfLen_um * r.uy; ez = r.cz + halfLen_um * r.uz;
        selfLpx = ex - cp.monoR * r.ux; selfLpy = ey - cp.monoR * r.uy; selfLpz = ez - cp.monoR * r.uz;
    } else {
        ex = r.cx - halfLen_um * r.ux; ey = r.cy - halfLen_um * r.uy; ez = r.cz - halfLen_um * r.uz;
        selfLpx = ex + cp.monoR * r.ux; selfLpy = ey + cp.monoR * r.uy; selfLpz = ez + cp.monoR * r.uz;
    }
    double tipx, tipy, tipz, nlpx, nlpy, nlpz;
    if (nside == 0) {
        tipx = nb.cx - nHalfLen_um * nb.ux; tipy = nb.cy - nHalfLen_um * nb.uy; tipz = nb.cz - nHalfLen_um * nb.uz;
        nlpx = tipx + cp.monoR * nb.ux; nlpy = tipy + cp.monoR * nb.uy; nlpz = tipz + cp.monoR * nb.uz;
    } else {
        tipx = nb.cx + nHalfLen_um * nb.ux; tipy = nb.cy + nHalfLen_um * nb.uy; tipz = nb.cz + nHalfLen_um * nb.uz;
        nlpx = tipx - cp.monoR * nb.ux; nlpy = tipy - cp.monoR * nb.uy; nlpz = tipz - cp.monoR * nb.uz;
    }
    bool owner = i < slot;
    double lpx = owner ? selfLpx : nlpx, lpy = owner ? selfLpy : nlpy, lpz = owner ? selfLpz : nlpz;
    double pex = owner ? tipx : ex, pey = owner ? tipy : ey, pez = owner ? tipz : ez;
    double dx = pex - lpx, dy = pey - lpy, dz = pez - lpz;
    G.strainDist = sqrt(dx * dx + dy * dy + dz * dz);
    double invStrain = (G.strainDist > 0.0) ? (1.0 / G.strainDist) : 0.0;
    G.luX = dx * invStrain; G.luY = dy * invStrain; G.luZ = dz * invStrain;
    double cosB1 = r.ux * G.luX + r.uy * G.luY + r.uz * G.luZ;
    if (cosB1 > 1.0) cosB1 = 1.0;
    if (cosB1 < -1.0) cosB1 = -1.0;
    double cosB2 = nb.ux * G.luX + nb.uy * G.luY + nb.uz * G.luZ;
    if (cosB2 > 1.0) cosB2 = 1.0;
    if (cosB2 < -1.0) cosB2 = -1.0;
    G.cosB1 = cosB1;
    G.cosB2 = cosB2;
    return G;
}

// One rod's mobility term along the strain (the moveC of :191-200 / :277-286)
SBX_DEV double chain_move_c(double cosB, const RodGeom& r) {
    double lSq = 1.0e-12 * r.len * r.len;
    double cosA = sbxm::sin(accurate_acos(cosB));
    double cosA_2 = cosA * cosA;
    return cosB * cosB / r.bTGx + cosA_2 / r.bTGy + lSq * cosA_2 / (4.0 * r.bRGy);
}

SBX_DEV double chain_force_mag(const ChainParams& cp, double strainDist, double moveC1, double moveC2) {
    double denom = cp.dt * (moveC1 + moveC2);
    return (denom > 0.0) ? (cp.fracMove * 1.0e-6 * strainDist / denom) : 0.0;
}

// The joint's torsion (:203-233 / :289-319): tvOK, 1/|tv| and the torsion magnitude
SBX_DEV void chain_torsion(const ChainParams& cp, int side, int nside, const RodGeom& r, const RodGeom& nb, int* tvOK,
                           double* invMag, double* torsionMag) {
    const double RAD2DEG = 180.0 / PI_D;
    const double DEG2RAD = PI_D / 180.0;
    double nxE = (nside == 0) ? nb.ux : -nb.ux, nyE = (nside == 0) ? nb.uy : -nb.uy, nzE = (nside == 0) ? nb.uz : -nb.uz;
    double mux = (side == 0) ? r.ux : -r.ux, muy = (side == 0) ? r.uy : -r.uy, muz = (side == 0) ? r.uz : -r.uz;
    double tvx = muy * nzE - muz * nyE, tvy = muz * nxE - mux * nzE, tvz = mux * nyE - muy * nxE;
    double tvMag2 = tvx * tvx + tvy * tvy + tvz * tvz;
    *tvOK = tvMag2 > 1.0e-30;
    *invMag = 0.0;
    *torsionMag = 0.0;
    if (*tvOK) {
        *invMag = 1.0 / sqrt(tvMag2);
        double dotV = mux * nxE + muy * nyE + muz * nzE;
        if (dotV > 1.0) dotV = 1.0;
        if (dotV < -1.0) dotV = -1.0;
        double angTween = angle_from_sin_cos(tvMag2, dotV) * RAD2DEG;
        if (cp.springActive > 0.5) {
            *torsionMag = cp.fracMoveTorq * cp.spring * angTween;
        } else {
            double invBRG = 1.0 / r.bRGy + 1.0 / nb.bRGy;
            *torsionMag = cp.fracMoveTorq * DEG2RAD * angTween / (invBRG * cp.dt);
        }
    }
}

SBX_DEV ChainJoint chain_joint(const ChainParams& cp, int i, int side, int slot, int nside, const RodGeom& r,
                               const RodGeom& nb) {
    JointGeom G = chain_joint_geom(cp, i, side, slot, nside, r, nb);
    ChainJoint J;
    J.forceMag = chain_force_mag(cp, G.strainDist, chain_move_c(G.cosB1, r), chain_move_c(G.cosB2, nb));
    J.luX = G.luX; J.luY = G.luY; J.luZ = G.luZ;
    chain_torsion(cp, side, nside, r, nb, &J.tvOK, &J.invMag, &J.torsionMag);
    return J;
}

// Accumulates joint J into rod i's double force/torque sums from its own side.
SBX_DEV void chain_apply(const ChainParams& cp, int i, int side, int slot, int nside, const RodGeom& r,
                         const RodGeom& nb, const ChainJoint& J, double f[3], double t[3]) {
    bool owner = i < slot;
    double fSign = owner ? 1.0 : -1.0;
    double Fx = fSign * J.forceMag * J.luX, Fy = fSign * J.forceMag * J.luY, Fz = fSign * J.forceMag * J.luZ;
    f[0] += Fx; f[1] += Fy; f[2] += Fz;
    double Rscale = (side == 0) ? (0.5e-6 * r.len * cp.fracR) : (-0.5e-6 * r.len * cp.fracR);
    double Rx = Rscale * r.ux, Ry = Rscale * r.uy, Rz = Rscale * r.uz;
    t[0] += Ry * Fz - Rz * Fy; t[1] += Rz * Fx - Rx * Fz; t[2] += Rx * Fy - Ry * Fx;
    if (J.tvOK) {
        double nxE = (nside == 0) ? nb.ux : -nb.ux, nyE = (nside == 0) ? nb.uy : -nb.uy,
               nzE = (nside == 0) ? nb.uz : -nb.uz;
        double mux = (side == 0) ? r.ux : -r.ux, muy = (side == 0) ? r.uy : -r.uy, muz = (side == 0) ? r.uz : -r.uz;
        double tvx = muy * nzE - muz * nyE, tvy = muz * nxE - mux * nzE, tvz = mux * nyE - muy * nxE;
        tvx *= J.invMag; tvy *= J.invMag; tvz *= J.invMag;
        t[0] += tvx * J.torsionMag; t[1] += tvy * J.torsionMag; t[2] += tvz * J.torsionMag;
    }
}

// One joint side of rod i, accumulated into f/t (ChainBendingForceSystem.java:152-321)
SBX_DEV void chain_side(const ChainParams& cp, int i, int side, int slot, int nside, const RodGeom& r,
                        const RodGeom& nb, double f[3], double t[3]) {
    ChainJoint J = chain_joint(cp, i, side, slot, nside, r, nb);
    chain_apply(cp, i, side, slot, nside, r, nb, J, f, t);
}

SBX_DEV RodGeom load_rod(int n, int i, const float* coord, const float* uVec, const float* segLength,
                         const float* bTG, const float* bRG) {
    RodGeom r;
    r.cx = coord[i]; r.cy = coord[n + i]; r.cz = coord[2 * n + i];
    r.ux = uVec[i]; r.uy = uVec[n + i]; r.uz = uVec[2 * n + i];
    r.len = segLength[i];
    r.bTGx = bTG[i]; r.bTGy = bTG[n + i]; r.bRGy = bRG[n + i];
    return r;
}

// ---------------------------------------------------------------- binding predicate
// BindingDetectionSystem.java:59-85 (== the inlined form at :197-219)
SBX_DEV float reach_test_dist_sq(float mx, float my, float mz, float mux, float muy, float muz, float rux,
                                 float ruy, float ruz, float e1x, float e1y, float e1z, float e2x, float e2y,
                                 float e2z, float myoColTol, float alignTol) {
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
    float inv = 1.0f / fsqrt(denom);
    float fux = r1x * inv, fuy = r1y * inv, fuz = r1z * inv;
    float motDotFil = mux * fux + muy * fuy + muz * fuz;
    if (motDotFil < alignTol) return -1.f;
    float rodDotFil = rux * fux + ruy * fuy + ruz * fuz;
    if (rodDotFil < 0.f) return -1.f;
    return conDistSq;
}

// bind-site arc of BindingDetectionSystem.java:378-383
SBX_DEV float bind_arc(float mx, float my, float mz, float e1x, float e1y, float e1z, float e2x, float e2y,
                       float e2z) {
    float r1x = e2x - e1x, r1y = e2y - e1y, r1z = e2z - e1z;
    float denom = r1x * r1x + r1y * r1y + r1z * r1z;
    float numer = (mx - e1x) * r1x + (my - e1y) * r1y + (mz - e1z) * r1z;
    return numer / fsqrt(denom);
}

// SpatialGrid.java:67-73 / BindingDetectionSystem.java:167-172: clamp-binned cell coordinate
SBX_DEV int cell_coord(float x, float xMin, float invCell, int nX) {
    int ix = (int)((x - xMin) * invCell);
    if (ix < 0) ix = 0;
    if (ix >= nX) ix = nX - 1;
    return ix;
}

// ---------------------------------------------------------------- nucleotide / release
SBX_DEV float unit_salted(int32_t m, int32_t step, int32_t seed, uint32_t salt) {
    return sbxm::unit_from_hash(sbxm::wang_hash(sbxm::rng_base(m, step, seed) ^ salt));
}

// NucleotideCycleSystem.java:44-67
SBX_DEV int cycle_one(int32_t m, int state, bool bound, const float* hist10, const float* np, int32_t step,
                      int32_t seed) {
    float dt = np[0], atpOn = np[1];
    float u = unit_salted(m, step, seed, 0x4E55u);
    if (state == NUC_NONE) {
        if (u < atpOn * dt) state = NUC_ATP;
    } else if (state == NUC_ATP) {
        float rate = bound ? np[2] : np[3];
        if (u < rate * dt) state = NUC_ADPPI;
    } else if (state == NUC_ADPPI) {
        float rate = bound ? np[4] : np[5];
        if (u < rate * dt) state = NUC_ADP;
    } else {
        float avg = 0.f;
        for (int k = 0; k < 10; k++) avg += hist10[k];
        avg *= 0.1f;
        if (avg <= 0.f) {
            float rate = bound ? np[6] : np[7];
            if (u < rate * dt) state = NUC_NONE;
        }
    }
    return state;
}

// NucleotideCycleSystem.java:89-132 for one motor; updates bs/cooldown/stats in place
SBX_DEV void release_one(int32_t m, int& bs, int& cooldown, int& statBound, int& statRel, int& capStat,
                         float forceDotFil, float forceMag, const float* kp, int32_t step, int32_t seed) {
    if (bs >= 0) {
        float kOff = kp[0], aCatch = kp[1], aSlip = kp[2];
        float xCatch = kp[3], xSlip = kp[4], kT = kp[5], dt = kp[6];
        int refractorySteps = (int)kp[10];
        float breakForceN = kp[11];
        bool capOn = kp[12] > 0.5f;
        float blockProb = kp[13];
        statBound += 1;
        bool enterRefractory = refractorySteps > 0;
        if (blockProb < 1.0f) {
            float ru = unit_salted(m, step, seed, 0x52465241u);
            enterRefractory = enterRefractory && (ru < blockProb);
        }
        if (capOn && forceMag > breakForceN) {
            capStat += 1;
            if (enterRefractory) { bs = FREE_COOLDOWN; cooldown = refractorySteps; }
            else bs = FREE_BINDABLE;
            return;
        }
        float F = forceDotFil;
        float rate = kOff * (aCatch * (float)sbxm::exp((double)(-F * xCatch / kT)) +
                             aSlip * (float)sbxm::exp((double)(F * xSlip / kT)));
        float u = unit_salted(m, step, seed, 0x4D54u);
        if (u < rate * dt) {
            statRel += 1;
            if (enterRefractory) { bs = FREE_COOLDOWN; cooldown = refractorySteps; }
            else bs = FREE_BINDABLE;
        }
    } else if (bs == FREE_COOLDOWN) {
        int c = cooldown - 1;
        if (c <= 0) bs = FREE_BINDABLE;
        else cooldown = c;
    }
}

}  // namespace sbx

// ============================================================================
// Slot functions used by both the per-system and the fused kernels
// ============================================================================
namespace sbx {

// BindingDetectionSystem.gridReachable per motor (BindingDetectionSystem.java:161-227):
// 27-cell walk z->y->x in CSR order, exact predicate, owned output slice; returns count
SBX_DEV int grid_reach_walk(int m, int nM, const float* head, const float* uVec, const float* rodUVec, int nSeg,
                            const float* e1, const float* e2, const float* gp, const int* gd, const int* offsets,
                            const int* contents, const int* ownerStore, const int* ownerSlot, int* outSlice,
                            float myoColTol, float alignTol) {
    float mx = head[m], my = head[nM + m], mz = head[2 * nM + m];
    float mux = uVec[m], muy = uVec[nM + m], muz = uVec[2 * nM + m];
    float rux = rodUVec[m], ruy = rodUVec[nM + m], ruz = rodUVec[2 * nM + m];
    int nX = gd[0], nY = gd[1], nZ = gd[2], nXY = nX * nY;
    int cx = cell_coord(mx, gp[0], gp[4], nX);
    int cy = cell_coord(my, gp[1], gp[4], nY);
    int cz = cell_coord(mz, gp[2], gp[4], nZ);
    int x0 = max(cx - 1, 0), x1 = min(cx + 1, nX - 1);
    int y0 = max(cy - 1, 0), y1 = min(cy + 1, nY - 1);
    int z0 = max(cz - 1, 0), z1 = min(cz + 1, nZ - 1);
    int out = 0;
    for (int zz = z0; zz <= z1; zz++)
        for (int yy = y0; yy <= y1; yy++)
            for (int xx = x0; xx <= x1; xx++) {
                int cc = xx + yy * nX + zz * nXY;
                int start = offsets[cc], end = offsets[cc + 1];
                for (int idx = start; idx < end; idx++) {
                    int j = contents[idx];
                    if (ownerStore[j] != STORE_FILAMENT) continue;
                    int s = ownerSlot[j];
                    float d = reach_test_dist_sq(mx, my, mz, mux, muy, muz, rux, ruy, ruz, e1[s], e1[nSeg + s],
                                                 e1[2 * nSeg + s], e2[s], e2[nSeg + s], e2[2 * nSeg + s], myoColTol,
                                                 alignTol);
                    if (d >= 0.f) {
                        if (out < MAX_CAND) outSlice[out] = s;
                        out++;
                    }
                }
            }
    return out;
}

// grid_reach_walk over cell-ordered endpoints: cellE1[idx] / cellE2[idx] hold the segment
// endpoints of grid entry idx (the slot in cellE1[idx].w as int bits, -1 for an entry that is
// not a filament segment). The three x-neighbour cells of a (y, z) row are consecutive cell
// ids, so their entries are one contiguous range [offsets[x0 + row], offsets[x1 + 1 + row]),
// walked in the same order as cell by cell: the reach list is the same.
SBX_DEV int grid_reach_walk_cells(int m, int nM, const float* head, const float* uVec, const float* rodUVec,
                                  const float* gp, const int* gd, const int* offsets, const float4* cellE1,
                                  const float4* cellE2, int* outSlice, float myoColTol, float alignTol) {
    float mx = head[m], my = head[nM + m], mz = head[2 * nM + m];
    float mux = uVec[m], muy = uVec[nM + m], muz = uVec[2 * nM + m];
    float rux = rodUVec[m], ruy = rodUVec[nM + m], ruz = rodUVec[2 * nM + m];
    int nX = gd[0], nY = gd[1], nZ = gd[2], nXY = nX * nY;
    int cx = cell_coord(mx, gp[0], gp[4], nX);
    int cy = cell_coord(my, gp[1], gp[4], nY);
    int cz = cell_coord(mz, gp[2], gp[4], nZ);
    int x0 = max(cx - 1, 0), x1 = min(cx + 1, nX - 1);
    int y0 = max(cy - 1, 0), y1 = min(cy + 1, nY - 1);
    int z0 = max(cz - 1, 0), z1 = min(cz + 1, nZ - 1);
    // the (up to) nine row ranges as one sequence k = 0..total-1 (row order, then index
    // order), taken four entries at a time so that their loads are in flight together
    int rs[9], pre[10];
    pre[0] = 0;
#pragma unroll
    for (int r = 0; r < 9; r++) {
        int zz = z0 + r / 3, yy = y0 + r % 3;
        bool ok = zz <= z1 && yy <= y1;
        int row = yy * nX + zz * nXY;
        rs[r] = ok ? offsets[x0 + row] : 0;
        pre[r + 1] = pre[r] + (ok ? offsets[x1 + 1 + row] - rs[r] : 0);
    }
    const int total = pre[9];
    int out = 0;
    for (int k0 = 0; k0 < total; k0 += 4) {
        float4 a[4], b[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            int k = k0 + q;
            if (k < total) {
                int idx = rs[0] + k;
#pragma unroll
                for (int r = 1; r < 9; r++)
                    if (k >= pre[r]) idx = rs[r] + (k - pre[r]);
                a[q] = cellE1[idx];
                b[q] = cellE2[idx];
            }
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            if (k0 + q >= total) break;
            int s = __float_as_int(a[q].w);
            if (s < 0) continue;
            float d = reach_test_dist_sq(mx, my, mz, mux, muy, muz, rux, ruy, ruz, a[q].x, a[q].y, a[q].z, b[q].x,
                                         b[q].y, b[q].z, myoColTol, alignTol);
            if (d >= 0.f) {
                if (out < MAX_CAND) outSlice[out] = s;
                out++;
            }
        }
    }
    return out;
}

// BindingDetectionSystem.bindNearest per motor (BindingDetectionSystem.java:366-388):
// strict < keeps the first nearest in list order; true when a segment was found
SBX_DEV bool bind_nearest_scan(int m, int nM, const float* head, const float* uVec, const float* rodUVec, int nSeg,
                               const float* e1, const float* e2, const int* candSlice, int cnt, float myoColTol,
                               float alignTol, int* bestSeg, float* bestArc) {
    float mx = head[m], my = head[nM + m], mz = head[2 * nM + m];
    float mux = uVec[m], muy = uVec[nM + m], muz = uVec[2 * nM + m];
    float rux = rodUVec[m], ruy = rodUVec[nM + m], ruz = rodUVec[2 * nM + m];
    if (cnt > MAX_CAND) cnt = MAX_CAND;
    int best = -1;
    float bestD = 1.0e30f, arc = 0.f;
    for (int k = 0; k < cnt; k++) {
        int s = candSlice[k];
        float e1x = e1[s], e1y = e1[nSeg + s], e1z = e1[2 * nSeg + s];
        float e2x = e2[s], e2y = e2[nSeg + s], e2z = e2[2 * nSeg + s];
        float d = reach_test_dist_sq(mx, my, mz, mux, muy, muz, rux, ruy, ruz, e1x, e1y, e1z, e2x, e2y, e2z,
                                     myoColTol, alignTol);
        if (d >= 0.f && d < bestD) {
            bestD = d;
            best = s;
            arc = bind_arc(mx, my, mz, e1x, e1y, e1z, e2x, e2y, e2z);
        }
    }
    *bestSeg = best;
    *bestArc = arc;
    return best >= 0;
}

// CrossBridgeSystem.bondForces per motor (CrossBridgeSystem.java:72-141) -> 13 floats
SBX_DEV void bond_one(int m, int nB, const float* mC, const float* mU, const float* mY, const float* mBRG, int nSeg,
                      const float* fC, const float* fU, const float* fY, const float* fBRG, const float* fLen, int s,
                      float bindArcM, int nucState, const float* xb, float out[XB_STRIDE]) {
    for (int k = 0; k < XB_STRIDE; k++) out[k] = 0.f;
    if (s < 0) return;
    const double DEG2RAD = PI_D / 180.0, RAD2DEG = 180.0 / PI_D;
    double myoSpring = xb[0], j1FMT = xb[2], dt = xb[3], headLen = xb[4], xbias = xb[5];
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
    double aOff = bindArcM - 0.5 * slen;
    double apx = scx + aOff * sux, apy = scy + aOff * suy, apz = scz + aOff * suz;
    double dx = apx - htipx, dy = apy - htipy, dz = apz - htipz;
    double dist = sqrt(dx * dx + dy * dy + dz * dz);
    double fmag = myoSpring * dist;
    double Fx = 0, Fy = 0, Fz = 0;
    if (dist > 0.0) { double inv = fmag / dist; Fx = inv * dx; Fy = inv * dy; Fz = inv * dz; }
    double RHx = (htipx - hcx) * 1e-6, RHy = (htipy - hcy) * 1e-6, RHz = (htipz - hcz) * 1e-6;
    double THx = RHy * Fz - RHz * Fy, THy = RHz * Fx - RHx * Fz, THz = RHx * Fy - RHy * Fx;
    double RSx = (apx - scx) * 1e-6, RSy = (apy - scy) * 1e-6, RSz = (apz - scz) * 1e-6;
    double nFx = -Fx, nFy = -Fy, nFz = -Fz;
    double TSx = RSy * nFz - RSz * nFy, TSy = RSz * nFx - RSx * nFz, TSz = RSx * nFy - RSy * nFx;
    double restF9 = (nucState != NUC_ADPPI) ? 120.0 : 90.0;
    double t9x = suy * huz - suz * huy, t9y = suz * hux - sux * huz, t9z = sux * huy - suy * hux;
    double m9 = t9x * t9x + t9y * t9y + t9z * t9z;
    double T9x = 0, T9y = 0, T9z = 0;
    if (m9 > 1.0e-30) {
        double im = 1.0 / sqrt(m9);
        t9x *= im; t9y *= im; t9z *= im;
        double dot = sux * hux + suy * huy + suz * huz;
        if (dot > 1) dot = 1;
        if (dot < -1) dot = -1;
        double angD = accurate_acos(dot) * RAD2DEG - restF9;
        double tm = j1FMT * DEG2RAD * angD / ((1.0 / hbRGy + 1.0 / sbRGy) * dt);
        T9x = tm * t9x; T9y = tm * t9y; T9z = tm * t9z;
    }
    double t10x = syy * hyz - syz * hyy, t10y = syz * hyx - syx * hyz, t10z = syx * hyy - syy * hyx;
    double m10 = t10x * t10x + t10y * t10y + t10z * t10z;
    double T10x = 0, T10y = 0, T10z = 0;
    if (m10 > 1.0e-30) {
        double im = 1.0 / sqrt(m10);
        t10x *= im; t10y *= im; t10z *= im;
        double dot = syx * hyx + syy * hyy + syz * hyz;
        if (dot > 1) dot = 1;
        if (dot < -1) dot = -1;
        double ang = accurate_acos(dot) * RAD2DEG;
        double tm = j1FMT * DEG2RAD * ang / ((1.0 / hbRGx + 1.0 / sbRGx) * dt);
        T10x = tm * t10x; T10y = tm * t10y; T10z = tm * t10z;
    }
    out[0] = (float)Fx; out[1] = (float)Fy; out[2] = (float)Fz;
    out[3] = (float)(THx - T9x - T10x);
    out[4] = (float)(THy - T9y - T10y);
    out[5] = (float)(THz - T9z - T10z);
    out[6] = (float)(nFx - xbias); out[7] = (float)nFy; out[8] = (float)nFz;
    out[9] = (float)(TSx + T9x + T10x);
    out[10] = (float)(TSy + T9y + T10y);
    out[11] = (float)(TSz + T9z + T10z);
    out[12] = (float)(Fx * sux + Fy * suy + Fz * suz);
}

// CrossBridgeSystem.registerForceDot per motor (CrossBridgeSystem.java:169-185)
SBX_DEV void register_force_dot_one(int m, const float* bondData, bool bound, float* fdf, float* fm, float* hist,
                                    int* place) {
    if (bound) {
        int d = m * XB_STRIDE;
        float fd = bondData[d + 12];
        fdf[m] = fd;
        float fx = bondData[d], fy = bondData[d + 1], fz = bondData[d + 2];
        fm[m] = fsqrt(fx * fx + fy * fy + fz * fz);
        int p = place[m];
        hist[m * 10 + p] = fd;
        place[m] = (p + 1) % 10;
    } else {
        fdf[m] = 0.f;
        fm[m] = 0.f;
        place[m] = 0;
        for (int k = 0; k < 10; k++) hist[m * 10 + k] = 0.f;
    }
}

// CSR gather of one row (CrossBridgeSystem.java:305-312, CrosslinkerSystem.java:132-142,
// MiniFilamentSystem.java:140-147): FP64 sums of float payloads in list order
SBX_DEV void csr_gather_row(int s, const int* offsets, const int* list, const float* payload, int stride, int off,
                            const int* guard, double f[3], double t[3]) {
    f[0] = f[1] = f[2] = 0.0;
    t[0] = t[1] = t[2] = 0.0;
    int start = offsets[s], end = offsets[s + 1];
    for (int k = start; k < end; k++) {
        int li = list[k];
        if (guard && guard[li] < 0) continue;
        const float* p = payload + (int64_t)li * stride + off;
        f[0] += p[0]; f[1] += p[1]; f[2] += p[2];
        t[0] += p[3]; t[1] += p[4]; t[2] += p[5];
    }
}

// CrosslinkerSystem.linkForces per link (CrosslinkerSystem.java:61-123) -> 12 floats
SBX_DEV void link_forces_one(int k, int nSeg, const float* fC, const float* fU, const float* fE1, const float* fBTG,
                             int a, int b, float loc1k, float loc2k, const int* ct, const float* xp,
                             float out[XL_STRIDE]) {
    for (int j = 0; j < XL_STRIDE; j++) out[j] = 0.f;
    if (a < 0 || b < 0) return;
    double restLength = xp[0], fracMoveBase = xp[1], dt = xp[2];
    double l1 = loc1k;
    double uax = fU[a], uay = fU[nSeg + a], uaz = fU[2 * nSeg + a];
    double p1x = fE1[a] + l1 * uax;
    double p1y = fE1[nSeg + a] + l1 * uay;
    double p1z = fE1[2 * nSeg + a] + l1 * uaz;
    double l2 = loc2k;
    double ubx = fU[b], uby = fU[nSeg + b], ubz = fU[2 * nSeg + b];
    double p2x = fE1[b] + l2 * ubx;
    double p2y = fE1[nSeg + b] + l2 * uby;
    double p2z = fE1[2 * nSeg + b] + l2 * ubz;
    double lvx = p2x - p1x, lvy = p2y - p1y, lvz = p2z - p1z;
    double linkLength = sqrt(lvx * lvx + lvy * lvy + lvz * lvz);
    double stretch = linkLength - restLength;
    if (stretch < 0.0) stretch = 0.0;
    int ctA = ct[a], ctB = ct[b];
    int maxLinks = ctA > ctB ? ctA : ctB;
    if (maxLinks < 1) maxLinks = 1;
    double fracMove = fracMoveBase / maxLinks;
    double g1 = fBTG[a], g2 = fBTG[b];
    double curForceMag = (fracMove * 1.0e-6 * stretch / dt) / (1.0 / g1 + 1.0 / g2);
    double Fx = curForceMag * lvx, Fy = curForceMag * lvy, Fz = curForceMag * lvz;
    double rax = (p1x - fC[a]) * 1e-6, ray = (p1y - fC[nSeg + a]) * 1e-6, raz = (p1z - fC[2 * nSeg + a]) * 1e-6;
    double TAx = ray * Fz - raz * Fy, TAy = raz * Fx - rax * Fz, TAz = rax * Fy - ray * Fx;
    double nFx = -Fx, nFy = -Fy, nFz = -Fz;
    double rbx = (p2x - fC[b]) * 1e-6, rby = (p2y - fC[nSeg + b]) * 1e-6, rbz = (p2z - fC[2 * nSeg + b]) * 1e-6;
    double TBx = rby * nFz - rbz * nFy, TBy = rbz * nFx - rbx * nFz, TBz = rbx * nFy - rby * nFx;
    out[0] = (float)Fx; out[1] = (float)Fy; out[2] = (float)Fz;
    out[3] = (float)TAx; out[4] = (float)TAy; out[5] = (float)TAz;
    out[6] = (float)nFx; out[7] = (float)nFy; out[8] = (float)nFz;
    out[9] = (float)TBx; out[10] = (float)TBy; out[11] = (float)TBz;
}

// CrosslinkerSystem.linkTorsion per link (CrosslinkerSystem.java:777-806); adds into xd row k
SBX_DEV void link_torsion_one(int k, int nSeg, const float* fU, int a, int b, int state, int orient, float* hist,
                              int* place, float* xd, double spring) {
    if (state < 0) return;
    if (a < 0 || b < 0) return;
    double uax = fU[a], uay = fU[nSeg + a], uaz = fU[2 * nSeg + a];
    double ubx = fU[b], uby = fU[nSeg + b], ubz = fU[2 * nSeg + b];
    bool same = orient != 0;
    double vbx = same ? ubx : -ubx, vby = same ? uby : -uby, vbz = same ? ubz : -ubz;
    double tx = uay * vbz - uaz * vby, ty = uaz * vbx - uax * vbz, tz = uax * vby - uay * vbx;
    double m2 = tx * tx + ty * ty + tz * tz;
    if (!(m2 > 1.0e-30)) return;
    double im = 1.0 / sqrt(m2);
    tx *= im; ty *= im; tz *= im;
    double dot = uax * ubx + uay * uby + uaz * ubz;
    if (dot > 1.0) dot = 1.0;
    if (dot < -1.0) dot = -1.0;
    double angT = same ? fast_acos(dot) : fabs(fast_acos(dot) - PI_D);
    double curMag = spring * angT;
    int base = k * TORQUE_WIN;
    int p = place[k];
    hist[base + p] = (float)curMag;
    place[k] = (p + 1) % TORQUE_WIN;
    double avg = 0.0;
    for (int j = 0; j < TORQUE_WIN; j++) avg += hist[base + j];
    avg /= TORQUE_WIN;
    double Tx = avg * tx, Ty = avg * ty, Tz = avg * tz;
    float* r = xd + (int64_t)k * XL_STRIDE;
    r[3] = (float)(r[3] + Tx);
    r[4] = (float)(r[4] + Ty);
    r[5] = (float)(r[5] + Tz);
    r[9] = (float)(r[9] - Tx);
    r[10] = (float)(r[10] - Ty);
    r[11] = (float)(r[11] - Tz);
}

// CrosslinkerSystem.unbind per ACTIVE link (CrosslinkerSystem.java:245-280); true = break
SBX_DEV bool unbind_one(int k, int nSeg, const float* fU, const float* fE1, int a, int b, float loc1k, float loc2k,
                        float* hist, int* place, const float* op, int32_t step, int32_t seed) {
    double offConst = op[0], offCoeff = op[1], offExp = op[2], dt = op[3], restLength = op[4];
    double l1 = loc1k;
    double uax = fU[a], uay = fU[nSeg + a], uaz = fU[2 * nSeg + a];
    double p1x = fE1[a] + l1 * uax, p1y = fE1[nSeg + a] + l1 * uay, p1z = fE1[2 * nSeg + a] + l1 * uaz;
    double l2 = loc2k;
    double ubx = fU[b], uby = fU[nSeg + b], ubz = fU[2 * nSeg + b];
    double p2x = fE1[b] + l2 * ubx, p2y = fE1[nSeg + b] + l2 * uby, p2z = fE1[2 * nSeg + b] + l2 * ubz;
    double lvx = p2x - p1x, lvy = p2y - p1y, lvz = p2z - p1z;
    double linkLength = sqrt(lvx * lvx + lvy * lvy + lvz * lvz);
    double stretch = linkLength - restLength;
    if (stretch < 0.0) stretch = 0.0;
    double strain = stretch / restLength;
    int base = k * STRAIN_WIN;
    int p = place[k];
    // the window with this step's entry replaced, summed in slot order
    float w[STRAIN_WIN];
    for (int j = 0; j < STRAIN_WIN; j++) w[j] = hist[base + j];
    hist[base + p] = (float)strain;
    place[k] = (p + 1) % STRAIN_WIN;
    double ave = 0.0;
    for (int j = 0; j < STRAIN_WIN; j++) ave += (j == p) ? (float)strain : w[j];
    ave /= STRAIN_WIN;
    double kOff = offConst + offCoeff * sbxm::exp(ave * offExp);
    double pBreak = kOff * dt;
    float u = unit_salted(k, step, seed, 0x584C4B42u);
    return u < pBreak;
}

// One motor joint (MotorJointSystem.java:86-197): which = 0 is joint 2 (rod-lever),
// which = 1 is joint 1 (lever-head). The position-only part, shared by the joint's two
// bodies; tm[0] / tm[1] are the torsion magnitudes for a nucleotide state other than /
// equal to ADP.Pi (joint 1's rest angle 60 / 0 degrees; joint 2 has one rest angle).
struct MotorJoint {
    double forceMag, lx, ly, lz, tvx, tvy, tvz, tm[2];
};

SBX_DEV MotorJoint motor_joint(int m, int which, int nB, const float* coord, const float* uVec,
                               const float* segLength, const float* bTG, const float* bRG, const float* jp) {
    const double DEG2RAD = PI_D / 180.0, RAD2DEG = 180.0 / PI_D;
    double dt = jp[0];
    int a = 3 * m + which, b = a + 1;           // (rod, lever) or (lever, head)
    double fracMove = which == 0 ? (double)jp[5] : (double)jp[1];
    double fracMoveTorq = which == 0 ? (double)jp[7] : (double)jp[3];
    double acx = coord[a], acy = coord[nB + a], acz = coord[2 * nB + a];
    double aux = uVec[a], auy = uVec[nB + a], auz = uVec[2 * nB + a];
    double alen = segLength[a];
    double bcx = coord[b], bcy = coord[nB + b], bcz = coord[2 * nB + b];
    double bux = uVec[b], buy = uVec[nB + b], buz = uVec[2 * nB + b];
    double blen = segLength[b];
    MotorJoint J;
    double aEx = acx + 0.5 * alen * aux, aEy = acy + 0.5 * alen * auy, aEz = acz + 0.5 * alen * auz;
    double bEx = bcx - 0.5 * blen * bux, bEy = bcy - 0.5 * blen * buy, bEz = bcz - 0.5 * blen * buz;
    double dx = aEx - bEx, dy = aEy - bEy, dz = aEz - bEz;
    double strain = sqrt(dx * dx + dy * dy + dz * dz);
    double inv = (strain > 0.0) ? 1.0 / strain : 0.0;
    double lx = dx * inv, ly = dy * inv, lz = dz * inv;
    double mcA = move_c(aux, auy, auz, lx, ly, lz, bTG[a], bTG[nB + a], bRG[nB + a], alen);
    double mcB = move_c(bux, buy, buz, lx, ly, lz, bTG[b], bTG[nB + b], bRG[nB + b], blen);
    double denom = dt * (mcA + mcB);
    J.forceMag = (denom > 0.0) ? (fracMove * 1.0e-6 * strain / denom) : 0.0;
    J.lx = lx; J.ly = ly; J.lz = lz;
    double tvx = auy * buz - auz * buy, tvy = auz * bux - aux * buz, tvz = aux * buy - auy * bux;
    double tvm2 = tvx * tvx + tvy * tvy + tvz * tvz;
    J.tm[0] = J.tm[1] = 0.0;
    if (tvm2 > 1.0e-30) {
        double im = 1.0 / sqrt(tvm2);
        tvx *= im; tvy *= im; tvz *= im;
        double dotV = aux * bux + auy * buy + auz * buz;
        if (dotV > 1.0) dotV = 1.0;
        if (dotV < -1.0) dotV = -1.0;
        double ang = accurate_acos(dotV) * RAD2DEG;
        double invBRG = 1.0 / bRG[nB + a] + 1.0 / bRG[nB + b];
        if (which == 0) {
            double j2Rest = jp[8];
            J.tm[0] = J.tm[1] = fracMoveTorq * DEG2RAD * (ang - j2Rest) / (invBRG * dt);
        } else {
            double maxMag = (double)jp[10] * 0.5 * blen * 1.0e-18;
            for (int r = 0; r < 2; r++) {
                double j1Rest = r == 0 ? 60.0 : 0.0;
                double tmag = fracMoveTorq * DEG2RAD * (ang - j1Rest) / (invBRG * dt);
                if (tmag > maxMag) tmag = maxMag;
                J.tm[r] = tmag;
            }
        }
    }
    J.tvx = tvx; J.tvy = tvy; J.tvz = tvz;
    return J;
}

// Adds joint J to body `s` (one of its two bodies; `second` = the lever of joint 2 or the
// head of joint 1) in double, the sequence of MotorJointSystem.java:124-137 / :175-188.
SBX_DEV void motor_joint_apply(const MotorJoint& J, int which, bool second, int nucState, int s, int nB,
                               const float* uVec, const float* segLength, const float* jp, double f[3],
                               double t[3]) {
    double fracR = which == 0 ? (double)jp[6] : (double)jp[2];
    double tm = J.tm[(which == 1 && nucState == NUC_ADPPI) ? 1 : 0];
    double ux = uVec[s], uy = uVec[nB + s], uz = uVec[2 * nB + s];
    double len = segLength[s];
    if (!second) {
        double Fx = -J.forceMag * J.lx, Fy = -J.forceMag * J.ly, Fz = -J.forceMag * J.lz;
        f[0] += Fx; f[1] += Fy; f[2] += Fz;
        double Rs = 0.5e-6 * len * fracR, Rx = Rs * ux, Ry = Rs * uy, Rz = Rs * uz;
        t[0] += Ry * Fz - Rz * Fy; t[1] += Rz * Fx - Rx * Fz; t[2] += Rx * Fy - Ry * Fx;
        t[0] += J.tvx * tm; t[1] += J.tvy * tm; t[2] += J.tvz * tm;
    } else {
        double Fx = J.forceMag * J.lx, Fy = J.forceMag * J.ly, Fz = J.forceMag * J.lz;
        f[0] += Fx; f[1] += Fy; f[2] += Fz;
        double Rs = -0.5e-6 * len * fracR, Rx = Rs * ux, Ry = Rs * uy, Rz = Rs * uz;
        t[0] += Ry * Fz - Rz * Fy; t[1] += Rz * Fx - Rx * Fz; t[2] += Rx * Fy - Ry * Fx;
        t[0] -= J.tvx * tm; t[1] -= J.tvy * tm; t[2] -= J.tvz * tm;
    }
}

// MotorJointSystem.joints for one sub-body (role 0 rod, 1 lever, 2 head), from zero
SBX_DEV void joints_one(int s, int nB, const float* coord, const float* uVec, const float* segLength,
                        const float* bTG, const float* bRG, int nucState, const float* jp, double f[3], double t[3]) {
    int m = s / 3, role = s - 3 * m;
    f[0] = f[1] = f[2] = 0.0;
    t[0] = t[1] = t[2] = 0.0;
    if (role == 0 || role == 1) {
        MotorJoint J = motor_joint(m, 0, nB, coord, uVec, segLength, bTG, bRG, jp);
        motor_joint_apply(J, 0, role == 1, nucState, s, nB, uVec, segLength, jp, f, t);
    }
    if (role == 1 || role == 2) {
        MotorJoint J = motor_joint(m, 1, nB, coord, uVec, segLength, bTG, bRG, jp);
        motor_joint_apply(J, 1, role == 2, nucState, s, nB, uVec, segLength, jp, f, t);
    }
}

// DimerCouplingSystem.couple per dimer (DimerCouplingSystem.java:99-182); self-writes rods/levers
// Force/torque accumulators addressed as (component k, body s): planar global arrays or a
// shared-memory window of them (the fused kernels keep a minifilament's sums on chip).
struct GlobalAcc {
    float* F; float* T; int n;
    SBX_DEV float& f(int k, int s) const { return F[k * n + s]; }
    SBX_DEV float& t(int k, int s) const { return T[k * n + s]; }
};
struct LocalAcc {
    float* F; float* T; int base, stride;
    SBX_DEV float& f(int k, int s) const { return F[k * stride + (s - base)]; }
    SBX_DEV float& t(int k, int s) const { return T[k * stride + (s - base)]; }
};

// DimerCouplingSystem.couple split into its position-only terms and their ordered
// accumulation: two end variants (rod-rod pull) and the lever torsion.
struct CoupleTerm {
    double FAx, FAy, FAz, TAx, TAy, TAz, TBx, TBy, TBz;
    int ok;                                      // strain > 0
};
struct LeverTerm {
    double px, py, pz;                           // tv * torsionMag
    int ok;                                      // tvm2 > 1e-30
};

SBX_DEV CoupleTerm couple_variant(int nB, const float* coord, const float* uVec, const float* segLength,
                                  const float* bTG, const float* bRG, int mA, int mB, bool par, const float* dp,
                                  int variant) {
    double dt = dp[0], fracMove = dp[1], rodLen = dp[4];
    int rodA = 3 * mA, rodB = 3 * mB;
    CoupleTerm C;
    double endSelA = (variant == 0) ? -1.0 : 1.0;
    double endSelB = par ? endSelA : -endSelA;
    double aCx = coord[rodA], aCy = coord[nB + rodA], aCz = coord[2 * nB + rodA];
    double aUx = uVec[rodA], aUy = uVec[nB + rodA], aUz = uVec[2 * nB + rodA];
    double bCx = coord[rodB], bCy = coord[nB + rodB], bCz = coord[2 * nB + rodB];
    double bUx = uVec[rodB], bUy = uVec[nB + rodB], bUz = uVec[2 * nB + rodB];
    double aLen = segLength[rodA], bLen = segLength[rodB];
    double pAx = aCx + endSelA * 0.5 * aLen * aUx, pAy = aCy + endSelA * 0.5 * aLen * aUy,
           pAz = aCz + endSelA * 0.5 * aLen * aUz;
    double pBx = bCx + endSelB * 0.5 * bLen * bUx, pBy = bCy + endSelB * 0.5 * bLen * bUy,
           pBz = bCz + endSelB * 0.5 * bLen * bUz;
    double dx = pBx - pAx, dy = pBy - pAy, dz = pBz - pAz;
    double strain = sqrt(dx * dx + dy * dy + dz * dz);
    C.ok = strain > 0.0;
    if (C.ok) {
        double inv = 1.0 / strain;
        double lx = dx * inv, ly = dy * inv, lz = dz * inv;
        double mcA = move_c(aUx, aUy, aUz, lx, ly, lz, bTG[rodA], bTG[nB + rodA], bRG[nB + rodA], aLen);
        double mcB = move_c(bUx, bUy, bUz, lx, ly, lz, bTG[rodB], bTG[nB + rodB], bRG[nB + rodB], bLen);
        double denom = dt * (mcA + mcB);
        double forceMag = (denom > 0.0) ? (fracMove * 1.0e-6 * strain / denom) : 0.0;
        double FAx = forceMag * lx, FAy = forceMag * ly, FAz = forceMag * lz;
        double RsA = 0.5e-6 * rodLen * endSelA;
        C.TAx = (RsA * aUy) * FAz - (RsA * aUz) * FAy;
        C.TAy = (RsA * aUz) * FAx - (RsA * aUx) * FAz;
        C.TAz = (RsA * aUx) * FAy - (RsA * aUy) * FAx;
        double RsB = 0.5e-6 * rodLen * endSelB;
        C.TBx = (RsB * bUy) * (-FAz) - (RsB * bUz) * (-FAy);
        C.TBy = (RsB * bUz) * (-FAx) - (RsB * bUx) * (-FAz);
        C.TBz = (RsB * bUx) * (-FAy) - (RsB * bUy) * (-FAx);
        C.FAx = FAx; C.FAy = FAy; C.FAz = FAz;
    }
    return C;
}

SBX_DEV LeverTerm couple_lever(int nB, const float* uVec, const float* bRG, int mA, int mB, const float* dp) {
    double dt = dp[0], leverTorq = dp[2], leverDeg = dp[3];
    int leverA = 3 * mA + 1, leverB = 3 * mB + 1;
    LeverTerm L;
    double u1x = uVec[leverA], u1y = uVec[nB + leverA], u1z = uVec[2 * nB + leverA];
    double u2x = uVec[leverB], u2y = uVec[nB + leverB], u2z = uVec[2 * nB + leverB];
    double tvx = u1y * u2z - u1z * u2y, tvy = u1z * u2x - u1x * u2z, tvz = u1x * u2y - u1y * u2x;
    double tvm2 = tvx * tvx + tvy * tvy + tvz * tvz;
    L.ok = tvm2 > 1.0e-30;
    if (L.ok) {
        double im = 1.0 / sqrt(tvm2);
        tvx *= im; tvy *= im; tvz *= im;
        double dot = u1x * u2x + u1y * u2y + u1z * u2z;
        if (dot > 1.0) dot = 1.0;
        if (dot < -1.0) dot = -1.0;
        double ang = accurate_acos(dot) * 180.0 / PI_D;
        double invBRG = 1.0 / bRG[nB + leverA] + 1.0 / bRG[nB + leverB];
        double torsionMag = leverTorq * (PI_D / 180.0) * (ang - leverDeg) / (invBRG * dt);
        L.px = tvx * torsionMag; L.py = tvy * torsionMag; L.pz = tvz * torsionMag;
    }
    return L;
}

// the variant's float accumulation into rod A (sign +) or rod B (force -, torque TB)
template <class Acc>
SBX_DEV void couple_apply_rod(const Acc& acc, int body, bool isA, const CoupleTerm& C) {
    if (!C.ok) return;
    if (isA) {
        acc.f(0, body) = (float)(acc.f(0, body) + C.FAx);
        acc.f(1, body) = (float)(acc.f(1, body) + C.FAy);
        acc.f(2, body) = (float)(acc.f(2, body) + C.FAz);
        acc.t(0, body) = (float)(acc.t(0, body) + C.TAx);
        acc.t(1, body) = (float)(acc.t(1, body) + C.TAy);
        acc.t(2, body) = (float)(acc.t(2, body) + C.TAz);
    } else {
        acc.f(0, body) = (float)(acc.f(0, body) - C.FAx);
        acc.f(1, body) = (float)(acc.f(1, body) - C.FAy);
        acc.f(2, body) = (float)(acc.f(2, body) - C.FAz);
        acc.t(0, body) = (float)(acc.t(0, body) + C.TBx);
        acc.t(1, body) = (float)(acc.t(1, body) + C.TBy);
        acc.t(2, body) = (float)(acc.t(2, body) + C.TBz);
    }
}

template <class Acc>
SBX_DEV void couple_apply_lever(const Acc& acc, int body, bool isA, const LeverTerm& L) {
    if (!L.ok) return;
    if (isA) {
        acc.t(0, body) = (float)(acc.t(0, body) + L.px);
        acc.t(1, body) = (float)(acc.t(1, body) + L.py);
        acc.t(2, body) = (float)(acc.t(2, body) + L.pz);
    } else {
        acc.t(0, body) = (float)(acc.t(0, body) - L.px);
        acc.t(1, body) = (float)(acc.t(1, body) - L.py);
        acc.t(2, body) = (float)(acc.t(2, body) - L.pz);
    }
}

// DimerCouplingSystem.couple per dimer (DimerCouplingSystem.java:99-182); self-writes rods/levers
template <class Acc>
SBX_DEV void couple_one(int nB, const float* coord, const float* uVec, const float* segLength, const float* bTG,
                        const float* bRG, const Acc& acc, int mA, int mB, bool par, const float* dp,
                        const int* boundSeg) {
    for (int variant = 0; variant < 2; variant++) {
        CoupleTerm C = couple_variant(nB, coord, uVec, segLength, bTG, bRG, mA, mB, par, dp, variant);
        couple_apply_rod(acc, 3 * mA, true, C);
        couple_apply_rod(acc, 3 * mB, false, C);
    }
    bool bothBound = boundSeg[mA] >= 0 && boundSeg[mB] >= 0;
    if (par && !bothBound) {
        LeverTerm L = couple_lever(nB, uVec, bRG, mA, mB, dp);
        couple_apply_lever(acc, 3 * mA + 1, true, L);
        couple_apply_lever(acc, 3 * mB + 1, false, L);
    }
}

// MiniFilamentSystem.tether per dimer (MiniFilamentSystem.java:77-131): the rod-A terms
// (force if strain > 0, torque tv * tmag if tvm2 > 1e-30) and the backbone reaction row.
struct TetherTerm {
    double Fx, Fy, Fz, Tx, Ty, Tz;
    int fOK, tOK;
    float row[6];                                // miniData row (reaction on the backbone)
};

SBX_DEV TetherTerm tether_terms(int nMB, const float* mC, const float* mU, const float* mL, const float* mBTG,
                                const float* mBRG, int nBb, const float* bbC, const float* bbU, const float* inv,
                                int bb, int mA, float axf, const float* mp) {
    double dt = mp[0], fracMove = mp[1], align = mp[2];
    int rodA = 3 * mA;
    double ax = axf;
    TetherTerm T;
    double bcx = bbC[bb], bcy = bbC[nBb + bb], bcz = bbC[2 * nBb + bb];
    double bux = bbU[bb], buy = bbU[nBb + bb], buz = bbU[2 * nBb + bb];
    double pax = bcx + ax * bux, pay = bcy + ax * buy, paz = bcz + ax * buz;
    double rcx = mC[rodA], rcy = mC[nMB + rodA], rcz = mC[2 * nMB + rodA];
    double rux = mU[rodA], ruy = mU[nMB + rodA], ruz = mU[2 * nMB + rodA];
    double rlen = mL[rodA];
    double re1x = rcx - 0.5 * rlen * rux, re1y = rcy - 0.5 * rlen * ruy, re1z = rcz - 0.5 * rlen * ruz;
    double fbx = 0, fby = 0, fbz = 0, tbx = 0, tby = 0, tbz = 0;
    double dx = pax - re1x, dy = pay - re1y, dz = paz - re1z;
    double strain = sqrt(dx * dx + dy * dy + dz * dz);
    T.fOK = strain > 0.0;
    if (T.fOK) {
        double iv = 1.0 / strain;
        double lx = dx * iv, ly = dy * iv, lz = dz * iv;
        double denom = dt * (1.0 / mBTG[nMB + rodA] + inv[bb]);
        double forceMag = (denom > 0.0) ? (fracMove * 1.0e-6 * strain / denom) : 0.0;
        T.Fx = forceMag * lx; T.Fy = forceMag * ly; T.Fz = forceMag * lz;
        fbx = -T.Fx; fby = -T.Fy; fbz = -T.Fz;
    }
    double alignSign = (ax < 0.0) ? -1.0 : 1.0;
    double tux = alignSign * bux, tuy = alignSign * buy, tuz = alignSign * buz;
    double tvx = ruy * tuz - ruz * tuy, tvy = ruz * tux - rux * tuz, tvz = rux * tuy - ruy * tux;
    double tvm2 = tvx * tvx + tvy * tvy + tvz * tvz;
    T.tOK = tvm2 > 1.0e-30;
    if (T.tOK) {
        double im = 1.0 / sqrt(tvm2);
        tvx *= im; tvy *= im; tvz *= im;
        double dot = rux * tux + ruy * tuy + ruz * tuz;
        if (dot > 1.0) dot = 1.0;
        if (dot < -1.0) dot = -1.0;
        double angDeg = accurate_acos(dot) * 180.0 / PI_D;
        double denomR = (1.0 / mBRG[nMB + rodA] + inv[nBb + bb]) * dt;
        double tmag = align * (PI_D / 180.0) * angDeg / denomR;
        T.Tx = tvx * tmag; T.Ty = tvy * tmag; T.Tz = tvz * tmag;
        tbx = -tvx * tmag; tby = -tvy * tmag; tbz = -tvz * tmag;
    }
    T.row[0] = (float)fbx; T.row[1] = (float)fby; T.row[2] = (float)fbz;
    T.row[3] = (float)tbx; T.row[4] = (float)tby; T.row[5] = (float)tbz;
    return T;
}

template <class Acc>
SBX_DEV void tether_apply(const Acc& acc, int rodA, const TetherTerm& T) {
    if (T.fOK) {
        acc.f(0, rodA) = (float)(acc.f(0, rodA) + T.Fx);
        acc.f(1, rodA) = (float)(acc.f(1, rodA) + T.Fy);
        acc.f(2, rodA) = (float)(acc.f(2, rodA) + T.Fz);
    }
    if (T.tOK) {
        acc.t(0, rodA) = (float)(acc.t(0, rodA) + T.Tx);
        acc.t(1, rodA) = (float)(acc.t(1, rodA) + T.Ty);
        acc.t(2, rodA) = (float)(acc.t(2, rodA) + T.Tz);
    }
}

template <class Acc>
SBX_DEV void tether_one(int d, int nMB, const float* mC, const float* mU, const float* mL, const float* mBTG,
                        const float* mBRG, const Acc& acc, int nBb, const float* bbC, const float* bbU,
                        const float* inv, int bb, int mA, float axf, float* miniData, const float* mp) {
    TetherTerm T = tether_terms(nMB, mC, mU, mL, mBTG, mBRG, nBb, bbC, bbU, inv, bb, mA, axf, mp);
    tether_apply(acc, 3 * mA, T);
    float* o = miniData + (int64_t)MINI_STRIDE * d;
    for (int k = 0; k < 6; k++) o[k] = T.row[k];
}

// integrate + derive one body slot from accumulated F/T (registers), the slot's stored
// Brownian draws and drag, then store pose, derived geometry and the final F/T sums
// (MechanicsFusion.integDerive, MechanicsFusion.java:129-200)
SBX_DEV void integrate_derive_store(const sbx_rigid_body& b, int s, const float F[3], const float T[3], float dt) {
    const int n = b.n;
    Pose p, q;
    float rf[3], rt[3], gT[3], gR[3], dc[3];
    // every input read up front, so that the loads are in flight together
    double c64[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < 3; k++) {
        p.c[k] = b.coord[k * n + s]; p.u[k] = b.uVec[k * n + s]; p.y[k] = b.yVec[k * n + s];
        rf[k] = b.randForce[k * n + s]; rt[k] = b.randTorque[k * n + s];
        gT[k] = b.bTransGam[k * n + s]; gR[k] = b.bRotGam[k * n + s];
        if (b.coord64) c64[k] = b.coord64[k * n + s];
    }
    const float len = b.segLength[s];
    integrate_pose(p, F, T, rf, rt, gT, gR, dt, q, dc);
    if (b.coord64) {
        for (int k = 0; k < 3; k++) {
            double c = c64[k] + (double)dc[k];
            b.coord64[k * n + s] = c;
            q.c[k] = (float)c;
        }
    }
    float z[3], e1[3], e2[3];
    derive_pose(q.c, q.u, q.y, z, e1, e2, len);
    for (int k = 0; k < 3; k++) {
        b.coord[k * n + s] = q.c[k]; b.uVec[k * n + s] = q.u[k]; b.yVec[k * n + s] = q.y[k];
        b.zVec[k * n + s] = z[k]; b.end1[k * n + s] = e1[k]; b.end2[k * n + s] = e2[k];
        b.forceSum[k * n + s] = F[k]; b.torqueSum[k * n + s] = T[k];
    }
}

}  // namespace sbx
