"""The reference harnesses' physics gates, as scene builders and step sequences that run on
either the CPU oracle or the CUDA library (the same sequence, the same arguments).

  * motor off-rate (MotorBindingHarness.reportOffRate, MotorBindingHarness.java:437-458):
    bound heads released by NucleotideCycleSystem.catchSlipRelease; the empirical per-step
    release probability releases / bound-steps equals k_off(F) dt, with
    k_off(F) = kOff (aCatch e^(-F xCatch / kT) + aSlip e^(F xSlip / kT)) (NucleotideCycleSystem.java:116);
    F = 0 is the reference's gate (k_off = kOff).
  * confined-rod equipartition (ThermostatDiag.confinedRodVar, ThermostatDiag.java:84-124):
    <theta^2> of a rod held to +z by the torsional fracMove restore equals the discrete AR(1)
    value 4 kT dt / (gamma c (2 - c)) (ThermostatDiag.java:56-58).
  * crosslinker rest hold and stretch relaxation (CrosslinkerHarness.check1RestHold and
    check2Relax, CrosslinkerHarness.java:279-347): two parallel single-segment filaments and
    one link; at rest length with Brownian off nothing moves (max |d coord| == 0); stretched,
    the centre of mass stays put while the separation relaxes; a small stretch decays per
    step by k = fracMove (gamma_par / gamma_perp) L, independently of dt.
"""
import math

import numpy as np

from softbox_b200 import scenes

F32, I32 = np.float32, np.int32


# ----------------------------------------------------------------------------- backends
class OracleBackend:
    """Host arrays, the oracle's methods."""

    def __init__(self, orc):
        self.o = orc

    def put(self, d):
        return d

    def get(self, a):
        return np.asarray(a)

    def sync(self):
        pass

    def release(self, m):
        self.o.catch_slip_release(m["n"], m["boundSeg"], m["forceDotFil"], m["forceMag"], m["cooldown"], m["stats"],
                                  m["capStats"], m["kinParams"], m["counts"])

    def rebind(self, m, seg):
        bs = m["boundSeg"]
        bs[bs == -1] = seg

    def set_step(self, counts, t):
        counts[1] = t

    def zero(self, b):
        self.o.zero_accumulators(b["n"], b["forceSum"], b["torqueSum"])

    def brownian(self, b, params, counts):
        self.o.brownian_force(b["n"], b["randForce"], b["randTorque"], b["bTransGam"], b["bRotGam"],
                              b["brownTransScale"], b["brownRotScale"], params, counts)

    def restore(self, b, reps, coeff, dt):
        self.o.torsional_restore(reps, b["uVec"], b["bRotGam"], b["torqueSum"], coeff, dt)

    def integrate_derive(self, b, params):
        self.o.integrate(b["n"], b["coord"], None, b["uVec"], b["yVec"], b["forceSum"], b["torqueSum"],
                         b["randForce"], b["randTorque"], b["bTransGam"], b["bRotGam"], params)
        self.o.derive(b["n"], b["coord"], b["uVec"], b["yVec"], b["zVec"], b["end1"], b["end2"], b["segLength"])

    def links(self, b, x):
        n, k = b["n"], x["nLinks"]
        self.o.link_forces(n, b["coord"], b["uVec"], b["end1"], b["bTransGam"], k, x["linkFilA"], x["linkFilB"],
                           x["loc1"], x["loc2"], x["filLinkCt"], x["xlinkData"], x["xlParams"])
        for side, key in ((0, "linkFilA"), (1, "linkFilB")):
            cnt, off, lst = x["cnt"][side], x["off"][side], x["lst"][side]
            self.o.csr_histogram(x[key], k, n, cnt)
            self.o.csr_scan(n, cnt, off)
            self.o.csr_scatter(x[key], k, off, cnt, lst)
            g = self.o.seg_gather_a if side == 0 else self.o.seg_gather_b
            g(n, off, lst, x["xlinkData"], x["linkState"], b["forceSum"], b["torqueSum"])


class GpuBackend:
    """torch CUDA tensors, the library's entry points (softbox_b200.systems)."""

    def __init__(self):
        import torch
        from softbox_b200 import systems
        self.torch, self.S = torch, systems

    def put(self, d):
        from softbox_b200 import device as D
        return D.to_device(d)

    def get(self, a):
        return a.detach().cpu().numpy()

    def sync(self):
        self.torch.cuda.synchronize()

    def release(self, m):
        self.S.NucleotideCycleSystem.catchSlipRelease(m["boundSeg"], m["forceDotFil"], m["forceMag"], m["cooldown"],
                                                      m["stats"], m["capStats"], m["kinParams"], m["counts"])

    def rebind(self, m, seg):
        bs = m["boundSeg"]
        bs.masked_fill_(bs == -1, seg)

    def set_step(self, counts, t):
        counts[1] = t

    def zero(self, b):
        self.S.ChainBendingForceSystem.zeroAccumulators(b["forceSum"], b["torqueSum"])

    def brownian(self, b, params, counts):
        self.S.BrownianForceSystem.brownianForce(b["randForce"], b["randTorque"], b["bTransGam"], b["bRotGam"],
                                                 b["brownTransScale"], b["brownRotScale"], params, counts)

    def restore(self, b, reps, coeff, dt):
        self.S.ThermostatDiag.torsionalRestore(b["uVec"], b["bRotGam"], b["torqueSum"], reps, coeff, dt)

    def integrate_derive(self, b, params):
        S = self.S
        S.RigidRodLangevinIntegrationSystem.integrate(b["coord"], b["uVec"], b["yVec"], b["forceSum"], b["torqueSum"],
                                                      b["randForce"], b["randTorque"], b["bTransGam"], b["bRotGam"],
                                                      params)
        S.DerivedGeometrySystem.derive(b["coord"], b["uVec"], b["yVec"], b["zVec"], b["end1"], b["end2"],
                                       b["segLength"])

    def links(self, b, x):
        S = self.S
        S.CrosslinkerSystem.linkForces(b["coord"], b["uVec"], b["end1"], b["bTransGam"], x["linkFilA"], x["linkFilB"],
                                       x["loc1"], x["loc2"], x["filLinkCt"], x["xlinkData"], x["xlParams"])
        n = b["segLength"].numel()
        for side, key in ((0, "linkFilA"), (1, "linkFilB")):
            cnt, off, lst = x["cnt"][side], x["off"][side], x["lst"][side]
            S.CrossBridgeSystem.csrBuild(x[key], n, cnt, off, lst)
            g = S.CrosslinkerSystem.segGatherA if side == 0 else S.CrosslinkerSystem.segGatherB
            g(off, lst, x["xlinkData"], x["linkState"], b["forceSum"], b["torqueSum"])


# ----------------------------------------------------------------------------- motor off-rate
KOFF, A_CATCH, A_SLIP, X_CATCH, X_SLIP = 100.0, 0.92, 0.08, 2.5e-9, 0.4e-9   # MotorStore.java:191-195


def release_bed(n=6400, force=0.0, dt=1.0e-5, seed=0x4A11):
    """n heads bound to segment 0 with a fixed force-dot F (N) and forceMag 0, the reference's
    kinParams (MotorStore.setKinParams, MotorStore.java:190-212: 1-step refractory, cap off)."""
    kp = np.zeros(14, F32)
    kp[:7] = [KOFF, A_CATCH, A_SLIP, X_CATCH, X_SLIP, scenes.KT, dt]
    kp[10], kp[11], kp[12], kp[13] = math.ceil(scenes.MYO_REBIND_TIME / dt), 12.0e-12, 0.0, 1.0
    return {"n": n, "boundSeg": np.zeros(n, I32), "forceDotFil": np.full(n, force, F32),
            "forceMag": np.zeros(n, F32), "cooldown": np.zeros(n, I32), "stats": np.zeros(2 * n, I32),
            "capStats": np.zeros(n, I32), "kinParams": kp, "counts": np.array([n, 0, seed, 1], I32)}


def run_release(be, m, steps):
    """Release each step; a head whose refractory has elapsed rebinds to segment 0 (the
    deterministic bind of the reference's gate scene)."""
    for t in range(steps):
        be.set_step(m["counts"], t)
        be.release(m)
        be.rebind(m, 0)
    be.sync()


def off_rate(stats, force=0.0, dt=1.0e-5):
    """(empirical p, analytic k_off(F) dt, binomial standard error of p)."""
    s = np.asarray(stats, np.int64).reshape(-1, 2)
    bound, rel = int(s[:, 0].sum()), int(s[:, 1].sum())
    kT = float(F32(scenes.KT))
    k = KOFF * (A_CATCH * math.exp(-force * X_CATCH / kT) + A_SLIP * math.exp(force * X_SLIP / kT))
    p = k * dt
    return rel / bound, p, math.sqrt(p * (1 - p) / bound)


# ----------------------------------------------------------------------------- equipartition
def confined_rods(reps=2000, dt=1.0e-5, seed=0x7E120D):
    """ThermostatDiag.confinedRodVar's scene: per motor slot a rod at the origin along +z with
    rotational Brownian only, its lever and head parked and inert."""
    nB = 3 * reps
    b = scenes.rigid_body(nB)
    for mm in range(reps):
        r, lv, hd = 3 * mm, 3 * mm + 1, 3 * mm + 2
        scenes.set_vec(b["uVec"], nB, r, 0, 0, 1)
        scenes.set_vec(b["yVec"], nB, r, 1, 0, 0)
        scenes.set_vec(b["coord"], nB, lv, 10, 0, 0)
        scenes.set_vec(b["uVec"], nB, lv, 1, 0, 0)
        scenes.set_vec(b["yVec"], nB, lv, 0, 1, 0)
        scenes.set_vec(b["coord"], nB, hd, 20, 0, 0)
        scenes.set_vec(b["uVec"], nB, hd, 1, 0, 0)
        scenes.set_vec(b["yVec"], nB, hd, 0, 1, 0)
        b["brownRotScale"][r] = 1.0
        b["segLength"][r] = F32(scenes.ROD_LEN)
        scenes.store_drag(b, r, scenes.rod_drag_si(scenes.ROD_LEN, scenes.ROD_R, 0.1))
        scenes.store_drag(b, lv, scenes.rod_drag_si(scenes.LEVER_LEN, scenes.LEVER_R, 0.1))
        scenes.store_drag(b, hd, scenes.sphere_drag_si(scenes.HEAD_R, 0.1))
    params = np.array([dt, np.sqrt(2 * scenes.KT / dt)], F32)
    counts = np.array([reps, 0, seed, 0], I32)
    return {"b": b, "params": params, "counts": counts, "reps": reps, "dt": dt}


def run_equipartition(be, sc, burn, steps, every, coeff=0.4):
    """Runs the confined-rod steps; returns (<theta^2> over samples, prediction)."""
    b, params, counts = sc["b"], sc["params"], sc["counts"]
    reps, dt = sc["reps"], sc["dt"]
    nB = 3 * reps
    s2, n = 0.0, 0
    for t in range(burn + steps):
        be.set_step(counts, t)
        be.zero(b)
        be.brownian(b, params, counts)
        be.restore(b, reps, coeff, dt)
        be.integrate_derive(b, params)
        if t >= burn and (t - burn) % every == 0:
            uz = np.clip(np.asarray(be.get(b["uVec"]), np.float64)[2 * nB:][0::3], -1.0, 1.0)
            s2 += float((np.arccos(uz) ** 2).sum())
            n += reps
    bRGy = float(np.asarray(be.get(b["bRotGam"]))[nB + 0])
    pred = 4.0 * scenes.KT * dt / (bRGy * coeff * (2.0 - coeff))
    return s2 / n, pred


# ----------------------------------------------------------------------------- crosslinker pair
XL_REST = 0.0125            # CrosslinkerHarness.REST_LEN (CrosslinkerHarness.java:51)
XL_FRAC_MOVE = 0.4          # CrosslinkerHarness.FRAC_MOVE (:52)


def xlink_pair(sep, dt=1.0e-5, shear_x=0.0):
    """CrosslinkerHarness.buildScene (CrosslinkerHarness.java:147-178): two 32-monomer
    single-segment filaments along x, the second at (shearX, 0, sep), Brownian off, one link
    midpoint to midpoint."""
    f = scenes.filament_store(2)
    b = f["body"]
    f["monomerCount"][:] = scenes.STD_SEG_LENGTH
    for s in range(2):
        scenes.set_vec(b["uVec"], 2, s, 1, 0, 0)
        scenes.set_vec(b["yVec"], 2, s, 0, 1, 0)
    b["brownTransScale"][:] = 0.0
    b["brownRotScale"][:] = 0.0
    scenes.set_vec(b["coord"], 2, 0, 0, 0, 0)
    scenes.set_vec(b["coord"], 2, 1, shear_x, 0, sep)
    scenes.drag_run_filament(f, 0.1)
    params = np.array([dt, math.sqrt(2.0 * scenes.KT / dt)], F32)
    counts = np.array([2, 0, 0x5A11, 1], I32)
    scenes.derive_host(b)
    L = (scenes.STD_SEG_LENGTH + 1) * scenes.ACTIN_MONO_RADIUS
    x = {"nLinks": 1, "linkFilA": np.array([0], I32), "linkFilB": np.array([1], I32),
         "loc1": np.array([0.5 * L], F32), "loc2": np.array([0.5 * L], F32), "linkState": np.array([0], I32),
         "filLinkCt": np.array([1, 1], I32), "xlinkData": np.zeros(12, F32),
         "xlParams": np.array([XL_REST, XL_FRAC_MOVE, dt], F32),
         "cnt": [np.zeros(2, I32), np.zeros(2, I32)], "off": [np.zeros(3, I32), np.zeros(3, I32)],
         "lst": [np.zeros(1, I32), np.zeros(1, I32)]}
    return {"b": b, "x": x, "params": params, "counts": counts}


def put_pair(be, sc):
    out = dict(sc)
    out["b"] = be.put(sc["b"])
    x = dict(sc["x"])
    for k in ("cnt", "off", "lst"):
        x[k] = [be.put(a) for a in sc["x"][k]]
    out["x"] = {k: (be.put(v) if isinstance(v, np.ndarray) else v) for k, v in x.items()}
    out["x"].update({k: x[k] for k in ("cnt", "off", "lst")})
    out["params"] = be.put(sc["params"])
    out["counts"] = be.put(sc["counts"])
    return out


def step_pair(be, sc, t):
    """CrosslinkerHarness.cpuStep (CrosslinkerHarness.java:186-214), unbinding off."""
    b = sc["b"]
    be.set_step(sc["counts"], t)
    be.zero(b)
    be.brownian(b, sc["params"], sc["counts"])
    be.links(b, sc["x"])
    be.integrate_derive(b, sc["params"])


def coords(be, sc):
    return np.asarray(be.get(sc["b"]["coord"]), np.float64)


def rest_hold(be, dt=1.0e-5, M=1000):
    """(a) max |d coord| at exact rest; (b) stretched release: (COM-z drift relative to the
    relaxation, start separation, end separation)."""
    a = put_pair(be, xlink_pair(XL_REST, dt))
    c0 = coords(be, a)
    for t in range(M):
        step_pair(be, a, t)
    be.sync()
    drift = float(np.abs(coords(be, a) - c0).max())
    s = put_pair(be, xlink_pair(2.0 * XL_REST, dt))
    c = coords(be, s)
    com0, sep0 = 0.5 * (c[4] + c[5]), c[5] - c[4]
    worst = 0.0
    for t in range(M):
        step_pair(be, s, t)
        c = coords(be, s)
        worst = max(worst, abs(0.5 * (c[4] + c[5]) - com0))
    sep_end = c[5] - c[4]
    return drift, worst / abs(sep0 - sep_end), sep0, sep_end


def stretch_decay(be, dt, M=2000, floor=1.0e-5):
    """CrosslinkerHarness.measureDecay (CrosslinkerHarness.java:325-344): mean observed and
    predicted per-step decay rates of a small perpendicular stretch over the clean window."""
    eps0 = 0.05 * XL_REST
    s = put_pair(be, xlink_pair(XL_REST + eps0, dt))
    bh = {k: np.asarray(be.get(v)) for k, v in s["b"].items() if k in ("bTransGam",)}
    g_par, g_perp = float(bh["bTransGam"][0]), float(bh["bTransGam"][2])
    c = coords(be, s)
    eps = [c[5] - c[4] - XL_REST]
    for t in range(M):
        step_pair(be, s, t)
        c = coords(be, s)
        eps.append(c[5] - c[4] - XL_REST)
    ko, kp = [], []
    for t in range(M):
        e, e1 = eps[t], eps[t + 1]
        if e < floor or e1 <= 0:
            continue
        ko.append((e - e1) / e)
        kp.append(XL_FRAC_MOVE * (g_par / g_perp) * (e + XL_REST))
    return float(np.mean(ko)), float(np.mean(kp)), len(ko)


# ----------------------------------------------------------------------------- crowded reach
def crowded_dense():
    """A small dense network (8,000 rods, 128 heads) packed into a 1 x 1 x 0.5 um slab with a
    0.5 um binding reach: a head has about 230 reachable segments on average and a few dozen
    have more than SpatialGrid.MAX_CAND (256)."""
    from dataclasses import replace
    cfg = replace(scenes.C1, n_fil=800, n_mini=4, n_links=100, side=1.0, myo_col_tol=0.5)
    return scenes.dense_contractile(cfg)
