"""Many independent dense networks advanced together: packing, the batched plan, unpacking.

    packed, info = pack_networks([scenes.dense_contractile(c) for c in configs])
    ens = BatchedNetworks(packed, info)
    ens.run(0, 1000)                          # one launch per step phase for every network
    fil_k = ens.network(k)["fil"]             # network k's arrays, as if it ran alone

Network k owns a contiguous index range of every store (segments, motors and their three
bodies, dimers, backbones, links) and its own grid cells; cross-store indices (chain
neighbours, bound segments, link ends, dimer motors, backbone slots) are offset by the
packer. The library's batched kernels key every draw by the item's local index and its
network's seed and use the network's own grid and walls (sbx_batch), so each network's
trajectory is the one it has when run alone, bit for bit.
"""
import ctypes as C

import numpy as np

from . import abi_types as T
from . import device as D
from .device import DeviceFill

I32, F32 = np.int32, np.float32

# arrays whose items are stored planar: [3][n] (or [2][n]) with n the store's item count
_PLANAR3 = ("coord", "uVec", "yVec", "zVec", "end1", "end2", "bTransGam", "bRotGam", "bTransDiff", "bRotDiff",
            "forceSum", "torqueSum", "randForce", "randTorque")


def _planar(arrs, ns, width):
    return np.concatenate([a.reshape(width, n) for a, n in zip(arrs, ns)], axis=1).reshape(-1)


def _offset(arrs, bases):
    out = []
    for a, b in zip(arrs, bases):
        a = a.copy()
        a[a >= 0] += b
        out.append(a)
    return np.concatenate(out)


def _same(arrs, what):
    for a in arrs[1:]:
        if not np.array_equal(a, arrs[0]):
            raise ValueError(f"{what} differs between networks; the batch shares it")
    return arrs[0].copy()


def _body(bodies):
    ns = [b["n"] for b in bodies]
    out = {"n": int(sum(ns)), "coord64": None}
    for k in _PLANAR3:
        out[k] = _planar([b[k] for b in bodies], ns, 3)
    for k in ("segLength", "brownTransScale", "brownRotScale"):
        out[k] = np.concatenate([b[k] for b in bodies])
    return out


def _bases(ns):
    return np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)


def _keys(ns):
    return np.concatenate([np.stack([np.full(n, k, I32), np.arange(n, dtype=I32)], axis=1).reshape(-1)
                           for k, n in enumerate(ns)]).astype(I32) if len(ns) else np.zeros(0, I32)


def pack_networks(scenes_):
    """One packed dense scene and the batch tables for a list of dense scenes
    (scenes.dense_contractile); the networks share every parameter array (dt, chain,
    kinetics, link and containment laws) and differ in size, composition and seeds."""
    S = list(scenes_)
    nS = [s["fil"]["body"]["n"] for s in S]
    nM = [s["mot"]["nMotors"] for s in S]
    nBb = [s["mini"]["nBackbones"] for s in S]
    nD = [s["dim"]["nDimers"] for s in S]
    nL = [s["xl"]["nLinks"] for s in S]
    cells = [s["grid"]["totalCells"] for s in S]
    sB, mB, bbB, dB, cB = _bases(nS), _bases(nM), _bases(nBb), _bases(nD), _bases(cells)
    NS, NM, NBB, ND, NL, NC = (int(sum(x)) for x in (nS, nM, nBb, nD, nL, cells))

    fil = {"body": _body([s["fil"]["body"] for s in S])}
    for k in ("monomerCount", "filState", "end1NbrSide", "end2NbrSide"):
        fil[k] = np.concatenate([s["fil"][k] for s in S])
    for k in ("end1NbrSlot", "end2NbrSlot"):
        fil[k] = _offset([s["fil"][k] for s in S], sB)
    fil["params"] = _same([s["fil"]["params"] for s in S], "fil.params")
    fil["chainParams"] = _same([s["fil"]["chainParams"] for s in S], "fil.chainParams")
    fil["counts"] = np.array([NS, 0, S[0]["fil"]["counts"][2], S[0]["fil"]["counts"][3]], I32)
    fil["extForce"] = _planar([s["fil"]["extForce"] for s in S], nS, 3)

    mot = {"body": _body([s["mot"]["body"] for s in S]), "nMotors": NM}
    for k in ("head", "uVec", "rodUVec"):
        mot[k] = _planar([s["mot"][k] for s in S], nM, 3)
    for k in ("reach", "bindArc", "capStats", "cooldown", "nucleotideState", "forceDotPlace", "forceDotFil",
              "forceMag", "stats", "forceDotHist"):
        mot[k] = np.concatenate([s["mot"][k] for s in S])
    mot["boundSeg"] = _offset([s["mot"]["boundSeg"] for s in S], sB)
    for k in ("bodyParams", "jointParams", "kinParams", "nucParams"):
        mot[k] = _same([s["mot"][k] for s in S], "mot." + k)
    mot["counts"] = np.array([NM, 0, S[0]["seed"], NS], I32)
    mot["publishParams"] = np.array([NS], I32)

    dim = {"nDimers": ND, "motorA": _offset([s["dim"]["motorA"] for s in S], mB),
           "motorB": _offset([s["dim"]["motorB"] for s in S], mB),
           "parallel": np.concatenate([s["dim"]["parallel"] for s in S]),
           "dimerParams": _same([s["dim"]["dimerParams"] for s in S], "dim.dimerParams")}

    mini = {"backbone": _body([s["mini"]["backbone"] for s in S]), "nBackbones": NBB, "nDimers": ND,
            "headBackboneSlot": _offset([s["mini"]["headBackboneSlot"] for s in S], bbB),
            "motorA": _offset([s["mini"]["motorA"] for s in S], mB),
            "attachAxial": np.concatenate([s["mini"]["attachAxial"] for s in S]),
            "miniData": np.concatenate([s["mini"]["miniData"] for s in S]),
            "bbInvDragY": _planar([s["mini"]["bbInvDragY"] for s in S], nBb, 2),
            "bbDimerCount": np.zeros(NBB, I32), "bbDimerOffsets": np.zeros(NBB + 1, I32),
            "bbDimerList": np.zeros(max(ND, 1), I32),
            "miniParams": _same([s["mini"]["miniParams"] for s in S], "mini.miniParams"),
            "bbBodyParams": _same([s["mini"]["bbBodyParams"] for s in S], "mini.bbBodyParams"),
            "bbCounts": np.array([NBB, 0, S[0]["seedBb"], NBB], I32)}

    xl = {"nLinks": NL, "linkFilA": _offset([s["xl"]["linkFilA"] for s in S], sB),
          "linkFilB": _offset([s["xl"]["linkFilB"] for s in S], sB)}
    for k in ("linkState", "linkOrientSame", "loc1", "loc2", "xlinkData", "strainHist", "torqueMagHist",
              "strainPlace", "torqueMagPlace", "activeLinkCount"):
        xl[k] = np.concatenate([s["xl"][k] for s in S])
    for k in ("xlParams", "offParams", "torsionParams"):
        xl[k] = _same([s["xl"][k] for s in S], "xl." + k)
    xl["counts"] = np.array([NL, 0, S[0]["seed"], NS], I32)
    for k in ("segCountA", "segCountB"):
        xl[k] = np.zeros(NS, I32)
    for k in ("segOffsetsA", "segOffsetsB"):
        xl[k] = np.zeros(NS + 1, I32)
    for k in ("segIdxA", "segIdxB"):
        xl[k] = np.zeros(max(NL, 1), I32)
    xl["placed"] = int(sum(s["xl"].get("placed", 0) for s in S))

    cap = NS + NM
    chunk = 512
    # per-step scratch lives on the device only
    grid = {"cap": cap, "totalCells": NC, "center": DeviceFill(3 * cap, 0, F32),
            "boundingRadius": DeviceFill(cap, 0, F32), "ownerStore": DeviceFill(cap, -1, I32),
            "ownerSlot": DeviceFill(cap, -1, I32), "gridParams": S[0]["grid"]["gridParams"].copy(),
            "viewParams": _same([s["grid"]["viewParams"] for s in S], "grid.viewParams"),
            "gridDims": np.array([0, 0, 0, NC], I32), "gridCounts": np.array([0, cap, 0, 0], I32),
            "bodyCell": DeviceFill(cap, -1, I32), "cellCount": DeviceFill(NC, 0, I32),
            "chunkSum": DeviceFill((NC + chunk - 1) // chunk + 1, 0, I32),
            "gridCellOffsets": DeviceFill(NC + 1, 0, I32), "gridCellContents": DeviceFill(cap, -1, I32),
            "reachSeg": DeviceFill(NM * 256, -1, I32), "reachCount": DeviceFill(NM, 0, I32)}

    xon = {int(s["xlinkOn"]) for s in S}
    xun = {int(s["xlUnbind"]) for s in S}
    if len(xon) != 1 or len(xun) != 1:
        raise ValueError("xlinkOn / xlUnbind differ between networks")
    packed = {"fil": fil, "mot": mot, "dim": dim, "mini": mini, "xl": xl, "grid": grid,
              "bondData": np.concatenate([s["bondData"] for s in S]),
              "xbParams": _same([s["xbParams"] for s in S], "xbParams"),
              "boxParams": S[0]["boxParams"].copy(),
              "segMotorCount": np.zeros(NS, I32), "segMotorOffsets": np.zeros(NS + 1, I32),
              "segMotorMyo": np.zeros(max(NM, 1), I32), "seed": int(S[0]["seed"]), "seedBb": int(S[0]["seedBb"]),
              "xlinkOn": xon.pop(), "xlUnbind": xun.pop()}
    box = [s["boxParams"] for s in S]
    if len({b[6] for b in box}) != 1 or len({b[7] for b in box}) != 1:
        raise ValueError("the containment cadence and dt must be shared")
    batch = {"segKey": _keys(nS), "motKey": _keys(nM), "bbKey": _keys(nBb), "linkKey": _keys(nL),
             "seeds": np.array([[s["seed"], s["seedBb"], s["fil"]["counts"][2]] for s in S], I32).reshape(-1),
             "gridParams": np.concatenate([s["grid"]["gridParams"] for s in S]).astype(F32),
             "gridDims": np.array([[*s["grid"]["gridDims"][:3], cB[k]] for k, s in enumerate(S)], I32).reshape(-1),
             "boxParams": np.concatenate(box).astype(F32)}
    info = {"nNet": len(S), "seg": sB, "mot": mB, "bb": bbB, "dim": dB, "link": _bases(nL), "cells": cB,
            "nS": nS, "nM": nM, "nBb": nBb, "nD": nD, "nL": nL}
    packed["batch"] = batch
    if all("turnover" in s for s in S):
        _pack_turnover(S, packed, info)
    return packed, info


def _pack_turnover(S, packed, info):
    """The networks' turnover arrays packed like their filament stores, plus the per-network
    tables of sbx_turnover_batch (rates, seeds, pools, birth request ranges)."""
    T_ = [s["turnover"] for s in S]
    cfgs = [s["tcfg"] for s in S]
    if len({c.check_int for c in cfgs}) != 1 or len({c.polyboost for c in cfgs}) != 1:
        raise ValueError("the biochem cadence and growth rounds must be shared")
    nS = info["nS"]
    sB = info["seg"]
    R = [t["birthAccept"].size for t in T_]
    rB = _bases(R)
    NS, NR = int(sB[-1]), int(rB[-1])
    t = {}
    for k in ("seedNode", "cofFrac", "grewFlag", "returnedMon", "deathFlag", "severDeathFlag", "severReturnedMon",
              "acceptFlag", "freeCount", "freeList", "filID", "filIDTmp"):
        t[k] = np.concatenate([x[k] for x in T_])
    t["nucFrac"] = _planar([x["nucFrac"] for x in T_], nS, 3)
    for k in ("reqCoord", "reqUVec", "reqYVec"):
        t[k] = _planar([x[k] for x in T_], nS, 3)
    for k in ("grewOffsets", "returnedOffsets", "severReturnedOffsets", "freeOffsets", "rankOffsets"):
        t[k] = np.zeros(NS + 1, I32)
    for k in ("splitParams", "dragParams", "birthParams", "seedParams"):
        t[k] = _same([x[k] for x in T_], "turnover." + k)
    seed_mon = _same([x["birthBox"][3:4] for x in T_], "turnover.birthBox[3]")
    t["growCounts"] = np.array([NS, 0, 0, 0], I32)
    t["depolyCounts"] = np.array([NS, 0, 0, 0], I32)
    t["agingCounts"] = np.array([NS, 0], I32)
    t["severCounts"] = np.array([NS, 0], I32)
    t["birthAccept"] = np.zeros(NR, I32)
    t["birthRankOffsets"] = np.zeros(NR + 1, I32)
    for k in ("birthReqCoord", "birthReqUVec", "birthReqYVec"):
        t[k] = np.zeros(3 * NR, F32)
    # per-network tables
    t["tbSeeds"] = np.array([c.seed for c in cfgs], I32)
    for k, w in (("growParams", 3), ("depolyParams", 3), ("depolyRateParams", 2), ("agingParams", 2),
                 ("cofilinParams", 2), ("birthBox", 4)):
        t["tb_" + k] = np.concatenate([x[k].reshape(-1)[:w] for x in T_]).astype(F32)
    t["tbOnRate"] = np.array([c.on_rate for c in cfgs], np.float64)
    t["tbPools"] = np.concatenate([x["pool"] for x in T_]).astype(np.float64)
    t["tbSlotBase"] = sB.astype(I32)
    t["tbBirthNet"] = np.concatenate([np.full(r, k, I32) for k, r in enumerate(R)])
    t["tbBirthBase"] = rB.astype(I32)
    packed["turnover"] = t
    packed["tcfg"] = cfgs[0]
    info["birth"] = rB
    info["seed_mon"] = int(seed_mon[0])


def _unplanar(a, base, n, total, width):
    return a.reshape(width, total)[:, base:base + n].reshape(-1)


def _unoffset(a, base):
    a = a.copy()
    a[a >= 0] -= base
    return a


def unpack_network(packed, info, k):
    """Network k's state arrays from a (host) packed scene, in its own indexing: the
    arrays its run alone holds (per-step scratch such as CSRs and the grid is left out)."""
    s0, n = int(info["seg"][k]), info["nS"][k]
    m0, nm = int(info["mot"][k]), info["nM"][k]
    b0, nb = int(info["bb"][k]), info["nBb"][k]
    d0, nd = int(info["dim"][k]), info["nD"][k]
    l0, nl = int(info["link"][k]), info["nL"][k]
    NS, NM, NBB = int(info["seg"][-1]), int(info["mot"][-1]), int(info["bb"][-1])

    def body(b, base, cnt, total):
        out = {key: _unplanar(b[key], base, cnt, total, 3) for key in _PLANAR3}
        for key in ("segLength", "brownTransScale", "brownRotScale"):
            out[key] = b[key][base:base + cnt]
        return out

    f, mo, mi, xl = packed["fil"], packed["mot"], packed["mini"], packed["xl"]
    fil = {"body": body(f["body"], s0, n, NS)}
    for key in ("monomerCount", "filState", "end1NbrSide", "end2NbrSide"):
        fil[key] = f[key][s0:s0 + n]
    for key in ("end1NbrSlot", "end2NbrSlot"):
        fil[key] = _unoffset(f[key][s0:s0 + n], s0)
    mot = {"body": body(mo["body"], 3 * m0, 3 * nm, 3 * NM)}
    for key in ("head", "uVec", "rodUVec"):
        mot[key] = _unplanar(mo[key], m0, nm, NM, 3)
    for key in ("reach", "bindArc", "capStats", "cooldown", "nucleotideState", "forceDotPlace", "forceDotFil",
                "forceMag"):
        mot[key] = mo[key][m0:m0 + nm]
    mot["stats"] = mo["stats"][2 * m0:2 * (m0 + nm)]
    mot["forceDotHist"] = mo["forceDotHist"][10 * m0:10 * (m0 + nm)]
    mot["boundSeg"] = _unoffset(mo["boundSeg"][m0:m0 + nm], s0)
    mini = {"backbone": body(mi["backbone"], b0, nb, NBB), "miniData": mi["miniData"][6 * d0:6 * (d0 + nd)]}
    x = {"linkFilA": _unoffset(xl["linkFilA"][l0:l0 + nl], s0), "linkFilB": _unoffset(xl["linkFilB"][l0:l0 + nl], s0)}
    for key in ("linkState", "linkOrientSame", "loc1", "loc2", "strainPlace", "torqueMagPlace"):
        x[key] = xl[key][l0:l0 + nl]
    x["xlinkData"] = xl["xlinkData"][12 * l0:12 * (l0 + nl)]
    x["strainHist"] = xl["strainHist"][10 * l0:10 * (l0 + nl)]
    x["torqueMagHist"] = xl["torqueMagHist"][5 * l0:5 * (l0 + nl)]
    x["activeLinkCount"] = xl["activeLinkCount"][s0:s0 + n]
    out = {"fil": fil, "mot": mot, "mini": mini, "xl": x, "bondData": packed["bondData"][13 * m0:13 * (m0 + nm)]}
    if "turnover" in packed:
        t = packed["turnover"]
        out["turnover"] = {"seedNode": t["seedNode"][s0:s0 + n], "cofFrac": t["cofFrac"][s0:s0 + n],
                           "nucFrac": _unplanar(t["nucFrac"], s0, n, NS, 3),
                           "pool": t["tbPools"][4 * k:4 * k + 4]}
    return out


def batch_desc(b):
    d = T.BatchDesc()
    T.fill(d, b)
    d.nNet = int(b["seeds"].numel() // 3) if hasattr(b["seeds"], "numel") else int(b["seeds"].size // 3)
    return d


class BatchedNetworks:
    """Packed networks on the device with one CUDA-graph step for all of them."""

    MODES = {"unfused": 0, "graph": 1}

    def __init__(self, packed, info, ctx=None, fp64_coords=False, device="cuda"):
        from .runtime import LIB, SbxError, default_context
        self.ctx = ctx or default_context()
        self.info = info
        self.dev = D.to_device({k: v for k, v in packed.items() if k not in ("cfg", "tcfg")}, device)
        if fp64_coords:
            for path in (("fil", "body"), ("mot", "body"), ("mini", "backbone")):
                D.add_coord64(self.dev[path[0]][path[1]])
        self.desc = D.dense_desc(self.dev)
        self.bdesc = batch_desc(self.dev["batch"])
        self.plan = C.c_void_p()
        st = LIB.sbx_dense_plan_create_batched(self.ctx.h, C.byref(self.desc), C.byref(self.bdesc),
                                               C.byref(self.plan))
        if st != 0:
            raise SbxError(st, "sbx_dense_plan_create_batched: " + self.ctx.last_error())

    def run(self, t0, nsteps, mode="graph"):
        from .runtime import LIB, SbxError
        st = LIB.sbx_dense_plan_run(self.plan, int(t0), int(nsteps), self.MODES[mode])
        if st != 0:
            raise SbxError(st, "sbx_dense_plan_run: " + self.ctx.last_error())

    @property
    def kernels_per_step(self):
        from .runtime import LIB
        return LIB.sbx_dense_plan_kernels_per_step(self.plan)

    def pull_all(self):
        return D.to_host(self.dev)

    def network(self, k, host=None):
        return unpack_network(host if host is not None else self.pull_all(), self.info, k)

    def close(self):
        from .runtime import LIB
        if self.plan:
            LIB.sbx_dense_plan_destroy(self.plan)
            self.plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchedTurnoverNetworks(BatchedNetworks):
    """Packed dense networks with actin turnover (each packed from scenes.dense_turnover):
    at each biochem cadence the batched turnover block and births run for every network,
    then the packed mechanics up to the next cadence; each network's arrays equal those of
    its engine.TurnoverNetwork run alone."""

    def __init__(self, packed, info, ctx=None, fp64_coords=False, device="cuda"):
        from .turnover import BatchedTurnover
        super().__init__(packed, info, ctx=ctx, fp64_coords=fp64_coords, device=device)
        d = self.dev
        self.tcfg = packed["tcfg"]
        xl = d["xl"]
        self.turnover = BatchedTurnover(d["fil"], d["turnover"], self.tcfg, info,
                                        links=(xl["linkFilA"], xl["linkFilB"], xl["linkState"]),
                                        boundSeg=d["mot"]["boundSeg"], segKey=d["batch"]["segKey"])

    def run(self, t0, nsteps, mode="graph"):
        t, end = int(t0), int(t0) + int(nsteps)
        ci = self.tcfg.check_int
        while t < end:
            if self.tcfg.fires_at(t):
                self.turnover.cadence(t)
                self.turnover.births(t)
            nxt = min(end, (t // ci + 1) * ci)
            super().run(t, nxt - t, mode)
            t = nxt
