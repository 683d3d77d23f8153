"""Actin turnover on the device: barbed-end growth and the split at 2 stdSegLength,
pointed-end depolymerisation and death, nucleotide aging, cofilin severing, birth into
free slots, and filament identity by pointer doubling.

Per-slot state stays in the filament store's planar arrays (FilamentStore.java:29-199)
plus the turnover arrays below; every per-slot update is a library kernel
(systems.GrowthSystem, DepolySystem, AgingSystem, SeveringSystem, FilamentBirthSystem,
FilIDSystem). The host scalars of the reference -- the actin pool (ActinPool.java) and the
per-cadence growth probability that reads it (GrowthStore.refreshRate) -- live in device
memory too (sbx_actin_pool, sbx_turnover_begin), so a cadence issues launches only: no
host read-back, no synchronisation, and it can be captured in a CUDA graph.

`Turnover.cadence(t)` is the turnover block of FullSystemDemoHarness.cpuStep
(FullSystemDemoHarness.java:648-683): age -> depolyProxy -> return scan -> death ->
{grow -> grew scan -> growthAtp -> pool take} x boost -> cofilin accumulate/dissolve ->
sever return scan -> death -> markSplits -> split allocation -> splitWire ->
splitInheritNuc -> nucleateFreshCofilin -> recomputeDrag. Node nucleation, which follows
it in that harness, is not part of this module.
"""
import math
from dataclasses import dataclass

import numpy as np

from . import scenes

F32, I32 = np.float32, np.int32

# Constants.java:70-103
ACTIN_SEED = 3
ACTIN_CONC_INIT = 15.0
BIOCHEM_DT = 1.0e-3
K_ATP_ON2_WITH_FORMIN = 11.6
MIN_MONOMER_CT = 30
K_ATP_OFF1, K_ADP_OFF1 = 0.8, 2.7
K_HYDROLYSIS, K_DISSOCIATION = 0.3, 1.0
COFILIN_RATE, COFILIN_CONC, COFILIN_RATIO = 0.1, 3.0, 1.0
AVOGADRO = 6.022e23
AETA = 0.1                                   # Constants.aeta, the recomputeDrag viscosity
FIL_FREE, FIL_ACTIVE = -1, 0                 # FilamentStore.java:112-113
TURNOVER_SEED = 0x0F0501                     # FullSystemDemoHarness.java:57


def um_per_monomer(box_vol_um3):
    """ActinPool.java:37-40 (v1 Chamber.java:52)."""
    return (1e5 * 1e5 * 1e5 * 1e6) / (box_vol_um3 * AVOGADRO)


def pool_array(conc, box_vol_um3):
    """An sbx_actin_pool as a float64[4] host array ([2], [3] hold the int64 ledger)."""
    a = np.zeros(4, np.float64)
    a[0] = conc
    a[1] = um_per_monomer(box_vol_um3)
    return a


def pool_fields(a):
    """(conc, uMPerMonomer, totalTaken, totalReturned) of a pool array."""
    a = np.asarray(a)
    led = a.view(np.int64)
    return float(a[0]), float(a[1]), int(led[2]), int(led[3])


@dataclass
class TurnoverConfig:
    """The turnover switches of FullSystemDemoHarness (:102-117) and the stores they build."""
    dt: float = 1.0e-5
    aging_on: bool = True
    sever_on: bool = True
    cof_ratio: float = 0.5
    kin: float = 1.0                  # biochem kinetic speed-up (1 = faithful)
    polyboost: int = 1                # grow rounds per cadence
    pool0_um: float = -1.0            # initial [actin]; < 0 = the critical concentration
    box_vol_um3: float = 3.6 * 3.6 * 0.5
    seed: int = TURNOVER_SEED
    aeta: float = AETA
    born_trans: float = scenes.BTRANS_COEFF
    born_rot: float = scenes.BROT_COEFF

    @property
    def check_int(self):
        """biochemCheckInt = max(1, round(biochemDeltaT / dt)) (GrowthStore.java:47)."""
        return max(1, int(math.floor(BIOCHEM_DT / self.dt + 0.5)))

    def fires_at(self, step):
        return step % self.check_int == 0

    @property
    def on_rate(self):
        return K_ATP_ON2_WITH_FORMIN * self.kin

    @property
    def pool0(self):
        """FullSystemDemoHarness.java:116-117,360: C_c of the (aging) off-rate."""
        if self.pool0_um > 0:
            return self.pool0_um
        s, a = scenes.STD_SEG_LENGTH, ACTIN_SEED
        k_off = K_ADP_OFF1 if self.aging_on else K_ATP_OFF1
        return (float(s) / (s - (a - 1))) * (k_off / K_ATP_ON2_WITH_FORMIN)

    def params(self):
        """The float parameter arrays of the stores (GrowthStore.java:53-76, DepolyStore.java:57-59,
        AgingStore.java:59-76, SeverStore.java:60-64, FilamentStore.setBirthParams) with the
        harness's kin scaling (FullSystemDemoHarness.java:365-375)."""
        h, s = scenes.ACTIN_MONO_RADIUS, scenes.STD_SEG_LENGTH
        p = {}
        p["growParams"] = np.array([0.0, h, 2 * s], F32)
        p["splitParams"] = np.array([h, 2 * s, s], F32)
        p["dragParams"] = np.array([h, self.aeta, scenes.ACTIN_RADIUS, scenes.KT, scenes.A_PARALLEL, scenes.A_ORTHOG,
                                    scenes.A_TURNING, s, MIN_MONOMER_CT], F32)
        p["depolyParams"] = np.array([K_ATP_OFF1 * self.kin * BIOCHEM_DT, h, ACTIN_SEED], F32)
        ph = K_HYDROLYSIS * BIOCHEM_DT if self.aging_on else 0.0
        pd = K_DISSOCIATION * BIOCHEM_DT if self.aging_on else 0.0
        p["agingParams"] = np.array([float(F32(ph)) * self.kin, float(F32(pd)) * self.kin], F32)   # float x double
        p["depolyRateParams"] = np.array([K_ATP_OFF1 * BIOCHEM_DT * self.kin, K_ADP_OFF1 * BIOCHEM_DT * self.kin],
                                         F32)
        pc = COFILIN_CONC * COFILIN_RATE * BIOCHEM_DT if self.sever_on else 0.0
        ratio = self.cof_ratio if self.sever_on else 1.0
        p["cofilinParams"] = np.array([float(F32(pc)) * self.kin, ratio], F32)
        p["birthParams"] = np.array([self.born_trans, self.born_rot], F32)
        return p


def turnover_arrays(C, cfg, seedNode=None, nucFrac=None, cofFrac=None):
    """The per-slot turnover arrays and the stores' parameter/count arrays (host numpy):
    the state a cadence reads and writes, next to a FilamentStore of capacity C."""
    t = {k: np.zeros(C, I32) for k in ("grewFlag", "returnedMon", "deathFlag", "severDeathFlag", "severReturnedMon",
                                        "acceptFlag", "freeCount", "freeList")}
    for k in ("grewOffsets", "returnedOffsets", "severReturnedOffsets", "freeOffsets", "rankOffsets"):
        t[k] = np.zeros(C + 1, I32)
    for k in ("reqCoord", "reqUVec", "reqYVec"):
        t[k] = np.zeros(3 * C, F32)
    t["seedNode"] = np.full(C, -1, I32) if seedNode is None else np.asarray(seedNode, I32).copy()
    if nucFrac is None:
        nucFrac = np.zeros(3 * C, F32)
        nucFrac[:C] = 1.0
    t["nucFrac"] = np.asarray(nucFrac, F32).copy()
    t["cofFrac"] = np.zeros(C, F32) if cofFrac is None else np.asarray(cofFrac, F32).copy()
    t.update(cfg.params())
    t["growCounts"] = np.array([C, 0, cfg.seed, 0], I32)
    t["depolyCounts"] = np.array([C, 0, cfg.seed, 0], I32)
    t["agingCounts"] = np.array([C, 0], I32)
    t["severCounts"] = np.array([C, 0], I32)
    t["pool"] = pool_array(cfg.pool0, cfg.box_vol_um3)
    t["filID"] = np.zeros(C, I32)
    t["filIDTmp"] = np.zeros(C, I32)
    return t


def birth_arrays(t, req_cap, box_half, seed_mon):
    """Adds the constant-actin birth requests to turnover arrays `t`: request buffers of
    capacity req_cap, the birth box [hx, hy, hz, monomers per newborn] and the newborn's
    [monomerCount, segLength] (NodeNucleationStore.seedParams)."""
    t["birthAccept"] = np.zeros(req_cap, I32)
    t["birthRankOffsets"] = np.zeros(req_cap + 1, I32)
    for k in ("birthReqCoord", "birthReqUVec", "birthReqYVec"):
        t[k] = np.zeros(3 * req_cap, F32)
    t["birthBox"] = np.array([box_half[0], box_half[1], box_half[2], seed_mon], F32)
    t["seedParams"] = np.array([seed_mon, (seed_mon + 1) * scenes.ACTIN_MONO_RADIUS], F32)
    return t


class Turnover:
    """Device turnover over a device filament store `fil` (dict of torch tensors as made by
    device.to_device from scenes.filament_store) and device turnover arrays `t` (from
    turnover_arrays). All calls launch on the library's default context.

    In a network (`links` = (linkFilA, linkFilB, linkState) of a crosslinker store,
    `boundSeg` of a motor store), every death is followed by sbx_turnover_release_dead, so
    no link or head stays on a FREE slot, and one that a split or birth reuses later in the
    same cadence starts unattached."""

    def __init__(self, fil, t, cfg, links=None, boundSeg=None):
        self.f, self.t, self.cfg = fil, t, cfg
        self.C = int(fil["filState"].numel())
        self.links, self.boundSeg = links, boundSeg
        # monomers per newborn, read once here so that a cadence never reads device memory
        self.seed_mon = int(np.asarray(t["birthBox"].cpu())[3]) if "birthBox" in t else 0

    def begin(self, step):
        from .systems import _ctx
        t, cfg = self.t, self.cfg
        fires = 1 if cfg.fires_at(step) else 0
        _ctx()("sbx_turnover_begin", step, cfg.seed, fires, float(cfg.on_rate), float(BIOCHEM_DT), t["pool"],
               t["growParams"], t["growCounts"], t["depolyCounts"], t["agingCounts"], t["severCounts"])
        return fires

    def _scan(self, counts, offsets):
        from .systems import _ctx
        _ctx()("sbx_csr_scan", self.C, counts, offsets)

    def _death(self, flag):
        from .systems import DepolySystem, _ctx
        f, b, t = self.f, self.f["body"], self.t
        DepolySystem.applyDeath(f["filState"], f["monomerCount"], t["seedNode"], f["end1NbrSlot"], f["end1NbrSide"],
                                f["end2NbrSlot"], f["end2NbrSide"], b["brownTransScale"], b["brownRotScale"], flag)
        if self.links is not None or self.boundSeg is not None:
            la, lb, ls = self.links if self.links is not None else (None, None, None)
            _ctx()("sbx_turnover_release_dead", f["filState"], 0 if ls is None else ls.numel(), la, lb, ls,
                   0 if self.boundSeg is None else self.boundSeg.numel(), self.boundSeg)

    def allocate(self, acceptFlag, reqCoord, reqUVec, reqYVec, rankOffsets, K=None):
        """FullSystemDemoHarness.allocCpu (:950-957): free list over filState, dense ranks of the
        accepted requests, rank r claims freeList[r] below nFree."""
        from .systems import FilamentBirthSystem as B
        f, b, t = self.f, self.f["body"], self.t
        K = acceptFlag.numel() if K is None else K
        B.freeFlags(f["filState"], t["freeCount"])
        self._scan(t["freeCount"], t["freeOffsets"])
        B.freeScatter(f["filState"], t["freeOffsets"], t["freeList"])
        from .systems import _ctx
        _ctx()("sbx_csr_scan", K, acceptFlag, rankOffsets)
        B.allocate(reqCoord, reqUVec, reqYVec, rankOffsets, t["freeList"], t["freeOffsets"], b["coord"], b["uVec"],
                   b["yVec"], b["brownTransScale"], b["brownRotScale"], f["filState"], t["birthParams"],
                   allocCounts=(self.C, K))

    def cadence(self, step):
        """One step's turnover block; returns False (and launches only the prologue) off-cadence,
        where every kernel of the block is a no-op in the reference."""
        from .systems import AgingSystem as A, DepolySystem as D, GrowthSystem as G, SeveringSystem as S, _ctx
        if not self.cfg.fires_at(step):
            return False
        self.begin(step)
        f, b, t = self.f, self.f["body"], self.t
        C = self.C
        A.age(f["filState"], t["nucFrac"], t["agingParams"], t["agingCounts"])
        D.depolyProxy(f["filState"], f["monomerCount"], b["coord"], b["uVec"], f["end1NbrSlot"], t["nucFrac"],
                      t["returnedMon"], t["deathFlag"], t["depolyParams"], t["depolyRateParams"], t["depolyCounts"])
        self._scan(t["returnedMon"], t["returnedOffsets"])
        self._death(t["deathFlag"])
        _ctx()("sbx_actin_pool_put_total", t["pool"], t["returnedOffsets"], C)
        for _ in range(max(1, self.cfg.polyboost)):
            G.grow(t["seedNode"], f["monomerCount"], b["coord"], b["uVec"], t["grewFlag"], t["growParams"],
                   t["growCounts"])
            self._scan(t["grewFlag"], t["grewOffsets"])
            A.growthAtp(t["grewFlag"], f["monomerCount"], t["nucFrac"])
            _ctx()("sbx_actin_pool_take_total", t["pool"], t["grewOffsets"], C)
        S.cofilinAccumulate(f["filState"], t["nucFrac"], t["cofFrac"], t["cofilinParams"], t["severCounts"])
        S.cofilinDissolve(f["filState"], f["monomerCount"], t["cofFrac"], t["severDeathFlag"], t["severReturnedMon"],
                          t["cofilinParams"], t["severCounts"])
        self._scan(t["severReturnedMon"], t["severReturnedOffsets"])
        self._death(t["severDeathFlag"])
        _ctx()("sbx_actin_pool_put_total", t["pool"], t["severReturnedOffsets"], C)
        G.markSplits(t["seedNode"], f["monomerCount"], b["coord"], b["uVec"], b["yVec"], t["acceptFlag"],
                     t["reqCoord"], t["reqUVec"], t["reqYVec"], t["splitParams"], t["growCounts"])
        self.allocate(t["acceptFlag"], t["reqCoord"], t["reqUVec"], t["reqYVec"], t["rankOffsets"])
        G.splitWire(t["rankOffsets"], t["freeList"], t["freeOffsets"], f["monomerCount"], b["coord"], b["uVec"],
                    f["end1NbrSlot"], f["end1NbrSide"], f["end2NbrSlot"], f["end2NbrSide"], t["seedNode"],
                    t["splitParams"], allocCounts=(C, C))
        A.splitInheritNuc(t["rankOffsets"], t["freeList"], t["freeOffsets"], t["nucFrac"], allocCounts=(C, C))
        S.nucleateFreshCofilin(t["rankOffsets"], t["freeList"], t["freeOffsets"], t["cofFrac"], allocCounts=(C, C))
        G.recomputeDrag(f["monomerCount"], b["segLength"], f["end1NbrSlot"], f["end2NbrSlot"], b["bTransGam"],
                        b["bRotGam"], b["bTransDiff"], b["bRotDiff"], t["dragParams"], t["growCounts"])
        return True

    def births(self, step):
        """Constant-actin births after the turnover block (in the place of the node nucleation
        of FullSystemDemoHarness.cpuStep, :685-692): requests for the polymer deficit, the
        allocator, initNewborn, tagSeeds (a newborn is a growing tip), fresh ATP and cofilin,
        and the pool debit of the formed births."""
        from .systems import AgingSystem as A, SeveringSystem as S, _ctx
        if not self.cfg.fires_at(step) or "birthBox" not in self.t:
            return False
        f, t, C = self.f, self.t, self.C
        K = t["birthAccept"].numel()
        _ctx()("sbx_birth_emit_constant_actin", K, t["pool"], t["birthBox"], step, self.cfg.seed, t["birthAccept"],
               t["birthReqCoord"], t["birthReqUVec"], t["birthReqYVec"])
        self.allocate(t["birthAccept"], t["birthReqCoord"], t["birthReqUVec"], t["birthReqYVec"],
                      t["birthRankOffsets"], K=K)
        ro, fl, fo = t["birthRankOffsets"], t["freeList"], t["freeOffsets"]
        _ctx()("sbx_birth_init_newborn", K, C, ro, fl, fo, f["monomerCount"], f["body"]["segLength"],
               t["seedParams"])
        _ctx()("sbx_birth_tag_seeds", K, C, ro, fl, fo, t["seedNode"])
        A.nucleateFreshAtp(ro, fl, fo, t["nucFrac"], allocCounts=(C, K))
        S.nucleateFreshCofilin(ro, fl, fo, t["cofFrac"], allocCounts=(C, K))
        _ctx()("sbx_actin_pool_take_births", t["pool"], ro, K, fo, C, self.seed_mon)
        return True

    def filament_ids(self):
        """FilIDSystem init + rounds(C) jumps into t['filID'] (the chain's end2 terminal)."""
        from .systems import FilIDSystem
        return FilIDSystem.compute(self.f["filState"], self.f["end2NbrSlot"], self.t["filID"], self.t["filIDTmp"])

    def pool(self):
        """(conc, uMPerMonomer, totalTaken, totalReturned), read back (synchronises)."""
        return pool_fields(self.t["pool"].cpu().numpy())


class BatchedTurnover:
    """The turnover block and births of packed networks (batch.pack_networks of
    scenes.dense_turnover scenes): the same sequence as Turnover.cadence / births, with the
    sbx_tb_* kernels where a rate, a draw, a pool or the allocator is involved and the
    single-network kernels elsewhere."""

    def __init__(self, fil, t, cfg, info, links, boundSeg, segKey):
        from . import abi_types as T
        self.f, self.t, self.cfg, self.info = fil, t, cfg, info
        self.C = int(fil["filState"].numel())
        self.R = int(t["birthAccept"].numel())
        self.links, self.boundSeg = links, boundSeg
        self.seed_mon = int(info["seed_mon"])
        d = T.TurnoverBatchDesc()
        T.fill(d, {"slotKey": segKey, "slotBase": t["tbSlotBase"], "seeds": t["tbSeeds"],
                   "growParams": t["tb_growParams"], "depolyParams": t["tb_depolyParams"],
                   "depolyRateParams": t["tb_depolyRateParams"], "agingParams": t["tb_agingParams"],
                   "cofilinParams": t["tb_cofilinParams"], "birthBox": t["tb_birthBox"], "onRate": t["tbOnRate"],
                   "pools": t["tbPools"], "birthNet": t["tbBirthNet"], "birthBase": t["tbBirthBase"]})
        d.nNet = int(info["nNet"])
        self.desc = d

    def _ctx(self):
        from .systems import _ctx
        return _ctx()

    def _scan(self, n, counts, offsets):
        self._ctx()("sbx_csr_scan", n, counts, offsets)

    def _death(self, flag):
        f, b, t = self.f, self.f["body"], self.t
        ctx = self._ctx()
        ctx("sbx_depoly_apply_death", self.C, f["filState"], f["monomerCount"], t["seedNode"], f["end1NbrSlot"],
            f["end1NbrSide"], f["end2NbrSlot"], f["end2NbrSide"], b["brownTransScale"], b["brownRotScale"], flag)
        la, lb, ls = self.links
        ctx("sbx_turnover_release_dead", f["filState"], ls.numel(), la, lb, ls, self.boundSeg.numel(), self.boundSeg)

    def _free_list(self):
        f, t = self.f, self.t
        ctx = self._ctx()
        ctx("sbx_xlink_free_flags", self.C, f["filState"], t["freeCount"])
        self._scan(self.C, t["freeCount"], t["freeOffsets"])
        ctx("sbx_xlink_free_scatter", self.C, f["filState"], t["freeOffsets"], t["freeList"])

    def cadence(self, step):
        import ctypes as C
        if not self.cfg.fires_at(step):
            return False
        f, b, t, n = self.f, self.f["body"], self.t, self.C
        ctx = self._ctx()
        tb = C.byref(self.desc)
        ctx("sbx_turnover_begin", step, 0, 1, 0.0, float(BIOCHEM_DT), None, None, t["growCounts"], t["depolyCounts"],
            t["agingCounts"], t["severCounts"])
        ctx("sbx_tb_begin", tb, 1, float(BIOCHEM_DT))
        ctx("sbx_tb_age", tb, n, f["filState"], t["nucFrac"], t["agingCounts"])
        ctx("sbx_tb_depoly_proxy", tb, n, f["filState"], f["monomerCount"], b["coord"], b["uVec"], f["end1NbrSlot"],
            t["nucFrac"], t["returnedMon"], t["deathFlag"], t["depolyCounts"])
        self._scan(n, t["returnedMon"], t["returnedOffsets"])
        self._death(t["deathFlag"])
        ctx("sbx_tb_pool", tb, t["returnedOffsets"], 0)
        for _ in range(max(1, self.cfg.polyboost)):
            ctx("sbx_tb_grow", tb, n, t["seedNode"], f["monomerCount"], b["coord"], b["uVec"], t["grewFlag"],
                t["growCounts"])
            self._scan(n, t["grewFlag"], t["grewOffsets"])
            ctx("sbx_aging_growth_atp", n, t["grewFlag"], f["monomerCount"], t["nucFrac"])
            ctx("sbx_tb_pool", tb, t["grewOffsets"], 1)
        ctx("sbx_tb_cofilin", tb, n, 0, f["filState"], t["nucFrac"], t["cofFrac"], None, None, None, t["severCounts"])
        ctx("sbx_tb_cofilin", tb, n, 1, f["filState"], None, t["cofFrac"], f["monomerCount"], t["severDeathFlag"],
            t["severReturnedMon"], t["severCounts"])
        self._scan(n, t["severReturnedMon"], t["severReturnedOffsets"])
        self._death(t["severDeathFlag"])
        ctx("sbx_tb_pool", tb, t["severReturnedOffsets"], 0)
        ctx("sbx_growth_mark_splits", n, t["seedNode"], f["monomerCount"], b["coord"], b["uVec"], b["yVec"],
            t["acceptFlag"], t["reqCoord"], t["reqUVec"], t["reqYVec"], n, t["splitParams"], t["growCounts"])
        self._free_list()
        self._scan(n, t["acceptFlag"], t["rankOffsets"])
        ctx("sbx_tb_birth_allocate", tb, 0, n, n, n, t["reqCoord"], t["reqUVec"], t["reqYVec"], t["rankOffsets"],
            t["freeList"], t["freeOffsets"], b["coord"], b["uVec"], b["yVec"], b["brownTransScale"],
            b["brownRotScale"], f["filState"], t["birthParams"])
        ctx("sbx_tb_split_wire", tb, n, t["rankOffsets"], t["freeList"], t["freeOffsets"], f["monomerCount"],
            b["coord"], b["uVec"], f["end1NbrSlot"], f["end1NbrSide"], f["end2NbrSlot"], f["end2NbrSide"],
            t["seedNode"], t["splitParams"])
        ctx("sbx_tb_formed_init", tb, 0, n, n, t["rankOffsets"], t["freeList"], t["freeOffsets"], t["nucFrac"], 2)
        ctx("sbx_tb_formed_init", tb, 0, n, n, t["rankOffsets"], t["freeList"], t["freeOffsets"], t["cofFrac"], 0)
        ctx("sbx_growth_recompute_drag", n, f["monomerCount"], b["segLength"], f["end1NbrSlot"], f["end2NbrSlot"],
            b["bTransGam"], b["bRotGam"], b["bTransDiff"], b["bRotDiff"], t["dragParams"], t["growCounts"])
        return True

    def births(self, step):
        import ctypes as C
        if not self.cfg.fires_at(step):
            return False
        f, b, t, n, R = self.f, self.f["body"], self.t, self.C, self.R
        ctx = self._ctx()
        tb = C.byref(self.desc)
        ctx("sbx_tb_birth_emit", tb, R, step, t["birthAccept"], t["birthReqCoord"], t["birthReqUVec"],
            t["birthReqYVec"])
        self._free_list()
        self._scan(R, t["birthAccept"], t["birthRankOffsets"])
        ro = t["birthRankOffsets"]
        ctx("sbx_tb_birth_allocate", tb, 1, R, n, R, t["birthReqCoord"], t["birthReqUVec"], t["birthReqYVec"], ro,
            t["freeList"], t["freeOffsets"], b["coord"], b["uVec"], b["yVec"], b["brownTransScale"],
            b["brownRotScale"], f["filState"], t["birthParams"])
        ctx("sbx_tb_newborn", tb, R, ro, t["freeList"], t["freeOffsets"], f["monomerCount"], b["segLength"],
            t["seedNode"], t["seedParams"])
        ctx("sbx_tb_formed_init", tb, 1, R, n, ro, t["freeList"], t["freeOffsets"], t["nucFrac"], 1)
        ctx("sbx_tb_formed_init", tb, 1, R, n, ro, t["freeList"], t["freeOffsets"], t["cofFrac"], 0)
        ctx("sbx_tb_pool_births", tb, ro, t["freeOffsets"], self.seed_mon)
        return True
