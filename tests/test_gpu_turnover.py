"""GPU actin turnover against the oracle, bit for bit, through the C ABI.

Scene: formin-pinned chains in random slots of a 4,096-slot store (a quarter FREE), with
random nucleotide and cofilin fractions, taken through a few oracle cadences at a raised
kinetic rate so that growth, depolymerisation, death, dissolves and splits all occur. Each
turnover entry point is then compared with the oracle on identical inputs, and whole
cadences (the turnover block of FullSystemDemoHarness.cpuStep) are run side by side.
"""
import copy

import numpy as np
import pytest

from helpers import (assert_same, chain_walk_ids, flat_arrays, oracle_filament_ids, oracle_turnover_allocate,
                     oracle_turnover_cadence)
from softbox_b200 import device as D, scenes
from softbox_b200.turnover import BIOCHEM_DT, Turnover, TurnoverConfig, pool_fields

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

CAP = 4096


@pytest.fixture(scope="module")
def seeded(orc_dm):
    cfg = TurnoverConfig(kin=60.0, polyboost=2)
    sc = scenes.turnover_chains(n_chains=420, cap=CAP, cfg=cfg, cofilin_high=0.4, seed=9)
    for step in (0, 100, 200):
        oracle_turnover_cadence(orc_dm, sc, step)
    return sc


def _dev(sc):
    return D.to_device(sc["fil"]), D.to_device(sc["t"])


def _compare(sc, fil, t, what=""):
    torch.cuda.synchronize()
    for name, a in flat_arrays(sc["fil"], "fil."):
        dev = fil
        for k in name.split(".")[1:]:
            dev = dev[k]
        assert_same(a, dev.cpu().numpy(), what + name)
    for k, a in sc["t"].items():
        if isinstance(a, np.ndarray):
            assert_same(a, t[k].cpu().numpy(), what + "t." + k)


def test_whole_cadences_bitwise(orc_dm, seeded):
    sc = copy.deepcopy(seeded)
    fil, t = _dev(sc)
    tv = Turnover(fil, t, sc["cfg"])
    events = {"split": 0, "death": 0, "dissolve": 0}
    for step in range(300, 300 + 100 * 12, 50):       # off-cadence steps interleaved
        fired = oracle_turnover_cadence(orc_dm, sc, step)
        assert tv.cadence(step) == fired
        _compare(sc, fil, t, f"step {step}: ")
        if fired:
            h = sc["t"]
            events["split"] += int(min(h["rankOffsets"][CAP], h["freeOffsets"][CAP]))
            events["death"] += int(h["deathFlag"].sum())
            events["dissolve"] += int(h["severDeathFlag"].sum())
    assert min(events.values()) > 0, events
    assert tv.pool() == pool_fields(sc["t"]["pool"])


def test_cadence_captures_in_a_cuda_graph(seeded, monkeypatch):
    """A cadence issues kernels only (no host read-back, no allocation once the context's
    scratch exists): captured in a CUDA graph, its replay equals eager execution."""
    import softbox_b200.runtime as R
    sc = copy.deepcopy(seeded)
    fil_e, t_e = _dev(sc)
    fil_w, t_w = _dev(sc)
    fil_g, t_g = _dev(sc)
    Turnover(fil_e, t_e, sc["cfg"]).cadence(300)
    s = torch.cuda.Stream()
    ctx = R.Context(0, stream=s.cuda_stream)
    try:
        monkeypatch.setattr(R, "_default", ctx)
        with torch.cuda.stream(s):
            Turnover(fil_w, t_w, sc["cfg"]).cadence(300)          # warm-up: sizes the scan scratch
        s.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            Turnover(fil_g, t_g, sc["cfg"]).cadence(300)
        g.replay()
        torch.cuda.synchronize()
        for name, a in flat_arrays(D.to_host(fil_e), "fil."):
            dev = fil_g
            for k in name.split(".")[1:]:
                dev = dev[k]
            assert_same(a, dev.cpu().numpy(), "graph " + name)
        for k, v in t_e.items():
            if hasattr(v, "data_ptr"):
                assert_same(v.cpu().numpy(), t_g[k].cpu().numpy(), "graph t." + k)
        del g
    finally:
        monkeypatch.undo()
        ctx.close()


def _begin(orc_dm, sc, step):
    t, cfg = sc["t"], sc["cfg"]
    orc_dm.turnover_begin(step, cfg.seed, 1, float(cfg.on_rate), float(BIOCHEM_DT), t["pool"], t["growParams"],
                          t["growCounts"], t["depolyCounts"], t["agingCounts"], t["severCounts"])


def test_entry_points_bitwise(orc_dm, seeded):
    from softbox_b200.systems import (AgingSystem as A, DepolySystem as Dp, GrowthSystem as G, SeveringSystem as S,
                                      _ctx)
    sc = copy.deepcopy(seeded)
    f, t, C = sc["fil"], sc["t"], CAP
    b = f["body"]
    _begin(orc_dm, sc, 400)
    fil, dt = _dev(sc)
    db = fil["body"]
    Turnover(fil, dt, sc["cfg"]).begin(400)

    orc_dm.aging_age(C, f["filState"], t["nucFrac"], t["agingParams"], t["agingCounts"])
    A.age(fil["filState"], dt["nucFrac"], dt["agingParams"], dt["agingCounts"])
    orc_dm.depoly(C, f["filState"], f["monomerCount"], b["coord"], b["uVec"], f["end1NbrSlot"], t["returnedMon"],
                  t["deathFlag"], t["depolyParams"], t["depolyCounts"])
    Dp.depoly(fil["filState"], fil["monomerCount"], db["coord"], db["uVec"], fil["end1NbrSlot"], dt["returnedMon"],
              dt["deathFlag"], dt["depolyParams"], dt["depolyCounts"])
    _compare(sc, fil, dt, "depoly: ")
    orc_dm.depoly_proxy(C, f["filState"], f["monomerCount"], b["coord"], b["uVec"], f["end1NbrSlot"], t["nucFrac"],
                        t["returnedMon"], t["deathFlag"], t["depolyParams"], t["depolyRateParams"], t["depolyCounts"])
    Dp.depolyProxy(fil["filState"], fil["monomerCount"], db["coord"], db["uVec"], fil["end1NbrSlot"], dt["nucFrac"],
                   dt["returnedMon"], dt["deathFlag"], dt["depolyParams"], dt["depolyRateParams"], dt["depolyCounts"])
    _compare(sc, fil, dt, "depolyProxy: ")
    assert t["deathFlag"].sum() > 0 and (t["returnedMon"] == 1).sum() > 0
    # death on random flags over the chain topology, adjacent pairs included
    rng = np.random.default_rng(4)
    flag = ((rng.random(C) < 0.15) & (f["filState"] >= 0)).astype(np.int32)
    e1 = f["end1NbrSlot"]
    pairs = np.flatnonzero(flag.astype(bool) & (e1 >= 0))
    assert pairs.size > 0
    flag[e1[pairs[:20]]] = 1
    dflag = torch.from_numpy(flag).cuda()
    orc_dm.apply_death(C, f["filState"], f["monomerCount"], t["seedNode"], f["end1NbrSlot"], f["end1NbrSide"],
                       f["end2NbrSlot"], f["end2NbrSide"], b["brownTransScale"], b["brownRotScale"], flag)
    Dp.applyDeath(fil["filState"], fil["monomerCount"], dt["seedNode"], fil["end1NbrSlot"], fil["end1NbrSide"],
                  fil["end2NbrSlot"], fil["end2NbrSide"], db["brownTransScale"], db["brownRotScale"], dflag)
    _compare(sc, fil, dt, "applyDeath: ")
    orc_dm.growth_grow(C, t["seedNode"], f["monomerCount"], b["coord"], b["uVec"], t["grewFlag"], t["growParams"],
                       t["growCounts"])
    G.grow(dt["seedNode"], fil["monomerCount"], db["coord"], db["uVec"], dt["grewFlag"], dt["growParams"],
           dt["growCounts"])
    assert t["grewFlag"].sum() > 0
    orc_dm.aging_growth_atp(C, t["grewFlag"], f["monomerCount"], t["nucFrac"])
    A.growthAtp(dt["grewFlag"], fil["monomerCount"], dt["nucFrac"])
    _compare(sc, fil, dt, "grow + growthAtp: ")
    orc_dm.cofilin_accumulate(C, f["filState"], t["nucFrac"], t["cofFrac"], t["cofilinParams"], t["severCounts"])
    S.cofilinAccumulate(fil["filState"], dt["nucFrac"], dt["cofFrac"], dt["cofilinParams"], dt["severCounts"])
    orc_dm.cofilin_dissolve(C, f["filState"], f["monomerCount"], t["cofFrac"], t["severDeathFlag"],
                            t["severReturnedMon"], t["cofilinParams"], t["severCounts"])
    S.cofilinDissolve(fil["filState"], fil["monomerCount"], dt["cofFrac"], dt["severDeathFlag"],
                      dt["severReturnedMon"], dt["cofilinParams"], dt["severCounts"])
    _compare(sc, fil, dt, "cofilin: ")
    assert t["severDeathFlag"].sum() > 0
    # force split-ready tips: every tip at the threshold
    tips = np.flatnonzero(t["seedNode"] >= 0)
    f["monomerCount"][tips[::2]] = 64
    fil["monomerCount"].copy_(torch.from_numpy(f["monomerCount"]).cuda())
    orc_dm.growth_mark_splits(C, t["seedNode"], f["monomerCount"], b["coord"], b["uVec"], b["yVec"], t["acceptFlag"],
                              t["reqCoord"], t["reqUVec"], t["reqYVec"], C, t["splitParams"], t["growCounts"])
    G.markSplits(dt["seedNode"], fil["monomerCount"], db["coord"], db["uVec"], db["yVec"], dt["acceptFlag"],
                 dt["reqCoord"], dt["reqUVec"], dt["reqYVec"], dt["splitParams"], dt["growCounts"])
    _compare(sc, fil, dt, "markSplits: ")
    oracle_turnover_allocate(orc_dm, sc, t["acceptFlag"], t["reqCoord"], t["reqUVec"], t["reqYVec"],
                             t["rankOffsets"])
    Turnover(fil, dt, sc["cfg"]).allocate(dt["acceptFlag"], dt["reqCoord"], dt["reqUVec"], dt["reqYVec"],
                                          dt["rankOffsets"])
    _compare(sc, fil, dt, "allocate: ")
    assert t["rankOffsets"][C] > 0
    orc_dm.growth_split_wire(C, C, t["rankOffsets"], t["freeList"], t["freeOffsets"], f["monomerCount"], b["coord"],
                             b["uVec"], f["end1NbrSlot"], f["end1NbrSide"], f["end2NbrSlot"], f["end2NbrSide"],
                             t["seedNode"], t["splitParams"])
    G.splitWire(dt["rankOffsets"], dt["freeList"], dt["freeOffsets"], fil["monomerCount"], db["coord"], db["uVec"],
                fil["end1NbrSlot"], fil["end1NbrSide"], fil["end2NbrSlot"], fil["end2NbrSide"], dt["seedNode"],
                dt["splitParams"], allocCounts=(C, C))
    orc_dm.aging_split_inherit_nuc(C, C, t["rankOffsets"], t["freeList"], t["freeOffsets"], t["nucFrac"])
    A.splitInheritNuc(dt["rankOffsets"], dt["freeList"], dt["freeOffsets"], dt["nucFrac"], allocCounts=(C, C))
    orc_dm.nucleate_fresh_cofilin(C, C, t["rankOffsets"], t["freeList"], t["freeOffsets"], t["cofFrac"])
    S.nucleateFreshCofilin(dt["rankOffsets"], dt["freeList"], dt["freeOffsets"], dt["cofFrac"], allocCounts=(C, C))
    _compare(sc, fil, dt, "split: ")
    orc_dm.aging_nucleate_fresh_atp(C, C, t["rankOffsets"], t["freeList"], t["freeOffsets"], t["nucFrac"])
    A.nucleateFreshAtp(dt["rankOffsets"], dt["freeList"], dt["freeOffsets"], dt["nucFrac"], allocCounts=(C, C))
    orc_dm.growth_recompute_drag(C, f["monomerCount"], b["segLength"], f["end1NbrSlot"], f["end2NbrSlot"],
                                 b["bTransGam"], b["bRotGam"], b["bTransDiff"], b["bRotDiff"], t["dragParams"],
                                 t["growCounts"])
    G.recomputeDrag(fil["monomerCount"], db["segLength"], fil["end1NbrSlot"], fil["end2NbrSlot"], db["bTransGam"],
                    db["bRotGam"], db["bTransDiff"], db["bRotDiff"], dt["dragParams"], dt["growCounts"])
    _compare(sc, fil, dt, "recomputeDrag: ")
    for op in ("put", "take"):
        getattr(orc_dm, f"pool_{op}_total")(t["pool"], t["rankOffsets"], C)
        _ctx()(f"sbx_actin_pool_{op}_total", dt["pool"], dt["rankOffsets"], C)
    _compare(sc, fil, dt, "pool: ")


def test_filament_ids_bitwise(orc_dm, seeded):
    sc = copy.deepcopy(seeded)
    fil, t = _dev(sc)
    ids = Turnover(fil, t, sc["cfg"]).filament_ids()
    want = oracle_filament_ids(orc_dm, sc)
    torch.cuda.synchronize()
    assert_same(want, ids.cpu().numpy(), "filID")
    assert np.array_equal(want, chain_walk_ids(sc))
    assert len(set(want[want >= 0].tolist())) > 100


def test_birth_allocation_overflow_and_reuse(orc_dm):
    """More birth requests than free slots: the lowest ranks form, in free-list order."""
    from helpers import turnover_store
    cfg = TurnoverConfig()
    C = 1024
    sc = turnover_store(C, cfg)
    rng = np.random.default_rng(1)
    f, t = sc["fil"], sc["t"]
    f["filState"][rng.random(C) < 0.9] = 0
    t["acceptFlag"][rng.random(C) < 0.3] = 1
    t["reqCoord"][:] = rng.normal(size=3 * C).astype(np.float32)
    t["reqUVec"][:] = rng.normal(size=3 * C).astype(np.float32)
    t["reqYVec"][:] = rng.normal(size=3 * C).astype(np.float32)
    fil, dt = _dev(sc)
    oracle_turnover_allocate(orc_dm, sc, t["acceptFlag"], t["reqCoord"], t["reqUVec"], t["reqYVec"], t["rankOffsets"])
    Turnover(fil, dt, cfg).allocate(dt["acceptFlag"], dt["reqCoord"], dt["reqUVec"], dt["reqYVec"],
                                    dt["rankOffsets"])
    _compare(sc, fil, dt, "birth: ")
    assert t["rankOffsets"][C] > t["freeOffsets"][C] > 0
    assert (f["filState"] >= 0).all()


def test_empty_and_rejected_calls():
    from softbox_b200.runtime import SbxError
    from softbox_b200.systems import _ctx
    ctx = _ctx()
    n = None
    assert ctx.raw("sbx_growth_grow", 0, n, n, n, n, n, n, n) == 0
    assert ctx.raw("sbx_depoly", 0, n, n, n, n, n, n, n, n, n) == 0
    assert ctx.raw("sbx_aging_age", 0, n, n, n, n) == 0
    assert ctx.raw("sbx_filid_init", 0, n, n, n) == 0
    buf = torch.zeros(8, dtype=torch.int32, device="cuda")
    with pytest.raises(SbxError):
        ctx("sbx_filid_jump", 8, buf, buf, buf)          # an in-place jump is rejected
    with pytest.raises(SbxError):
        ctx("sbx_growth_mark_splits", 8, buf, buf, buf, buf, buf, buf, buf, buf, buf, 4, buf, buf)   # reqCap < C
    ctx.sync()
