"""The turnover oracle against the reference harnesses' known answers (CPU only).

Each case restates a check of the reference's own validation harnesses on the same
scene: FilamentBirthHarness.checkAllocator (:118-192), DepolyHarness.checkSlotRecycle /
checkLinkBreak (:323-394), SeveringHarness.checkTrigger (:190-231), AgingHarness
.checkAgingKinetics (:186-232), GrowthHarness.checkLengthen / checkSplit (:241-352), the
integer conservation ledger (AgingHarness.conservationOk, :180-183) and FilIDSystem against
the host chain walk it replaces (FullSystemDemoHarness.computeFilID).
"""
import copy
import math

import numpy as np
import pytest

from helpers import (chain_walk_ids, link, oracle_filament_ids, oracle_growth_cadence, oracle_turnover_allocate,
                     oracle_turnover_cadence, set_segment, turnover_store)
from softbox_b200 import scenes
from softbox_b200.turnover import (BIOCHEM_DT, COFILIN_CONC, COFILIN_RATE, K_ATP_ON2_WITH_FORMIN, K_DISSOCIATION,
                                   K_HYDROLYSIS, TurnoverConfig, pool_fields)

F32 = np.float32


def _birth_scene(orc):
    """C=16: odd slots ACTIVE at x = 10 + s, even slots FREE; requests 0..2 at x = 0.10 + 0.01 q."""
    sc = turnover_store(16, TurnoverConfig())
    f, t = sc["fil"], sc["t"]
    b = f["body"]
    for s in range(16):
        scenes.set_vec(b["uVec"], 16, s, 1.0, 0.0, 0.0)
        scenes.set_vec(b["yVec"], 16, s, 0.0, 1.0, 0.0)
        if s & 1:
            f["filState"][s] = 0
            scenes.set_vec(b["coord"], 16, s, 10.0 + s, 0.0, 0.0)
            b["brownTransScale"][s] = 1.0
    for q in range(3):
        _request(t, 16, q, 0.10 + 0.01 * q)
    return sc


def _request(t, RC, r, x):
    t["acceptFlag"][r] = 1
    scenes.set_vec(t["reqCoord"], RC, r, x, 0.0, 0.0)
    scenes.set_vec(t["reqUVec"], RC, r, 1.0, 0.0, 0.0)
    scenes.set_vec(t["reqYVec"], RC, r, 0.0, 1.0, 0.0)


def _alloc(orc, sc):
    t = sc["t"]
    oracle_turnover_allocate(orc, sc, t["acceptFlag"], t["reqCoord"], t["reqUVec"], t["reqYVec"], t["rankOffsets"])


def test_birth_allocator_free_list_payload_and_stability(orc):
    sc = _birth_scene(orc)
    _alloc(orc, sc)
    f, t = sc["fil"], sc["t"]
    b = f["body"]
    assert t["freeOffsets"][16] == 8 and list(t["freeList"][:8]) == list(range(0, 16, 2))
    for q, s in enumerate((0, 2, 4)):
        assert f["filState"][s] == 0
        assert b["coord"][s] == F32(0.10 + 0.01 * q) and b["uVec"][s] == 1.0
        assert b["brownTransScale"][s] == F32(scenes.BTRANS_COEFF) and b["brownRotScale"][s] == F32(scenes.BROT_COEFF)
    for s in range(1, 16, 2):
        assert b["coord"][s] == F32(10 + s) and f["filState"][s] == 0
    for s in range(6, 16, 2):
        assert f["filState"][s] < 0 and b["brownTransScale"][s] == 0


def test_birth_overflow_clamp(orc):
    """C=8, 6 ACTIVE + 2 FREE, 5 requests: only the two lowest ranks form."""
    sc = turnover_store(8, TurnoverConfig())
    f, t = sc["fil"], sc["t"]
    f["filState"][:6] = 0
    for q in range(5):
        _request(t, 8, q, 0.2 + 0.01 * q)
    _alloc(orc, sc)
    assert (f["filState"] >= 0).sum() == 8
    assert f["body"]["coord"][6] == F32(0.2) and f["body"]["coord"][7] == F32(0.21)


def test_birth_same_step_reuse(orc):
    """A slot freed this step is in the free list rebuilt the same step: rank 0 takes slot 0."""
    sc = _birth_scene(orc)
    f, t = sc["fil"], sc["t"]
    flag = np.zeros(16, np.int32)
    flag[1] = 1
    orc.apply_death(16, f["filState"], f["monomerCount"], t["seedNode"], f["end1NbrSlot"], f["end1NbrSide"],
                    f["end2NbrSlot"], f["end2NbrSide"], f["body"]["brownTransScale"], f["body"]["brownRotScale"], flag)
    t["acceptFlag"][:] = 0
    _request(t, 16, 0, 0.5)
    _alloc(orc, sc)
    assert list(t["freeList"][:4]) == [0, 1, 2, 4]
    assert f["filState"][0] == 0 and f["body"]["coord"][0] == F32(0.5)


def _chain3():
    """A(0)-B(1)-C(2): A.end1 <-> B.end2, B.end1 <-> C.end2; C the pointed tip."""
    sc = turnover_store(8, TurnoverConfig())
    for s in range(3):
        set_segment(sc, s, 32, x=0.1 * s)
    link(sc, 0, 1, 1, 2)
    link(sc, 1, 1, 2, 2)
    return sc


def _death(orc, sc, slots):
    f, t = sc["fil"], sc["t"]
    flag = np.zeros(sc["C"], np.int32)
    flag[list(slots)] = 1
    orc.apply_death(sc["C"], f["filState"], f["monomerCount"], t["seedNode"], f["end1NbrSlot"], f["end1NbrSide"],
                    f["end2NbrSlot"], f["end2NbrSide"], f["body"]["brownTransScale"], f["body"]["brownRotScale"], flag)
    return f


def test_death_pointed_tip_and_interior(orc):
    f = _death(orc, _chain3(), [2])
    assert f["filState"][2] < 0 and f["end1NbrSlot"][1] == -1
    assert f["end1NbrSlot"][0] == 1 and f["end2NbrSlot"][1] == 0
    f = _death(orc, _chain3(), [1])
    assert f["filState"][1] < 0 and f["end1NbrSlot"][0] == -1 and f["end2NbrSlot"][2] == -1
    assert f["end1NbrSlot"][1] == -1 and f["end2NbrSlot"][1] == -1
    assert f["monomerCount"][1] == 0 and f["body"]["brownTransScale"][1] == 0


def test_death_of_adjacent_segments(orc):
    """Two neighbours dying together (severing can flag both): every link to either is gone."""
    f = _death(orc, _chain3(), [0, 1])
    assert (f["end1NbrSlot"][:3] == -1).all() and (f["end2NbrSlot"][:3] == -1).all()
    assert f["filState"][2] == 0


def test_slot_recycle_death_then_split(orc):
    """Slot 0 (a free filament at 2 monomers) dies; the 64-monomer tip in slot 1 splits into it."""
    cfg = TurnoverConfig(kin=1.0, pool0_um=1.0e30)
    sc = turnover_store(4, cfg)
    f, t = sc["fil"], sc["t"]
    set_segment(sc, 0, 2)
    set_segment(sc, 1, 64, seed_node=0)
    set_segment(sc, 2, 32, x=0.2)
    set_segment(sc, 3, 32, x=0.5)
    link(sc, 1, 1, 2, 2)
    b = f["body"]
    orc.turnover_begin(0, cfg.seed, 1, float(cfg.on_rate), float(BIOCHEM_DT), t["pool"], t["growParams"],
                       t["growCounts"], t["depolyCounts"], t["agingCounts"], t["severCounts"])
    orc.depoly(4, f["filState"], f["monomerCount"], b["coord"], b["uVec"], f["end1NbrSlot"], t["returnedMon"],
               t["deathFlag"], t["depolyParams"], t["depolyCounts"])
    assert t["deathFlag"][0] == 1 and t["returnedMon"][0] == 2
    _death(orc, sc, [0])
    assert f["filState"][0] < 0
    oracle_growth_cadence(orc, sc, 0)
    assert f["end1NbrSlot"][1] == 0 and f["filState"][0] == 0 and f["monomerCount"][0] == 32
    assert f["end1NbrSlot"][0] == 2 and f["end2NbrSlot"][2] == 0


def test_cofilin_accumulation_and_dissolve_threshold(orc):
    p_cof = COFILIN_CONC * COFILIN_RATE * BIOCHEM_DT
    cfg = TurnoverConfig(cof_ratio=0.5)
    for n in (1000, 3000, 10000):
        sc = turnover_store(4, cfg)
        f, t = sc["fil"], sc["t"]
        f["filState"][0] = 0
        t["nucFrac"][:] = 0
        t["nucFrac"][2 * 4 + 0] = 1.0
        t["severCounts"][1] = 1
        for _ in range(n):
            orc.cofilin_accumulate(4, f["filState"], t["nucFrac"], t["cofFrac"], t["cofilinParams"], t["severCounts"])
        assert abs(float(t["cofFrac"][0]) - (1.0 - (1.0 - p_cof) ** n)) < 1e-4
    n_star = math.ceil(math.log(1.0 - 0.5) / math.log(1.0 - p_cof))
    sc = turnover_store(4, cfg)
    f, t = sc["fil"], sc["t"]
    f["filState"][0] = 0
    f["monomerCount"][0] = 32
    t["nucFrac"][:] = 0
    t["nucFrac"][8] = 1.0
    t["severCounts"][1] = 1
    fired = -1
    for step in range(1, n_star + 6):
        orc.cofilin_accumulate(4, f["filState"], t["nucFrac"], t["cofFrac"], t["cofilinParams"], t["severCounts"])
        orc.cofilin_dissolve(4, f["filState"], f["monomerCount"], t["cofFrac"], t["severDeathFlag"],
                             t["severReturnedMon"], t["cofilinParams"], t["severCounts"])
        if t["severDeathFlag"][0] == 1:
            fired = step
            break
    assert fired == n_star and t["severReturnedMon"][0] == 32


def test_aging_kinetics_match_two_step_solution(orc):
    kH, kD = K_HYDROLYSIS, K_DISSOCIATION
    cfg = TurnoverConfig()
    for T in (1.0, 3.0, 5.0, 10.0):
        sc = turnover_store(8, cfg)
        f, t = sc["fil"], sc["t"]
        f["filState"][0] = 0
        t["agingCounts"][1] = 1
        for _ in range(int(round(T / BIOCHEM_DT))):
            orc.aging_age(8, f["filState"], t["nucFrac"], t["agingParams"], t["agingCounts"])
        atp = math.exp(-kH * T)
        adppi = kH / (kD - kH) * (math.exp(-kH * T) - math.exp(-kD * T))
        got = t["nucFrac"].reshape(3, 8)[:, 0].astype(np.float64)
        assert np.abs(got - [atp, adppi, 1.0 - atp - adppi]).max() < 0.01
    sc = turnover_store(4, cfg)
    f, t = sc["fil"], sc["t"]
    f["filState"][0] = 0
    t["nucFrac"][[0, 4, 8]] = [0.4, 0.35, 0.25]
    t["agingCounts"][1] = 1
    for _ in range(5000):
        orc.aging_age(4, f["filState"], t["nucFrac"], t["agingParams"], t["agingCounts"])
    assert abs(float(t["nucFrac"][0]) + float(t["nucFrac"][4]) + float(t["nucFrac"][8]) - 1.0) < 1e-5


def test_recompute_drag_matches_host_drag_law(orc):
    cfg = TurnoverConfig()
    for mc in (3, 20, 32, 40, 64, 100):
        sc = turnover_store(1, cfg)
        f, t = sc["fil"], sc["t"]
        f["monomerCount"][0] = mc
        ref = copy.deepcopy(f)
        scenes.drag_run_filament(ref, 0.1)
        t["growCounts"][3] = 1
        b = f["body"]
        orc.growth_recompute_drag(1, f["monomerCount"], b["segLength"], f["end1NbrSlot"], f["end2NbrSlot"],
                                  b["bTransGam"], b["bRotGam"], b["bTransDiff"], b["bRotDiff"], t["dragParams"],
                                  t["growCounts"])
        rb = ref["body"]
        for got, want in ((b["segLength"][0], rb["segLength"][0]), (b["bTransGam"][0], rb["bTransGam"][0]),
                          (b["bTransGam"][1], rb["bTransGam"][1]), (b["bRotGam"][1], rb["bRotGam"][1])):
            assert abs(float(got) - float(want)) / abs(float(want)) < 1e-6


def test_growth_rate_matches_on_rate(orc):
    """64 tips from 3 monomers, 3000 cadences, [actin] frozen: P_emp within 5 % of k_on c dt."""
    cfg = TurnoverConfig(pool0_um=15.0)
    N, C = 64, 4096
    sc = turnover_store(C, cfg)
    for k in range(N):
        set_segment(sc, k, 3, x=0.5 * k, seed_node=k)
    m0 = int(sc["fil"]["monomerCount"].sum())
    pool0 = sc["t"]["pool"].copy()
    for step in range(3000):
        sc["t"]["pool"][:] = pool0                    # conc frozen (no depletion)
        oracle_growth_cadence(orc, sc, step)
    grown = int(sc["fil"]["monomerCount"].sum()) - m0
    p_emp = grown / (N * 3000)
    p_th = K_ATP_ON2_WITH_FORMIN * 15.0 * BIOCHEM_DT
    assert abs(p_emp - p_th) / p_th < 0.05
    assert (sc["fil"]["filState"] >= 0).sum() > N


def test_split_lone_tip_and_inserted_child(orc):
    h = scenes.ACTIN_MONO_RADIUS
    cfg = TurnoverConfig(pool0_um=1.0e30)
    sc = turnover_store(8, cfg)
    set_segment(sc, 0, 64, seed_node=0)
    f, b = sc["fil"], sc["fil"]["body"]
    node0 = b["coord"][0] - F32(0.5) * b["segLength"][0]
    oracle_growth_cadence(orc, sc, 0)
    G, Cs = 0, int(f["end1NbrSlot"][0])
    assert Cs >= 1 and f["filState"][Cs] >= 0
    assert f["monomerCount"][G] == 32 and f["monomerCount"][Cs] == 32
    assert f["end1NbrSide"][G] == 1 and f["end2NbrSlot"][Cs] == G and f["end2NbrSide"][Cs] == 0
    assert f["end1NbrSlot"][Cs] == -1
    assert abs(float(b["coord"][G] - F32(0.5) * b["segLength"][G] - node0)) < 1e-5
    g_out = b["coord"][G] + F32(0.5) * b["segLength"][G]
    c_node = b["coord"][Cs] - F32(0.5) * b["segLength"][Cs]
    assert b["coord"][Cs] > b["coord"][G] and abs(float(c_node - g_out)) < 1.5 * h

    sc = turnover_store(8, cfg)
    set_segment(sc, 0, 64, seed_node=0)
    L0, L7 = (64 + 1) * h, (32 + 1) * h
    set_segment(sc, 7, 32, x=float(sc["fil"]["body"]["coord"][0]) + 0.5 * L0 + 0.5 * L7)
    link(sc, 0, 1, 7, 2)
    oracle_growth_cadence(orc, sc, 0)
    f = sc["fil"]
    Cs = int(f["end1NbrSlot"][0])
    assert Cs not in (-1, 7) and f["end2NbrSlot"][Cs] == 0 and f["end2NbrSide"][Cs] == 0
    assert f["end1NbrSlot"][Cs] == 7 and f["end1NbrSide"][Cs] == 1
    assert f["end2NbrSlot"][7] == Cs and f["end2NbrSide"][7] == 0
    assert f["monomerCount"][0] == f["monomerCount"][Cs] == f["monomerCount"][7] == 32


@pytest.fixture(scope="module")
def turnover_run(orc_dm):
    cfg = TurnoverConfig(kin=60.0, polyboost=2)
    sc = scenes.turnover_chains(n_chains=200, cap=2048, cfg=cfg, cofilin_high=0.4)
    m0 = int(sc["fil"]["monomerCount"].sum())
    start = copy.deepcopy(sc)
    stats = {"deaths": 0, "dissolves": 0, "splits": 0}
    for step in range(0, 3000, 100):
        oracle_turnover_cadence(orc_dm, sc, step)
        t = sc["t"]
        stats["deaths"] += int(t["deathFlag"].sum())
        stats["dissolves"] += int(t["severDeathFlag"].sum())
        stats["splits"] += int(min(t["rankOffsets"][sc["C"]], t["freeOffsets"][sc["C"]]))
    return start, sc, m0, stats


def test_turnover_conserves_monomers_exactly(turnover_run):
    _, sc, m0, stats = turnover_run
    _, _, taken, returned = pool_fields(sc["t"]["pool"])
    assert int(sc["fil"]["monomerCount"].sum()) == m0 + taken - returned
    assert stats["deaths"] > 0 and stats["dissolves"] > 0 and stats["splits"] > 0
    f = sc["fil"]
    act = f["filState"] >= 0
    assert (f["monomerCount"][~act] == 0).all() and (f["monomerCount"][act] >= 0).all()
    # every link is reciprocal
    for end in (1, 2):
        nb, side = f[f"end{end}NbrSlot"], f[f"end{end}NbrSide"]
        for s in np.flatnonzero(nb >= 0):
            back = f[f"end{side[s] + 1}NbrSlot"][nb[s]]
            assert back == s


def test_filament_ids_match_chain_walk(orc, turnover_run):
    _, sc, _, _ = turnover_run
    sc = copy.deepcopy(sc)
    ids = oracle_filament_ids(orc, sc)
    assert np.array_equal(ids, chain_walk_ids(sc))


def test_growth_atp_is_inert_after_the_grew_scan(orc_dm):
    """The harness order scans grewFlag (which clears it) before growthAtp reads it, so the
    composition of a grown tip is not reweighted; the kernel itself reweights when called
    on the flags directly."""
    cfg = TurnoverConfig(pool0_um=1.0e30)
    sc = turnover_store(4, cfg)
    set_segment(sc, 0, 10, seed_node=0)
    t = sc["t"]
    t["nucFrac"][[0, 4, 8]] = [0.2, 0.3, 0.5]
    before = t["nucFrac"].copy()
    orc_dm.turnover_begin(0, cfg.seed, 1, float(cfg.on_rate), float(BIOCHEM_DT), t["pool"], t["growParams"],
                          t["growCounts"], t["depolyCounts"], t["agingCounts"], t["severCounts"])
    f = sc["fil"]
    orc_dm.growth_grow(4, t["seedNode"], f["monomerCount"], f["body"]["coord"], f["body"]["uVec"], t["grewFlag"],
                       t["growParams"], t["growCounts"])
    assert t["grewFlag"][0] == 1 and f["monomerCount"][0] == 11
    flags = t["grewFlag"].copy()
    orc_dm.csr_scan(4, t["grewFlag"], t["grewOffsets"])
    orc_dm.aging_growth_atp(4, t["grewFlag"], f["monomerCount"], t["nucFrac"])
    assert np.array_equal(t["nucFrac"], before) and t["grewOffsets"][4] == 1
    orc_dm.aging_growth_atp(4, flags, f["monomerCount"], t["nucFrac"])
    w = F32(10) / F32(11)
    assert t["nucFrac"][0] == F32(F32(0.2) * w + F32(1) / F32(11))
