"""Shared test helpers: scene copies, oracle stepping and bitwise comparison."""
import copy

import numpy as np

from softbox_b200 import device as D, scenes


def host_copy(sc):
    return copy.deepcopy(sc)


def oracle_dense_run(orc, sc, t0, nsteps):
    """Advance a host scene with the oracle's DenseContractileHarness.cpuStep restatement."""
    desc = D.dense_desc(sc)
    orc.dense_run(desc, t0, nsteps)
    return sc


def assert_same(a, b, what=""):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    if a.dtype.kind == "f":
        ok = np.array_equal(a.view(np.uint32 if a.dtype == np.float32 else np.uint64),
                            b.view(np.uint32 if b.dtype == np.float32 else np.uint64))
    else:
        ok = np.array_equal(a, b)
    if not ok:
        diff = np.flatnonzero(a != b)
        raise AssertionError(f"{what}: {diff.size} of {a.size} entries differ; first at {diff[:5]}: "
                             f"{a.reshape(-1)[diff[:5]]} vs {b.reshape(-1)[diff[:5]]}")


def flat_arrays(sc, prefix=""):
    """(name, array) for every numpy array in a (nested) scene dict."""
    out = []
    for k, v in sc.items():
        if isinstance(v, dict):
            out += flat_arrays(v, prefix + k + ".")
        elif isinstance(v, np.ndarray):
            out.append((prefix + k, v))
    return out


def compare_scenes(host, dev_host, skip=()):
    """Bitwise comparison of every array of two host scenes; returns the names compared."""
    names = []
    dmap = dict(flat_arrays(dev_host))
    for name, arr in flat_arrays(host):
        if any(name.endswith(s) for s in skip) or name not in dmap:
            continue
        assert_same(arr, dmap[name], name)
        names.append(name)
    return names


def small_dense(scale=0.05, **kw):
    return scenes.dense_contractile(scenes.dense_small(scale, **kw))


# ---------------------------------------------------------------- crosslinker formation
def oracle_formation_grid(orc, sc):
    """FormationGrid.buildCpu (FormationGrid.java:90-101) on host arrays; returns the grid."""
    f = sc["fil"]
    b = f["body"]
    n = b["n"]
    g = sc["grid"]
    half, cell = g["half"], g["cell"]
    nX = 1 + int(np.ceil(2 * half / cell))
    total = nX ** 3
    grid = {"gridParams": np.array([-half, -half, -half, cell, 1.0 / cell, g["grab"]], np.float32),
            "gridDims": np.array([nX, nX, nX, total], np.int32),
            "center": np.zeros(3 * n, np.float32), "R": np.zeros(n, np.float32),
            "ownerStore": np.zeros(n, np.int32), "ownerSlot": np.zeros(n, np.int32),
            "bodyCell": np.full(n, -1, np.int32), "cellCount": np.zeros(total, np.int32),
            "chunkSum": np.zeros((total + 511) // 512 + 1, np.int32),
            "offsets": np.zeros(total + 1, np.int32), "contents": np.full(n, -1, np.int32),
            "candCountSeg": np.zeros(n, np.int32), "candBaseSeg": np.zeros(n + 1, np.int32)}
    vp = np.array([g["radius"]], np.float32)
    orc.fil_publish(n, b["coord"], b["segLength"], n, grid["center"], grid["R"], grid["ownerStore"],
                    grid["ownerSlot"], vp, None)
    orc.body_cell(n, grid["center"], grid["gridParams"], grid["gridDims"], n, grid["bodyCell"])
    orc.grid_zero(total, grid["cellCount"])
    orc.grid_histogram(grid["bodyCell"], n, grid["cellCount"])
    orc.grid_scan_local(total, grid["cellCount"], grid["offsets"], grid["chunkSum"])
    orc.grid_scan_chunks(total, grid["chunkSum"])
    orc.grid_scan_add(total, grid["offsets"], n, grid["cellCount"], grid["chunkSum"])
    orc.grid_scatter(grid["bodyCell"], n, grid["offsets"], grid["contents"], n, grid["cellCount"])
    return grid


def oracle_formation(orc, sc, step, use_grid=True):
    """CrosslinkerBundleHarness.formationCpu (CrosslinkerBundleHarness.java:451-507) on host
    arrays: counts, candidates, gates, admission, free list, ranks, allocate, orientation."""
    f, xl = sc["fil"], sc["xl"]
    b = f["body"]
    n, C, K = b["n"], sc["C"], sc["reqCap"]
    xl["formCounts"][1] = step
    orc.count_active_links(C, xl["linkState"], xl["linkFilA"], xl["linkFilB"], n, xl["activeLinkCount"])
    if use_grid:
        g = oracle_formation_grid(orc, sc)
        orc.xl_grid_form_count(n, b["coord"], b["segLength"], sc["filID"], g["gridParams"], g["gridDims"],
                               g["offsets"], g["contents"], g["candCountSeg"], xl["formParams"])
        orc.xl_grid_form_scan(n, g["candCountSeg"], g["candBaseSeg"], K, xl["reqFilA"], xl["reqFilB"],
                              xl["formCounts"])
        orc.xl_grid_form_emit(n, b["coord"], b["segLength"], sc["filID"], g["gridParams"], g["gridDims"],
                              g["offsets"], g["contents"], g["candBaseSeg"], g["candCountSeg"], K, xl["reqFilA"],
                              xl["reqFilB"], xl["formParams"])
    else:
        orc.xl_fil_fil_candidates(n, b["coord"], b["segLength"], sc["filID"], K, xl["reqFilA"], xl["reqFilB"],
                                  xl["formParams"], xl["formCounts"])
    orc.xl_form_gates(n, b["uVec"], b["end1"], b["end2"], b["segLength"], K, xl["reqFilA"], xl["reqFilB"],
                      xl["reqLoc1"], xl["reqLoc2"], xl["reqOrient"], xl["gatePass"], xl["formParams"],
                      xl["formCounts"])
    orc.xl_form_admit_reduce(K, xl["reqFilA"], xl["reqFilB"], xl["gatePass"], n, xl["minCand"])
    orc.xl_form_admit(K, xl["reqFilA"], xl["reqFilB"], xl["reqLoc1"], xl["reqLoc2"], xl["gatePass"], xl["minCand"],
                      xl["activeLinkCount"], C, xl["linkState"], xl["linkFilA"], xl["linkFilB"], xl["loc1"],
                      xl["loc2"], xl["acceptFlag"], xl["formParams"])
    orc.xl_free_flags(C, xl["linkState"], xl["freeCount"])
    orc.csr_scan(C, xl["freeCount"], xl["freeOffsets"])
    orc.xl_free_scatter(C, xl["linkState"], xl["freeOffsets"], xl["freeList"])
    orc.csr_scan(K, xl["acceptFlag"], xl["rankOffsets"])
    orc.xl_allocate(K, xl["reqFilA"], xl["reqFilB"], xl["reqLoc1"], xl["reqLoc2"], xl["rankOffsets"],
                    xl["freeList"], xl["freeOffsets"], C, xl["linkFilA"], xl["linkFilB"], xl["loc1"], xl["loc2"],
                    xl["linkState"], xl["strainHist"], xl["strainPlace"])
    orc.xl_place_orient(K, xl["reqOrient"], xl["rankOffsets"], xl["freeList"], xl["freeOffsets"], C,
                        xl["linkOrientSame"], xl["torqueMagHist"], xl["torqueMagPlace"])
    return sc


def oracle_turnover_allocate(orc, sc, accept, req_coord, req_u, req_y, rank_offsets, K=None):
    """FullSystemDemoHarness.allocCpu (:950-957) on host arrays."""
    f, t, C = sc["fil"], sc["t"], sc["C"]
    b = f["body"]
    K = C if K is None else K
    orc.xl_free_flags(C, f["filState"], t["freeCount"])
    orc.csr_scan(C, t["freeCount"], t["freeOffsets"])
    orc.xl_free_scatter(C, f["filState"], t["freeOffsets"], t["freeList"])
    orc.csr_scan(K, accept, rank_offsets)
    orc.birth_allocate(K, C, req_coord.size // 3, req_coord, req_u, req_y, rank_offsets, t["freeList"],
                       t["freeOffsets"], b["coord"], b["uVec"], b["yVec"], b["brownTransScale"], b["brownRotScale"],
                       f["filState"], t["birthParams"])


def oracle_turnover_cadence(orc, sc, step):
    """The turnover block of FullSystemDemoHarness.cpuStep (:648-683) on host arrays; returns
    False off-cadence (every kernel of the block is then a no-op)."""
    cfg = sc["cfg"]
    if not cfg.fires_at(step):
        return False
    from softbox_b200.turnover import BIOCHEM_DT
    f, t, C = sc["fil"], sc["t"], sc["C"]
    b = f["body"]
    orc.turnover_begin(step, cfg.seed, 1, float(cfg.on_rate), float(BIOCHEM_DT), t["pool"], t["growParams"],
                       t["growCounts"], t["depolyCounts"], t["agingCounts"], t["severCounts"])

    def death(flag):
        orc.apply_death(C, f["filState"], f["monomerCount"], t["seedNode"], f["end1NbrSlot"], f["end1NbrSide"],
                        f["end2NbrSlot"], f["end2NbrSide"], b["brownTransScale"], b["brownRotScale"], flag)
        if sc.get("release") is not None:
            la, lb, ls, bs = sc["release"]
            orc.turnover_release_dead(f["filState"], ls.size, la, lb, ls, bs.size, bs)

    orc.aging_age(C, f["filState"], t["nucFrac"], t["agingParams"], t["agingCounts"])
    orc.depoly_proxy(C, f["filState"], f["monomerCount"], b["coord"], b["uVec"], f["end1NbrSlot"], t["nucFrac"],
                     t["returnedMon"], t["deathFlag"], t["depolyParams"], t["depolyRateParams"], t["depolyCounts"])
    orc.csr_scan(C, t["returnedMon"], t["returnedOffsets"])
    death(t["deathFlag"])
    orc.pool_put_total(t["pool"], t["returnedOffsets"], C)
    for _ in range(max(1, cfg.polyboost)):
        orc.growth_grow(C, t["seedNode"], f["monomerCount"], b["coord"], b["uVec"], t["grewFlag"], t["growParams"],
                        t["growCounts"])
        orc.csr_scan(C, t["grewFlag"], t["grewOffsets"])
        orc.aging_growth_atp(C, t["grewFlag"], f["monomerCount"], t["nucFrac"])
        orc.pool_take_total(t["pool"], t["grewOffsets"], C)
    orc.cofilin_accumulate(C, f["filState"], t["nucFrac"], t["cofFrac"], t["cofilinParams"], t["severCounts"])
    orc.cofilin_dissolve(C, f["filState"], f["monomerCount"], t["cofFrac"], t["severDeathFlag"],
                         t["severReturnedMon"], t["cofilinParams"], t["severCounts"])
    orc.csr_scan(C, t["severReturnedMon"], t["severReturnedOffsets"])
    death(t["severDeathFlag"])
    orc.pool_put_total(t["pool"], t["severReturnedOffsets"], C)
    orc.growth_mark_splits(C, t["seedNode"], f["monomerCount"], b["coord"], b["uVec"], b["yVec"], t["acceptFlag"],
                           t["reqCoord"], t["reqUVec"], t["reqYVec"], C, t["splitParams"], t["growCounts"])
    oracle_turnover_allocate(orc, sc, t["acceptFlag"], t["reqCoord"], t["reqUVec"], t["reqYVec"], t["rankOffsets"])
    orc.growth_split_wire(C, C, t["rankOffsets"], t["freeList"], t["freeOffsets"], f["monomerCount"], b["coord"],
                          b["uVec"], f["end1NbrSlot"], f["end1NbrSide"], f["end2NbrSlot"], f["end2NbrSide"],
                          t["seedNode"], t["splitParams"])
    orc.aging_split_inherit_nuc(C, C, t["rankOffsets"], t["freeList"], t["freeOffsets"], t["nucFrac"])
    orc.nucleate_fresh_cofilin(C, C, t["rankOffsets"], t["freeList"], t["freeOffsets"], t["cofFrac"])
    orc.growth_recompute_drag(C, f["monomerCount"], b["segLength"], f["end1NbrSlot"], f["end2NbrSlot"],
                              b["bTransGam"], b["bRotGam"], b["bTransDiff"], b["bRotDiff"], t["dragParams"],
                              t["growCounts"])
    return True


def oracle_filament_ids(orc, sc):
    """FilIDSystem init + rounds(C) ping-pong jumps; the ids end in t['filID']."""
    from softbox_b200.systems import FilIDSystem
    f, t, C = sc["fil"], sc["t"], sc["C"]
    orc.filid_init(C, f["filState"], f["end2NbrSlot"], t["filID"])
    for r in range(FilIDSystem.rounds(C)):
        src, dst = (t["filID"], t["filIDTmp"]) if r % 2 == 0 else (t["filIDTmp"], t["filID"])
        orc.filid_jump(C, src, dst, f["filState"])
    return t["filID"]


def chain_walk_ids(sc):
    """Filament ids by walking end2 links to the chain terminal (the host chain walk that
    FilIDSystem replaces): an independent check of the pointer doubling."""
    f = sc["fil"]
    st, e2 = f["filState"], f["end2NbrSlot"]
    out = np.empty(st.size, np.int32)
    for s in range(st.size):
        if st[s] < 0:
            out[s] = -s - 2
            continue
        cur, seen = s, 0
        while True:
            nx = e2[cur]
            if nx < 0 or nx == cur or st[nx] < 0:
                break
            cur = nx
            seen += 1
            assert seen <= st.size, "cycle in the end2 links"
        out[s] = cur
    return out


def turnover_store(C, cfg, seed_conc=None):
    """A turnover scene of capacity C with every slot FREE (the harnesses' small stores)."""
    from softbox_b200 import scenes
    from softbox_b200.turnover import pool_array, turnover_arrays
    f = scenes.filament_store(C)
    f["filState"][:] = -1
    t = turnover_arrays(C, cfg)
    if seed_conc is not None:
        t["pool"][:] = pool_array(seed_conc, cfg.box_vol_um3)
    return {"fil": f, "t": t, "cfg": cfg, "C": C}


def set_segment(sc, s, mono, x=0.0, u=(-1.0, 0.0, 0.0), seed_node=-1):
    """Slot s ACTIVE with `mono` monomers at (x, 0, 0) along u, y = +y; drag from the length."""
    from softbox_b200 import scenes
    f, C = sc["fil"], sc["C"]
    b = f["body"]
    f["filState"][s] = 0
    f["monomerCount"][s] = mono
    scenes.set_vec(b["coord"], C, s, x, 0.0, 0.0)
    scenes.set_vec(b["uVec"], C, s, *u)
    scenes.set_vec(b["yVec"], C, s, 0.0, 1.0, 0.0)
    b["brownTransScale"][s] = np.float32(1.0)
    sc["t"]["seedNode"][s] = seed_node
    b["segLength"][s] = np.float32((mono + 1) * scenes.ACTIN_MONO_RADIUS)


def link(sc, a, a_end, b, b_end):
    """Glue end a_end (1 or 2) of slot a to end b_end of slot b, both directions."""
    f = sc["fil"]
    f[f"end{a_end}NbrSlot"][a], f[f"end{a_end}NbrSide"][a] = b, b_end - 1
    f[f"end{b_end}NbrSlot"][b], f[f"end{b_end}NbrSide"][b] = a, a_end - 1


def oracle_growth_cadence(orc, sc, step):
    """The growth-only cadence of GrowthHarness (grow -> grew scan -> markSplits -> split
    allocation -> splitWire -> recomputeDrag) on host arrays."""
    from softbox_b200.turnover import BIOCHEM_DT
    f, t, C, cfg = sc["fil"], sc["t"], sc["C"], sc["cfg"]
    b = f["body"]
    orc.turnover_begin(step, cfg.seed, 1, float(cfg.on_rate), float(BIOCHEM_DT), t["pool"], t["growParams"],
                       t["growCounts"], t["depolyCounts"], t["agingCounts"], t["severCounts"])
    orc.growth_grow(C, t["seedNode"], f["monomerCount"], b["coord"], b["uVec"], t["grewFlag"], t["growParams"],
                    t["growCounts"])
    orc.csr_scan(C, t["grewFlag"], t["grewOffsets"])
    orc.growth_mark_splits(C, t["seedNode"], f["monomerCount"], b["coord"], b["uVec"], b["yVec"], t["acceptFlag"],
                           t["reqCoord"], t["reqUVec"], t["reqYVec"], C, t["splitParams"], t["growCounts"])
    oracle_turnover_allocate(orc, sc, t["acceptFlag"], t["reqCoord"], t["reqUVec"], t["reqYVec"], t["rankOffsets"])
    orc.growth_split_wire(C, C, t["rankOffsets"], t["freeList"], t["freeOffsets"], f["monomerCount"], b["coord"],
                          b["uVec"], f["end1NbrSlot"], f["end1NbrSide"], f["end2NbrSlot"], f["end2NbrSide"],
                          t["seedNode"], t["splitParams"])
    orc.growth_recompute_drag(C, f["monomerCount"], b["segLength"], f["end1NbrSlot"], f["end2NbrSlot"],
                              b["bTransGam"], b["bRotGam"], b["bTransDiff"], b["bRotDiff"], t["dragParams"],
                              t["growCounts"])


def oracle_births(orc, sc, step):
    """Turnover.births on host arrays."""
    cfg = sc["cfg"]
    t, f, C = sc["t"], sc["fil"], sc["C"]
    if not cfg.fires_at(step) or "birthBox" not in t:
        return False
    K = t["birthAccept"].size
    orc.birth_emit_constant_actin(K, t["pool"], t["birthBox"], step, cfg.seed, t["birthAccept"], t["birthReqCoord"],
                                  t["birthReqUVec"], t["birthReqYVec"])
    oracle_turnover_allocate(orc, sc, t["birthAccept"], t["birthReqCoord"], t["birthReqUVec"], t["birthReqYVec"],
                             t["birthRankOffsets"], K=K)
    ro, fl, fo = t["birthRankOffsets"], t["freeList"], t["freeOffsets"]
    orc.birth_init_newborn(K, C, ro, fl, fo, f["monomerCount"], f["body"]["segLength"], t["seedParams"])
    orc.birth_tag_seeds(K, C, ro, fl, fo, t["seedNode"])
    orc.aging_nucleate_fresh_atp(K, C, ro, fl, fo, t["nucFrac"])
    orc.nucleate_fresh_cofilin(K, C, ro, fl, fo, t["cofFrac"])
    orc.pool_take_births(t["pool"], ro, K, fo, C, int(t["birthBox"][3]))
    return True


def turnover_view(sc):
    """The turnover arrays of a dense turnover scene as the cadence helpers take them."""
    xl, mot = sc["xl"], sc["mot"]
    return {"fil": sc["fil"], "t": sc["turnover"], "C": sc["fil"]["body"]["n"], "cfg": sc["tcfg"],
            "release": (xl["linkFilA"], xl["linkFilB"], xl["linkState"], mot["boundSeg"])}


def oracle_turnover_network_run(orc, sc, t0, nsteps):
    """TurnoverNetwork.run on host arrays: the turnover cadence and births at each biochem
    cadence, then the dense steps up to the next one."""
    view = turnover_view(sc)
    cfg = sc["tcfg"]
    t, end, ci = t0, t0 + nsteps, cfg.check_int
    while t < end:
        if cfg.fires_at(t):
            oracle_turnover_cadence(orc, view, t)
            oracle_births(orc, view, t)
        nxt = min(end, (t // ci + 1) * ci)
        oracle_dense_run(orc, sc, t, nxt - t)
        t = nxt
    return sc


def oracle_observables(orc, sc, seg_base=None, link_base=None, mot_base=None, volume=None, rounds=None):
    """The sbx_obs_* restatements on a host dense scene: (extent[nNet,2], stress[nNet],
    clusters[nNet,2], label)."""
    from softbox_b200.observables import HEAD_LEN, motor_backbones
    f, xl, mot = sc["fil"], sc["xl"], sc["mot"]
    fb = f["body"]
    nS, nM, nL, nBb = fb["n"], mot["nMotors"], xl["nLinks"], sc["mini"]["nBackbones"]
    seg = np.asarray(seg_base if seg_base is not None else [0, nS], np.int32)
    lnk = np.asarray(link_base if link_base is not None else [0, nL], np.int32)
    mtb = np.asarray(mot_base if mot_base is not None else [0, nM], np.int32)
    nNet = seg.size - 1
    if volume is None:
        b = sc["boxParams"]
        volume = [b[1] * b[2] * b[3]]
    vol = np.asarray(volume, np.float32)
    ext = np.zeros(2 * nNet)
    orc.obs_extent(nNet, seg, nS, fb["coord"], fb.get("coord64"), f["filState"], ext)
    st = np.zeros(nNet)
    orc.obs_stress(nNet, nS, fb["coord"], fb["uVec"], fb["end1"], fb["segLength"], lnk, xl["linkFilA"],
                   xl["linkFilB"], xl["linkState"], xl["loc1"], xl["loc2"], xl["xlinkData"], nM, mtb,
                   mot["body"]["coord"], mot["body"]["uVec"], mot["boundSeg"], mot["bindArc"], sc["bondData"],
                   HEAD_LEN, vol, st)
    mb = motor_backbones(sc["dim"], sc["mini"], nM)
    label = np.zeros(nS + nBb, np.int32)
    size = np.zeros(nS + nBb, np.int32)
    cl = np.zeros(2 * nNet, np.int32)
    orc.obs_clusters(nNet, seg, nS, f["filState"], f["end2NbrSlot"], nL, xl["linkFilA"], xl["linkFilB"],
                     xl["linkState"], nM, mot["boundSeg"], mb, nBb, label, size, cl)
    return ext.reshape(-1, 2), st, cl.reshape(-1, 2), label
