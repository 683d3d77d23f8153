"""GPU parity: every CUDA path against the CPU oracle, bit for bit.

The oracle is built with the same portable transcendentals as the kernels
(liboracle_dm.so), so identical inputs must give identical bits: integers (cells, CSR
offsets and lists, pair and reach lists, bound segments, nucleotide states, link states)
and floats (forces, poses) alike. Inputs are seeded scenes of the reference harnesses'
composition, taken to a realistic mid-run state by the oracle before each comparison.
"""
import copy

import numpy as np
import pytest

from helpers import assert_same, compare_scenes, oracle_dense_run, small_dense, flat_arrays
from softbox_b200 import device as D, scenes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def warm_scene(orc_dm):
    """A small dense network after 300 oracle steps (motors bound, nucleotides cycling)."""
    sc = small_dense(0.05)
    oracle_dense_run(orc_dm, sc, 0, 300)
    assert (sc["mot"]["boundSeg"] >= 0).sum() > 5
    return sc


def dev(x):
    return D.to_device(x)


def host(x):
    return D.to_host(x)


# ----------------------------------------------------------------------------- whole step
@pytest.mark.parametrize("mode", ["unfused", "graph", "fused", "auto"])
def test_dense_steps_bitwise(orc_dm, warm_scene, mode):
    from softbox_b200.engine import DenseNetwork
    ref = copy.deepcopy(warm_scene)
    net = DenseNetwork(copy.deepcopy(warm_scene))
    nsteps = 40
    if mode == "unfused":
        for t in range(300, 300 + nsteps):
            net.step_unfused(t)
    else:
        assert mode != "fused" or net.fused_available
        net.run(300, nsteps, mode=mode)
        assert net.status() == 0
    torch.cuda.synchronize()
    oracle_dense_run(orc_dm, ref, 300, nsteps)
    got = host(net.dev)
    names = compare_scenes({k: v for k, v in ref.items() if k != "cfg"}, got)
    assert len(names) > 80


@pytest.mark.parametrize("mode", ["unfused", "graph", "fused"])
def test_dense_supplied_noise_bitwise(orc, warm_scene, mode):
    """Supplied-noise mode of the dense step (every path) against the libm oracle fed the
    same Gaussian array: the same bits."""
    from softbox_b200.engine import DenseNetwork
    ref = copy.deepcopy(warm_scene)
    net = DenseNetwork(copy.deepcopy(warm_scene))
    rng = np.random.default_rng(21)
    nsteps = 40
    nf = rng.standard_normal((nsteps, 6, ref["fil"]["body"]["n"]), dtype=np.float32)
    nm = rng.standard_normal((nsteps, 6, ref["mot"]["body"]["n"]), dtype=np.float32)
    nb = rng.standard_normal((nsteps, 6, ref["mini"]["backbone"]["n"]), dtype=np.float32)
    net.set_noise(dev(nf), dev(nm), dev(nb), 300)
    net.run(300, nsteps, mode=mode)
    assert net.status() == 0
    torch.cuda.synchronize()
    orc.dense_run_supplied(D.dense_desc(ref), 300, nsteps, nf, nm, nb)
    names = compare_scenes({k: v for k, v in ref.items() if k != "cfg"}, host(net.dev))
    assert len(names) > 80


@pytest.mark.parametrize("mode", ["graph", "fused"])
def test_dense_fp64_coords(orc_dm, warm_scene, mode):
    from softbox_b200.engine import DenseNetwork
    ref = copy.deepcopy(warm_scene)
    for s, b in (("fil", "body"), ("mot", "body"), ("mini", "backbone")):
        D.add_coord64(ref[s][b])
    net = DenseNetwork(copy.deepcopy(warm_scene), fp64_coords=True)
    net.run(300, 25, mode=mode)
    torch.cuda.synchronize()
    oracle_dense_run(orc_dm, ref, 300, 25)
    got = host(net.dev)
    for s, b in (("fil", "body"), ("mot", "body"), ("mini", "backbone")):
        assert_same(ref[s][b]["coord64"], got[s][b]["coord64"], s + ".coord64")
        assert_same(ref[s][b]["coord"], got[s][b]["coord"], s + ".coord")


# ----------------------------------------------------------------------------- free rods
@pytest.mark.parametrize("mode", ["wang", "philox", "supplied"])
@pytest.mark.parametrize("fp64", [False, True])
def test_free_rods_bitwise(orc_dm, mode, fp64):
    from softbox_b200.engine import FreeRods
    f = scenes.free_rods_box(n=1024)
    nsteps = 60
    noise = None
    if mode == "supplied":
        noise = np.random.default_rng(7).standard_normal((nsteps, 6, 1024)).astype(np.float32)
    ref = copy.deepcopy(f)
    if fp64:
        D.add_coord64(ref["body"])
    rods = FreeRods(copy.deepcopy(f), fp64_coords=fp64)
    rods.run(0, nsteps, noise=mode, philox_seed=0xABCDEF12345, supplied=dev(noise) if noise is not None else None)
    torch.cuda.synchronize()
    b = ref["body"]
    n = b["n"]
    for t in range(nsteps):
        ref["counts"][1] = t
        if mode == "wang":
            orc_dm.brownian_force(n, b["randForce"], b["randTorque"], b["bTransGam"], b["bRotGam"],
                                  b["brownTransScale"], b["brownRotScale"], ref["params"], ref["counts"])
        elif mode == "philox":
            orc_dm.brownian_force_philox(n, b["randForce"], b["randTorque"], b["bTransGam"], b["bRotGam"],
                                         b["brownTransScale"], b["brownRotScale"], ref["params"], ref["counts"],
                                         0xABCDEF12345)
        else:
            orc_dm.brownian_force_supplied(n, b["randForce"], b["randTorque"], b["bTransGam"], b["bRotGam"],
                                           b["brownTransScale"], b["brownRotScale"], ref["params"],
                                           np.ascontiguousarray(noise[t]))
        orc_dm.integrate(n, b["coord"], b["coord64"], b["uVec"], b["yVec"], b["forceSum"], b["torqueSum"],
                         b["randForce"], b["randTorque"], b["bTransGam"], b["bRotGam"], ref["params"])
        orc_dm.derive(n, b["coord"], b["uVec"], b["yVec"], b["zVec"], b["end1"], b["end2"], b["segLength"])
    got = host(rods.dev)
    for k in ("coord", "uVec", "yVec", "zVec", "end1", "end2", "randForce", "randTorque") + (("coord64",) if fp64 else ()):
        assert_same(b[k], got["body"][k], k)


def test_supplied_noise_nonfinite_rejected():
    from softbox_b200.engine import FreeRods
    from softbox_b200.runtime import SbxError
    f = scenes.free_rods_box(n=64)
    rods = FreeRods(f)
    noise = np.zeros((3, 6, 64), np.float32)
    noise[1, 4, 17] = np.nan
    before = rods.pull("coord").copy()
    with pytest.raises(SbxError) as e:
        rods.run(0, 3, noise="supplied", supplied=dev(noise))
    assert e.value.code == -6
    assert_same(before, rods.pull("coord"), "coord untouched")


def test_fdt_golden_on_gpu():
    """The reference's published FDT numbers (JOURNAL.md:2249-2251), reproduced on the B200."""
    from softbox_b200.engine import FreeRods
    n, m = 2048, 8000
    rods = FreeRods(scenes.free_rods_fdt(n, trans_scale=1.0, rot_scale=0.0, seed=12345))
    ts, msd = [], [[], [], []]
    for step in range(0, m + 1, 200):
        c = rods.pull("coord").astype(np.float64).reshape(3, n)
        ts.append(step * 1e-4)
        for k in range(3):
            msd[k].append((c[k] ** 2).sum() / n)
        if step < m:
            rods.run(step, 200)
    ts = np.array(ts)
    D_ = [float((ts * np.array(v)).sum() / (ts * ts).sum() / 2) for v in msd]
    rods = FreeRods(scenes.free_rods_fdt(n, trans_scale=0.0, rot_scale=1.0, seed=67890))
    ts, cs = [], []
    for step in range(0, m // 5 + 1, 20):
        ts.append(step * 1e-4)
        cs.append(rods.pull("uVec")[:n].astype(np.float64).sum() / n)
        if step < m // 5:
            rods.run(step, 20)
    ts, cs = np.array(ts), np.array(cs)
    w = (cs > 0.2) & (cs < 0.95)
    x, y = ts[w], np.log(cs[w])
    k = len(x)
    slope = (k * (x * y).sum() - x.sum() * y.sum()) / (k * (x * x).sum() - x.sum() ** 2)
    got = D_ + [-slope / 2]
    for g, w_ in zip(got, [1.11676e-1, 7.36203e-2, 7.53293e-2, 1.89712e1]):
        assert float(f"{g:.5e}") == w_, got


# ----------------------------------------------------------------------------- per system
def _s(warm):
    return copy.deepcopy(warm)


def test_grid_build_and_broad_phase(orc_dm, warm_scene):
    from softbox_b200.systems import SpatialGrid
    sc = _s(warm_scene)
    g = sc["grid"]
    rng = np.random.default_rng(3)
    # perturb the published centres so the build is not the scene's last one
    g["center"][:] += rng.normal(scale=0.05, size=g["center"].shape).astype(np.float32)
    d = dev(g)
    SpatialGrid.bodyCell(d["center"], d["gridParams"], d["gridDims"], d["gridCounts"], d["bodyCell"])
    SpatialGrid.build(d["bodyCell"], d["gridCounts"], d["gridDims"], d["cellCount"], d["chunkSum"],
                      d["gridCellOffsets"], d["gridCellContents"])
    cap, S = g["cap"], int(g["gridCounts"][1])
    orc_dm.body_cell(cap, g["center"], g["gridParams"], g["gridDims"], S, g["bodyCell"])
    C_ = g["totalCells"]
    orc_dm.grid_zero(C_, g["cellCount"])
    orc_dm.grid_histogram(g["bodyCell"], S, g["cellCount"])
    orc_dm.grid_scan_local(C_, g["cellCount"], g["gridCellOffsets"], g["chunkSum"])
    orc_dm.grid_scan_chunks(C_, g["chunkSum"])
    orc_dm.grid_scan_add(C_, g["gridCellOffsets"], cap, g["cellCount"], g["chunkSum"])
    orc_dm.grid_scatter(g["bodyCell"], S, g["gridCellOffsets"], g["gridCellContents"], cap, g["cellCount"])
    h = host(d)
    for k in ("bodyCell", "cellCount", "chunkSum", "gridCellOffsets", "gridCellContents"):
        assert_same(g[k], h[k], k)
    # broad phase: bitwise vs the oracle (order included) and set-equal to O(N^2) brute force
    cand = torch.full((cap * 256,), -1, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(cap, dtype=torch.int32, device="cuda")
    SpatialGrid.broadPhase(d["center"], d["boundingRadius"], d["bodyCell"], d["gridCellOffsets"],
                           d["gridCellContents"], d["gridDims"], d["gridParams"], d["gridCounts"], cand, cnt)
    bcand = torch.full((cap * 256,), -1, dtype=torch.int32, device="cuda")
    bcnt = torch.zeros(cap, dtype=torch.int32, device="cuda")
    SpatialGrid.bruteForce(d["center"], d["boundingRadius"], d["gridParams"], d["gridCounts"], bcand, bcnt)
    ocand = np.full(cap * 256, -1, np.int32)
    ocnt = np.zeros(cap, np.int32)
    orc_dm.broad_phase(cap, g["center"], g["boundingRadius"], g["bodyCell"], g["gridCellOffsets"],
                       g["gridCellContents"], g["gridDims"], g["gridParams"], S, ocand, ocnt)
    assert_same(ocand, host(cand), "candPartner")
    assert_same(ocnt, host(cnt), "candCount")
    hc, hcnt, hb, hbcnt = host(cand), host(cnt), host(bcand), host(bcnt)
    assert np.array_equal(hcnt, hbcnt)
    assert hcnt.sum() > 0 and hcnt.max() <= 256
    for i in range(cap):
        k = hcnt[i]
        assert np.array_equal(np.sort(hc[i * 256:i * 256 + k]), np.sort(hb[i * 256:i * 256 + k]))


def test_grid_degenerate_single_cell(orc_dm):
    """All bodies in one clamped cell (and padding slots): the stable order must survive."""
    from softbox_b200.systems import SpatialGrid
    cap, S = 3000, 2500
    center = np.zeros(3 * cap, np.float32)
    gp = np.array([0, 0, 0, 1.0, 1.0, 0.1], np.float32)
    gd = np.array([4, 4, 4, 64], np.int32)
    counts = np.array([0, S, 0, 0], np.int32)
    arrays = {"center": center, "gp": gp, "gd": gd, "counts": counts, "bodyCell": np.full(cap, -7, np.int32),
              "cellCount": np.zeros(64, np.int32), "chunkSum": np.zeros(2, np.int32),
              "off": np.zeros(65, np.int32), "cont": np.full(cap, -1, np.int32)}
    d = dev(arrays)
    SpatialGrid.bodyCell(d["center"], d["gp"], d["gd"], d["counts"], d["bodyCell"])
    SpatialGrid.build(d["bodyCell"], d["counts"], d["gd"], d["cellCount"], d["chunkSum"], d["off"], d["cont"])
    h = host(d)
    assert_same(np.concatenate([np.zeros(S, np.int32), np.full(cap - S, -1, np.int32)]), h["bodyCell"], "bodyCell")
    assert_same(np.arange(S, dtype=np.int32), h["cont"][:S], "contents")
    assert h["off"][0] == 0 and h["off"][64] == S and h["cellCount"][0] == S


@pytest.mark.parametrize("which", ["motor", "linkA", "linkB", "backbone"])
def test_csr_build_matches_serial_and_chunked(orc_dm, warm_scene, which):
    from softbox_b200.systems import CrossBridgeSystem
    sc = _s(warm_scene)
    keys, rows = {
        "motor": (sc["mot"]["boundSeg"], sc["fil"]["body"]["n"]),
        "linkA": (sc["xl"]["linkFilA"], sc["fil"]["body"]["n"]),
        "linkB": (sc["xl"]["linkFilB"], sc["fil"]["body"]["n"]),
        "backbone": (sc["mini"]["headBackboneSlot"], sc["mini"]["nBackbones"]),
    }[which]
    n = keys.size
    cnt, off, lst = np.zeros(rows, np.int32), np.zeros(rows + 1, np.int32), np.full(max(n, 1), -1, np.int32)
    orc_dm.csr_histogram(keys, n, rows, cnt)
    orc_dm.csr_scan(rows, cnt, off)
    orc_dm.csr_scatter(keys, n, off, cnt, lst)
    # the chunked (parallel) reference variant produces the same offsets and list
    cs = orc_dm.body_chunk_size(n, rows)
    nch = (n + cs - 1) // cs
    mtx = np.zeros(nch * rows, np.int32)
    cnt2, off2, lst2 = np.zeros(rows, np.int32), np.zeros(rows + 1, np.int32), np.full(max(n, 1), -1, np.int32)
    orc_dm.csr_chunk_zero(nch, rows, mtx)
    orc_dm.csr_chunk_histogram(keys, n, rows, cs, nch, mtx)
    orc_dm.csr_chunk_reduce(rows, nch, mtx, cnt2)
    orc_dm.csr_scan(rows, cnt2, off2)
    orc_dm.csr_chunk_scatter(keys, n, rows, cs, nch, off2, lst2, mtx)
    assert_same(off, off2, "chunked offsets")
    assert_same(lst, lst2, "chunked list")
    d = dev({"k": keys, "c": np.zeros(rows, np.int32), "o": np.zeros(rows + 1, np.int32),
             "l": np.full(max(n, 1), -1, np.int32)})
    CrossBridgeSystem.csrBuild(d["k"], rows, d["c"], d["o"], d["l"])
    h = host(d)
    assert_same(off, h["o"], "offsets")
    assert_same(lst, h["l"], "list")
    assert_same(cnt, h["c"], "rowCount")


@pytest.mark.parametrize("entry", ["sbx_csr_build", "sbx_csr_build_payload"])
def test_csr_build_out_of_range_key_is_skipped_and_reported(orc_dm, warm_scene, entry):
    """A key >= the row count (the reference's Java would throw) touches no row: the item
    is skipped, the next sync reports SBX_EINVAL once, and offsets/list/counts equal the
    oracle's build of the same keys with that item unbound."""
    from softbox_b200.runtime import default_context
    sc = _s(warm_scene)
    rows = sc["fil"]["body"]["n"]
    keys = sc["mot"]["boundSeg"].copy()
    keys[3] = rows
    keys[-1] = rows + 1000
    n = keys.size
    fixed = np.where(keys >= rows, -1, keys).astype(np.int32)
    cnt, off, lst = np.zeros(rows, np.int32), np.zeros(rows + 1, np.int32), np.full(n, -1, np.int32)
    orc_dm.csr_histogram(fixed, n, rows, cnt)
    orc_dm.csr_scan(rows, cnt, off)
    orc_dm.csr_scatter(fixed, n, off, cnt, lst)
    d = dev({"k": keys, "c": np.zeros(rows, np.int32), "o": np.zeros(rows + 1, np.int32),
             "l": np.full(n, -1, np.int32), "p": np.ones(13 * n, np.float32), "rp": np.zeros(6 * n, np.float32)})
    ctx = default_context()
    ctx.sync()
    args = [d["k"], n, rows, d["c"], d["o"], d["l"]]
    if entry == "sbx_csr_build_payload":
        args += [d["p"], 13, 6, None, d["rp"]]
    assert ctx.raw(entry, *args) == 0
    assert ctx.raw("sbx_ctx_sync") == -1
    assert ctx.raw("sbx_ctx_sync") == 0
    h = host(d)
    assert_same(off, h["o"], "offsets")
    assert_same(lst, h["l"], "list")
    assert_same(cnt, h["c"], "rowCount")


def test_binding_systems(orc_dm, warm_scene):
    from softbox_b200.systems import BindingDetectionSystem, NucleotideCycleSystem
    sc = _s(warm_scene)
    m, g, fb = sc["mot"], sc["grid"], sc["fil"]["body"]
    nM, nSeg = m["nMotors"], fb["n"]
    m["counts"][1] = 300
    d = dev({"m": m, "g": g, "e1": fb["end1"], "e2": fb["end2"]})
    dm, dg = d["m"], d["g"]
    BindingDetectionSystem.gridReachable(dm["head"], dm["uVec"], dm["rodUVec"], d["e1"], d["e2"], dg["gridParams"],
                                         dg["gridDims"], dg["gridCellOffsets"], dg["gridCellContents"],
                                         dg["ownerStore"], dg["ownerSlot"], dg["reachSeg"], dg["reachCount"],
                                         dm["kinParams"])
    orc_dm.grid_reachable(nM, m["head"], m["uVec"], m["rodUVec"], nSeg, fb["end1"], fb["end2"], g["gridParams"],
                          g["gridDims"], g["gridCellOffsets"], g["gridCellContents"], g["ownerStore"],
                          g["ownerSlot"], g["reachSeg"], g["reachCount"], m["kinParams"])
    hg = host(dg)
    assert_same(g["reachCount"], hg["reachCount"], "reachCount")
    assert_same(g["reachSeg"], hg["reachSeg"], "reachSeg")
    # grid reach == O(N*M) brute reach (as sets)
    bs = torch.full((nM * 256,), -1, dtype=torch.int32, device="cuda")
    bc = torch.zeros(nM, dtype=torch.int32, device="cuda")
    BindingDetectionSystem.bruteReachable(dm["head"], dm["uVec"], dm["rodUVec"], d["e1"], d["e2"], bs, bc,
                                          dm["kinParams"])
    hbs, hbc = host(bs), host(bc)
    assert np.array_equal(hbc, hg["reachCount"])
    for i in range(nM):
        k = hbc[i]
        assert np.array_equal(np.sort(hbs[i * 256:i * 256 + k]), np.sort(hg["reachSeg"][i * 256:i * 256 + k]))
    # release -> bind -> cycle
    NucleotideCycleSystem.catchSlipRelease(dm["boundSeg"], dm["forceDotFil"], dm["forceMag"], dm["cooldown"],
                                           dm["stats"], dm["capStats"], dm["kinParams"], dm["counts"])
    BindingDetectionSystem.bindNearest(dm["head"], dm["uVec"], dm["rodUVec"], d["e1"], d["e2"], dg["reachSeg"],
                                       dg["reachCount"], dm["boundSeg"], dm["bindArc"], dm["kinParams"])
    NucleotideCycleSystem.cycle(dm["nucleotideState"], dm["boundSeg"], dm["forceDotHist"], dm["nucParams"],
                                dm["counts"])
    orc_dm.catch_slip_release(nM, m["boundSeg"], m["forceDotFil"], m["forceMag"], m["cooldown"], m["stats"],
                              m["capStats"], m["kinParams"], m["counts"])
    orc_dm.bind_nearest(nM, m["head"], m["uVec"], m["rodUVec"], nSeg, fb["end1"], fb["end2"], g["reachSeg"],
                        g["reachCount"], m["boundSeg"], m["bindArc"], m["kinParams"])
    orc_dm.cycle(nM, m["nucleotideState"], m["boundSeg"], m["forceDotHist"], m["nucParams"], m["counts"])
    hm = host(dm)
    for k in ("boundSeg", "bindArc", "cooldown", "stats", "capStats", "nucleotideState"):
        assert_same(m[k], hm[k], k)


def test_force_systems(orc_dm, warm_scene):
    """chain, crosslinker forces/torsion/unbind, cross-bridge, joints, dimer, tether, gathers."""
    from softbox_b200 import systems as S
    sc = _s(warm_scene)
    f, fb, m, mb, xl, mini = sc["fil"], sc["fil"]["body"], sc["mot"], sc["mot"]["body"], sc["xl"], sc["mini"]
    bb = mini["backbone"]
    nSeg, nB, nM, nBb = fb["n"], mb["n"], m["nMotors"], bb["n"]
    xl["counts"][1] = 300
    rng = np.random.default_rng(11)
    for b in (fb, mb, bb):
        b["forceSum"][:] = rng.normal(scale=1e-12, size=b["forceSum"].shape).astype(np.float32)
        b["torqueSum"][:] = rng.normal(scale=1e-20, size=b["torqueSum"].shape).astype(np.float32)
    d = dev({k: sc[k] for k in ("fil", "mot", "dim", "mini", "xl")} | {"bondData": sc["bondData"],
                                                                         "xbParams": sc["xbParams"]})
    df, dfb, dmo, dmb, dxl, dmi, ddi = d["fil"], d["fil"]["body"], d["mot"], d["mot"]["body"], d["xl"], d["mini"], \
        d["dim"]
    dbb = dmi["backbone"]
    S.ChainBendingForceSystem.chainForces(dfb["coord"], dfb["uVec"], dfb["segLength"], df["end2NbrSlot"],
                                          df["end2NbrSide"], df["end1NbrSlot"], df["end1NbrSide"], dfb["bTransGam"],
                                          dfb["bRotGam"], dfb["forceSum"], dfb["torqueSum"], df["chainParams"])
    orc_dm.chain_forces(nSeg, fb["coord"], fb["uVec"], fb["segLength"], f["end2NbrSlot"], f["end2NbrSide"],
                        f["end1NbrSlot"], f["end1NbrSide"], fb["bTransGam"], fb["bRotGam"], fb["forceSum"],
                        fb["torqueSum"], f["chainParams"])
    S.CrosslinkerSystem.unbind(dfb["coord"], dfb["uVec"], dfb["end1"], dxl["linkFilA"], dxl["linkFilB"], dxl["loc1"],
                               dxl["loc2"], dxl["linkState"], dxl["strainHist"], dxl["strainPlace"],
                               dxl["offParams"], dxl["counts"])
    S.CrosslinkerSystem.countActiveLinks(dxl["linkState"], dxl["linkFilA"], dxl["linkFilB"], dxl["activeLinkCount"])
    S.CrosslinkerSystem.linkForces(dfb["coord"], dfb["uVec"], dfb["end1"], dfb["bTransGam"], dxl["linkFilA"],
                                   dxl["linkFilB"], dxl["loc1"], dxl["loc2"], dxl["activeLinkCount"],
                                   dxl["xlinkData"], dxl["xlParams"])
    S.CrosslinkerSystem.linkTorsion(dfb["uVec"], dxl["linkFilA"], dxl["linkFilB"], dxl["linkState"],
                                    dxl["linkOrientSame"], dxl["torqueMagHist"], dxl["torqueMagPlace"],
                                    dxl["xlinkData"], dxl["torsionParams"])
    nL = xl["nLinks"]
    orc_dm.xl_unbind(nSeg, fb["uVec"], fb["end1"], nL, xl["linkFilA"], xl["linkFilB"], xl["loc1"], xl["loc2"],
                     xl["linkState"], xl["strainHist"], xl["strainPlace"], xl["offParams"], xl["counts"])
    orc_dm.count_active_links(nL, xl["linkState"], xl["linkFilA"], xl["linkFilB"], nSeg, xl["activeLinkCount"])
    orc_dm.link_forces(nSeg, fb["coord"], fb["uVec"], fb["end1"], fb["bTransGam"], nL, xl["linkFilA"],
                       xl["linkFilB"], xl["loc1"], xl["loc2"], xl["activeLinkCount"], xl["xlinkData"], xl["xlParams"])
    orc_dm.link_torsion(nSeg, fb["uVec"], nL, xl["linkFilA"], xl["linkFilB"], xl["linkState"], xl["linkOrientSame"],
                        xl["torqueMagHist"], xl["torqueMagPlace"], xl["xlinkData"], xl["torsionParams"])
    # gathers over the reference CSR (built by the oracle, uploaded)
    for side, key in ((0, "linkFilA"), (1, "linkFilB")):
        cnt, off, lst = np.zeros(nSeg, np.int32), np.zeros(nSeg + 1, np.int32), np.zeros(nL, np.int32)
        orc_dm.csr_histogram(xl[key], nL, nSeg, cnt)
        orc_dm.csr_scan(nSeg, cnt, off)
        orc_dm.csr_scatter(xl[key], nL, off, cnt, lst)
        do, dl = dev(off), dev(lst)
        (S.CrosslinkerSystem.segGatherA if side == 0 else S.CrosslinkerSystem.segGatherB)(
            do, dl, dxl["xlinkData"], dxl["linkState"], dfb["forceSum"], dfb["torqueSum"])
        (orc_dm.seg_gather_a if side == 0 else orc_dm.seg_gather_b)(nSeg, off, lst, xl["xlinkData"],
                                                                    xl["linkState"], fb["forceSum"], fb["torqueSum"])
    # myosin structure + cross-bridge
    S.MotorJointSystem.joints(dmb["coord"], dmb["uVec"], dmb["segLength"], dmb["bTransGam"], dmb["bRotGam"],
                              dmb["forceSum"], dmb["torqueSum"], dmo["nucleotideState"], dmo["jointParams"])
    S.DimerCouplingSystem.couple(dmb["coord"], dmb["uVec"], dmb["segLength"], dmb["bTransGam"], dmb["bRotGam"],
                                 dmb["forceSum"], dmb["torqueSum"], ddi["motorA"], ddi["motorB"], ddi["parallel"],
                                 ddi["dimerParams"], dmo["boundSeg"])
    S.MiniFilamentSystem.tether(dmb["coord"], dmb["uVec"], dmb["segLength"], dmb["bTransGam"], dmb["bRotGam"],
                                dmb["forceSum"], dmb["torqueSum"], dbb["coord"], dbb["uVec"], dmi["bbInvDragY"],
                                dmi["headBackboneSlot"], dmi["motorA"], dmi["attachAxial"], dmi["miniData"],
                                dmi["miniParams"])
    S.CrossBridgeSystem.bondForces(dmb["coord"], dmb["uVec"], dmb["yVec"], dmb["bRotGam"], dfb["coord"], dfb["uVec"],
                                   dfb["yVec"], dfb["bRotGam"], dfb["segLength"], dmo["boundSeg"], dmo["bindArc"],
                                   dmo["nucleotideState"], d["bondData"], d["xbParams"])
    S.CrossBridgeSystem.applyHeadForce(d["bondData"], dmb["forceSum"], dmb["torqueSum"])
    S.CrossBridgeSystem.registerForceDot(d["bondData"], dmo["boundSeg"], dmo["forceDotFil"], dmo["forceMag"],
                                         dmo["forceDotHist"], dmo["forceDotPlace"])
    orc_dm.joints(nB, mb["coord"], mb["uVec"], mb["segLength"], mb["bTransGam"], mb["bRotGam"], mb["forceSum"],
                  mb["torqueSum"], m["nucleotideState"], m["jointParams"])
    dim = sc["dim"]
    orc_dm.dimer_couple(nB, mb["coord"], mb["uVec"], mb["segLength"], mb["bTransGam"], mb["bRotGam"],
                        mb["forceSum"], mb["torqueSum"], dim["nDimers"], dim["motorA"], dim["motorB"],
                        dim["parallel"], dim["dimerParams"], m["boundSeg"])
    orc_dm.mini_tether(nB, mb["coord"], mb["uVec"], mb["segLength"], mb["bTransGam"], mb["bRotGam"], mb["forceSum"],
                       mb["torqueSum"], nBb, bb["coord"], bb["uVec"], mini["bbInvDragY"], mini["nDimers"],
                       mini["headBackboneSlot"], mini["motorA"], mini["attachAxial"], mini["miniData"],
                       mini["miniParams"])
    orc_dm.bond_forces(nB, mb["coord"], mb["uVec"], mb["yVec"], mb["bRotGam"], nSeg, fb["coord"], fb["uVec"],
                       fb["yVec"], fb["bRotGam"], fb["segLength"], m["boundSeg"], m["bindArc"], m["nucleotideState"],
                       sc["bondData"], sc["xbParams"])
    orc_dm.apply_head_force(nB, sc["bondData"], mb["forceSum"], mb["torqueSum"])
    orc_dm.register_force_dot(nM, sc["bondData"], m["boundSeg"], m["forceDotFil"], m["forceMag"], m["forceDotHist"],
                              m["forceDotPlace"])
    got = host(d)
    names = compare_scenes({k: sc[k] for k in ("fil", "mot", "dim", "mini", "xl", "bondData")}, got)
    assert len(names) > 40
    # gathers equal their O(N^2) brute references (bitwise, same summation order)
    bF = torch.zeros_like(dfb["forceSum"])
    bT = torch.zeros_like(dfb["torqueSum"])
    S.CrossBridgeSystem.bruteGather(dmo["boundSeg"], d["bondData"], bF, bT)
    cnt, off, lst = np.zeros(nSeg, np.int32), np.zeros(nSeg + 1, np.int32), np.zeros(nM, np.int32)
    orc_dm.csr_histogram(m["boundSeg"], nM, nSeg, cnt)
    orc_dm.csr_scan(nSeg, cnt, off)
    orc_dm.csr_scatter(m["boundSeg"], nM, off, cnt, lst)
    gF = torch.zeros_like(bF)
    gT = torch.zeros_like(bT)
    S.CrossBridgeSystem.segGather(dev(off), dev(lst), d["bondData"], gF, gT)
    assert_same(host(bF), host(gF), "segGather == bruteGather (force)")
    assert_same(host(bT), host(gT), "segGather == bruteGather (torque)")


def test_integration_systems(orc_dm, warm_scene):
    from softbox_b200 import systems as S
    sc = _s(warm_scene)
    fb, f = sc["fil"]["body"], sc["fil"]
    n = fb["n"]
    f["counts"][1] = 300     # a containment-cadence step (300 % 10 == 0)
    rng = np.random.default_rng(5)
    fb["forceSum"][:] = rng.normal(scale=1e-12, size=3 * n).astype(np.float32)
    fb["torqueSum"][:] = rng.normal(scale=1e-20, size=3 * n).astype(np.float32)
    fb["coord"][:n] *= np.float32(1.2)      # push some rods through the walls
    d = dev({"fil": f, "box": sc["boxParams"]})
    db = d["fil"]["body"]
    S.MechanicsFusion.forceBuild(db["randForce"], db["randTorque"], torch.zeros_like(db["randForce"]),
                                 torch.zeros_like(db["randTorque"]), db["bTransGam"], db["bRotGam"],
                                 db["brownTransScale"], db["brownRotScale"], d["fil"]["params"], d["fil"]["counts"])
    S.BrownianForceSystem.brownianForce(db["randForce"], db["randTorque"], db["bTransGam"], db["bRotGam"],
                                        db["brownTransScale"], db["brownRotScale"], d["fil"]["params"],
                                        d["fil"]["counts"])
    S.ContainmentSystem.confine(db["coord"], db["uVec"], db["segLength"], db["bTransGam"], db["forceSum"],
                                db["torqueSum"], d["box"], d["fil"]["counts"])
    S.RigidRodLangevinIntegrationSystem.integrate(db["coord"], db["uVec"], db["yVec"], db["forceSum"],
                                                  db["torqueSum"], db["randForce"], db["randTorque"], db["bTransGam"],
                                                  db["bRotGam"], d["fil"]["params"])
    S.DerivedGeometrySystem.derive(db["coord"], db["uVec"], db["yVec"], db["zVec"], db["end1"], db["end2"],
                                   db["segLength"])
    orc_dm.brownian_force(n, fb["randForce"], fb["randTorque"], fb["bTransGam"], fb["bRotGam"],
                          fb["brownTransScale"], fb["brownRotScale"], f["params"], f["counts"])
    orc_dm.confine(n, fb["coord"], fb["uVec"], fb["segLength"], fb["bTransGam"], fb["forceSum"], fb["torqueSum"],
                   sc["boxParams"], f["counts"])
    orc_dm.integrate(n, fb["coord"], None, fb["uVec"], fb["yVec"], fb["forceSum"], fb["torqueSum"], fb["randForce"],
                     fb["randTorque"], fb["bTransGam"], fb["bRotGam"], f["params"])
    orc_dm.derive(n, fb["coord"], fb["uVec"], fb["yVec"], fb["zVec"], fb["end1"], fb["end2"], fb["segLength"])
    got = host(db)
    for k in ("coord", "uVec", "yVec", "zVec", "end1", "end2", "forceSum", "torqueSum", "randForce", "randTorque"):
        assert_same(fb[k], got[k], k)
    # the fused integDeriveConfined equals confine -> integrate -> derive
    sc2 = _s(warm_scene)
    fb2, f2 = sc2["fil"]["body"], sc2["fil"]
    f2["counts"][1] = 300
    fb2["coord"][:n] *= np.float32(1.2)
    d2 = dev({"fil": f2, "box": sc2["boxParams"]})
    b2 = d2["fil"]["body"]
    S.MechanicsFusion.integDeriveConfined(b2["coord"], b2["uVec"], b2["yVec"], b2["zVec"], b2["segLength"],
                                          b2["end1"], b2["end2"], b2["forceSum"], b2["torqueSum"], b2["randForce"],
                                          b2["randTorque"], b2["bTransGam"], b2["bRotGam"], d2["box"],
                                          d2["fil"]["counts"])
    orc_dm.confine(n, fb2["coord"], fb2["uVec"], fb2["segLength"], fb2["bTransGam"], fb2["forceSum"],
                   fb2["torqueSum"], sc2["boxParams"], f2["counts"])
    orc_dm.integ_derive(n, fb2["coord"], None, fb2["uVec"], fb2["yVec"], fb2["zVec"], fb2["segLength"], fb2["end1"],
                        fb2["end2"], fb2["forceSum"], fb2["torqueSum"], fb2["randForce"], fb2["randTorque"],
                        fb2["bTransGam"], fb2["bRotGam"], f2["params"])
    got2 = host(b2)
    for k in ("coord", "uVec", "yVec", "zVec", "end1", "end2", "forceSum", "torqueSum"):
        assert_same(fb2[k], got2[k], "fused " + k)


def test_drag_kernels_match_oracle(orc_dm):
    from softbox_b200 import systems as S
    f = scenes.deflection_chain(11)
    n = 11
    out = {k: np.zeros(3 * n, np.float32) for k in ("tg", "rg", "td", "rd")}
    out["seg"] = np.zeros(n, np.float32)
    d = dev(out)
    di = dev({k: f[k] for k in ("monomerCount", "end1NbrSlot", "end2NbrSlot")})
    S.DragTensorSystem.run_filament(di["monomerCount"], di["end1NbrSlot"], di["end2NbrSlot"], 0.1, d["seg"], d["tg"],
                                    d["rg"], d["td"], d["rd"])
    orc_dm.drag_run_filament(n, f["monomerCount"], f["end1NbrSlot"], f["end2NbrSlot"], 0.1, out["seg"], out["tg"],
                             out["rg"], out["td"], out["rd"])
    h = host(d)
    for k in out:
        assert_same(out[k], h[k], k)
    nM = 7
    o2 = {k: np.zeros(9 * nM, np.float32) for k in ("tg", "rg", "td", "rd")}
    o2["seg"] = np.zeros(3 * nM, np.float32)
    d2 = dev(o2)
    S.DragTensorSystem.run_motor(nM, 0.1, d2["seg"], d2["tg"], d2["rg"], d2["td"], d2["rd"])
    orc_dm.drag_run_motor(nM, 0.1, o2["seg"], o2["tg"], o2["rg"], o2["td"], o2["rd"])
    h2 = host(d2)
    for k in o2:
        assert_same(o2[k], h2[k], "motor " + k)


def test_thermostat_equipartition():
    """ThermostatDiag Cut 3 (ThermostatDiag.java:41-58): a single rod held to +z by the
    fracMove torsional restore sits at the discrete AR(1) equipartition
    <theta^2> = 4 kT dt / (gamma c (2 - c)), within 2 % (measured 0.992)."""
    from softbox_b200 import systems as S
    reps, dt, coeff = 2000, 1.0e-5, 0.4
    nB = 3 * reps
    b = scenes.rigid_body(nB)
    for mm in range(reps):
        r, lv, hd = 3 * mm, 3 * mm + 1, 3 * mm + 2
        scenes.set_vec(b["uVec"], nB, r, 0, 0, 1); scenes.set_vec(b["yVec"], nB, r, 1, 0, 0)
        scenes.set_vec(b["coord"], nB, lv, 10, 0, 0); scenes.set_vec(b["uVec"], nB, lv, 1, 0, 0)
        scenes.set_vec(b["yVec"], nB, lv, 0, 1, 0)
        scenes.set_vec(b["coord"], nB, hd, 20, 0, 0); scenes.set_vec(b["uVec"], nB, hd, 1, 0, 0)
        scenes.set_vec(b["yVec"], nB, hd, 0, 1, 0)
        b["brownRotScale"][r] = 1.0
        b["segLength"][r] = np.float32(scenes.ROD_LEN)
        scenes.store_drag(b, r, scenes.rod_drag_si(scenes.ROD_LEN, scenes.ROD_R, 0.1))
        scenes.store_drag(b, lv, scenes.rod_drag_si(scenes.LEVER_LEN, scenes.LEVER_R, 0.1))
        scenes.store_drag(b, hd, scenes.sphere_drag_si(scenes.HEAD_R, 0.1))
    params = np.array([dt, np.sqrt(2 * scenes.KT / dt)], np.float32)
    counts = np.array([reps, 0, 0x7E120D, 0], np.int32)
    d = dev({"b": b, "p": params, "c": counts})
    db = d["b"]
    burn, M = 2000, 4000
    s2 = 0.0
    nsamp = 0
    for t in range(burn + M):
        d["c"][1] = t
        S.ChainBendingForceSystem.zeroAccumulators(db["forceSum"], db["torqueSum"])
        S.BrownianForceSystem.brownianForce(db["randForce"], db["randTorque"], db["bTransGam"], db["bRotGam"],
                                            db["brownTransScale"], db["brownRotScale"], d["p"], d["c"])
        S.ThermostatDiag.torsionalRestore(db["uVec"], db["bRotGam"], db["torqueSum"], reps, coeff, dt)
        S.RigidRodLangevinIntegrationSystem.integrate(db["coord"], db["uVec"], db["yVec"], db["forceSum"],
                                                      db["torqueSum"], db["randForce"], db["randTorque"],
                                                      db["bTransGam"], db["bRotGam"], d["p"])
        S.DerivedGeometrySystem.derive(db["coord"], db["uVec"], db["yVec"], db["zVec"], db["end1"], db["end2"],
                                       db["segLength"])
        if t >= burn and t % 4 == 0:
            uz = db["uVec"][2 * nB:][0::3].double().clamp(-1, 1)
            s2 += float((torch.acos(uz) ** 2).sum())
            nsamp += reps
    meas = s2 / nsamp
    bRGy = float(b["bRotGam"][nB + 0])
    pred = 4.0 * scenes.KT * dt / (bRGy * coeff * (2.0 - coeff))
    assert abs(meas / pred - 1.0) < 0.02, (meas, pred)


def test_fused_equals_graph_on_full_network():
    """The full 20,000-rod network: 60 fused steps (one launch) == 60 graph-replayed steps."""
    from softbox_b200.engine import DenseNetwork
    sc = scenes.dense_contractile(scenes.C1)
    a = DenseNetwork(copy.deepcopy(sc))
    b = DenseNetwork(copy.deepcopy(sc))
    assert a.fused_available, "fused path must qualify for the benchmark network"
    a.run(0, 60, mode="fused")
    b.run(0, 60, mode="graph")
    assert a.status() == 0
    torch.cuda.synchronize()
    names = compare_scenes(host(a.dev), host(b.dev))
    assert len(names) > 80


def test_fused_barrier_timeout_reports_and_recovers(warm_scene):
    """Failure detection without a GPU fault: the test hook makes the grid barrier wait for
    an arrival that never comes; the bounded wait runs out, every CTA returns, the run
    reports SBX_ETIMEOUT, and the context and plan stay usable."""
    from softbox_b200.engine import DenseNetwork
    from softbox_b200.runtime import LIB, SbxError
    net = DenseNetwork(copy.deepcopy(warm_scene))
    assert LIB.sbx_dense_plan_test_barrier_extra(net.plan, 1) == 0
    net.run(300, 1, mode="fused")
    with pytest.raises(SbxError) as e:
        net.status()
    assert e.value.code == -4
    assert LIB.sbx_dense_plan_test_barrier_extra(net.plan, 0) == 0
    fresh = DenseNetwork(copy.deepcopy(warm_scene))
    fresh.run(300, 5, mode="fused")
    assert fresh.status() == 0
    ref = DenseNetwork(copy.deepcopy(warm_scene))
    ref.run(300, 5, mode="graph")
    torch.cuda.synchronize()
    compare_scenes(host(ref.dev), host(fresh.dev))


def test_async_download_and_stream_markers():
    """sbx_download_async + sbx_ctx_mark / sbx_ctx_wait_mark: the bytes are on the host once
    the marker recorded after the copy has been passed; invalid slots are refused."""
    import ctypes as C
    from softbox_b200.runtime import Context, LIB
    ctx = Context(0)
    src = torch.arange(4096, dtype=torch.int32, device="cuda")
    dst = [torch.zeros(4096, dtype=torch.int32).pin_memory() for _ in range(2)]
    for k in range(6):
        b = k & 1
        ctx("sbx_memset", C.c_void_p(src.data_ptr()), k, 4 * 4096)
        ctx("sbx_download_async", C.c_void_p(dst[b].data_ptr()), C.c_void_p(src.data_ptr()), 4 * 4096)
        ctx("sbx_ctx_mark", b)
        ctx("sbx_ctx_wait_mark", b)
        want = int.from_bytes(bytes([k]) * 4, "little")
        assert (dst[b].numpy() == want).all()
    assert LIB.sbx_ctx_mark(ctx.h, 8) != 0
    assert LIB.sbx_ctx_wait_mark(ctx.h, 5) != 0          # never recorded


def test_side_copy_and_stream_wait_markers():
    """sbx_download_async_side + sbx_ctx_mark_side / sbx_ctx_stream_wait_mark /
    sbx_ctx_wait_mark: each step's copy runs on the copy stream after the step; the next step
    overwrites the source only after that copy (stream wait on its marker), so every copy
    holds its own step's bytes; sbx_ctx_sync also waits for the copy stream."""
    import ctypes as C
    from softbox_b200.runtime import Context, LIB
    ctx = Context(0)
    assert LIB.sbx_ctx_mark_side(ctx.h, 0) != 0           # no copy stream yet
    assert LIB.sbx_ctx_stream_wait_mark(ctx.h, 3) != 0     # never recorded
    n = 16 << 20                                           # 64 MB: the copy outlasts the memset
    src = torch.zeros(n, dtype=torch.int32, device="cuda")
    dst = [torch.zeros(n, dtype=torch.int32).pin_memory() for _ in range(2)]
    word = lambda k: int.from_bytes(bytes([k]) * 4, "little")
    for k in range(6):
        b = k & 1
        if k > 0:
            ctx("sbx_ctx_stream_wait_mark", 1 - b)         # after step k - 1's copy
        ctx("sbx_memset", C.c_void_p(src.data_ptr()), k + 1, 4 * n)
        ctx("sbx_download_async_side", C.c_void_p(dst[b].data_ptr()), C.c_void_p(src.data_ptr()), 4 * n)
        ctx("sbx_ctx_mark_side", b)
        if k > 0:
            ctx("sbx_ctx_wait_mark", 1 - b)
            v = dst[1 - b].numpy()
            assert v[0] == word(k) and v[-1] == word(k) and (v == word(k)).all()
    ctx("sbx_ctx_sync")
    assert (dst[1].numpy() == word(6)).all()
    assert LIB.sbx_ctx_mark_side(ctx.h, 8) != 0
