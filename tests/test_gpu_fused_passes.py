"""The fused passes of the dense step against the separate reference calls, bit for bit:

* sbx_csr_build_payload: offsets and lists equal the serial CSR build, and each row's
  payload copy equals the listed items' payload (zeros where the guard is negative);
* sbx_fusion_chain_gathers over those copies: the accumulators equal the oracle's
  chainForces followed by segGatherA, segGatherB and the cross-bridge segGather
  (ChainBendingForceSystem.java:105-331, CrosslinkerSystem.java:129-173,
  CrossBridgeSystem.java:302-320), with -0.0 accumulators and with the crosslinker
  gathers skipped;
* sbx_grid_cell_endpoints + sbx_fusion_grid_reachable (the reach walk over cell-ordered
  endpoints): reach lists and counts equal the oracle's gridReachable
  (BindingDetectionSystem.java:143-228).
"""
import copy

import numpy as np
import pytest

from helpers import assert_same, oracle_dense_run, small_dense
from softbox_b200 import device as D, scenes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

XL_STRIDE, XB_STRIDE = 12, 13


@pytest.fixture(scope="module")
def warm(orc_dm):
    sc = small_dense(0.05)
    oracle_dense_run(orc_dm, sc, 0, 300)
    assert (sc["mot"]["boundSeg"] >= 0).sum() > 5
    return sc


def _ctx():
    from softbox_b200.systems import _ctx as c
    return c()


def _oracle_csr(orc_dm, keys, n_items, n_rows):
    cnt, off, lst = np.zeros(n_rows, np.int32), np.zeros(n_rows + 1, np.int32), np.zeros(max(n_items, 1), np.int32)
    orc_dm.csr_histogram(keys, n_items, n_rows, cnt)
    orc_dm.csr_scan(n_rows, cnt, off)
    orc_dm.csr_scatter(keys, n_items, off, cnt, lst)
    return cnt, off, lst[:n_items]


def _payload_csr(keys, n_rows, payload, stride, offset, guard):
    n = keys.size
    dk = D.to_device(keys)
    cnt = torch.zeros(n_rows, dtype=torch.int32, device="cuda")
    off = torch.zeros(n_rows + 1, dtype=torch.int32, device="cuda")
    lst = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    rowp = torch.zeros(6 * max(n, 1), dtype=torch.float32, device="cuda")
    _ctx()("sbx_csr_build_payload", dk, n, n_rows, cnt, off, lst, D.to_device(payload), stride, offset,
           None if guard is None else D.to_device(guard), rowp)
    return off, lst, rowp


@pytest.mark.parametrize("offset,guarded", [(0, True), (6, True), (6, False)])
def test_csr_build_payload_rows(orc_dm, offset, guarded):
    rng = np.random.default_rng(5 + offset)
    n_rows, n_items = 3001, 7000
    keys = rng.integers(-1, n_rows, n_items).astype(np.int32)
    keys[:40] = 17                                           # one long row
    payload = rng.normal(size=n_items * XL_STRIDE).astype(np.float32)
    guard = rng.integers(-2, 3, n_items).astype(np.int32) if guarded else None
    off, lst, rowp = _payload_csr(keys, n_rows, payload, XL_STRIDE, offset, guard)
    torch.cuda.synchronize()
    _, r_off, r_lst = _oracle_csr(orc_dm, keys, n_items, n_rows)
    assert_same(r_off, D.to_host(off), "offsets")
    total = int(r_off[-1])
    assert_same(r_lst[:total], D.to_host(lst)[:total], "list")
    want = payload.reshape(n_items, XL_STRIDE)[r_lst[:total], offset:offset + 6].copy()
    if guarded:
        want[guard[r_lst[:total]] < 0] = 0.0
    assert_same(want.reshape(-1), D.to_host(rowp)[:6 * total], "row payload")


@pytest.mark.parametrize("xl_on", [True, False])
@pytest.mark.parametrize("neg_zero", [False, True])
def test_chain_gathers_equal_chain_then_gathers(orc_dm, warm, xl_on, neg_zero):
    sc = copy.deepcopy(warm)
    f, fb, m, xl = sc["fil"], sc["fil"]["body"], sc["mot"], sc["xl"]
    nSeg, nM, nL = fb["n"], m["nMotors"], xl["nLinks"]
    rng = np.random.default_rng(3)
    fb["forceSum"][:] = rng.normal(scale=1e-12, size=fb["forceSum"].shape).astype(np.float32)
    fb["torqueSum"][:] = rng.normal(scale=1e-20, size=fb["torqueSum"].shape).astype(np.float32)
    if neg_zero:                                             # accumulators that the sums must not flip
        fb["forceSum"][::7] = np.float32(-0.0)
        fb["torqueSum"][::5] = np.float32(-0.0)
    d = D.to_device({"fil": f, "xl": xl, "mot": m, "bondData": sc["bondData"]})
    df, dfb, dxl, dmo = d["fil"], d["fil"]["body"], d["xl"], d["mot"]

    # reference: oracle chain, then the three gathers over the oracle's CSRs
    orc_dm.chain_forces(nSeg, fb["coord"], fb["uVec"], fb["segLength"], f["end2NbrSlot"], f["end2NbrSide"],
                        f["end1NbrSlot"], f["end1NbrSide"], fb["bTransGam"], fb["bRotGam"], fb["forceSum"],
                        fb["torqueSum"], f["chainParams"])
    if xl_on:
        for side, key in ((0, "linkFilA"), (1, "linkFilB")):
            _, off, lst = _oracle_csr(orc_dm, xl[key], nL, nSeg)
            (orc_dm.seg_gather_a if side == 0 else orc_dm.seg_gather_b)(nSeg, off, lst, xl["xlinkData"],
                                                                        xl["linkState"], fb["forceSum"],
                                                                        fb["torqueSum"])
    _, off, lst = _oracle_csr(orc_dm, m["boundSeg"], nM, nSeg)
    orc_dm.seg_gather(nSeg, off, lst, sc["bondData"], fb["forceSum"], fb["torqueSum"])

    # fused pass over the row-ordered payload copies
    oA = pA = oB = pB = None
    if xl_on:
        oA, _, pA = _payload_csr(xl["linkFilA"], nSeg, xl["xlinkData"], XL_STRIDE, 0, xl["linkState"])
        oB, _, pB = _payload_csr(xl["linkFilB"], nSeg, xl["xlinkData"], XL_STRIDE, 6, xl["linkState"])
    oM, _, pM = _payload_csr(m["boundSeg"], nSeg, sc["bondData"], XB_STRIDE, 6, None)
    _ctx()("sbx_fusion_chain_gathers", nSeg, dfb["coord"], dfb["uVec"], dfb["segLength"], df["end2NbrSlot"],
           df["end2NbrSide"], df["end1NbrSlot"], df["end1NbrSide"], dfb["bTransGam"], dfb["bRotGam"],
           dfb["forceSum"], dfb["torqueSum"], df["chainParams"], oA, pA, oB, pB, oM, pM)
    torch.cuda.synchronize()
    assert_same(fb["forceSum"], D.to_host(dfb["forceSum"]), "forceSum")
    assert_same(fb["torqueSum"], D.to_host(dfb["torqueSum"]), "torqueSum")
    assert (xl["linkState"] < 0).any() and (xl["linkState"] >= 0).any()


def test_cell_endpoint_walk_equals_grid_reachable(orc_dm, warm):
    sc = copy.deepcopy(warm)
    m, g, fb = sc["mot"], sc["grid"], sc["fil"]["body"]
    nM, nSeg, cap = m["nMotors"], fb["n"], int(g["cap"])
    d = D.to_device({"m": m, "g": g, "e1": fb["end1"], "e2": fb["end2"]})
    dm, dg = d["m"], d["g"]
    orc_dm.grid_reachable(nM, m["head"], m["uVec"], m["rodUVec"], nSeg, fb["end1"], fb["end2"], g["gridParams"],
                          g["gridDims"], g["gridCellOffsets"], g["gridCellContents"], g["ownerStore"],
                          g["ownerSlot"], g["reachSeg"], g["reachCount"], m["kinParams"])
    ce1 = torch.zeros(4 * cap, dtype=torch.float32, device="cuda")
    ce2 = torch.zeros(4 * cap, dtype=torch.float32, device="cuda")
    dg["reachSeg"].fill_(-7)
    dg["reachCount"].fill_(-7)
    c = _ctx()
    c("sbx_grid_cell_endpoints", cap, int(g["totalCells"]), dg["gridCellOffsets"], dg["gridCellContents"],
      dg["ownerStore"], dg["ownerSlot"], nSeg, d["e1"], d["e2"], ce1, ce2)
    c("sbx_fusion_grid_reachable", dm["head"], dm["uVec"], dm["rodUVec"], dg["gridParams"], dg["gridDims"],
      dg["gridCellOffsets"], ce1, ce2, dg["reachSeg"], dg["reachCount"], dm["kinParams"], nM)
    torch.cuda.synchronize()
    hc = D.to_host(dg["reachCount"])
    assert_same(g["reachCount"], hc, "reachCount")
    hs = D.to_host(dg["reachSeg"]).reshape(nM, -1)
    want = g["reachSeg"].reshape(nM, -1)
    for i in range(nM):
        k = min(int(hc[i]), want.shape[1])
        assert_same(want[i, :k], hs[i, :k], f"reachSeg row {i}")
    assert hc.sum() > 0


def test_staged_tile_walk_equals_grid_reachable(orc_dm, warm):
    """sbx_fusion_grid_reachable_staged (one block per tile of cells, the neighbourhood staged in
    shared memory by bulk copies) gives the oracle's reach lists and counts."""
    sc = copy.deepcopy(warm)
    m, g, fb = sc["mot"], sc["grid"], sc["fil"]["body"]
    nM, nSeg, cap = m["nMotors"], fb["n"], int(g["cap"])
    d = D.to_device({"m": m, "g": g, "e1": fb["end1"], "e2": fb["end2"]})
    dm, dg = d["m"], d["g"]
    orc_dm.grid_reachable(nM, m["head"], m["uVec"], m["rodUVec"], nSeg, fb["end1"], fb["end2"], g["gridParams"],
                          g["gridDims"], g["gridCellOffsets"], g["gridCellContents"], g["ownerStore"],
                          g["ownerSlot"], g["reachSeg"], g["reachCount"], m["kinParams"])
    ce1 = torch.zeros(4 * cap, dtype=torch.float32, device="cuda")
    ce2 = torch.zeros(4 * cap, dtype=torch.float32, device="cuda")
    dg["reachSeg"].fill_(-7)
    dg["reachCount"].fill_(-7)
    c = _ctx()
    c("sbx_grid_cell_endpoints", cap, int(g["totalCells"]), dg["gridCellOffsets"], dg["gridCellContents"],
      dg["ownerStore"], dg["ownerSlot"], nSeg, d["e1"], d["e2"], ce1, ce2)
    nX, nY, nZ = (int(v) for v in g["gridDims"][:3])
    c("sbx_fusion_grid_reachable_staged", dm["head"], dm["uVec"], dm["rodUVec"], dg["gridParams"], dg["gridDims"],
      nX, nY, nZ, dg["gridCellOffsets"], dg["gridCellContents"], dg["ownerStore"], dg["ownerSlot"], dg["bodyCell"],
      cap, dm["publishParams"], ce1, ce2, dg["reachSeg"], dg["reachCount"], dm["kinParams"], nM)
    c.sync()
    hc = D.to_host(dg["reachCount"])
    assert_same(g["reachCount"], hc, "reachCount")
    hs = D.to_host(dg["reachSeg"]).reshape(nM, -1)
    want = g["reachSeg"].reshape(nM, -1)
    for i in range(nM):
        k = min(int(hc[i]), want.shape[1])
        assert_same(want[i, :k], hs[i, :k], f"reachSeg row {i}")
    assert hc.sum() > 0


def test_staged_tile_walk_at_scale_equals_plain_walk():
    """200,000 rods (about 18,000 tiles) after one step: the staged-tile walk and the per-head
    walk over the same grid and endpoints give the same reach lists and counts."""
    from softbox_b200.engine import DenseNetwork
    sc = scenes.dense_contractile(scenes.dense_scaled(200000))
    net = DenseNetwork(sc)
    net.run(0, 1, mode="graph")
    assert net.status() == 0
    d = net.dev
    m, g, fb = d["mot"], d["grid"], d["fil"]["body"]
    nM, nSeg, cap = sc["mot"]["nMotors"], sc["fil"]["body"]["n"], int(sc["grid"]["cap"])
    nX, nY, nZ = (int(v) for v in sc["grid"]["gridDims"][:3])
    ce1 = torch.zeros(4 * cap, dtype=torch.float32, device="cuda")
    ce2 = torch.zeros(4 * cap, dtype=torch.float32, device="cuda")
    c = net.ctx
    c("sbx_grid_cell_endpoints", cap, int(sc["grid"]["totalCells"]), g["gridCellOffsets"], g["gridCellContents"],
      g["ownerStore"], g["ownerSlot"], nSeg, fb["end1"], fb["end2"], ce1, ce2)
    out = []
    for staged in (False, True):
        seg = torch.full((nM * 256,), -7, dtype=torch.int32, device="cuda")
        cnt = torch.full((nM,), -7, dtype=torch.int32, device="cuda")
        if staged:
            c("sbx_fusion_grid_reachable_staged", m["head"], m["uVec"], m["rodUVec"], g["gridParams"], g["gridDims"],
              nX, nY, nZ, g["gridCellOffsets"], g["gridCellContents"], g["ownerStore"], g["ownerSlot"],
              g["bodyCell"], cap, m["publishParams"], ce1, ce2, seg, cnt, m["kinParams"], nM)
        else:
            c("sbx_fusion_grid_reachable", m["head"], m["uVec"], m["rodUVec"], g["gridParams"], g["gridDims"],
              g["gridCellOffsets"], ce1, ce2, seg, cnt, m["kinParams"], nM)
        c.sync()
        out.append((cnt.cpu().numpy(), seg.cpu().numpy().reshape(nM, 256)))
    (c0, s0), (c1, s1) = out
    assert_same(c0, c1, "reachCount")
    assert c0.sum() > 0
    filled = np.arange(256)[None, :] < np.minimum(c0, 256)[:, None]
    assert_same(s0[filled], s1[filled], "reachSeg")
