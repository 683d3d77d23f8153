"""GPU crosslinker formation and allocator against the oracle, bit for bit.

Scene: a dense bundle of single-segment filaments (the bundle harness's composition) taken
through a few oracle formation steps so that the link pool holds ACTIVE links; then each
formation entry point, and whole formation steps (CrosslinkerBundleHarness.formationCpu
order), are compared with the oracle on identical inputs.
"""
import copy

import numpy as np
import pytest

from helpers import assert_same, oracle_formation, oracle_formation_grid
from softbox_b200 import device as D, scenes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def seeded(orc_dm):
    sc = scenes.xlink_bundle(n_fil=160, seed=11, p_form=0.6)
    for step in (0, 100):
        oracle_formation(orc_dm, sc, step)
    assert (sc["xl"]["linkState"] >= 0).sum() > 0
    return sc


def _dev(sc):
    d = D.to_device({"fil": sc["fil"], "xl": sc["xl"]})
    d["filID"] = torch.from_numpy(sc["filID"]).cuda()
    return d


def _fgrid(sc):
    from softbox_b200.systems import FormationGrid
    g = sc["grid"]
    return FormationGrid(sc["fil"]["body"]["n"], g["half"], g["half"], g["half"], g["cell"], g["grab"], g["radius"])


def gpu_formation(d, fg, step, use_grid=True):
    from softbox_b200.systems import CrosslinkerSystem as X, _ctx
    f, xl = d["fil"], d["xl"]
    b = f["body"]
    C, K = xl["linkState"].numel(), xl["reqFilA"].numel()
    xl["formCounts"][1] = step
    X.countActiveLinks(xl["linkState"], xl["linkFilA"], xl["linkFilB"], xl["activeLinkCount"])
    if use_grid:
        fg.build(b["coord"], b["segLength"])
        fg.formCandidates(b["coord"], b["segLength"], d["filID"], xl["reqFilA"], xl["reqFilB"], xl["formParams"],
                          xl["formCounts"])
    else:
        X.filFilCandidates(b["coord"], b["segLength"], d["filID"], xl["reqFilA"], xl["reqFilB"], xl["formParams"],
                           xl["formCounts"])
    X.formGates(b["uVec"], b["end1"], b["end2"], b["segLength"], xl["reqFilA"], xl["reqFilB"], xl["reqLoc1"],
                xl["reqLoc2"], xl["reqOrient"], xl["gatePass"], xl["formParams"], xl["formCounts"])
    X.formAdmitReduce(xl["reqFilA"], xl["reqFilB"], xl["gatePass"], xl["minCand"])
    X.formAdmit(xl["reqFilA"], xl["reqFilB"], xl["reqLoc1"], xl["reqLoc2"], xl["gatePass"], xl["minCand"],
                xl["activeLinkCount"], xl["linkState"], xl["linkFilA"], xl["linkFilB"], xl["loc1"], xl["loc2"],
                xl["acceptFlag"], xl["formParams"])
    X.freeFlags(xl["linkState"], xl["freeCount"])
    _ctx()("sbx_csr_scan", C, xl["freeCount"], xl["freeOffsets"])
    X.freeScatter(xl["linkState"], xl["freeOffsets"], xl["freeList"])
    _ctx()("sbx_csr_scan", K, xl["acceptFlag"], xl["rankOffsets"])
    X.allocate(xl["reqFilA"], xl["reqFilB"], xl["reqLoc1"], xl["reqLoc2"], xl["rankOffsets"], xl["freeList"],
               xl["freeOffsets"], xl["linkFilA"], xl["linkFilB"], xl["loc1"], xl["loc2"], xl["linkState"],
               xl["strainHist"], xl["strainPlace"])
    X.placeOrient(xl["reqOrient"], xl["rankOffsets"], xl["freeList"], xl["freeOffsets"], xl["linkOrientSame"],
                  xl["torqueMagHist"], xl["torqueMagPlace"])


def _compare_xl(host_xl, dev_xl):
    for k, v in host_xl.items():
        if isinstance(v, np.ndarray):
            assert_same(v, dev_xl[k].cpu().numpy(), "xl." + k)


@pytest.mark.parametrize("use_grid", [True, False])
def test_formation_step_bitwise(orc_dm, seeded, use_grid):
    sc = copy.deepcopy(seeded)
    d = _dev(sc)
    fg = _fgrid(sc)
    for step in (200, 300, 400):
        oracle_formation(orc_dm, sc, step, use_grid=use_grid)
        gpu_formation(d, fg, step, use_grid=use_grid)
        torch.cuda.synchronize()
        _compare_xl(sc["xl"], d["xl"])
    assert (sc["xl"]["linkState"] >= 0).sum() > (seeded["xl"]["linkState"] >= 0).sum()


def test_formation_grid_and_candidates(orc_dm, seeded):
    sc = copy.deepcopy(seeded)
    d = _dev(sc)
    fg = _fgrid(sc)
    b = d["fil"]["body"]
    fg.build(b["coord"], b["segLength"])
    g = oracle_formation_grid(orc_dm, sc)
    torch.cuda.synchronize()
    for k_dev, k_host in (("bodyCell", "bodyCell"), ("gridCellOffsets", "offsets"), ("gridCellContents", "contents"),
                          ("cellCount", "cellCount"), ("chunkSum", "chunkSum"), ("center", "center")):
        assert_same(g[k_host], getattr(fg, k_dev).cpu().numpy(), "formation grid " + k_host)
    xl = d["xl"]
    fg.formCandidates(b["coord"], b["segLength"], d["filID"], xl["reqFilA"], xl["reqFilB"], xl["formParams"],
                      xl["formCounts"])
    hx = sc["xl"]
    n, K = sc["fil"]["body"]["n"], sc["reqCap"]
    fb = sc["fil"]["body"]
    orc_dm.xl_fil_fil_candidates(n, fb["coord"], fb["segLength"], sc["filID"], K, hx["reqFilA"], hx["reqFilB"],
                                 hx["formParams"], hx["formCounts"])
    torch.cuda.synchronize()
    assert_same(hx["reqFilA"], xl["reqFilA"].cpu().numpy(), "grid reqFilA == all-pairs")
    assert_same(hx["reqFilB"], xl["reqFilB"].cpu().numpy(), "grid reqFilB == all-pairs")
    assert_same(hx["formCounts"][:1], xl["formCounts"][:1].cpu().numpy(), "nCand")
    assert hx["formCounts"][0] > 100


def test_allocator_overflow_clamp(orc_dm, seeded):
    """More accepted requests than free slots: the lowest nFree ranks form, the rest do not."""
    sc = copy.deepcopy(seeded)
    xl = sc["xl"]
    K, C = sc["reqCap"], sc["C"]
    rng = np.random.default_rng(3)
    xl["linkState"][:] = 0
    free = rng.choice(C, 5, replace=False)
    xl["linkState"][free] = -1
    acc = np.zeros(K, np.int32)
    acc[rng.choice(200, 12, replace=False)] = 1
    xl["reqFilA"][:200] = rng.integers(0, 160, 200)
    xl["reqFilB"][:200] = rng.integers(0, 160, 200)
    d = _dev(sc)
    from softbox_b200.systems import CrosslinkerSystem as X, _ctx
    dx = d["xl"]
    dx["acceptFlag"].copy_(torch.from_numpy(acc).cuda())
    X.freeFlags(dx["linkState"], dx["freeCount"])
    _ctx()("sbx_csr_scan", C, dx["freeCount"], dx["freeOffsets"])
    X.freeScatter(dx["linkState"], dx["freeOffsets"], dx["freeList"])
    _ctx()("sbx_csr_scan", K, dx["acceptFlag"], dx["rankOffsets"])
    X.allocate(dx["reqFilA"], dx["reqFilB"], dx["reqLoc1"], dx["reqLoc2"], dx["rankOffsets"], dx["freeList"],
               dx["freeOffsets"], dx["linkFilA"], dx["linkFilB"], dx["loc1"], dx["loc2"], dx["linkState"],
               dx["strainHist"], dx["strainPlace"])
    xl["acceptFlag"][:] = acc
    orc_dm.xl_free_flags(C, xl["linkState"], xl["freeCount"])
    orc_dm.csr_scan(C, xl["freeCount"], xl["freeOffsets"])
    orc_dm.xl_free_scatter(C, xl["linkState"], xl["freeOffsets"], xl["freeList"])
    orc_dm.csr_scan(K, xl["acceptFlag"], xl["rankOffsets"])
    orc_dm.xl_allocate(K, xl["reqFilA"], xl["reqFilB"], xl["reqLoc1"], xl["reqLoc2"], xl["rankOffsets"],
                       xl["freeList"], xl["freeOffsets"], C, xl["linkFilA"], xl["linkFilB"], xl["loc1"], xl["loc2"],
                       xl["linkState"], xl["strainHist"], xl["strainPlace"])
    torch.cuda.synchronize()
    for k in ("freeCount", "freeOffsets", "freeList", "acceptFlag", "rankOffsets", "linkFilA", "linkFilB",
              "linkState", "strainHist", "strainPlace"):
        assert_same(xl[k], dx[k].cpu().numpy(), k)
    assert (xl["linkState"] >= 0).all()          # all 5 free slots claimed, 7 requests clamped
    assert xl["freeOffsets"][C] == 5 and xl["rankOffsets"][K] == 12
