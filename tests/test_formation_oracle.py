"""Crosslinker formation in the oracle: the reference's own relational gates.

FORMATION == BRUTE (the grid candidate query equals the all-pairs enumeration,
CrosslinkerSystem.java:405-427 vs :474-595), the allocator's slot stability (an ACTIVE
slot is never overwritten; CrosslinkerHarness.java:799-836), one new link per segment
per step, and saturation/spacing of the admitted links.
"""
import copy

import numpy as np
import pytest

from helpers import oracle_formation, oracle_formation_grid, assert_same
from softbox_b200 import scenes


@pytest.fixture(scope="module")
def bundle():
    return scenes.xlink_bundle(n_fil=160, seed=11, p_form=0.6)


def test_grid_candidates_equal_all_pairs(orc, bundle):
    sc = copy.deepcopy(bundle)
    f, xl = sc["fil"], sc["xl"]
    b = f["body"]
    n, K = b["n"], sc["reqCap"]
    a1, b1 = xl["reqFilA"].copy(), xl["reqFilB"].copy()
    fc1 = xl["formCounts"].copy()
    orc.xl_fil_fil_candidates(n, b["coord"], b["segLength"], sc["filID"], K, a1, b1, xl["formParams"], fc1)
    g = oracle_formation_grid(orc, sc)
    a2, b2 = xl["reqFilA"].copy(), xl["reqFilB"].copy()
    fc2 = xl["formCounts"].copy()
    orc.xl_grid_form_count(n, b["coord"], b["segLength"], sc["filID"], g["gridParams"], g["gridDims"], g["offsets"],
                           g["contents"], g["candCountSeg"], xl["formParams"])
    orc.xl_grid_form_scan(n, g["candCountSeg"], g["candBaseSeg"], K, a2, b2, fc2)
    orc.xl_grid_form_emit(n, b["coord"], b["segLength"], sc["filID"], g["gridParams"], g["gridDims"], g["offsets"],
                          g["contents"], g["candBaseSeg"], g["candCountSeg"], K, a2, b2, xl["formParams"])
    assert fc1[0] > 100
    assert fc1[0] == fc2[0]
    assert_same(a1, a2, "reqFilA")
    assert_same(b1, b2, "reqFilB")
    # lexicographic, distinct filaments, the coarse bound holds
    m = fc1[0]
    key = a1[:m].astype(np.int64) * n + b1[:m]
    assert np.all(np.diff(key) > 0) and np.all(a1[:m] < b1[:m])
    assert np.all(a1[m:] == -1) and np.all(b1[m:] == -1)


def test_formation_steps_allocate_stably(orc, bundle):
    sc = copy.deepcopy(bundle)
    xl = sc["xl"]
    C = sc["C"]
    formed_total = 0
    for step in range(0, 600, 100):
        before_state = xl["linkState"].copy()
        before = {k: xl[k].copy() for k in ("linkFilA", "linkFilB", "loc1", "loc2")}
        oracle_formation(orc, sc, step)
        active_before = before_state >= 0
        for k, v in before.items():          # slot stability
            assert_same(v[active_before], xl[k][active_before], k)
        new = (before_state < 0) & (xl["linkState"] >= 0)
        formed_total += int(new.sum())
        # one new link per segment per step, admitted links respect saturation
        segs = np.concatenate([xl["linkFilA"][new], xl["linkFilB"][new]])
        assert segs.size == np.unique(segs).size
        counts = np.bincount(np.concatenate([xl["linkFilA"][xl["linkState"] >= 0],
                                             xl["linkFilB"][xl["linkState"] >= 0]]), minlength=sc["fil"]["body"]["n"])
        assert counts.max() <= scenes.XL_MAX_LINKS_ON_SEG
        # the formed links carry fresh rings and the formation orientation
        assert np.all(xl["strainHist"].reshape(C, -1)[new] == 0) and np.all(xl["strainPlace"][new] == 0)
    assert formed_total >= 5
