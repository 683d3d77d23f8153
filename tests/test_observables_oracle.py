"""Observable restatements (CPU): the oracle's deterministic FP64 order against the
reference's serial sums, and its cluster labelling against an independent graph library."""
import math

import numpy as np
import pytest

from helpers import oracle_dense_run, oracle_observables, small_dense
from softbox_b200.observables import contraction_rate, motor_backbones


@pytest.fixture(scope="module")
def mid_run(orc):
    sc = small_dense(0.05)
    oracle_dense_run(orc, sc, 0, 200)
    sc["fil"]["filState"][[3, 17, 250]] = -1          # FREE slots are left out
    return sc


def test_extent_matches_serial_fil_rms(orc, mid_run):
    ext, _, _, _ = oracle_observables(orc, mid_run)
    f = mid_run["fil"]
    n = f["body"]["n"]
    c = f["body"]["coord"].reshape(3, n).astype(np.float64)
    act = f["filState"] >= 0
    cx, cy, cz, cnt = 0.0, 0.0, 0.0, 0          # FullSystemDemoHarness.filRms, serial
    for i in np.flatnonzero(act):
        cx += c[0, i]; cy += c[1, i]; cz += c[2, i]; cnt += 1
    cx /= cnt; cy /= cnt; cz /= cnt
    s2 = 0.0
    for i in np.flatnonzero(act):
        dx, dy, dz = c[0, i] - cx, c[1, i] - cy, c[2, i] - cz
        s2 += dx * dx + dy * dy + dz * dz
    want = math.sqrt(s2 / cnt)
    assert ext[0, 1] == cnt
    assert abs(ext[0, 0] - want) <= 1e-12 * want


def test_clusters_match_connected_components(orc, mid_run):
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    sc = mid_run
    _, _, cl, label = oracle_observables(orc, sc)
    f, xl, mot = sc["fil"], sc["xl"], sc["mot"]
    nS, nBb = f["body"]["n"], sc["mini"]["nBackbones"]
    live = np.concatenate([f["filState"] >= 0, np.ones(nBb, bool)])
    e = []
    for s in range(nS):
        t = f["end2NbrSlot"][s]
        if t >= 0 and live[s] and live[t]:
            e.append((s, t))
    for k in range(xl["nLinks"]):
        a, b = xl["linkFilA"][k], xl["linkFilB"][k]
        if xl["linkState"][k] >= 0 and live[a] and live[b]:
            e.append((a, b))
    mb = motor_backbones(sc["dim"], sc["mini"], mot["nMotors"])
    for m in range(mot["nMotors"]):
        s = mot["boundSeg"][m]
        if s >= 0 and mb[m] >= 0 and live[s]:
            e.append((s, nS + mb[m]))
    assert len(e) > nS // 2 and any(u >= nS or v >= nS for u, v in e)
    e = np.array(e)
    g = coo_matrix((np.ones(len(e)), (e[:, 0], e[:, 1])), shape=(nS + nBb, nS + nBb))
    _, comp = connected_components(g, directed=False)
    sizes = np.bincount(comp[:nS][live[:nS]])
    assert cl[0, 0] == sizes.max() and cl[0, 1] == live[:nS].sum()
    # same partition, labelled by the smallest member
    for c in np.unique(comp[:nS][live[:nS]]):
        members = np.flatnonzero((comp == c) & live)
        assert (label[members] == members.min()).all()
    assert (label[:nS][~live[:nS]] == -1).all()


def test_stress_matches_vectorised_virial(orc, mid_run):
    sc = mid_run
    _, st, _, _ = oracle_observables(orc, sc)
    f, xl, mot = sc["fil"], sc["xl"], sc["mot"]
    n = f["body"]["n"]
    e1 = f["body"]["end1"].reshape(3, n).astype(np.float64)
    u = f["body"]["uVec"].reshape(3, n).astype(np.float64)
    act = xl["linkState"] >= 0
    a, b = xl["linkFilA"][act], xl["linkFilB"][act]
    p1 = e1[:, a] + xl["loc1"][act].astype(np.float64) * u[:, a]
    p2 = e1[:, b] + xl["loc2"][act].astype(np.float64) * u[:, b]
    F = xl["xlinkData"].reshape(-1, 12)[act, :3].astype(np.float64).T
    w = (1e-6 * (p1 - p2)[:2] * F[:2]).sum()
    nM = mot["nMotors"]
    nB = 3 * nM
    bs = mot["boundSeg"]
    mm = np.flatnonzero(bs >= 0)
    h = 3 * mm + 2
    mc = mot["body"]["coord"].reshape(3, nB).astype(np.float64)
    mu = mot["body"]["uVec"].reshape(3, nB).astype(np.float64)
    tip = mc[:, h] + 0.5 * 0.020 * mu[:, h]
    s = bs[mm]
    c = f["body"]["coord"].reshape(3, n).astype(np.float64)
    off = mot["bindArc"][mm].astype(np.float64) - 0.5 * f["body"]["segLength"][s].astype(np.float64)
    ap = c[:, s] + off * u[:, s]
    Fh = sc["bondData"].reshape(-1, 13)[mm, :3].astype(np.float64).T
    w += (1e-6 * (tip - ap)[:2] * Fh[:2]).sum()
    bx = sc["boxParams"]
    vol = float(np.float32(bx[1] * bx[2] * bx[3]))
    want = -w / (2.0 * vol * 1e-18)
    assert act.sum() > 0 and mm.size > 0
    assert abs(st[0] - want) <= 1e-9 * abs(want)


def test_contraction_rate_fit():
    t = np.linspace(0, 2.0, 21)
    assert abs(contraction_rate(t, 3.0 * np.exp(-0.15 * t)) - 0.15) < 1e-12
