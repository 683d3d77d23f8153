"""The reference harnesses' physics gates on the CUDA library: each sequence of
tests/physics_gates.py runs through the library's entry points and must (1) give the
oracle's bits and (2) pass the gate itself. Plus the reach-list capacity gate of the fused
step: a head whose candidate count passes SBX_MAX_CAND keeps counting past the cap
(SpatialGrid.java:395-398) and the run reports SBX_EOVERFLOW."""
import copy

import numpy as np
import pytest

import physics_gates as G
from helpers import assert_same

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.mark.parametrize("force", [0.0, 2.0e-12])
def test_motor_off_rate_gate_gpu(orc_dm, force):
    host = G.release_bed(force=force)
    ref = copy.deepcopy(host)
    G.run_release(G.OracleBackend(orc_dm), ref, 3000)
    be = G.GpuBackend()
    m = be.put(host)
    G.run_release(be, m, 3000)
    for k in ("boundSeg", "cooldown", "stats"):
        assert_same(ref[k], be.get(m[k]), k)
    p, want, se = G.off_rate(be.get(m["stats"]), force)
    assert abs(p - want) / want < 0.05 and abs(p - want) < 5 * se, (p, want, se)


def test_confined_rod_equipartition_gate_gpu(orc_dm):
    sc = G.confined_rods(reps=2000)
    ref = copy.deepcopy(sc)
    want = G.run_equipartition(G.OracleBackend(orc_dm), ref, burn=4000, steps=8000, every=2)
    be = G.GpuBackend()
    d = dict(sc)
    d["b"], d["params"], d["counts"] = be.put(sc["b"]), be.put(sc["params"]), be.put(sc["counts"])
    got = G.run_equipartition(be, d, burn=4000, steps=8000, every=2)
    assert got == want
    assert_same(ref["b"]["uVec"], be.get(d["b"]["uVec"]), "uVec")
    assert abs(got[0] / got[1] - 1.0) < 0.02, got[0] / got[1]


def test_crosslinker_rest_hold_gate_gpu(orc_dm):
    want = G.rest_hold(G.OracleBackend(orc_dm))
    got = G.rest_hold(G.GpuBackend())
    assert got == want
    drift, rel, sep0, sep_end = got
    assert drift == 0.0
    assert rel < 1e-3 and sep_end < sep0 and sep_end > 0.9 * G.XL_REST


def test_crosslinker_stretch_relaxation_gate_gpu(orc_dm):
    be = G.GpuBackend()
    for dt in (1.0e-5, 1.0e-6):
        assert G.stretch_decay(be, dt) == G.stretch_decay(G.OracleBackend(orc_dm), dt)
    k_obs, k_pred, _ = G.stretch_decay(be, 1.0e-5)
    k10, _, _ = G.stretch_decay(be, 1.0e-6)
    assert abs(k_obs - k_pred) / k_pred < 1e-3 and abs(k_obs - k10) / k_obs < 1e-3


def test_fused_reach_list_past_cap_reports_overflow(orc_dm):
    """A crowded small network: every head sits among more than SBX_MAX_CAND reachable
    segments. The fused step counts past the cap like the reference (reachCount > 256, the
    stored slice holds the first 256 in walk order), binds like the oracle, and the run
    reports SBX_EOVERFLOW."""
    from helpers import oracle_dense_run
    from softbox_b200 import device as D
    from softbox_b200.engine import DenseNetwork
    from softbox_b200.runtime import SbxError
    sc = G.crowded_dense()
    ref = copy.deepcopy(sc)
    oracle_dense_run(orc_dm, ref, 0, 3)
    assert ref["grid"]["reachCount"].max() > 256
    net = DenseNetwork(copy.deepcopy(sc))
    assert net.fused_available, net
    net.run(0, 3, mode="fused")
    with pytest.raises(SbxError) as e:
        net.status()
    assert e.value.code == -3
    torch.cuda.synchronize()
    got = D.to_host(net.dev)
    for s, f in (("grid", "reachCount"), ("grid", "reachSeg"), ("mot", "boundSeg"), ("mot", "bindArc")):
        assert_same(ref[s][f], got[s][f], f"{s}.{f}")
    assert_same(ref["fil"]["body"]["coord"], got["fil"]["body"]["coord"], "fil.coord")
    assert net.fused_stats()["reach_over_cap"] > 0


def test_deflection_support_matches_oracle(orc_dm):
    """DeflectionSupport.seedAccumulators / pinEndpoints (the deflection benchmark's load and
    pins) on the GPU equal the oracle bit for bit, load on and off."""
    from softbox_b200 import device as D, scenes
    from softbox_b200.systems import DeflectionSupport
    rng = np.random.default_rng(5)
    n, P = 257, 9
    host = {"F": rng.standard_normal(3 * n).astype(np.float32), "T": rng.standard_normal(3 * n).astype(np.float32),
            "ext": rng.standard_normal(3 * n).astype(np.float32) * 1e-12, "c": np.array([n, 3, 0, 1], np.int32),
            "coord": rng.standard_normal(3 * n).astype(np.float32), "seg": rng.uniform(0.05, 0.2, n).astype(np.float32),
            "pinSeg": rng.choice(n, P, replace=False).astype(np.int32), "pinEnd": rng.integers(1, 3, P).astype(np.int32),
            "anchor": rng.standard_normal(3 * P).astype(np.float32)}
    u = rng.standard_normal((3, n))
    host["u"] = (u / np.linalg.norm(u, axis=0)).reshape(-1).astype(np.float32)
    for load in (1, 0):
        host["c"][3] = load
        ref = copy.deepcopy(host)
        d = D.to_device(host)
        DeflectionSupport.seedAccumulators(d["F"], d["T"], d["ext"], d["c"])
        DeflectionSupport.pinEndpoints(d["coord"], d["u"], d["seg"], d["pinSeg"], d["pinEnd"], d["anchor"])
        orc_dm.seed_accumulators(n, ref["F"], ref["T"], ref["ext"], ref["c"])
        orc_dm.pin_endpoints(n, ref["coord"], ref["u"], ref["seg"], P, ref["pinSeg"], ref["pinEnd"], ref["anchor"])
        h = D.to_host(d)
        for k in ("F", "T", "coord"):
            assert_same(ref[k], h[k], k)
