"""Precision statement: the FP32 arithmetic of the kernels against an FP64 build of the same
algorithm (oracle/liboracle_f64.so: the oracle's restatement with every float evaluated as
double). The CUDA kernels equal the FP32 oracle bit for bit (tests/test_gpu_*), so these
differences are the kernels' FP32 error. Bounds are stated with measured values:

  free rods (1,024 rods of 1 um, 1,000 steps, Wang noise): centres 2.9e-5 um (FP32
  centres), orientations 7.5e-6; the FP64-centre option of the kernels cuts the centre error;
  diffusion coefficients from the per-step body-frame displacements differ by < 1e-5 relative;
  dense contractile network (20,000 rods, 1,000 steps after 1,000, supplied noise): rod
  centres median 1.3e-6 um, 99th percentile 7.2e-6 um, largest 3.2e-4 um; rod orientations
  median 1.9e-6, 99th percentile 1.6e-5, largest 1.6e-3; myosin sub-bodies (short and stiffly
  jointed, so they amplify rounding) centres median 1.2e-6 um, 99th percentile 3.0e-5 um,
  orientations median 2.2e-5, 99th percentile 7.1e-4; one binding event of 6,400 heads differs
  at the end (a decision whose inputs sit within rounding of its threshold; the bodies it
  touches carry the largest differences, up to a different lever pose);
  confined-rod equipartition ratio: the same to 1e-4.
"""
import copy

import numpy as np
import pytest

import oracle
import physics_gates as G
from softbox_b200 import device as D, scenes


@pytest.fixture(scope="module")
def orc64():
    return oracle.get(fp64=True)


def _pose_err(a, b):
    c = np.abs(a["coord"].astype(np.float64) - b["coord"]).max()
    u = max(np.abs(a[k].astype(np.float64) - b[k]).max() for k in ("uVec", "yVec"))
    return float(c), float(u)


def _body_frame_d(coords, uvecs, yvecs, n, dt):
    """D_par, D_perp from per-step displacements projected on the body frame at step start."""
    dpar, dperp = [], []
    for t in range(len(coords) - 1):
        d = (coords[t + 1] - coords[t]).reshape(3, n)
        u, y = uvecs[t].reshape(3, n), yvecs[t].reshape(3, n)
        dpar.append(((d * u).sum(0) ** 2).mean())
        dperp.append(((d * y).sum(0) ** 2).mean())
    return np.mean(dpar) / (2 * dt), np.mean(dperp) / (2 * dt)


def test_free_rods_fp32_vs_fp64(orc_dm, orc64):
    f = scenes.free_rods_box(n=1024)
    n, dt = 1024, float(f["params"][0])
    runs = {}
    for name, orc, sc in (("fp32", orc_dm, copy.deepcopy(f)), ("fp64", orc64, oracle.to_fp64(f))):
        cs, us, ys = [], [], []
        b = sc["body"]
        for k in range(10):
            cs.append(b["coord"].astype(np.float64).copy())
            us.append(b["uVec"].astype(np.float64).copy())
            ys.append(b["yVec"].astype(np.float64).copy())
            orc.fdt_run(D.filament_desc(sc), 100 * k, 100)
        runs[name] = (sc, _body_frame_d(cs, us, ys, n, 100 * dt))
    c, u = _pose_err(runs["fp32"][0]["body"], runs["fp64"][0]["body"])
    assert c < 1e-4 and u < 5e-5, (c, u)
    for x, y in zip(runs["fp32"][1], runs["fp64"][1]):
        assert abs(x / y - 1.0) < 1e-4, (x, y)
    # the kernels' FP64-centre option: centres accumulated in double
    g = copy.deepcopy(f)
    D.add_coord64(g["body"])
    orc_dm.fdt_run(D.filament_desc(g), 0, 1000)
    c64 = float(np.abs(g["body"]["coord64"] - runs["fp64"][0]["body"]["coord"]).max())
    assert c64 < c, (c64, c)


# per store: centre median and 99th percentile (um), orientation median and 99th percentile
BOUNDS = {"fil": (5e-6, 5e-5, 5e-6, 1e-4), "mot": (5e-6, 2e-4, 1e-4, 5e-3), "mini": (5e-6, 2e-4, 5e-5, 1e-3)}


def test_dense_network_fp32_vs_fp64(orc_dm, orc64):
    sc = scenes.dense_contractile(scenes.C1)
    orc_dm.dense_run(D.dense_desc(sc), 0, 1000)
    a, b = copy.deepcopy(sc), oracle.to_fp64(sc)
    rng = np.random.default_rng(64)
    nF, nB, nBb = sc["fil"]["body"]["n"], sc["mot"]["body"]["n"], sc["mini"]["backbone"]["n"]
    for c in range(4):
        t0 = 1000 + 250 * c
        nf = rng.standard_normal((250, 6, nF), dtype=np.float32)
        nm = rng.standard_normal((250, 6, nB), dtype=np.float32)
        nb = rng.standard_normal((250, 6, nBb), dtype=np.float32)
        orc_dm.dense_run_supplied(D.dense_desc(a), t0, 250, nf, nm, nb)
        orc64.dense_run_supplied(D.dense_desc(b), t0, 250, nf.astype(np.float64), nm.astype(np.float64),
                                 nb.astype(np.float64))
    for s, bd in (("fil", "body"), ("mot", "body"), ("mini", "backbone")):
        x, y = a[s][bd], b[s][bd]
        n = x["n"]
        dc = np.abs(x["coord"].astype(np.float64) - y["coord"]).reshape(3, n).max(0)
        du = np.abs(x["uVec"].astype(np.float64) - y["uVec"]).reshape(3, n).max(0)
        print(s, "centres median %.2e p99 %.2e max %.2e; orientations median %.2e p99 %.2e max %.2e"
              % (np.median(dc), np.percentile(dc, 99), dc.max(), np.median(du), np.percentile(du, 99), du.max()))
        c_med, c_p99, u_med, u_p99 = BOUNDS[s]
        assert np.median(dc) < c_med and np.percentile(dc, 99) < c_p99, (s, np.median(dc), np.percentile(dc, 99))
        assert np.median(du) < u_med and np.percentile(du, 99) < u_p99, (s, np.median(du), np.percentile(du, 99))
    for s, k, most in (("mot", "boundSeg", 5), ("mot", "nucleotideState", 5), ("xl", "linkState", 5)):
        assert int((a[s][k] != b[s][k]).sum()) <= most, (s, k)


def test_equipartition_fp32_vs_fp64(orc_dm, orc64):
    r32 = G.run_equipartition(G.OracleBackend(orc_dm), G.confined_rods(reps=1000), burn=2000, steps=4000, every=2)
    sc = G.confined_rods(reps=1000)
    sc["b"] = oracle.to_fp64(sc["b"])
    sc["params"] = sc["params"].astype(np.float64)
    r64 = G.run_equipartition(G.OracleBackend(orc64), sc, burn=2000, steps=4000, every=2)
    assert abs(r32[0] / r32[1] - r64[0] / r64[1]) < 1e-3, (r32, r64)
