"""The index-checking debug build (libsoftbox_b200_check.so, -DSBX_CHECK): on valid scenes
its kernels find no index outside its array and give the same bits as the normal build, on
the fused, graph and per-system paths. It runs in a child process (SBX_LIB=check selects the
library at load time); the parent compares its results with the oracle."""
import copy
import os
import pickle
import subprocess
import sys

import numpy as np
import pytest

from helpers import compare_scenes, oracle_dense_run, small_dense
from softbox_b200 import scenes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECK_LIB = os.path.join(ROOT, "softbox_b200", "_lib", "libsoftbox_b200_check.so")

CHILD = r'''
import ctypes as C, pickle, sys
sys.path.insert(0, sys.argv[1])
import torch
from softbox_b200 import device as D
from softbox_b200.engine import DenseNetwork, TurnoverNetwork
from softbox_b200.runtime import LIB
assert LIB.sbx_check_build() == 1
job = pickle.load(open(sys.argv[2], "rb"))
out = {}
for mode in job["modes"]:
    cls = TurnoverNetwork if job.get("turnover") else DenseNetwork
    net = cls(job["scene"], fp64_coords=job.get("fp64", False))
    if mode == "unfused":
        for t in range(job["t0"], job["t0"] + job["n"]):
            net.step_unfused(t)
    else:
        net.run(job["t0"], job["n"], mode=mode)
        assert net.status() == 0
    torch.cuda.synchronize()
    c, s, i = C.c_int64(), C.c_int32(), C.c_int64()
    assert LIB.sbx_check_report(C.byref(c), C.byref(s), C.byref(i), 1) == 0
    out[mode] = {"scene": D.to_host(net.dev), "bad": (c.value, s.value, i.value)}
pickle.dump(out, open(sys.argv[3], "wb"))
'''


def run_checked(tmp_path, scene, t0, n, modes, fp64=False, turnover=False):
    job, res = tmp_path / "job.pkl", tmp_path / "res.pkl"
    pickle.dump({"scene": scene, "t0": t0, "n": n, "modes": modes, "fp64": fp64, "turnover": turnover},
                open(job, "wb"))
    env = dict(os.environ, SBX_LIB="check")
    subprocess.run([sys.executable, "-c", CHILD, ROOT, str(job), str(res)], check=True, env=env, cwd=ROOT,
                   timeout=600)
    return pickle.load(open(res, "rb"))


@pytest.fixture(scope="module")
def warm_small(orc_dm):
    sc = small_dense(0.05)
    oracle_dense_run(orc_dm, sc, 0, 300)
    return sc


@pytest.mark.skipif(not os.path.exists(CHECK_LIB), reason="check build missing")
def test_check_build_small_network_all_paths(orc_dm, warm_small, tmp_path):
    out = run_checked(tmp_path, copy.deepcopy(warm_small), 300, 40, ["fused", "graph", "unfused"])
    ref = copy.deepcopy(warm_small)
    oracle_dense_run(orc_dm, ref, 300, 40)
    for mode, r in out.items():
        assert r["bad"] == (0, 0, 0), (mode, r["bad"])
        names = compare_scenes({k: v for k, v in ref.items() if k != "cfg"}, r["scene"])
        assert len(names) > 80, mode


@pytest.mark.skipif(not os.path.exists(CHECK_LIB), reason="check build missing")
def test_check_build_benchmark_network_fused(tmp_path):
    """The 20,000-rod benchmark network, 200 fused steps in the check build: no bad index, and
    the same bits as the normal build in this process."""
    from softbox_b200 import device as D
    from softbox_b200.engine import DenseNetwork
    sc = scenes.dense_contractile(scenes.C1)
    out = run_checked(tmp_path, copy.deepcopy(sc), 0, 200, ["fused"], fp64=True)
    assert out["fused"]["bad"] == (0, 0, 0), out["fused"]["bad"]
    net = DenseNetwork(copy.deepcopy(sc), fp64_coords=True)
    net.run(0, 200, mode="fused")
    assert net.status() == 0
    torch.cuda.synchronize()
    names = compare_scenes({k: v for k, v in D.to_host(net.dev).items() if k != "cfg"}, out["fused"]["scene"])
    assert len(names) > 80


@pytest.mark.skipif(not os.path.exists(CHECK_LIB), reason="check build missing")
def test_check_build_turnover_network_fused(orc_dm, tmp_path):
    """A turnover network (deaths, splits, births into FREE slots: chain neighbours across the
    fused kernel's rod groups) for 500 fused steps in the check build: no bad index, and the
    oracle's bits."""
    from helpers import oracle_turnover_network_run
    sc = scenes.dense_turnover(scenes.dense_small(0.05), growth_rate=400.0, sever_rate=5.0)
    out = run_checked(tmp_path, copy.deepcopy(sc), 0, 500, ["fused"], turnover=True)
    assert out["fused"]["bad"] == (0, 0, 0), out["fused"]["bad"]
    ref = copy.deepcopy(sc)
    oracle_turnover_network_run(orc_dm, ref, 0, 500)
    names = compare_scenes({k: v for k, v in ref.items() if k != "tcfg"}, out["fused"]["scene"], skip=("coord64",))
    assert "fil.body.coord" in names
