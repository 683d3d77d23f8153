"""Sweep sharding across ranks (two gloo ranks on CPU): every point is run exactly once,
by rank (index mod world size), and the gathered outputs come back in the points' order."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp


def _fake_runner(points, steps, sample_every):
    # a deterministic per-point function stands in for the packed GPU run
    return {"contraction_rate": np.array([p.n_rods * 1e-5 + p.myo_ratio for p in points]),
            "largest_fraction": np.array([p.xl_ratio for p in points]),
            "stress_pa": np.array([float(p.chain_len) for p in points]), "gpu_ms": 1.0 + len(points)}


def _worker(rank, ws, port, q):
    import torch.distributed as dist
    from softbox_b200 import ensemble
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    pts = ensemble.sample_points(11, seed=4)
    seen = []

    def runner(p, s, e):
        seen.extend(p)
        return _fake_runner(p, s, e)
    out = ensemble.run_sharded(pts, 10, 5, runner=runner)
    q.put((rank, [x.seed for x in seen], {k: np.asarray(v).tolist() for k, v in out.items()}))
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_sharded_sweep_matches_single():
    from softbox_b200 import ensemble
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=100) for _ in procs]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    pts = ensemble.sample_points(11, seed=4)
    want = _fake_runner(pts, 10, 5)
    seeds = sorted(s for _, ss, _ in res for s in ss)
    assert seeds == sorted(p.seed for p in pts)                     # each point exactly once
    for rank, ss, out in res:
        assert ss == [pts[i].seed for i in range(rank, 11, 2)]
        for k in ("contraction_rate", "largest_fraction", "stress_pa"):
            assert np.array_equal(np.asarray(out[k]), want[k])
        assert out["gpu_ms_max_over_ranks"] == 1.0 + 6
