"""Parameter sweeps of independent dense networks run as one packed batch.

    pts = sample_points(256, seed=1)                  # the sweep distribution below
    res = run_ensemble(pts, steps=2000, sample_every=200)
    res["contraction_rate"], res["largest_fraction"], res["stress_pa"]     # one value per point

Sweep distribution (per point, seeded): actin rods log-uniform in [2,000, 80,000]; myosin
minifilaments per actin rod U(0.005, 0.05); crosslinkers per actin rod U(0, 0.5);
filament chain length U{5..20} rods of 0.1 um; turnover rate U(0, 0.02)/s (with
`turnover=True` each network runs scenes.dense_turnover's turnover with that rate as its
severing rate, its own turnover seed and actin pool; otherwise the rate is a surrogate
input only and the runs advance the mechanics); slab aspect
x:y log-uniform in [1/2, 2] at the benchmark density (20 x 20 um per 20,000 rods, depth
0.5 um). Every network has its own seeds. The network's other parameters are the
benchmark's (scenes.C1).

Outputs per point: the contraction rate -d ln R_rms/dt (least squares over the samples),
the largest-cluster fraction at the end and the mean network stress averaged over the
samples (softbox_b200.observables).
"""
import math
import time
from dataclasses import dataclass, replace

import numpy as np

from . import scenes

RODS_RANGE = (2000, 80000)
MYO_RANGE = (0.005, 0.05)
XL_RANGE = (0.0, 0.5)
CHAIN_RANGE = (5, 20)
TURNOVER_RANGE = (0.0, 0.02)
ASPECT_RANGE = (0.5, 2.0)


@dataclass(frozen=True)
class SweepPoint:
    n_rods: int
    myo_ratio: float
    xl_ratio: float
    chain_len: int
    turnover: float
    aspect: float
    seed: int


def sample_points(n, seed=0, rods_range=RODS_RANGE):
    rng = np.random.default_rng(seed)
    lo, hi = math.log(rods_range[0]), math.log(rods_range[1])
    out = []
    for k in range(n):
        chain = int(rng.integers(CHAIN_RANGE[0], CHAIN_RANGE[1] + 1))
        rods = int(round(math.exp(rng.uniform(lo, hi)) / chain)) * chain
        out.append(SweepPoint(n_rods=max(chain, rods), myo_ratio=float(rng.uniform(*MYO_RANGE)),
                              xl_ratio=float(rng.uniform(*XL_RANGE)), chain_len=chain,
                              turnover=float(rng.uniform(*TURNOVER_RANGE)),
                              aspect=float(math.exp(rng.uniform(math.log(ASPECT_RANGE[0]), math.log(ASPECT_RANGE[1])))),
                              seed=int(rng.integers(1, 2**31 - 1))))
    return out


def features(points, rods_range=RODS_RANGE):
    """The six surrogate inputs, each scaled to [0, 1]: the four sweep parameters (myosin
    ratio, crosslinker ratio, chain length, turnover rate), log rod count and log aspect."""
    lo, hi = math.log(rods_range[0]), math.log(rods_range[1])
    a0, a1 = math.log(ASPECT_RANGE[0]), math.log(ASPECT_RANGE[1])
    x = np.array([[(p.myo_ratio - MYO_RANGE[0]) / (MYO_RANGE[1] - MYO_RANGE[0]),
                   (p.xl_ratio - XL_RANGE[0]) / (XL_RANGE[1] - XL_RANGE[0]),
                   (p.chain_len - CHAIN_RANGE[0]) / (CHAIN_RANGE[1] - CHAIN_RANGE[0]),
                   (p.turnover - TURNOVER_RANGE[0]) / (TURNOVER_RANGE[1] - TURNOVER_RANGE[0]),
                   (math.log(p.n_rods) - lo) / (hi - lo),
                   (math.log(p.aspect) - a0) / (a1 - a0)] for p in points], np.float32)
    return x


def point_config(p, cell_scale=1.0):
    base = scenes.C1
    n_fil = max(1, p.n_rods // p.chain_len)
    n_rods = n_fil * p.chain_len
    rng = np.random.default_rng(p.seed)
    seeds = [int(s) for s in rng.integers(1, 2**31 - 1, 4)]
    return replace(base, n_fil=n_fil, segs_per_fil=p.chain_len, n_mini=max(1, int(round(p.myo_ratio * n_rods))),
                   n_links=int(round(p.xl_ratio * n_rods)), side=base.side * math.sqrt(n_rods / base.n_seg),
                   aspect=p.aspect, cell_scale=cell_scale, fast_links=True, seed=seeds[0], seed_bb=seeds[1],
                   seed_fil=seeds[2])


def build_batch(points, cell_scale=1.0, turnover=False):
    from .batch import pack_networks
    nets = []
    for p in points:
        cfg = point_config(p, cell_scale)
        if turnover:
            sc = scenes.dense_turnover(cfg, sever_rate=p.turnover, turnover_seed=p.seed ^ 0x0F0501)
        else:
            sc = scenes.dense_contractile(cfg)
        for k in ("reachSeg", "center", "gridCellContents", "bodyCell", "cellCount", "gridCellOffsets"):
            sc["grid"].pop(k, None)                 # per-step scratch: the packed scene makes its own
        nets.append(sc)
    return pack_networks(nets)


def autotune_cell(points, candidates=(1.0, 1.25, 1.5, 2.0), steps=20, fp64_coords=True, sample=32):
    """The grid cell (as a multiple of the completeness minimum) with the fastest batched
    step: each candidate is built for `sample` of the points (every k-th) and timed over
    `steps` graph steps after 3 warm-up steps. Larger cells keep every reachable pair (the
    stencil still covers the cutoff); the candidate list order differs, so the choice is a
    performance setting."""
    import torch
    from .batch import BatchedNetworks
    points = list(points)[::max(1, len(points) // sample)]
    timings = {}
    for c in candidates:
        packed, info = build_batch(points, c)
        ens = BatchedNetworks(packed, info, fp64_coords=fp64_coords)
        ens.run(0, 3)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(True), torch.cuda.Event(True)
        s.record()
        ens.run(3, steps)
        e.record()
        torch.cuda.synchronize()
        timings[c] = s.elapsed_time(e) / steps
        ens.close()
        del ens
    best = min(timings, key=timings.get)
    return best, timings


def run_ensemble(points, steps, sample_every, cell_scale=1.0, fp64_coords=True, t0=0, turnover=False):
    """Advances every point's network `steps` steps in one packed batch and returns the
    observables per point plus timing (`turnover`: with each point's actin turnover)."""
    import torch
    from .batch import BatchedNetworks, BatchedTurnoverNetworks
    from .observables import Observables, contraction_rate
    tb = time.perf_counter()
    packed, info = build_batch(points, cell_scale, turnover)
    build_s = time.perf_counter() - tb
    ens = (BatchedTurnoverNetworks if turnover else BatchedNetworks)(packed, info, fp64_coords=fp64_coords)
    obs = Observables(ens)
    dt = float(packed["fil"]["params"][0])
    times, rms, stress = [], [], []
    s0 = obs.sample()
    times.append(0.0)
    rms.append(s0["rms_um"])
    stress.append(s0["stress_pa"])
    ev0, ev1 = torch.cuda.Event(True), torch.cuda.Event(True)
    gpu_ms = 0.0
    done = 0
    while done < steps:
        k = min(sample_every, steps - done)
        ev0.record()
        ens.run(t0 + done, k)
        ev1.record()
        torch.cuda.synchronize()
        gpu_ms += ev0.elapsed_time(ev1)
        done += k
        s = obs.sample()
        times.append(done * dt)
        rms.append(s["rms_um"])
        stress.append(s["stress_pa"])
    rms = np.array(rms)
    rates = np.array([contraction_rate(times, rms[:, j]) for j in range(len(points))])
    out = {"contraction_rate": rates, "largest_fraction": s["largest_fraction"],
           "stress_pa": np.array(stress)[1:].mean(axis=0), "rms_um": rms, "times_s": np.array(times),
           "steps": steps, "gpu_ms": gpu_ms, "ms_per_step": gpu_ms / max(steps, 1), "build_s": build_s,
           "rods": int(packed["fil"]["body"]["n"]), "bodies": int(packed["fil"]["body"]["n"]
                                                                  + packed["mot"]["body"]["n"]
                                                                  + packed["mini"]["backbone"]["n"])}
    ens.close()
    return out


def main():
    import argparse
    import json
    ap = argparse.ArgumentParser(description="batched parameter sweep of dense networks")
    ap.add_argument("--points", type=int, default=256)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--sample-every", type=int, default=100)
    ap.add_argument("--run-steps", type=int, default=50000, help="steps of one sweep run (for points/s)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--turnover", action="store_true", help="run each point's actin turnover")
    a = ap.parse_args()
    pts = sample_points(a.points, a.seed)
    cell, tune = 1.0, None
    if a.autotune:
        cell, tune = autotune_cell(pts)
    r = run_ensemble(pts, a.steps, a.sample_every, cell_scale=cell, turnover=a.turnover)
    sec_per_run = r["ms_per_step"] * 1e-3 * a.run_steps
    print(json.dumps({"points": a.points, "rods": r["rods"], "bodies": r["bodies"], "steps_timed": a.steps,
                      "ms_per_step": r["ms_per_step"], "rod_steps_per_s": r["rods"] / (r["ms_per_step"] * 1e-3),
                      "body_steps_per_s": r["bodies"] / (r["ms_per_step"] * 1e-3), "run_steps": a.run_steps,
                      "sweep_points_per_s": a.points / sec_per_run, "cell_scale": cell, "autotune_ms": tune,
                      "turnover": a.turnover,
                      "build_s": r["build_s"],
                      "contraction_rate_mean": float(np.mean(r["contraction_rate"])),
                      "largest_fraction_mean": float(np.mean(r["largest_fraction"])),
                      "stress_pa_mean": float(np.mean(r["stress_pa"]))}), flush=True)


if __name__ == "__main__":
    main()


def run_sharded(points, steps, sample_every, runner=None, **kw):
    """A sweep over all ranks of the default process group: rank r runs points r, r + N,
    ... (one packed batch per rank), then the per-point outputs are gathered once and put
    back in the points' order. Without a process group it is `runner` on all points."""
    runner = runner or run_ensemble
    try:
        import torch.distributed as dist
        ws = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
        rank = dist.get_rank() if ws > 1 else 0
    except Exception:
        ws, rank = 1, 0
    if ws == 1:
        return runner(points, steps, sample_every, **kw)
    mine = list(range(rank, len(points), ws))
    r = runner([points[i] for i in mine], steps, sample_every, **kw) if mine else None
    part = {"index": mine}
    if r is not None:
        for k in ("contraction_rate", "largest_fraction", "stress_pa"):
            part[k] = np.asarray(r[k]).tolist()
        part["gpu_ms"] = float(r.get("gpu_ms", 0.0))
    parts = [None] * ws
    dist.all_gather_object(parts, part)
    out = {k: np.zeros(len(points)) for k in ("contraction_rate", "largest_fraction", "stress_pa")}
    gpu_ms = 0.0
    for p in parts:
        for j, i in enumerate(p["index"]):
            for k in out:
                out[k][i] = p[k][j]
        gpu_ms = max(gpu_ms, p.get("gpu_ms", 0.0))
    out["gpu_ms_max_over_ranks"] = gpu_ms
    return out
