"""Timing helpers for the fused dense step.

    python -m softbox_b200.profiling phases [--steps 200] [--warm 3000] [--fp64]   # per-phase times
    python -m softbox_b200.profiling onestep                 # two one-step fused launches (for ncu -s 1 -c 1)

`phases` switches on the plan's %globaltimer stamps (sbx_dense_plan_phase_times): the
fused kernel writes the device time after every grid barrier of every step, so the
difference of consecutive stamps is the duration of one phase (including its barrier).
"""
import argparse
import ctypes as C

import numpy as np

from . import scenes
from .engine import DenseNetwork
from .runtime import LIB

PHASES = ["A publish, bin, histograms + lists, crosslinker unbind",   # K(prev) -> A
          "B tile sums", "C scans + motor Brownian", "E stable placement",
          "B0 binding (8 lanes per head)",
          "F minifilaments + crosslinker forces + chain joints + filament Brownian",
          "K rods (+ motor CSR helpers, resets)"]


def phase_times(steps=200, fp64_coords=False, cfg=None, warm=20):
    """Median per-phase times (us) of `steps` fused steps after `warm` untimed ones."""
    import torch
    net = DenseNetwork(scenes.dense_contractile(cfg or scenes.C1), fp64_coords=fp64_coords)
    net.run(0, warm, mode="fused")
    torch.cuda.synchronize()
    nph = len(PHASES)
    times = torch.zeros(steps * nph, dtype=torch.int64, device="cuda")
    LIB.sbx_dense_plan_phase_times(net.plan, C.c_void_p(times.data_ptr()))
    s, e = torch.cuda.Event(True), torch.cuda.Event(True)
    s.record()
    net.run(warm, steps, mode="fused")
    e.record()
    torch.cuda.synchronize()
    net.status()
    LIB.sbx_dense_plan_phase_times(net.plan, None)
    t = times.cpu().numpy().reshape(steps, nph).astype(np.float64)
    out = {PHASES[0]: float(np.median(t[1:, 0] - t[:-1, nph - 1]) / 1e3)}
    d = np.diff(t, axis=1)
    for k in range(1, nph):
        out[PHASES[k]] = float(np.median(d[:, k - 1]) / 1e3)
    out["step"] = float(np.median(np.diff(t[:, 0])) / 1e3)
    out["ms_per_step_events"] = s.elapsed_time(e) / steps
    return out


def one_step_launches():
    import torch
    net = DenseNetwork(scenes.dense_contractile(scenes.C1))
    net.run(0, 1, mode="fused")
    net.run(1, 1, mode="fused")
    torch.cuda.synchronize()
    return net.status()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["phases", "onestep"])
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--fp64", action="store_true")
    ap.add_argument("--warm", type=int, default=3000)
    a = ap.parse_args()
    if a.what == "phases":
        for k, v in phase_times(a.steps, a.fp64, warm=a.warm).items():
            print(f"{k:48s} {v:9.2f} {'ms' if k.startswith('ms') else 'us'}")
    else:
        print("status", one_step_launches())


if __name__ == "__main__":
    main()
