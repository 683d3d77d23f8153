"""Scale sweep of the dense step: the benchmark network's composition at fixed density.

    python -m softbox_b200.scale [--rods 20000 100000 500000 2000000] [--steps 20] [--modes fused graph]
                                 [--turnover]

For every size: build the network (slab side scaled by sqrt(n / 20,000), crosslinkers by
the KD-tree builder), then time `steps` consecutive steps per path with CUDA events on the
library's stream after 3 warm-up steps, and report ms/step, rod-steps/s and the achieved
GB/s of the algorithmic byte model (softbox_b200.roofline.step_bytes) against the measured
HBM peak. At 5e5 rods and beyond the working set is several times the 126 MB L2, so the
figures are HBM-resident measurements; below it they run L2-warm. One JSON line per size
and path; FP64 rod centres throughout.

--turnover runs the same networks with actin turnover on (scenes.dense_turnover: growth
10 subunits/s at barbed ends, severing 0.01/s per rod, constant-actin births into dead
slots) on the graph path, timing whole 100-step biochem cadences (the turnover block, the
release of dead attachments, births, and 100 mechanics steps with the grid rebuilt every
step).
"""
import argparse
import json
import time

from . import scenes
from .roofline import peaks, step_bytes


def measure(n_rods, steps=20, modes=("fused", "graph")):
    import torch
    from .engine import DenseNetwork
    from .runtime import LIB
    t0 = time.perf_counter()
    sc = scenes.dense_contractile(scenes.dense_scaled(n_rods))
    build_s = time.perf_counter() - t0
    nbytes = step_bytes(sc, fp64=True)
    hbm, how = peaks()
    out = []
    for mode in modes:
        net = DenseNetwork(sc, fp64_coords=True)
        if mode == "fused" and not net.fused_available:
            out.append({"rods": n_rods, "mode": mode, "unavailable": "fused path not available for this scene"})
            continue
        stream = torch.cuda.ExternalStream(LIB.sbx_ctx_stream(net.ctx.h))
        net.run(0, 3, mode=mode)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(True), torch.cuda.Event(True)
        with torch.cuda.stream(stream):
            s.record(stream)
            net.run(3, steps, mode=mode)
            e.record(stream)
        torch.cuda.synchronize()
        net.status()
        ms = s.elapsed_time(e) / steps
        gbs = nbytes / (ms / 1e3) / 1e9
        out.append({"rods": n_rods, "mode": mode, "ms_per_step": ms, "rod_steps_per_s": n_rods / (ms / 1e3),
                    "algorithmic_bytes_per_step": nbytes, "achieved_gbs": gbs, "hbm_peak_gbs": hbm,
                    "frac": gbs / hbm, "peak_source": how, "grid_ctas": net.fused_grid,
                    "scene_build_s": build_s, "steps": steps})
        net.close()
        del net
        torch.cuda.empty_cache()
    return out


def measure_turnover(n_rods, steps=1000, mode="graph"):
    import torch
    from .engine import TurnoverNetwork
    from .runtime import LIB
    from .turnover import pool_fields
    t0 = time.perf_counter()
    sc = scenes.dense_turnover(scenes.dense_scaled(n_rods))
    build_s = time.perf_counter() - t0
    nbytes = step_bytes(sc, fp64=True)
    hbm, how = peaks()
    net = TurnoverNetwork(sc, fp64_coords=True)
    ci = net.tcfg.check_int
    steps = max(ci, steps // ci * ci)
    stream = torch.cuda.ExternalStream(LIB.sbx_ctx_stream(net.ctx.h))
    if mode == "fused" and not net.fused_available:
        net.close()
        return {"rods": n_rods, "mode": "fused+turnover", "unavailable": "fused path not available for this scene"}
    net.run(0, 3 * ci, mode=mode)
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(True), torch.cuda.Event(True)
    with torch.cuda.stream(stream):
        s.record(stream)
        net.run(3 * ci, steps, mode=mode)
        e.record(stream)
    torch.cuda.synchronize()
    net.status()
    ms = s.elapsed_time(e) / steps
    fs = net.pull("fil", "filState")
    conc, _, taken, returned = pool_fields(net.pull("turnover", "pool"))
    out = {"rods": n_rods, "mode": mode + "+turnover", "ms_per_step": ms, "rod_steps_per_s": n_rods / (ms / 1e3),
           "algorithmic_bytes_per_step": nbytes, "achieved_gbs": nbytes / (ms / 1e3) / 1e9, "hbm_peak_gbs": hbm,
           "frac": nbytes / (ms / 1e3) / 1e9 / hbm, "peak_source": how, "steps": steps, "cadence_steps": ci,
           "active_rods_end": int((fs >= 0).sum()), "pool_taken": taken, "pool_returned": returned,
           "scene_build_s": build_s}
    net.close()
    del net
    torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rods", type=int, nargs="+", default=[20000, 100000, 500000, 2000000])
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--modes", nargs="+", default=["fused", "graph"])
    ap.add_argument("--turnover", action="store_true")
    a = ap.parse_args()
    if a.turnover:
        for n in a.rods:
            for mode in a.modes:
                print(json.dumps(measure_turnover(n, a.steps, mode)), flush=True)
        return
    for n in a.rods:
        for line in measure(n, a.steps, tuple(a.modes)):
            print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
