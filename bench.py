"""Benchmark: rod-steps/s of the dense contractile network on B200.

Workload (one step = one DenseContractileHarness.cpuStep of the whole network):
2,000 filaments x 10 rigid rods of 0.1 um (20,000 rods), 200 minifilaments with a 0.8 um
backbone and 16 heads per end (6,400 heads, 19,200 myosin sub-bodies), 4,000
crosslinkers (Bell unbinding on), 20 x 20 x 0.5 um slab with confining walls, dt = 10 us,
forces FP32, rod centres accumulated in FP64. Synthetic seeded scene (the reference's
scene builder with these counts); no dataset.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Both arms first advance the network WARM_STEPS steps untimed, to the state where binding
has built up (about 700 bound heads; a fresh scene has about 120 in its first 25 steps),
then take W untimed warm-up steps and time K steps.
Our arm: each step is one launch of the fused persistent kernel; timed with CUDA events
on the library's stream, one step at a time, with L2 flushed (a 256 MiB write) between
timed steps. The reference arm times the reference's CPU path: the C++ restatement of
the Java System classes (oracle/), on all host threads, on the same workload, for at
least REF_MIN_STEPS timed steps.
Multi-GPU: one process per GPU (torchrun), each advancing its own independent network
(replicas; the single network does not shard), value = all ranks' rod-steps / max time.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "rod-steps/s"
WORKLOAD = ("dense contractile network: 2000 filaments x 10 rods of 0.1 um (20000 rods), 200 minifilaments "
            "(0.8 um backbone, 16 heads/end: 6400 heads), 4000 crosslinkers, 20x20x0.5 um slab with walls, "
            "dt 10 us, FP32 forces, FP64 rod centres")


from softbox_b200.roofline import peaks, step_bytes  # noqa: E402

WARM_STEPS = 3000      # untimed steps before the warm-up: bound heads have built up
REF_MIN_STEPS = 200    # the reference arm times at least this many steps
# DRAM bytes (read + write) of one launch of the fused kernel advancing one step of this
# workload (FP64 centres, warmed state, L2 flushed before the launch), from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum, mean of three launches of
# `python bench.py --steps 3 --warmup 3 --no-cpu --sweep-points 0` under
# `ncu --clock-control none -k regex:k_dense_fused -s 1 -c 3`)
FUSED_STEP_DRAM_BYTES = 12_302_000


def workload_config(sc_host, warmup):
    """The `config` object of the bench line: identical in both arms."""
    return {"workload": WORKLOAD, "rods": int(sc_host["fil"]["body"]["n"]), "heads": int(sc_host["mot"]["nMotors"]),
            "crosslinks": int(sc_host["xl"]["nLinks"]), "warm_steps": WARM_STEPS + warmup,
            "l2": "inputs (18 MB) below L2 size: L2 flushed between timed steps (256 MiB write) in the GPU arm"}


def bound_state(sc_or_dev):
    """Bound heads and active crosslinks of a host scene (numpy) or device scene (torch)."""
    bs, ls = sc_or_dev["mot"]["boundSeg"], sc_or_dev["xl"]["linkState"]
    return {"bound_heads": int((bs >= 0).sum()), "active_links": int((ls >= 0).sum())}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------------- CPU arm
def _oracle(threads):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    orc = oracle.get(devmath=False)
    orc.set_threads(threads)
    return orc


def cpu_oracle_rate(sc, t0, steps, threads, warmup=0):
    """rod-steps/s of the oracle (C++ restatement of the reference's Java System classes)
    advancing the host scene `sc` (FP64 centres attached) in place from step t0: `warmup`
    untimed steps, then `steps` timed ones. Returns (rate, seconds, next step)."""
    from softbox_b200 import device as D
    orc = _oracle(threads)
    desc = D.dense_desc(sc)
    if warmup:
        orc.dense_run(desc, t0, warmup)
    t0 += warmup
    s0 = time.perf_counter()
    orc.dense_run(desc, t0, steps)
    dt = time.perf_counter() - s0
    return sc["fil"]["body"]["n"] * steps / dt, dt, t0 + steps


def host_scene_fp64():
    """The benchmark scene on the host with FP64 centres attached."""
    from softbox_b200 import device as D, scenes
    sc = scenes.dense_contractile(scenes.C1)
    for s_, b_ in (("fil", "body"), ("mot", "body"), ("mini", "backbone")):
        D.add_coord64(sc[s_][b_])
    return sc


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from softbox_b200 import device as D
    sc = host_scene_fp64()
    threads = os.cpu_count() or 1
    steps = max(args.steps, REF_MIN_STEPS)
    warmup = max(3, args.warmup)
    _oracle(threads).dense_run(D.dense_desc(sc), 0, WARM_STEPS)      # to the warmed state, untimed
    rate, dt, _ = cpu_oracle_rate(sc, WARM_STEPS, steps, threads, warmup=warmup)
    line = {"metric": METRIC, "value": rate, "unit": "rod-steps/s", "n_gpus": args.gpus, "steps": steps,
            "warmup": warmup, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 forces, f64 centres", "data": "synthetic",
            "config": workload_config(sc, warmup), "impl": "reference",
            "arm": {"path": "C++ restatement of the Java System classes (oracle/, libm), OpenMP over slots",
                    "parallelism": f"{threads} host threads", "state_at_end": bound_state(sc)},
            "cpu_baseline": {"value": rate, "unit": "rod-steps/s", "cores": threads, "kind": "port",
                             "sample": f"{steps} full steps of the workload after {WARM_STEPS + warmup} untimed "
                                       f"steps, {dt:.1f} s, C++ restatement of the Java System classes "
                                       f"(no JVM on the box)"},
            "e2e": {"value": rate, "unit": "rod-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- GPU arm
def run_ours(args):
    import torch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    from softbox_b200 import scenes
    from softbox_b200.engine import DenseNetwork
    from softbox_b200.runtime import LIB, Context

    ctx = Context(local)
    sc_host = scenes.dense_contractile(scenes.C1)
    net = DenseNetwork(sc_host, ctx=ctx, fp64_coords=True)
    assert net.fused_available, "the benchmark network must qualify for the fused path"
    stream = torch.cuda.ExternalStream(LIB.sbx_ctx_stream(ctx.h))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    nrods = sc_host["fil"]["body"]["n"]

    def one_step(t):
        net.run(t, 1, mode="fused")

    # advance to the warmed state (one persistent launch), untimed
    net.run(0, WARM_STEPS, mode="fused")
    net.status()
    t = WARM_STEPS
    with torch.cuda.stream(stream):
        for _ in range(max(3, args.warmup)):
            flush.zero_()
            one_step(t)
            t += 1
    torch.cuda.synchronize()
    net.status()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        time.sleep(0.3)
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.zero_()
                starts[k].record(stream)
                one_step(t)
                ends[k].record(stream)
                t += 1
        torch.cuda.synchronize()
    net.status()
    state = bound_state(net.dev)
    step_ms = np.array([s.elapsed_time(e) for s, e in zip(starts, ends)])
    total_ms = float(step_ms.sum())
    if pg:
        tt = torch.tensor([total_ms], device=f"cuda:{local}", dtype=torch.float64)
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        total_ms = float(tt.item())
    value = ws * nrods * args.steps / (total_ms / 1e3)

    # e2e through the C ABI: per step, H2D of the step's counts blocks (the reference's
    # EVERY_EXECUTION upload: motor, backbone and filament counts, 3 x 16 B, contiguous on
    # the device, so one copy) from pinned memory, one fused step, D2H of the step's binding
    # state (boundSeg) into pinned memory.
    # Pipelined as a streaming host would run it: step k is queued (upload, launch, result
    # copy, marker) before the host waits for step k - 1's result; two pinned buffers each.
    # The result copy runs on the context's copy stream, so it overlaps the next step's
    # upload; the next step waits for it before it rewrites boundSeg.
    d = net.dev
    counts_host = [torch.zeros(12, dtype=torch.int32).pin_memory() for _ in range(2)]
    bound_host = [torch.empty(sc_host["mot"]["nMotors"], dtype=torch.int32).pin_memory() for _ in range(2)]
    cfg = sc_host["cfg"]
    h2d = 3 * 16
    d2h = bound_host[0].numel() * 4
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    e2e_steps = args.steps
    bound_sum = 0
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        b = k & 1
        c = counts_host[b].numpy()
        c[:] = [sc_host["mot"]["nMotors"], t, cfg.seed, nrods, sc_host["mini"]["nBackbones"], t, cfg.seed_bb,
                sc_host["mini"]["nBackbones"], nrods, t, cfg.seed_fil, 1]
        ctx("sbx_upload", C.c_void_p(net.counts_block.data_ptr()), C.c_void_p(counts_host[b].data_ptr()), h2d)
        if k > 0:
            ctx("sbx_ctx_stream_wait_mark", 1 - b)       # the step rewrites boundSeg: after k - 1's copy
        st = LIB.sbx_dense_plan_run(net.plan, t, 1, 2)
        assert st == 0, ctx.last_error()
        ctx("sbx_download_async_side", C.c_void_p(bound_host[b].data_ptr()),
            C.c_void_p(d["mot"]["boundSeg"].data_ptr()), d2h)
        ctx("sbx_ctx_mark_side", b)
        if k > 0:
            ctx("sbx_ctx_wait_mark", 1 - b)              # step k - 1's result is on the host
            bound_sum += int(bound_host[1 - b].numpy()[0])
        t += 1
    ctx("sbx_ctx_wait_mark", (e2e_steps - 1) & 1)
    bound_sum += int(bound_host[(e2e_steps - 1) & 1].numpy()[0])
    e2e_s = time.perf_counter() - t0
    if pg:
        tt = torch.tensor([e2e_s], device=f"cuda:{local}", dtype=torch.float64)
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        e2e_s = float(tt.item())
    e2e = ws * nrods * e2e_steps / e2e_s

    # roofline of the dominant (only) kernel: the fused step
    hbm, how = peaks()
    bytes_step = step_bytes(sc_host, fp64=True)
    achieved = bytes_step / (float(np.mean(step_ms)) / 1e3) / 1e9
    traffic = FUSED_STEP_DRAM_BYTES

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        # the same warmed state: the device arrays (bit-identical to the oracle's run)
        import copy
        sc_cpu = copy.deepcopy(sc_host)
        got = net.pull_all()
        for k in sc_cpu:
            if k in got:
                sc_cpu[k] = got[k]
        rate, dt, _ = cpu_oracle_rate(sc_cpu, t, args.cpu_steps, 1)
        cpu = {"value": rate, "unit": "rod-steps/s", "cores": 1, "kind": "port",
               "sample": f"{args.cpu_steps} full steps of the warmed workload on 1 host core ({dt:.1f} s), C++ "
                         f"restatement of the Java System classes' single-threaded -cpu runner"}
    clocks = clk.summary()
    sweep = None
    if ws == 1 and args.sweep_points > 0:
        sweep = sweep_measure(args.sweep_points, args.sweep_steps)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "rod-steps/s", "n_gpus": ws, "steps": args.steps,
                "warmup": max(3, args.warmup), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32 forces, f64 centres", "data": "synthetic",
                "config": workload_config(sc_host, max(3, args.warmup)),
                "arm": {"path": "fused persistent cooperative kernel, 1 launch per step",
                        "parallelism": f"replicas x{ws}", "grid_ctas": net.fused_grid, "state_at_timing": state},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                             "frac": achieved / hbm, "traffic": traffic, "peak_source": how,
                             "kernel": "k_dense_fused", "algorithmic_bytes_per_launch": bytes_step},
                "cpu_baseline": cpu,
                "e2e": {"value": e2e, "unit": "rod-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "host_loop": "C ABI from Python; each step's upload, launch and result copy (on the copy stream) queued "
                                     "before the host waits for the previous step's result (L2 not flushed)"},
                "gpu_launches": args.steps,
                "clocks": clocks,
                "step_ms_median": float(np.median(step_ms)), "step_ms_p90": float(np.percentile(step_ms, 90)),
                "sweep": sweep}
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def sweep_measure(n_points, steps, run_steps=50000):
    """The sweep side of the metric on this box: one packed batch of sampled sweep points
    advanced `steps` steps (CUDA events), extrapolated to sweep runs of `run_steps` steps,
    and the surrogate ensemble's inference rate (5 x 6-256x4-3 MLPs, tensor-core GEMMs) on
    100,000 points. The surrogate's error and fallback fraction come from the full pipeline
    (python -m softbox_b200.sweep_surrogate)."""
    import torch
    from softbox_b200 import ensemble
    from softbox_b200.surrogate import MLPEnsemble
    pts = ensemble.sample_points(n_points, seed=1)
    r = ensemble.run_ensemble(pts, steps, sample_every=steps)
    ens = MLPEnsemble(n_nets=5, seed=0)
    x = ensemble.features(ensemble.sample_points(100000, seed=2))
    ens.set_normalisation(x, np.zeros((1, 3)))
    ens.predict(x)                                  # warm-up: the inference buffers exist after it
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(True), torch.cuda.Event(True)
    s.record()
    ens.predict(x)
    e.record()
    torch.cuda.synchronize()
    infer_s = s.elapsed_time(e) / 1e3
    return {"points": n_points, "rods": r["rods"], "bodies": r["bodies"], "steps_timed": steps,
            "ms_per_packed_step": r["ms_per_step"], "rod_steps_per_s": r["rods"] / (r["ms_per_step"] / 1e3),
            "batched_points_per_s_at_run_steps": n_points / (r["ms_per_step"] / 1e3 * run_steps),
            "run_steps": run_steps, "surrogate_inference_points_per_s": 100000 / infer_s,
            "surrogate_error_source": "python -m softbox_b200.sweep_surrogate (not measured in this run)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=600)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--sweep-points", type=int, default=256,
                    help="packed sweep points timed beside the step: 256, the batched ensemble's size (0: off)")
    ap.add_argument("--sweep-steps", type=int, default=200)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
