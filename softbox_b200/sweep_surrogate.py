"""The surrogate sweep end to end: training data from packed batched runs, the MLP
ensemble trained on the GPU, fresh points predicted with the plain batched simulator as
the fallback where the ensemble disagrees, and the throughput against the plain per-run
GPU sweep.

    python -m softbox_b200.sweep_surrogate [--train 1024] [--heldout 512] [--fresh 100000]
                                           [--steps 2000] [--rods 2000 80000] [--epochs 200]

Points per second are whole-sweep figures for runs of `steps` steps:
* plain per-run: each point's network advanced alone by the single-network plan (the
  fused kernel where available), timed on a sample of the points and scaled to the sweep;
* plain batched: packed batches of up to 256 points (the timed training-data batches);
* surrogate: ensemble inference for every fresh point plus, for the points whose ensemble
  standard deviation exceeds the threshold on any output, a plain batched rerun charged at
  the measured batched cost per point (on the held-out points a fallback point takes its
  plain result, which gives the error of the whole rule).
Relative error on an output: mean |prediction - plain run| / mean |plain run| over the
held-out points.

Rule selection: the fallback rule (outputs checked: all three or the contraction rate alone;
threshold on std / |mean|; |mean| floored at a fraction of each output's training spread) is
chosen on the first half of the held-out runs as the fastest sweep whose contraction-rate
error there stays within --max-err, and its error is reported on the second half.
"""
import argparse
import json
import time

import numpy as np

from . import ensemble

OUTPUTS = ("contraction_rate", "largest_fraction", "stress_pa")


def _targets(r):
    return np.stack([r[k] for k in OUTPUTS], axis=1)


def generate(points, steps, sample_every, batch=256, turnover=False):
    """Plain batched runs of `points` in packs of `batch`; returns targets and GPU seconds."""
    ys, gpu_s, build_s = [], 0.0, 0.0
    for b0 in range(0, len(points), batch):
        r = ensemble.run_ensemble(points[b0:b0 + batch], steps, sample_every, turnover=turnover)
        ys.append(_targets(r))
        gpu_s += r["gpu_ms"] * 1e-3
        build_s += r["build_s"]
    return np.concatenate(ys), gpu_s, build_s


def per_run_seconds(points, steps, sample=8, turnover=False):
    """Mean GPU seconds of one point's run alone (single-network plan on the auto path,
    with or without turnover)."""
    import torch
    from .engine import DenseNetwork, TurnoverNetwork
    from . import scenes
    secs = []
    for p in points[:sample]:
        cfg = ensemble.point_config(p)
        if turnover:
            net = TurnoverNetwork(scenes.dense_turnover(cfg, sever_rate=p.turnover, turnover_seed=p.seed ^ 0x0F0501),
                                  fp64_coords=True)
        else:
            net = DenseNetwork(scenes.dense_contractile(cfg), fp64_coords=True)
        net.run(0, 3)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(True), torch.cuda.Event(True)
        s.record()
        net.run(3, steps)
        e.record()
        torch.cuda.synchronize()
        secs.append(s.elapsed_time(e) * 1e-3)
        net.close()
    return float(np.mean(secs)), secs


def rel_error(pred, true):
    return (np.abs(pred - true).mean(axis=0) / np.maximum(np.abs(true).mean(axis=0), 1e-30)).tolist()


def main():
    import torch
    from .surrogate import MLPEnsemble, fallback_mask
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=1024)
    ap.add_argument("--heldout", type=int, default=512)
    ap.add_argument("--fresh", type=int, default=100000)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--sample-every", type=int, default=250)
    ap.add_argument("--rods", type=int, nargs=2, default=list(ensemble.RODS_RANGE))
    ap.add_argument("--epochs", type=int, default=200)
    ap.add_argument("--threshold", type=float, default=0.10)
    ap.add_argument("--floor", type=float, default=0.0,
                    help="also report the rule with |mean| floored at this fraction of each output's training spread")
    ap.add_argument("--per-run-sample", type=int, default=8)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--turnover", action="store_true", help="every run with its point's actin turnover")
    ap.add_argument("--max-err", type=float, default=0.05, help="contraction-rate error bound of the selected rule")
    ap.add_argument("--save-data", default="", help="write the plain runs' targets and timings to this .npz")
    ap.add_argument("--retime-batched", type=int, default=0,
                    help="time the packed rerun cost on a fresh batch of this many training points")
    ap.add_argument("--load-data", default="", help="reuse the plain runs of a --save-data file (same settings)")
    ap.add_argument("--train-grid", action="store_true",
                    help="also train ensembles for 25/50/100/200 epochs, with and without bootstrap resampling, "
                         "and select training and rule together on the validation half")
    a = ap.parse_args()
    rr = tuple(a.rods)
    pts_train = ensemble.sample_points(a.train, a.seed, rr)
    pts_held = ensemble.sample_points(a.heldout, a.seed + 1, rr)
    pts_fresh = ensemble.sample_points(a.fresh, a.seed + 2, rr)

    sig = np.array([a.train, a.heldout, a.steps, a.sample_every, a.seed, rr[0], rr[1], int(a.turnover)], np.int64)
    if a.load_data:
        z = np.load(a.load_data)
        if not np.array_equal(z["sig"], sig):
            raise SystemExit(f"{a.load_data} was generated with other sweep settings")
        y_train, y_held = z["y_train"], z["y_held"]
        gen_gpu_s, held_gpu_s, gen_build_s = float(z["gen_gpu_s"]), float(z["held_gpu_s"]), float(z["gen_build_s"])
    else:
        y_train, gen_gpu_s, gen_build_s = generate(pts_train, a.steps, a.sample_every, turnover=a.turnover)
        y_held, held_gpu_s, _ = generate(pts_held, a.steps, a.sample_every, turnover=a.turnover)
        if a.save_data:
            np.savez(a.save_data, sig=sig, y_train=y_train, y_held=y_held, gen_gpu_s=gen_gpu_s,
                     held_gpu_s=held_gpu_s, gen_build_s=gen_build_s)
    batched_s_per_point = (gen_gpu_s + held_gpu_s) / (a.train + a.heldout)
    if a.retime_batched > 0:                 # the rerun cost from a fresh packed batch of this build
        _, rt_gpu_s, _ = generate(pts_train[:a.retime_batched], a.steps, a.sample_every, batch=a.retime_batched,
                                  turnover=a.turnover)
        batched_s_per_point = rt_gpu_s / a.retime_batched

    x_train = ensemble.features(pts_train, rr)
    x_held = ensemble.features(pts_held, rr)
    ens = MLPEnsemble(n_nets=5, seed=a.seed)
    t0 = time.perf_counter()
    hist = ens.fit(x_train, y_train, epochs=a.epochs)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0

    mean_h, std_h, _ = ens.predict(x_held)
    fb_h = fallback_mask(mean_h, std_h, a.threshold)
    blended = np.where(fb_h[:, None], y_held, mean_h)          # fallback points take the plain result
    err_surrogate = rel_error(mean_h, y_held)
    err_with_fallback = rel_error(blended, y_held)
    err_mean_predictor = rel_error(np.broadcast_to(y_train.mean(axis=0), y_held.shape), y_held)

    x_fresh = ensemble.features(pts_fresh, rr)
    ens.predict(x_fresh)                                        # warm-up: the inference buffers exist after it
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    mean_f, std_f, _ = ens.predict(x_fresh)
    torch.cuda.synchronize()
    infer_s = time.perf_counter() - t0
    fb_f = fallback_mask(mean_f, std_f, a.threshold)
    n_fb = int(fb_f.sum())
    surrogate_s = infer_s + n_fb * batched_s_per_point

    floored = {}
    if a.floor > 0:
        scale = a.floor * y_train.std(axis=0)
        fbh2 = (std_h > a.threshold * np.maximum(np.abs(mean_h), scale)).any(axis=1)
        fbf2 = (std_f > a.threshold * np.maximum(np.abs(mean_f), scale)).any(axis=1)
        s2 = infer_s + int(fbf2.sum()) * batched_s_per_point
        floored = {"floor": a.floor, "fallback_fraction": float(fbf2.mean()),
                   "heldout_fallback_fraction": float(fbh2.mean()),
                   "heldout_rel_error_with_fallback": rel_error(np.where(fbh2[:, None], y_held, mean_h), y_held),
                   "surrogate_sweep_points_per_s": a.fresh / s2}
    run_s, run_samples = per_run_seconds(pts_fresh, a.steps, a.per_run_sample, a.turnover)
    # rule selection on one half of the held-out runs, its error reported on the other half
    from .surrogate import fallback_mask as fbm, select_rule
    half = a.heldout // 2
    spread = y_train.std(axis=0)
    best, rules = select_rule(mean_h[:half], std_h[:half], y_held[:half], mean_f, std_f, spread, infer_s,
                              batched_s_per_point, run_s, target_col=0, max_err=a.max_err)
    selected = None
    if best is not None:
        sc = best["floor"] * spread if best["floor"] > 0 else None
        fb_t = fbm(mean_h[half:], std_h[half:], best["threshold"], best["outputs"], sc)
        blend_t = np.where(fb_t[:, None], y_held[half:], mean_h[half:])
        selected = dict(best, test_points=int(a.heldout - half), test_fallback=float(fb_t.mean()),
                        test_rel_error=rel_error(blend_t, y_held[half:]))
    grid, chosen = [], None
    if a.train_grid:
        for boot in (False, True):
            for ep in (25, 50, 100, 200):
                e2 = MLPEnsemble(n_nets=5, seed=a.seed)
                e2.fit(x_train, y_train, epochs=ep, bootstrap=boot)
                mh, sh, _ = e2.predict(x_held)
                mf, sf, _ = e2.predict(x_fresh)
                b2, _ = select_rule(mh[:half], sh[:half], y_held[:half], mf, sf, spread, infer_s,
                                    batched_s_per_point, run_s, target_col=0, max_err=a.max_err)
                row = {"epochs": ep, "bootstrap": boot, "validation_rel_error_surrogate": rel_error(mh[:half],
                                                                                                y_held[:half]),
                       "best_rule": b2}
                if b2 is not None:
                    sc = b2["floor"] * spread if b2["floor"] > 0 else None
                    fb_t = fbm(mh[half:], sh[half:], b2["threshold"], b2["outputs"], sc)
                    row["test_fallback"] = float(fb_t.mean())
                    row["test_rel_error"] = rel_error(np.where(fb_t[:, None], y_held[half:], mh[half:]),
                                                      y_held[half:])
                    row["test_rel_error_surrogate"] = rel_error(mh[half:], y_held[half:])
                grid.append(row)
        ok = [r for r in grid if r["best_rule"] is not None]
        chosen = max(ok, key=lambda r: r["best_rule"]["points_per_s"]) if ok else None
    out = {"steps_per_run": a.steps, "turnover": a.turnover, "train_grid": grid, "selected_training": chosen,
           "batched_s_per_point": batched_s_per_point, "batched_retimed_on": a.retime_batched, "rods_range": rr, "train_points": a.train, "heldout_points": a.heldout,
           "fresh_points": a.fresh, "outputs": OUTPUTS,
           "plain_per_run_points_per_s": 1.0 / run_s, "per_run_sample_s": run_samples,
           "plain_batched_points_per_s": 1.0 / batched_s_per_point,
           "surrogate_inference_points_per_s": a.fresh / infer_s,
           "fallback_fraction": n_fb / a.fresh, "threshold": a.threshold,
           "surrogate_sweep_points_per_s": a.fresh / surrogate_s,
           "gain_vs_plain_per_run": (a.fresh / surrogate_s) * run_s,
           "gain_vs_plain_batched": (a.fresh / surrogate_s) * batched_s_per_point,
           "heldout_rel_error_surrogate": err_surrogate, "heldout_rel_error_with_fallback": err_with_fallback,
           "heldout_rel_error_mean_predictor": err_mean_predictor, "heldout_fallback_fraction": float(fb_h.mean()),
           "floored_rule": floored,
           "selected_rule": selected, "max_err_contraction_rate": a.max_err, "rules": rules,
           "train_loss_first_last": [hist[0], hist[-1]], "train_s": train_s, "epochs": a.epochs,
           "data_gpu_s": gen_gpu_s + held_gpu_s, "data_build_s": gen_build_s}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
