"""What the trained surrogate gains over the sweep without it, on a small sweep run here:
plain batched runs generate the training and held-out data, the 5-member MLP ensemble is
trained on the GPU by the library's kernels, and fresh points are predicted, falling back to
a plain run wherever the ensemble disagrees. Reported and checked: the sweep rate (points/s)
of surrogate + fallback against the plain per-run GPU sweep (each point's network alone on
the single-network plan), and the contraction-rate error of surrogate + fallback against the
plain runs on held-out points, next to the error of predicting the training mean."""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def test_surrogate_gain_over_plain_per_run_sweep():
    from softbox_b200 import ensemble
    from softbox_b200.surrogate import MLPEnsemble, fallback_mask
    from softbox_b200.sweep_surrogate import generate, per_run_seconds, rel_error
    rr, steps, every = (2000, 6000), 400, 100
    pts_train = ensemble.sample_points(384, 31, rr)
    pts_held = ensemble.sample_points(96, 32, rr)
    pts_fresh = ensemble.sample_points(20000, 33, rr)
    y_train, gen_s, _ = generate(pts_train, steps, every)
    y_held, held_s, _ = generate(pts_held, steps, every)
    rerun_s = (gen_s + held_s) / (len(pts_train) + len(pts_held))      # plain batched cost per point
    ens = MLPEnsemble(n_nets=5, seed=3)
    ens.fit(ensemble.features(pts_train, rr), y_train, epochs=100, bootstrap=True)
    mean_h, std_h, _ = ens.predict(ensemble.features(pts_held, rr))
    spread = y_train.std(axis=0)
    rule = dict(threshold=0.2, outputs=(0,), scale=0.5 * spread)
    fb_h = fallback_mask(mean_h, std_h, **rule)
    blend = np.where(fb_h[:, None], y_held, mean_h)
    err_fb = rel_error(blend, y_held)
    err_sur = rel_error(mean_h, y_held)
    err_mean = rel_error(np.broadcast_to(y_train.mean(axis=0), y_held.shape), y_held)
    x_fresh = ensemble.features(pts_fresh, rr)
    ens.predict(x_fresh)
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(True), torch.cuda.Event(True)
    s.record()
    mean_f, std_f, _ = ens.predict(x_fresh)
    e.record()
    torch.cuda.synchronize()
    infer_s = s.elapsed_time(e) / 1e3
    n_fb = int(fallback_mask(mean_f, std_f, **rule).sum())
    sweep_rate = len(pts_fresh) / (infer_s + n_fb * rerun_s)
    per_run_s, _ = per_run_seconds(pts_fresh, steps, sample=4)
    gain = sweep_rate * per_run_s
    print(json.dumps({"gain_vs_plain_per_run": gain, "surrogate_sweep_points_per_s": sweep_rate,
                      "plain_per_run_points_per_s": 1.0 / per_run_s, "plain_batched_points_per_s": 1.0 / rerun_s,
                      "fresh_fallback_fraction": n_fb / len(pts_fresh), "heldout_fallback_fraction": float(fb_h.mean()),
                      "heldout_rel_error_with_fallback": err_fb, "heldout_rel_error_surrogate": err_sur,
                      "heldout_rel_error_mean_predictor": err_mean}))
    assert gain > 2.0, gain
    assert err_fb[0] < err_mean[0], (err_fb, err_mean)
