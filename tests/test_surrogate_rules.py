"""Fallback-rule selection of the surrogate sweep (CPU, synthetic ensemble outputs)."""
import numpy as np

from softbox_b200.surrogate import fallback_mask, select_rule


def test_fallback_mask_outputs_and_floor():
    mean = np.array([[1.0, 0.0, 5.0], [0.01, 2.0, 5.0]])
    std = np.array([[0.05, 0.01, 0.1], [0.005, 0.05, 0.1]])
    assert fallback_mask(mean, std, 0.1).tolist() == [True, True]           # output 1 / output 0 near zero
    assert fallback_mask(mean, std, 0.1, outputs=(0,)).tolist() == [False, True]
    assert fallback_mask(mean, std, 0.1, outputs=(0,), scale=[0.1, 1, 1]).tolist() == [False, False]


def test_select_rule_meets_the_bound_and_prefers_fewer_fallbacks():
    rng = np.random.default_rng(0)
    n = 400
    y = rng.normal(1.0, 0.5, size=(n, 3))
    noisy = rng.uniform(size=n) < 0.3                     # 30 % of points: wrong and uncertain
    mean = y + np.where(noisy[:, None], rng.normal(0, 1.0, size=(n, 3)), rng.normal(0, 0.01, size=(n, 3)))
    std = np.where(noisy[:, None], 0.8, 0.01) * np.ones((n, 3))
    best, rows = select_rule(mean[:200], std[:200], y[:200], mean[200:], std[200:], y.std(axis=0), 0.01, 0.1, 1.0,
                             max_err=0.05)
    assert best is not None and best["validation_rel_error"][0] <= 0.05
    assert 0.2 < best["fresh_fallback"] < 0.45                # the noisy points and little else
    assert all(r["points_per_s"] <= best["points_per_s"] for r in rows if r["validation_rel_error"][0] <= 0.05)
