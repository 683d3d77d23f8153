"""A small packed sweep end to end: sampled points, one batch, observables per point."""
import numpy as np
import pytest

from softbox_b200 import ensemble

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def test_small_sweep_runs_and_reports_every_point():
    pts = ensemble.sample_points(6, seed=3, rods_range=(2000, 5000))
    r = ensemble.run_ensemble(pts, steps=300, sample_every=100)
    for key in ("contraction_rate", "largest_fraction", "stress_pa"):
        assert r[key].shape == (6,) and np.isfinite(r[key]).all(), key
    assert (r["largest_fraction"] > 0).all() and (r["largest_fraction"] <= 1).all()
    assert r["rms_um"].shape == (4, 6) and r["ms_per_step"] > 0
    x = ensemble.features(pts)
    assert x.shape == (6, 6) and (x >= 0).all() and (x <= 1).all()


def test_sweep_with_turnover_runs_each_points_turnover():
    """turnover=True: each point's network runs its actin turnover (the per-network pools
    move: monomers taken by growth), the outputs stay finite, and the packed runs equal
    their turnover runs alone (checked at the array level by test_gpu_batch_turnover)."""
    pts = ensemble.sample_points(4, seed=5, rods_range=(2000, 4000))
    r = ensemble.run_ensemble(pts, steps=300, sample_every=100, turnover=True)
    for key in ("contraction_rate", "largest_fraction", "stress_pa"):
        assert r[key].shape == (4,) and np.isfinite(r[key]).all(), key
    assert (r["largest_fraction"] > 0).all() and (r["largest_fraction"] <= 1).all()
    plain = ensemble.run_ensemble(pts, steps=300, sample_every=100)
    assert not np.array_equal(r["rms_um"], plain["rms_um"])
