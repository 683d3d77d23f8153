"""Free-running rods against slender-rod theory (the free Brownian diffusion workload).

1,024 rods of 1.0 um, radius 4 nm, in water (eta = 1 mPa s), dt = 10 us, Philox noise.
Estimator: the per-step displacement of every rod projected on its start-of-step body
frame, so var(d . u) = 2 D_par dt, var(d . y) = var(d . z) = 2 D_perp dt and the rotation
of u about y / z gives 2 D_rot dt; about 1e6 samples per coefficient (0.14 % statistical
error). Theory: D = kT / gamma with the slender-rod drag of DragTensorSystem.rodDragSI
(DragTensorSystem.java:33-45); the coefficients must land within 2 % of it.
"""
import math

import numpy as np
import pytest

from softbox_b200 import scenes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _frame(b, n):
    c = b["coord"].reshape(3, n).astype(np.float64)
    u = b["uVec"].reshape(3, n).astype(np.float64)
    y = b["yVec"].reshape(3, n).astype(np.float64)
    z = np.cross(u.T, y.T).T
    return c, u, y, z


def test_free_rod_diffusion_matches_slender_rod_theory():
    from softbox_b200.engine import FreeRods
    n, dt, steps = 1024, 1.0e-5, 1000
    f = scenes.free_rods_box(n=n, length_um=1.0, radius_um=0.004, box_um=10.0, aeta=1.0e-3, dt=dt)
    rods = FreeRods(f)
    g = scenes.rod_drag_si(1.0, 0.004, 1.0e-3)
    d_par = scenes.KT / g[0] * 1e12           # um^2/s
    d_perp = scenes.KT / g[1] * 1e12
    d_rot = scenes.KT / g[4]                   # rad^2/s
    # the stated theory values of the workload (slender-rod law, water, kT = 4.11 pN nm)
    assert abs(d_par - 3.03) < 0.02 and abs(d_perp - 1.85) < 0.02 and abs(d_rot - 16.4) < 0.2
    par, perp, rot = [], [], []
    prev = {k: rods.pull(k) for k in ("coord", "uVec", "yVec")}
    for t in range(steps):
        rods.run(t, 1, noise="philox", philox_seed=0x5B0C0)
        cur = {k: rods.pull(k) for k in ("coord", "uVec", "yVec")}
        c0, u0, y0, z0 = _frame(prev, n)
        c1, u1, _, _ = _frame(cur, n)
        d = c1 - c0
        par.append((d * u0).sum(0))
        perp.append((d * y0).sum(0))
        perp.append((d * z0).sum(0))
        du = u1 - u0
        rot.append((du * y0).sum(0))
        rot.append((du * z0).sum(0))
        prev = cur
    est = {
        "D_par": np.var(np.concatenate(par)) / (2 * dt),
        "D_perp": np.var(np.concatenate(perp)) / (2 * dt),
        "D_rot": np.var(np.concatenate(rot)) / (2 * dt),
    }
    theory = {"D_par": d_par, "D_perp": d_perp, "D_rot": d_rot}
    for k in est:
        rel = est[k] / theory[k] - 1.0
        assert abs(rel) < 0.02, f"{k}: measured {est[k]:.5g}, theory {theory[k]:.5g} ({100 * rel:+.2f} %)"
    # the rods stay unit-length rigid bodies
    u = rods.pull("uVec").reshape(3, n)
    assert np.allclose(np.linalg.norm(u, axis=0), 1.0, atol=1e-5)
    assert math.isfinite(float(est["D_rot"]))
