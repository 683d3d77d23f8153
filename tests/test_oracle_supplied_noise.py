"""CPU checks of the oracle's supplied-noise mode of the dense step (test infrastructure).

(1) Noise equal to the Wang-hash Box-Muller draws of BrownianForceSystem.brownianForce
(BrownianForceSystem.java:44-106), fed through the supplied-noise path, reproduces the
ordinary step bit for bit: the noise layout ([step][6][body], stores in the step's order)
and the seeds per store are the ones the step uses.
(2) With the noise supplied, the libm build (the reference's platform math) and the build
on the kernels' portable transcendentals give the same bits: the draws are the only place
where the two math libraries disagree on this network.
"""
import copy

import numpy as np

from helpers import compare_scenes, small_dense
from softbox_b200 import device as D


def _wang_noise(orc, n, t0, nsteps, seed):
    out = np.zeros((nsteps, 6, n), np.float32)
    for k in range(nsteps):
        orc.gauss6_wang(n, t0 + k, seed, out[k])
    return out


def _strip(sc):
    return {k: v for k, v in sc.items() if k not in ("cfg", "tcfg")}


def test_supplied_wang_draws_reproduce_the_step(orc_dm):
    sc = small_dense(0.05)
    orc_dm.dense_run(D.dense_desc(sc), 0, 100)
    a, b = copy.deepcopy(sc), copy.deepcopy(sc)
    t0, n = 100, 60
    nf = _wang_noise(orc_dm, sc["fil"]["body"]["n"], t0, n, int(sc["fil"]["counts"][2]))
    nm = _wang_noise(orc_dm, sc["mot"]["body"]["n"], t0, n, int(sc["seed"]))
    nb = _wang_noise(orc_dm, sc["mini"]["backbone"]["n"], t0, n, int(sc["seedBb"]))
    orc_dm.dense_run(D.dense_desc(a), t0, n)
    orc_dm.dense_run_supplied(D.dense_desc(b), t0, n, nf, nm, nb)
    assert len(compare_scenes(_strip(a), _strip(b))) > 80


def test_supplied_noise_libm_equals_devmath(orc, orc_dm):
    sc = small_dense(0.05)
    orc_dm.dense_run(D.dense_desc(sc), 0, 200)
    for s, b in (("fil", "body"), ("mot", "body"), ("mini", "backbone")):
        D.add_coord64(sc[s][b])
    a, b = copy.deepcopy(sc), copy.deepcopy(sc)
    rng = np.random.default_rng(3)
    n = 400
    nf = rng.standard_normal((n, 6, sc["fil"]["body"]["n"]), dtype=np.float32)
    nm = rng.standard_normal((n, 6, sc["mot"]["body"]["n"]), dtype=np.float32)
    nb = rng.standard_normal((n, 6, sc["mini"]["backbone"]["n"]), dtype=np.float32)
    orc.dense_run_supplied(D.dense_desc(a), 200, n, nf, nm, nb)
    orc_dm.dense_run_supplied(D.dense_desc(b), 200, n, nf, nm, nb)
    assert (a["mot"]["boundSeg"] >= 0).sum() > 5
    assert len(compare_scenes(_strip(a), _strip(b))) > 80
