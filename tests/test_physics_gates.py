"""The reference harnesses' physics gates on the CPU oracle (the same sequences run on the
GPU in test_gpu_physics_gates.py, where they must also equal these results bit for bit).
Scenes and step sequences: tests/physics_gates.py."""
import math

import numpy as np
import pytest

import physics_gates as G


@pytest.mark.parametrize("force", [0.0, 2.0e-12])
def test_motor_off_rate_gate(orc_dm, force):
    """releases / bound-steps == k_off(F) dt (MotorBindingHarness.java:437-446: 5 %); here
    also within 5 binomial standard errors."""
    m = G.release_bed(force=force)
    G.run_release(G.OracleBackend(orc_dm), m, 3000)
    p, want, se = G.off_rate(m["stats"], force)
    assert abs(p - want) / want < 0.05, (p, want)
    assert abs(p - want) < 5 * se, (p, want, se)


def test_confined_rod_equipartition_gate(orc_dm):
    """<theta^2> == 4 kT dt / (gamma c (2 - c)) within 2 % (ThermostatDiag.java:45-58)."""
    sc = G.confined_rods(reps=2000)
    meas, pred = G.run_equipartition(G.OracleBackend(orc_dm), sc, burn=4000, steps=8000, every=2)
    assert abs(meas / pred - 1.0) < 0.02, meas / pred


def test_crosslinker_rest_hold_gate(orc_dm):
    """CrosslinkerHarness check #1: exact rest => max |d coord| == 0; stretched => the
    centre of mass stays put (< 1e-3 of the relaxation) and the separation relaxes toward
    rest (CrosslinkerHarness.java:279-297)."""
    drift, rel, sep0, sep_end = G.rest_hold(G.OracleBackend(orc_dm))
    assert drift == 0.0
    assert rel < 1e-3 and sep_end < sep0 and sep_end > 0.9 * G.XL_REST, (rel, sep0, sep_end)


def test_crosslinker_stretch_relaxation_gate(orc_dm):
    """CrosslinkerHarness check #2: measured per-step decay == fracMove (g_par/g_perp) L within
    0.1 %, and dt-independent within 0.1 % (CrosslinkerHarness.java:300-323)."""
    be = G.OracleBackend(orc_dm)
    k_obs, k_pred, n = G.stretch_decay(be, 1.0e-5)
    k10, _, n10 = G.stretch_decay(be, 1.0e-6)
    assert n > 100 and n10 > 100
    assert abs(k_obs - k_pred) / k_pred < 1e-3, (k_obs, k_pred)
    assert abs(k_obs - k10) / k_obs < 1e-3, (k_obs, k10)
