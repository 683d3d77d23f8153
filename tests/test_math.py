"""Accuracy of the portable double-precision transcendentals (softbox_b200/csrc/sbx_math.h)
that the CUDA kernels evaluate, against libm on the host."""
import numpy as np
import pytest


def ulp_err(y, ref):
    y = np.asarray(y, np.float64)
    ref = np.asarray(ref, np.float64)
    return np.abs(y - ref) / np.spacing(np.abs(ref))


def _eval(orc, which, x):
    x = np.ascontiguousarray(x, np.float64)
    y = np.empty_like(x)
    orc.m_eval(which, len(x), x, y)
    return y


@pytest.mark.parametrize("lo,hi", [(1e-7, 1.0), (1e-300, 1e300)])
def test_log_within_2ulp(orc, lo, hi):
    rng = np.random.default_rng(1)
    x = np.exp(rng.uniform(np.log(lo), np.log(hi), 200000))
    assert ulp_err(_eval(orc, 0, x), np.log(x)).max() <= 2.0


def test_exp_within_2ulp(orc):
    rng = np.random.default_rng(2)
    x = rng.uniform(-700, 700, 200000)
    x = np.concatenate([x, rng.uniform(-1, 1, 100000)])
    assert ulp_err(_eval(orc, 1, x), np.exp(x)).max() <= 2.0


@pytest.mark.parametrize("which,fn", [(2, np.sin), (3, np.cos)])
def test_sincos_within_2ulp(orc, which, fn):
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.uniform(0, 2 * np.pi, 200000), rng.uniform(-8, 8, 100000),
                        rng.uniform(-2.0 ** 20, 2.0 ** 20, 100000)])
    assert ulp_err(_eval(orc, which, x), fn(x)).max() <= 2.0


def test_boxmuller_float_results_match_libm(orc):
    """(float)Math.log/cos/sin of float arguments: the float results of the portable
    functions and of libm agree except in a vanishing fraction of cases."""
    rng = np.random.default_rng(4)
    u = rng.uniform(1e-7, 1.0, 1_000_000).astype(np.float32).astype(np.float64)
    th = (np.float32(2.0) * np.float32(3.14159265) * u.astype(np.float32)).astype(np.float64)
    diffs = 0
    for which, fn, x in ((0, np.log, u), (2, np.sin, th), (3, np.cos, th)):
        a = _eval(orc, which, x).astype(np.float32)
        b = fn(x).astype(np.float32)
        diffs += int((a != b).sum())
    assert diffs <= 3


def test_sincos_equals_sin_and_cos_bitwise(orc):
    """sincos (one argument reduction for both results, as the Box-Muller draws and the
    acos/asin Newton steps use it) gives the bits of sin and cos evaluated separately."""
    rng = np.random.default_rng(4)
    x = np.concatenate([rng.uniform(0, 2 * np.pi, 100000), rng.uniform(-8, 8, 50000),
                        rng.uniform(-2.0 ** 20, 2.0 ** 20, 50000), [0.0, -0.0, np.pi / 4, -np.pi / 2]])
    assert np.array_equal(_eval(orc, 4, x).view(np.uint64), _eval(orc, 2, x).view(np.uint64))
    assert np.array_equal(_eval(orc, 5, x).view(np.uint64), _eval(orc, 3, x).view(np.uint64))
