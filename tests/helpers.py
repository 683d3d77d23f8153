"""Shared test helpers: scene copies, oracle stepping and bitwise comparison."""
import copy

import numpy as np

from softbox_b200 import device as D, scenes


def host_copy(sc):
    return copy.deepcopy(sc)


def oracle_dense_run(orc, sc, t0, nsteps):
    """Advance a host scene with the oracle's DenseContractileHarness.cpuStep restatement."""
    desc = D.dense_desc(sc)
    orc.dense_run(desc, t0, nsteps)
    return sc


def assert_same(a, b, what=""):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    if a.dtype.kind == "f":
        ok = np.array_equal(a.view(np.uint32 if a.dtype == np.float32 else np.uint64),
                            b.view(np.uint32 if b.dtype == np.float32 else np.uint64))
    else:
        ok = np.array_equal(a, b)
    if not ok:
        diff = np.flatnonzero(a != b)
        raise AssertionError(f"{what}: {diff.size} of {a.size} entries differ; first at {diff[:5]}: "
                             f"{a.reshape(-1)[diff[:5]]} vs {b.reshape(-1)[diff[:5]]}")


def flat_arrays(sc, prefix=""):
    """(name, array) for every numpy array in a (nested) scene dict."""
    out = []
    for k, v in sc.items():
        if isinstance(v, dict):
            out += flat_arrays(v, prefix + k + ".")
        elif isinstance(v, np.ndarray):
            out.append((prefix + k, v))
    return out


def compare_scenes(host, dev_host, skip=()):
    """Bitwise comparison of every array of two host scenes; returns the names compared."""
    names = []
    dmap = dict(flat_arrays(dev_host))
    for name, arr in flat_arrays(host):
        if any(name.endswith(s) for s in skip) or name not in dmap:
            continue
        assert_same(arr, dmap[name], name)
        names.append(name)
    return names


def small_dense(scale=0.05, **kw):
    return scenes.dense_contractile(scenes.dense_small(scale, **kw))
