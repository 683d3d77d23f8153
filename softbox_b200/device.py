"""Moving host scenes (softbox_b200.scenes) to the device and describing them to the library.

A scene is a dict of stores; each store is a dict of planar-SoA numpy arrays named like
the reference store fields. `to_device` mirrors every array as a torch CUDA tensor (the
FIRST_EXECUTION upload of the reference's TaskGraphs); `to_host` pulls them back
(UNDER_DEMAND). The *_desc helpers fill the ctypes descriptors of include/softbox_b200.h.
"""
import numpy as np

from . import abi_types as T


class DeviceFill:
    """A scratch array that exists only on the device: to_device creates it filled with
    `value` (no host copy, no transfer)."""

    def __init__(self, n, value, dtype):
        self.n, self.value, self.dtype = int(n), value, np.dtype(dtype)


def to_device(obj, device="cuda"):
    import torch
    if isinstance(obj, dict):
        return {k: to_device(v, device) for k, v in obj.items()}
    if isinstance(obj, np.ndarray):
        return torch.from_numpy(np.ascontiguousarray(obj)).to(device)
    if isinstance(obj, DeviceFill):
        tdt = {np.dtype(np.int32): torch.int32, np.dtype(np.float32): torch.float32}[obj.dtype]
        return torch.full((obj.n,), obj.value, dtype=tdt, device=device)
    return obj


def counts_block(dev):
    """Moves the three per-execution counts blocks of a device dense scene (mot.counts,
    mini.bbCounts, fil.counts: 4 int32 each, the reference's EVERY_EXECUTION uploads) into
    one contiguous 12-int32 device tensor, points the scene at its three slices and returns
    it, so that a host uploads one step's counts with one 48-byte copy."""
    import torch
    slots = ((dev["mot"], "counts"), (dev["mini"], "bbCounts"), (dev["fil"], "counts"))
    assert all(s[k].numel() == 4 and s[k].dtype == torch.int32 for s, k in slots)
    block = torch.empty(12, dtype=torch.int32, device=slots[0][0][slots[0][1]].device)
    for j, (s, k) in enumerate(slots):
        block[4 * j:4 * j + 4].copy_(s[k])
        s[k] = block[4 * j:4 * j + 4]
    return block


def to_host(obj):
    if isinstance(obj, dict):
        return {k: to_host(v) for k, v in obj.items()}
    if hasattr(obj, "detach"):
        return obj.detach().cpu().numpy()
    return obj


def body_desc(b, d=None):
    d = d or T.RigidBody()
    T.fill(d, b)
    d.n = int(b["n"])
    return d


def filament_desc(f, d=None):
    d = d or T.FilamentStoreDesc()
    body_desc(f["body"], d.body)
    T.fill(d, f)
    return d


def dense_desc(sc):
    """DenseSceneDesc over a scene whose arrays are numpy (host) or torch (device)."""
    d = T.DenseSceneDesc()
    filament_desc(sc["fil"], d.fil)
    body_desc(sc["mot"]["body"], d.mot.body)
    T.fill(d.mot, sc["mot"])
    d.mot.nMotors = int(sc["mot"]["nMotors"])
    T.fill(d.dim, sc["dim"])
    d.dim.nDimers = int(sc["dim"]["nDimers"])
    body_desc(sc["mini"]["backbone"], d.mini.backbone)
    T.fill(d.mini, sc["mini"])
    d.mini.nBackbones = int(sc["mini"]["nBackbones"])
    d.mini.nDimers = int(sc["mini"]["nDimers"])
    T.fill(d.xl, sc["xl"])
    d.xl.nLinks = int(sc["xl"]["nLinks"])
    T.fill(d.grid, sc["grid"])
    d.grid.cap = int(sc["grid"]["cap"])
    d.grid.totalCells = int(sc["grid"]["totalCells"])
    T.fill(d, sc)
    d.seed, d.seedBb = int(sc["seed"]), int(sc["seedBb"])
    d.xlinkOn, d.xlUnbind = int(sc["xlinkOn"]), int(sc["xlUnbind"])
    return d


def add_coord64(store_body, device=None):
    """Attach an FP64 centre array initialised from the FP32 coord (numpy or torch)."""
    c = store_body["coord"]
    if hasattr(c, "double"):
        store_body["coord64"] = c.double().contiguous()
    else:
        store_body["coord64"] = c.astype(np.float64)
    return store_body
