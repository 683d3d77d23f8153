"""Precision of FP32 rod centres against FP64 centre accumulation (the same kernels, the
same noise): the free Brownian rods of the diffusion workload over 1,000 steps stay within
1e-5 relative of the FP64-centre run, and the FP64 centres' float projection is what the
FP32 store holds."""
import numpy as np
import pytest

from softbox_b200 import scenes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def test_fp32_centres_within_1e5_of_fp64_over_1000_steps():
    from softbox_b200.engine import FreeRods
    f = scenes.free_rods_box(n=1024, length_um=1.0, radius_um=0.004, box_um=10.0, aeta=1.0e-3, dt=1.0e-5)
    r32 = FreeRods(f)
    r64 = FreeRods(f, fp64_coords=True)
    r32.run(0, 1000, noise="philox", philox_seed=0x5B0C0)
    r64.run(0, 1000, noise="philox", philox_seed=0x5B0C0)
    torch.cuda.synchronize()
    c32 = r32.pull("coord").astype(np.float64)
    c64 = r64.dev["body"]["coord64"].cpu().numpy()
    scale = np.abs(c64).max()
    err = np.abs(c32 - c64).max() / scale
    assert err < 1e-5, err
    assert np.array_equal(r64.pull("coord"), c64.astype(np.float32))   # FP32 store = rounded FP64 centre
    moved = np.abs(c64 - f["body"]["coord"].astype(np.float64)).max()
    assert moved > 1e3 * err * scale                                    # the walk itself is far above the error
