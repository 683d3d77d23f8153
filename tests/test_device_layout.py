"""Host-side layout of a device dense scene (no GPU: the same helpers on CPU tensors)."""
import numpy as np
import torch

from softbox_b200 import device as D
from softbox_b200 import scenes


def test_counts_block_is_one_contiguous_copy_target():
    host = scenes.dense_contractile(scenes.dense_small(0.02))
    dev = D.to_device({k: v for k, v in host.items() if k not in ("cfg", "tcfg")}, "cpu")
    block = D.counts_block(dev)
    want = np.concatenate([host["mot"]["counts"], host["mini"]["bbCounts"], host["fil"]["counts"]])
    assert block.dtype == torch.int32 and block.is_contiguous() and block.numel() == 12
    assert np.array_equal(block.numpy(), want)
    # the scene's three arrays are views of the block: one 48-byte write updates all three
    for j, (s, k) in enumerate(((dev["mot"], "counts"), (dev["mini"], "bbCounts"), (dev["fil"], "counts"))):
        assert s[k].data_ptr() == block.data_ptr() + 16 * j
    block.copy_(torch.arange(12, dtype=torch.int32))
    assert dev["mini"]["bbCounts"].tolist() == [4, 5, 6, 7]
    assert dev["fil"]["counts"].tolist() == [8, 9, 10, 11]
