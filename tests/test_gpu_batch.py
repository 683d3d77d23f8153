"""Packed networks on the GPU: each network's trajectory equals its run alone, bit for bit.

Three networks of the benchmark composition at different sizes (600, 1,000 and 400 rods)
and seeds, packed into one scene and advanced 300 steps by the batched plan (one launch
per step phase for all three), against each network advanced alone by the single-network
plan (which equals the oracle, tests/test_gpu_parity.py).
"""
import numpy as np
import pytest

from helpers import assert_same, flat_arrays
from softbox_b200 import batch, scenes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _nets():
    return [scenes.dense_contractile(scenes.dense_small(s, seed=sd, seed_bb=sd + 1, seed_fil=sd + 2))
            for s, sd in ((0.03, 11), (0.05, 22), (0.02, 33))]


@pytest.mark.parametrize("mode", ["graph", "unfused"])
def test_batched_equals_each_network_alone(mode):
    from softbox_b200.engine import DenseNetwork
    nets = _nets()
    packed, info = batch.pack_networks(nets)
    ens = batch.BatchedNetworks(packed, info)
    ens.run(0, 300, mode=mode)
    alone = []
    for net in nets:
        d = DenseNetwork(net)
        d.run(0, 300, mode="graph")
        alone.append(d)
    torch.cuda.synchronize()
    host = ens.pull_all()
    moved = bound = 0
    for k, d in enumerate(alone):
        got = dict(flat_arrays(batch.unpack_network(host, info, k)))
        want = dict(flat_arrays(d.pull_all()))
        for name, arr in got.items():
            assert_same(want[name], arr, f"network {k} {name}")
        moved += int((want["fil.body.coord"] != nets[k]["fil"]["body"]["coord"]).sum())
        bound += int((want["mot.boundSeg"] >= 0).sum())
        d.close()
    assert moved > 0 and bound > 0
    ens.close()


def test_batched_launches_per_step_do_not_grow_with_networks():
    nets = _nets()
    one = batch.BatchedNetworks(*batch.pack_networks(nets[:1]))
    ens = batch.BatchedNetworks(*batch.pack_networks(nets))
    assert ens.kernels_per_step == one.kernels_per_step
    one.close()
    ens.close()
