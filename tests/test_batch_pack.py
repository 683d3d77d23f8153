"""Packing of independent networks (CPU): every network's arrays come back unchanged."""
import numpy as np

from helpers import flat_arrays
from softbox_b200 import batch, scenes


def _nets():
    return [scenes.dense_contractile(scenes.dense_small(s, seed=sd, seed_bb=sd + 1, seed_fil=sd + 2))
            for s, sd in ((0.03, 11), (0.05, 22), (0.02, 33))]


def test_pack_unpack_round_trip():
    nets = _nets()
    packed, info = batch.pack_networks(nets)
    assert info["nNet"] == 3
    assert packed["fil"]["body"]["n"] == sum(n["fil"]["body"]["n"] for n in nets)
    for k, net in enumerate(nets):
        got = dict(flat_arrays(batch.unpack_network(packed, info, k)))
        want = dict(flat_arrays(net))
        assert len(got) > 40
        for name, arr in got.items():
            assert np.array_equal(arr, want[name]), name


def test_pack_tables():
    nets = _nets()
    packed, info = batch.pack_networks(nets)
    b = packed["batch"]
    gd = b["gridDims"].reshape(-1, 4)
    assert list(gd[:, 3]) == list(info["cells"][:-1])
    assert packed["grid"]["totalCells"] == int(info["cells"][-1])
    seeds = b["seeds"].reshape(-1, 3)
    assert [int(s) for s in seeds[:, 0]] == [n["seed"] for n in nets]
    key = b["segKey"].reshape(-1, 2)
    assert (key[:600, 0] == 0).all() and key[600, 0] == 1 and key[600, 1] == 0
    # cross-store indices are offset into the packed ranges
    s1 = int(info["seg"][1])
    e2 = packed["fil"]["end2NbrSlot"][s1:s1 + 10]
    assert (e2[e2 >= 0] >= s1).all()
