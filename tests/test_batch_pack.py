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


def test_sweep_batch_with_turnover_packs_per_network_tables():
    """ensemble.build_batch(turnover=True): every point's network carries its own turnover
    seed, severing rate (its point's turnover rate), actin pool and birth request range, and
    each network unpacks to the arrays it was built with."""
    from softbox_b200 import ensemble
    pts = ensemble.sample_points(3, seed=4, rods_range=(2000, 3000))
    packed, info = ensemble.build_batch(pts, turnover=True)
    t = packed["turnover"]
    assert info["nNet"] == 3 and t["tbSeeds"].size == 3 and len(set(t["tbSeeds"].tolist())) == 3
    assert t["tbSlotBase"].tolist() == [int(v) for v in info["seg"]]
    assert t["tbBirthBase"][0] == 0 and np.all(np.diff(t["tbBirthBase"]) > 0)
    assert t["tbPools"].reshape(3, 4)[:, 0].min() > 0                     # initial [actin] per network
    for k, p in enumerate(pts):
        want = scenes.dense_turnover(ensemble.point_config(p), sever_rate=p.turnover,
                                     turnover_seed=p.seed ^ 0x0F0501)
        got = batch.unpack_network(packed, info, k)
        assert np.array_equal(got["turnover"]["seedNode"], want["turnover"]["seedNode"])
        assert np.array_equal(got["turnover"]["cofFrac"].view(np.uint32),
                              want["turnover"]["cofFrac"].view(np.uint32))
        assert np.array_equal(got["fil"]["body"]["coord"].view(np.uint32),
                              want["fil"]["body"]["coord"].view(np.uint32))
        assert np.float32(t["tb_cofilinParams"].reshape(3, 2)[k, 0]) == want["turnover"]["cofilinParams"][0]
