"""Device observables against the oracle's restatement (bit for bit), single and packed."""
import numpy as np
import pytest

from helpers import assert_same, oracle_observables, small_dense
from softbox_b200 import batch, scenes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def test_observables_bitwise_single(orc_dm):
    from softbox_b200.engine import DenseNetwork
    from softbox_b200.observables import Observables
    net = DenseNetwork(small_dense(0.05))
    net.run(0, 300, mode="graph")
    obs = Observables(net)
    s = obs.sample()
    host = net.pull_all()
    ext, st, cl, label = oracle_observables(orc_dm, host)
    assert_same(ext[:, 0], s["rms_um"], "R_rms")
    assert_same(st, s["stress_pa"], "stress")
    assert_same(cl[:, 0], s["largest"], "largest")
    assert_same(label, obs.label.cpu().numpy(), "labels")
    assert s["stress_pa"][0] != 0 and 0 < s["largest_fraction"][0] <= 1
    net.close()


def test_observables_batched_equal_single():
    from softbox_b200.engine import DenseNetwork
    from softbox_b200.observables import Observables
    nets = [scenes.dense_contractile(scenes.dense_small(sz, seed=sd, seed_bb=sd + 1, seed_fil=sd + 2))
            for sz, sd in ((0.03, 5), (0.05, 6))]
    packed, info = batch.pack_networks(nets)
    ens = batch.BatchedNetworks(packed, info)
    ens.run(0, 200)
    sb = Observables(ens).sample()
    for k, sc in enumerate(nets):
        d = DenseNetwork(sc)
        d.run(0, 200, mode="graph")
        s1 = Observables(d).sample()
        for key in ("rms_um", "stress_pa", "largest", "active"):
            assert_same(np.asarray(s1[key])[:1], np.asarray(sb[key])[k:k + 1], f"network {k} {key}")
        d.close()
    ens.close()
