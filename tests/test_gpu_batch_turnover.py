"""Packed networks with actin turnover: each network's arrays, turnover state and actin
pool after 600 steps (6 biochem cadences) equal its TurnoverNetwork run alone, bit for bit
(three networks of different sizes, seeds, turnover seeds and severing rates, rates raised
so that deaths, releases, splits and births occur)."""
import copy

import numpy as np
import pytest

from helpers import assert_same, flat_arrays
from softbox_b200 import batch, scenes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _nets():
    out = []
    for k, (sz, sd, sev) in enumerate(((0.03, 11, 4.0), (0.05, 22, 6.0), (0.02, 33, 8.0))):
        cfg = scenes.dense_small(sz, seed=sd, seed_bb=sd + 1, seed_fil=sd + 2)
        out.append(scenes.dense_turnover(cfg, growth_rate=400.0, sever_rate=sev, turnover_seed=1000 + k))
    return out


def test_batched_turnover_equals_each_network_alone():
    from softbox_b200.engine import TurnoverNetwork
    nets = _nets()
    packed, info = batch.pack_networks(copy.deepcopy(nets))
    ens = batch.BatchedTurnoverNetworks(packed, info)
    ens.run(0, 600)
    alone = []
    for net in nets:
        d = TurnoverNetwork(copy.deepcopy(net))
        d.run(0, 600)
        alone.append(d)
    torch.cuda.synchronize()
    host = ens.pull_all()
    deaths = births = 0
    for k, d in enumerate(alone):
        got = dict(flat_arrays(batch.unpack_network(host, info, k)))
        want_all = d.pull_all()
        want = dict(flat_arrays(want_all))
        for name, arr in got.items():
            assert_same(want[name], arr, f"network {k} {name}")
        deaths += int((want_all["fil"]["filState"] < 0).sum())
        births += int((want_all["turnover"]["seedNode"] >= 0).sum() - (nets[k]["turnover"]["seedNode"] >= 0).sum())
        d.close()
    assert deaths > 0 and births > 0
    ens.close()
