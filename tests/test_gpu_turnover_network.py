"""A dense network with actin turnover (scenes.dense_turnover) on the GPU against the oracle.

1,000-rod network (the benchmark composition at 5 %), rates raised so that growth,
depolymerisation, severing, deaths with link and head release, splits and constant-actin
births all occur within 1,000 steps (10 biochem cadences). The graph path, the per-system
path and the fused kernel (its plan re-reading the chain topology after every cadence:
births into FREE slots put chain neighbours across its rod groups) are compared with the
oracle's TurnoverNetwork restatement array by array, bit for bit, after every 250 steps.
"""
import copy

import numpy as np
import pytest

from helpers import compare_scenes, oracle_turnover_network_run
from softbox_b200 import scenes
from softbox_b200.turnover import pool_fields

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def scene():
    return scenes.dense_turnover(scenes.dense_small(0.05), growth_rate=400.0, sever_rate=5.0)


@pytest.mark.parametrize("mode", ["graph", "unfused", "fused"])
def test_turnover_network_bitwise(orc_dm, scene, mode):
    from softbox_b200.engine import TurnoverNetwork
    host = copy.deepcopy(scene)
    net = TurnoverNetwork(copy.deepcopy(scene))
    assert mode != "fused" or net.fused_available
    m0 = int(host["fil"]["monomerCount"].sum())
    for t0 in range(0, 1000, 250):
        oracle_turnover_network_run(orc_dm, host, t0, 250)
        net.run(t0, 250, mode=mode)
        assert net.status() == 0
        torch.cuda.synchronize()
        names = compare_scenes({k: v for k, v in host.items() if k != "tcfg"}, net.pull_all(), skip=("coord64",))
        assert "turnover.pool" in names and "fil.body.coord" in names and "xl.linkState" in names
    t = host["turnover"]
    _, _, taken, returned = pool_fields(t["pool"])
    assert int(host["fil"]["monomerCount"].sum()) == m0 + taken - returned
    assert (t["seedNode"] >= 0).sum() > (scene["turnover"]["seedNode"] >= 0).sum()      # births happened
    assert (host["fil"]["filState"] < 0).any()                                           # deaths happened
    dead = host["fil"]["filState"] < 0
    xl = host["xl"]
    act = xl["linkState"] >= 0
    assert not dead[xl["linkFilA"][act]].any() and not dead[xl["linkFilB"][act]].any()
    bs = host["mot"]["boundSeg"]
    assert not dead[bs[bs >= 0]].any()
    net.close()
