"""GPU parity on the benchmark network itself: the dense contractile network of 2,000
filaments x 10 rods (20,000 rods), 200 minifilaments (6,400 heads) and 4,000 crosslinkers
with FP64 centres, the configuration bench.py times.

The network is first advanced 2,000 steps by the oracle, so that about 700 heads are bound
(the count is still near 120 at step 20), then 1,000 more steps run on the fused
persistent kernel and on the CUDA-graph path and every store array is compared with the
oracle bit for bit every 250 steps (DenseContractileHarness.cpuStep,
DenseContractileHarness.java:350-429). The fused kernel's fixed-capacity fallbacks (row
overflow lists, payloads read from global memory past the staging buffers, the
repeated-minimum walk of long motor rows) are forced on the same network by lowering the
capacities, and must give the same bits.

The supplied-noise test is the oracle contract of the benchmark: both implementations
consume the same seeded Gaussian array (the draws of BrownianForceSystem.brownianForce,
BrownianForceSystem.java:44-106, are replaced), and the CUDA path is compared with the oracle
built on the platform libm (the reference's Math.* functions) for 1,000 steps: integer
arrays exactly, centres and orientations within 1e-5 relative.
"""
import copy

import numpy as np
import pytest

from helpers import compare_scenes, oracle_dense_run
from softbox_b200 import device as D, scenes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

WARM = 2000      # oracle steps before the comparison window
NSTEPS = 1000    # compared steps
CHECK = 250      # comparison interval


def _strip(sc):
    return {k: v for k, v in sc.items() if k not in ("cfg", "tcfg")}


@pytest.fixture(scope="module")
def warm_c1(orc_dm):
    sc = scenes.dense_contractile(scenes.C1)
    for s, b in (("fil", "body"), ("mot", "body"), ("mini", "backbone")):
        D.add_coord64(sc[s][b])
    oracle_dense_run(orc_dm, sc, 0, WARM)
    return sc


@pytest.fixture(scope="module")
def oracle_checkpoints(orc_dm, warm_c1):
    ref = copy.deepcopy(warm_c1)
    out = []
    for c in range(NSTEPS // CHECK):
        oracle_dense_run(orc_dm, ref, WARM + c * CHECK, CHECK)
        out.append(copy.deepcopy(_strip(ref)))
    return out


def test_warm_state_is_representative(warm_c1):
    """The comparison window starts where binding has built up (the bench's warm state)."""
    assert warm_c1["fil"]["body"]["n"] == 20000
    assert warm_c1["mot"]["nMotors"] == 6400
    assert (warm_c1["mot"]["boundSeg"] >= 0).sum() > 600
    assert (warm_c1["xl"]["linkState"] >= 0).sum() > 3800


@pytest.mark.parametrize("mode", ["fused", "graph"])
def test_benchmark_network_1000_steps_bitwise(warm_c1, oracle_checkpoints, mode):
    from softbox_b200.engine import DenseNetwork
    net = DenseNetwork(copy.deepcopy(warm_c1))
    assert mode != "fused" or net.fused_available
    net.fused_stats(reset=True)
    for c in range(NSTEPS // CHECK):
        net.run(WARM + c * CHECK, CHECK, mode=mode)
        assert net.status() == 0
        torch.cuda.synchronize()
        names = compare_scenes(oracle_checkpoints[c], D.to_host(net.dev))
        assert len(names) > 80
        assert "fil.body.coord64" in names and "grid.reachSeg" in names and "mot.boundSeg" in names
    if mode == "fused":
        st = net.fused_stats()
        # at the compiled capacities the benchmark network overflows a few grid cells'
        # fixed slots; it never needs the payload fallbacks
        assert st["cell_list"] > 0, st
        assert st["reach_over_cap"] == 0, st


ALL = ("cell_list", "link_list", "motor_list", "link_payload_global", "motor_row_walk")


@pytest.mark.parametrize("caps,paths", [((0, 0, 0, 0, 0), ALL),
                                        ((8, 1, 2, 1, 1), ALL + ("motor_payload_global",))],
                         ids=["all-fallback", "mixed"])
def test_benchmark_network_fallback_paths_bitwise(warm_c1, oracle_checkpoints, caps, paths):
    """The fused kernel with its capacities lowered: rows spill to their overflow lists,
    link payloads are read from global memory past the staging, motor rows longer than the
    sorted slots take the repeated-minimum walk and (mixed capacities) motor reactions past
    the staged ones are read from global memory; same bits as the oracle."""
    from softbox_b200.engine import DenseNetwork
    net = DenseNetwork(copy.deepcopy(warm_c1))
    ent, mot, ids, row, cell = caps
    net.test_caps(ent=ent, motor=mot, motor_ids=ids, row_slots=row, cell_slots=cell)
    net.fused_stats(reset=True)
    net.run(WARM, CHECK, mode="fused")
    assert net.status() == 0
    torch.cuda.synchronize()
    compare_scenes(oracle_checkpoints[0], D.to_host(net.dev))
    st = net.fused_stats()
    for k in paths:
        assert st[k] > 0, (k, st)


@pytest.mark.parametrize("mode", ["fused", "graph"])
def test_benchmark_network_supplied_noise_vs_libm_oracle(orc, warm_c1, mode):
    from softbox_b200.engine import DenseNetwork
    ref = copy.deepcopy(warm_c1)
    net = DenseNetwork(copy.deepcopy(warm_c1))
    nF, nB, nBb = ref["fil"]["body"]["n"], ref["mot"]["body"]["n"], ref["mini"]["backbone"]["n"]
    rng = np.random.default_rng(0x5EED)
    tol = 1e-5
    worst = {}
    for c in range(NSTEPS // CHECK):
        t0 = WARM + c * CHECK
        nf = rng.standard_normal((CHECK, 6, nF), dtype=np.float32)
        nm = rng.standard_normal((CHECK, 6, nB), dtype=np.float32)
        nb = rng.standard_normal((CHECK, 6, nBb), dtype=np.float32)
        net.set_noise(D.to_device(nf), D.to_device(nm), D.to_device(nb), t0)
        net.run(t0, CHECK, mode=mode)
        assert net.status() == 0
        orc.dense_run_supplied(D.dense_desc(ref), t0, CHECK, nf, nm, nb)
        torch.cuda.synchronize()
        got = D.to_host(net.dev)
        # integer outputs: cells, CSR, reach lists, binding, nucleotide and link states, exact
        for s, f in (("grid", "bodyCell"), ("grid", "gridCellOffsets"), ("grid", "gridCellContents"),
                     ("grid", "reachSeg"), ("grid", "reachCount"), ("mot", "boundSeg"), ("mot", "nucleotideState"),
                     ("mot", "stats"), ("xl", "linkState"), ("xl", "segOffsetsA"), ("xl", "segIdxA"),
                     ("xl", "segOffsetsB"), ("xl", "segIdxB"), ("segMotorOffsets", None), ("segMotorMyo", None)):
            want = ref[s][f] if f else ref[s]
            have = got[s][f] if f else got[s]
            assert np.array_equal(want, have), (s, f, int((want != have).sum()))
        # centres (FP64 and the FP32 store) and orientations of every body, within 1e-5
        # relative (lengths in um; a 1 um floor keeps centres near the origin meaningful)
        for s, b in (("fil", "body"), ("mot", "body"), ("mini", "backbone")):
            for f in ("coord64", "coord", "uVec", "yVec"):
                want = np.asarray(ref[s][b][f], np.float64)
                have = np.asarray(got[s][b][f], np.float64)
                err = float(np.max(np.abs(have - want) / np.maximum(np.abs(want), 1.0)))
                worst[(s, f)] = max(worst.get((s, f), 0.0), err)
                assert err <= tol, (s, f, err)
    net.set_noise(None, None, None, 0)
    print("max relative deviation over 1,000 steps:", {f"{k[0]}.{k[1]}": v for k, v in worst.items()})


def test_supplied_noise_range_and_nonfinite_rejected(warm_c1):
    from softbox_b200.engine import DenseNetwork
    from softbox_b200.runtime import SbxError
    net = DenseNetwork(copy.deepcopy(warm_c1))
    nF, nB, nBb = (warm_c1["fil"]["body"]["n"], warm_c1["mot"]["body"]["n"], warm_c1["mini"]["backbone"]["n"])
    nf = torch.zeros((4, 6, nF), device="cuda")
    nm = torch.zeros((4, 6, nB), device="cuda")
    nb = torch.zeros((4, 6, nBb), device="cuda")
    net.set_noise(nf, nm, nb, 100)
    for t0, n in ((99, 2), (103, 2)):
        with pytest.raises(SbxError) as e:
            net.run(t0, n, mode="fused")
        assert e.value.code == -1
    net.run(100, 4, mode="graph")
    assert net.status() == 0
    bad = nm.clone()
    bad[2, 3, 17] = float("inf")
    with pytest.raises(SbxError) as e:
        net.set_noise(nf, bad, nb, 0)
    assert e.value.code == -6
