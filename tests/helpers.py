"""Shared test helpers: scene copies, oracle stepping and bitwise comparison."""
import copy

import numpy as np

from softbox_b200 import device as D, scenes


def host_copy(sc):
    return copy.deepcopy(sc)


def oracle_dense_run(orc, sc, t0, nsteps):
    """Advance a host scene with the oracle's DenseContractileHarness.cpuStep restatement."""
    desc = D.dense_desc(sc)
    orc.dense_run(desc, t0, nsteps)
    return sc


def assert_same(a, b, what=""):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    if a.dtype.kind == "f":
        ok = np.array_equal(a.view(np.uint32 if a.dtype == np.float32 else np.uint64),
                            b.view(np.uint32 if b.dtype == np.float32 else np.uint64))
    else:
        ok = np.array_equal(a, b)
    if not ok:
        diff = np.flatnonzero(a != b)
        raise AssertionError(f"{what}: {diff.size} of {a.size} entries differ; first at {diff[:5]}: "
                             f"{a.reshape(-1)[diff[:5]]} vs {b.reshape(-1)[diff[:5]]}")


def flat_arrays(sc, prefix=""):
    """(name, array) for every numpy array in a (nested) scene dict."""
    out = []
    for k, v in sc.items():
        if isinstance(v, dict):
            out += flat_arrays(v, prefix + k + ".")
        elif isinstance(v, np.ndarray):
            out.append((prefix + k, v))
    return out


def compare_scenes(host, dev_host, skip=()):
    """Bitwise comparison of every array of two host scenes; returns the names compared."""
    names = []
    dmap = dict(flat_arrays(dev_host))
    for name, arr in flat_arrays(host):
        if any(name.endswith(s) for s in skip) or name not in dmap:
            continue
        assert_same(arr, dmap[name], name)
        names.append(name)
    return names


def small_dense(scale=0.05, **kw):
    return scenes.dense_contractile(scenes.dense_small(scale, **kw))


# ---------------------------------------------------------------- crosslinker formation
def oracle_formation_grid(orc, sc):
    """FormationGrid.buildCpu (FormationGrid.java:90-101) on host arrays; returns the grid."""
    f = sc["fil"]
    b = f["body"]
    n = b["n"]
    g = sc["grid"]
    half, cell = g["half"], g["cell"]
    nX = 1 + int(np.ceil(2 * half / cell))
    total = nX ** 3
    grid = {"gridParams": np.array([-half, -half, -half, cell, 1.0 / cell, g["grab"]], np.float32),
            "gridDims": np.array([nX, nX, nX, total], np.int32),
            "center": np.zeros(3 * n, np.float32), "R": np.zeros(n, np.float32),
            "ownerStore": np.zeros(n, np.int32), "ownerSlot": np.zeros(n, np.int32),
            "bodyCell": np.full(n, -1, np.int32), "cellCount": np.zeros(total, np.int32),
            "chunkSum": np.zeros((total + 511) // 512 + 1, np.int32),
            "offsets": np.zeros(total + 1, np.int32), "contents": np.full(n, -1, np.int32),
            "candCountSeg": np.zeros(n, np.int32), "candBaseSeg": np.zeros(n + 1, np.int32)}
    vp = np.array([g["radius"]], np.float32)
    orc.fil_publish(n, b["coord"], b["segLength"], n, grid["center"], grid["R"], grid["ownerStore"],
                    grid["ownerSlot"], vp, None)
    orc.body_cell(n, grid["center"], grid["gridParams"], grid["gridDims"], n, grid["bodyCell"])
    orc.grid_zero(total, grid["cellCount"])
    orc.grid_histogram(grid["bodyCell"], n, grid["cellCount"])
    orc.grid_scan_local(total, grid["cellCount"], grid["offsets"], grid["chunkSum"])
    orc.grid_scan_chunks(total, grid["chunkSum"])
    orc.grid_scan_add(total, grid["offsets"], n, grid["cellCount"], grid["chunkSum"])
    orc.grid_scatter(grid["bodyCell"], n, grid["offsets"], grid["contents"], n, grid["cellCount"])
    return grid


def oracle_formation(orc, sc, step, use_grid=True):
    """CrosslinkerBundleHarness.formationCpu (CrosslinkerBundleHarness.java:451-507) on host
    arrays: counts, candidates, gates, admission, free list, ranks, allocate, orientation."""
    f, xl = sc["fil"], sc["xl"]
    b = f["body"]
    n, C, K = b["n"], sc["C"], sc["reqCap"]
    xl["formCounts"][1] = step
    orc.count_active_links(C, xl["linkState"], xl["linkFilA"], xl["linkFilB"], n, xl["activeLinkCount"])
    if use_grid:
        g = oracle_formation_grid(orc, sc)
        orc.xl_grid_form_count(n, b["coord"], b["segLength"], sc["filID"], g["gridParams"], g["gridDims"],
                               g["offsets"], g["contents"], g["candCountSeg"], xl["formParams"])
        orc.xl_grid_form_scan(n, g["candCountSeg"], g["candBaseSeg"], K, xl["reqFilA"], xl["reqFilB"],
                              xl["formCounts"])
        orc.xl_grid_form_emit(n, b["coord"], b["segLength"], sc["filID"], g["gridParams"], g["gridDims"],
                              g["offsets"], g["contents"], g["candBaseSeg"], g["candCountSeg"], K, xl["reqFilA"],
                              xl["reqFilB"], xl["formParams"])
    else:
        orc.xl_fil_fil_candidates(n, b["coord"], b["segLength"], sc["filID"], K, xl["reqFilA"], xl["reqFilB"],
                                  xl["formParams"], xl["formCounts"])
    orc.xl_form_gates(n, b["uVec"], b["end1"], b["end2"], b["segLength"], K, xl["reqFilA"], xl["reqFilB"],
                      xl["reqLoc1"], xl["reqLoc2"], xl["reqOrient"], xl["gatePass"], xl["formParams"],
                      xl["formCounts"])
    orc.xl_form_admit_reduce(K, xl["reqFilA"], xl["reqFilB"], xl["gatePass"], n, xl["minCand"])
    orc.xl_form_admit(K, xl["reqFilA"], xl["reqFilB"], xl["reqLoc1"], xl["reqLoc2"], xl["gatePass"], xl["minCand"],
                      xl["activeLinkCount"], C, xl["linkState"], xl["linkFilA"], xl["linkFilB"], xl["loc1"],
                      xl["loc2"], xl["acceptFlag"], xl["formParams"])
    orc.xl_free_flags(C, xl["linkState"], xl["freeCount"])
    orc.csr_scan(C, xl["freeCount"], xl["freeOffsets"])
    orc.xl_free_scatter(C, xl["linkState"], xl["freeOffsets"], xl["freeList"])
    orc.csr_scan(K, xl["acceptFlag"], xl["rankOffsets"])
    orc.xl_allocate(K, xl["reqFilA"], xl["reqFilB"], xl["reqLoc1"], xl["reqLoc2"], xl["rankOffsets"],
                    xl["freeList"], xl["freeOffsets"], C, xl["linkFilA"], xl["linkFilB"], xl["loc1"], xl["loc2"],
                    xl["linkState"], xl["strainHist"], xl["strainPlace"])
    orc.xl_place_orient(K, xl["reqOrient"], xl["rankOffsets"], xl["freeList"], xl["freeOffsets"], C,
                        xl["linkOrientSame"], xl["torqueMagHist"], xl["torqueMagPlace"])
    return sc
