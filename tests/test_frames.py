"""Headless frames (CPU): java.util.Formatter's %g layout and FrameWriter's schema."""
import json

import numpy as np

from softbox_b200 import scenes
from softbox_b200.frames import FrameWriter, java_g


def test_java_general_format():
    cases = [(1.0, 5, "1.0000"), (0.0, 5, "0.0000"), (-0.0, 5, "-0.0000"), (1.23456e-5, 5, "1.2346e-05"),
             (123456.0, 5, "1.2346e+05"), (-0.00012345, 5, "-0.00012345"), (0.5, 3, "0.500"),
             (99999.5, 5, "1.0000e+05"), (0.0001, 5, "0.00010000"), (2.5, 1, "3"), (0.125, 2, "0.13"),
             (12.345, 5, "12.345"), (0.0035, 5, "0.0035000"), (1e-300, 5, "1.0000e-300"), (42.0, 6, "42.0000"),
             (9.99995, 5, "10.000"), (-7.25e21, 6, "-7.25000e+21")]
    for v, p, want in cases:
        assert java_g(v, p) == want, (v, p, java_g(v, p), want)


def test_frame_schema_and_geometry(tmp_path):
    sc = scenes.turnover_chains(n_chains=20, cap=256, seed=2)
    f = sc["fil"]
    fw = FrameWriter(str(tmp_path / "run"), 4.0, 4.0, 0.5)
    p0 = fw.write_frame(f, 0.0)
    p1 = fw.write_frame(f, 1.5e-3, nuc_frac=sc["t"]["nucFrac"])
    assert p0.endswith("frame_000000.json") and p1.endswith("frame_000001.json")
    a, b = json.load(open(p0)), json.load(open(p1))
    assert a["frame"] == 0 and b["frame"] == 1 and b["t"] == 0.0015
    assert a["bounds"] == {"xDim": 4.0, "yDim": 4.0, "zDim": 0.5}
    assert len(a["segments"]) == 256                                   # every slot
    act = np.flatnonzero(f["filState"] >= 0)
    assert [s["id"] for s in b["segments"]] == act.tolist()           # ACTIVE slots only
    n = f["body"]["n"]
    c = f["body"]["coord"].reshape(3, n).astype(np.float64)
    u = f["body"]["uVec"].reshape(3, n).astype(np.float64)
    L = f["body"]["segLength"].astype(np.float64)
    for s in b["segments"][:10]:
        i = s["id"]
        assert np.allclose(s["end1"], c[:, i] - 0.5 * L[i] * u[:, i], rtol=1e-4, atol=1e-6)
        assert np.allclose(s["end2"], c[:, i] + 0.5 * L[i] * u[:, i], rtol=1e-4, atol=1e-6)
        assert s["isBarbedEnd"] == bool(f["end2NbrSlot"][i] < 0)
        nf = sc["t"]["nucFrac"].reshape(3, n)
        assert abs(s["notADPRatio"] - (nf[0, i] + nf[1, i])) < 6e-3
    text = open(p0).read()
    assert '"r":0.0035000' in text and '"notADPRatio":1.00,"cofilinCount":0' in text
    fw2 = FrameWriter(str(tmp_path / "run"), 1, 1, 1)
    assert fw2.dir.endswith("run.001")
