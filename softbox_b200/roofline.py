"""Roofline helpers of the dense step: the algorithmic byte model and the measured peak.

The byte model counts every array one step reads once at its stored size and every array it
writes once (the compulsory traffic of the step); achieved GB/s = bytes / step time.
"""
import json
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def peaks():
    """HBM copy bandwidth measured on this pool (GB/s) and its source."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def step_bytes(sc, fp64=True):
    """Algorithmic bytes of one step: every array the step reads counted once at its stored
    size, every array it writes counted once (the compulsory traffic of the step)."""
    f, m, mini, xl, g = sc["fil"], sc["mot"], sc["mini"], sc["xl"], sc["grid"]
    fb, mb, bb = f["body"], m["body"], mini["backbone"]
    nb = lambda a: int(a.nbytes)
    total = 0
    for b in (fb, mb, bb):
        rd = ["coord", "uVec", "yVec", "segLength", "bTransGam", "bRotGam", "brownTransScale", "brownRotScale"]
        wr = ["coord", "uVec", "yVec", "zVec", "end1", "end2", "forceSum", "torqueSum", "randForce", "randTorque"]
        total += sum(nb(b[k]) for k in rd) + sum(nb(b[k]) for k in wr)
        if fp64:
            total += 2 * 8 * b["coord"].size
    total += sum(nb(f[k]) for k in ("end1NbrSlot", "end1NbrSide", "end2NbrSlot", "end2NbrSide"))
    total += nb(fb["end1"]) + nb(fb["end2"])                      # read by binding and links
    mot_rw = ["boundSeg", "bindArc", "stats", "capStats", "cooldown", "nucleotideState", "forceDotPlace",
              "forceDotFil", "forceMag", "forceDotHist"]
    total += 2 * sum(nb(m[k]) for k in mot_rw) + 3 * nb(m["head"]) + nb(m["reach"])
    total += nb(sc["bondData"]) * 2 + nb(mini["miniData"]) * 2 + nb(mini["attachAxial"])
    total += 2 * sum(nb(xl[k]) for k in ("linkState", "strainHist", "strainPlace", "torqueMagHist",
                                          "torqueMagPlace", "xlinkData"))
    total += sum(nb(xl[k]) for k in ("linkFilA", "linkFilB", "loc1", "loc2", "linkOrientSame"))
    # grid + CSRs (written once, read once)
    total += 2 * sum(nb(g[k]) for k in ("center", "boundingRadius", "ownerStore", "ownerSlot", "bodyCell",
                                         "cellCount", "gridCellOffsets", "gridCellContents"))
    total += 2 * (4 * m["nMotors"] * 4)                           # reach lists actually used (~4 per head)
    for k in ("segCountA", "segOffsetsA", "segIdxA", "segCountB", "segOffsetsB", "segIdxB"):
        total += 2 * nb(xl[k])
    for k in ("segMotorCount", "segMotorOffsets", "segMotorMyo"):
        total += 2 * nb(sc[k])
    return total
