"""ctypes mirrors of the store descriptors declared in include/softbox_b200.h.

The same structs describe host arrays (for the CPU oracle's step driver) and device
arrays (for the fused CUDA step plans); only the pointer values differ.
"""
import ctypes as C

f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
i32p = C.POINTER(C.c_int32)


class RigidBody(C.Structure):          # RigidRodBody.java:26-84
    _fields_ = [("n", C.c_int32)] + [(k, f32p) for k in (
        "coord", "uVec", "yVec", "zVec", "end1", "end2", "segLength",
        "bTransGam", "bRotGam", "bTransDiff", "bRotDiff",
        "forceSum", "torqueSum", "randForce", "randTorque",
        "brownTransScale", "brownRotScale")] + [("coord64", f64p)]


class FilamentStoreDesc(C.Structure):   # FilamentStore.java:29-199
    _fields_ = [("body", RigidBody)] + [(k, i32p) for k in (
        "monomerCount", "end1NbrSlot", "end1NbrSide", "end2NbrSlot", "end2NbrSide", "filState")] + [
        ("params", f32p), ("chainParams", f32p), ("counts", i32p)]


class MotorStoreDesc(C.Structure):      # MotorStore.java:32-161
    _fields_ = [("body", RigidBody), ("nMotors", C.c_int32)] + [(k, f32p) for k in (
        "head", "uVec", "rodUVec", "reach", "bindArc")] + [(k, i32p) for k in (
        "boundSeg", "stats", "capStats", "cooldown", "nucleotideState", "forceDotPlace")] + [
        (k, f32p) for k in ("forceDotFil", "forceMag", "forceDotHist",
                            "bodyParams", "jointParams", "kinParams", "nucParams")] + [
        ("counts", i32p), ("publishParams", i32p)]


class DimerStoreDesc(C.Structure):      # DimerStore.java:26-67
    _fields_ = [("nDimers", C.c_int32), ("motorA", i32p), ("motorB", i32p), ("parallel", i32p),
                ("dimerParams", f32p)]


class MiniStoreDesc(C.Structure):       # MiniFilamentStore.java:28-135
    _fields_ = [("backbone", RigidBody), ("nBackbones", C.c_int32), ("nDimers", C.c_int32),
                ("bbBodyParams", f32p), ("bbCounts", i32p), ("headBackboneSlot", i32p), ("motorA", i32p),
                ("attachAxial", f32p), ("miniData", f32p), ("bbInvDragY", f32p), ("miniParams", f32p),
                ("bbDimerCount", i32p), ("bbDimerOffsets", i32p), ("bbDimerList", i32p)]


class CrosslinkerStoreDesc(C.Structure):  # CrosslinkerStore.java:31-179
    _fields_ = [("nLinks", C.c_int32)] + [(k, i32p) for k in (
        "linkFilA", "linkFilB", "linkState", "linkOrientSame", "activeLinkCount")] + [
        (k, f32p) for k in ("loc1", "loc2", "xlinkData", "strainHist", "torqueMagHist")] + [
        ("strainPlace", i32p), ("torqueMagPlace", i32p)] + [
        (k, f32p) for k in ("xlParams", "offParams", "torsionParams")] + [("counts", i32p)] + [
        (k, i32p) for k in ("segCountA", "segOffsetsA", "segIdxA", "segCountB", "segOffsetsB", "segIdxB")]


class GridStateDesc(C.Structure):       # SpatialBodyView.java:29-56 + grid arrays
    _fields_ = [("cap", C.c_int32), ("totalCells", C.c_int32), ("center", f32p), ("boundingRadius", f32p),
                ("ownerStore", i32p), ("ownerSlot", i32p), ("gridParams", f32p), ("viewParams", f32p),
                ("gridDims", i32p), ("gridCounts", i32p)] + [(k, i32p) for k in (
                    "bodyCell", "cellCount", "chunkSum", "gridCellOffsets", "gridCellContents",
                    "reachSeg", "reachCount")]


class DenseSceneDesc(C.Structure):      # DenseContractileHarness.Scene
    _fields_ = [("fil", FilamentStoreDesc), ("mot", MotorStoreDesc), ("dim", DimerStoreDesc),
                ("mini", MiniStoreDesc), ("xl", CrosslinkerStoreDesc), ("grid", GridStateDesc),
                ("bondData", f32p), ("xbParams", f32p), ("boxParams", f32p),
                ("segMotorCount", i32p), ("segMotorOffsets", i32p), ("segMotorMyo", i32p),
                ("seed", C.c_int32), ("seedBb", C.c_int32), ("xlinkOn", C.c_int32), ("xlUnbind", C.c_int32)]


def _ptr(arr, ctype):
    """Pointer of a numpy array (host) or a torch tensor (device); None -> NULL."""
    if arr is None:
        return C.cast(None, C.POINTER(ctype))
    if hasattr(arr, "data_ptr"):
        return C.cast(C.c_void_p(arr.data_ptr()), C.POINTER(ctype))
    return arr.ctypes.data_as(C.POINTER(ctype))


def fill(struct, arrays, prefix=""):
    """Fill pointer fields of `struct` from the mapping `arrays` (name -> array)."""
    for name, ftype in struct._fields_:
        if isinstance(ftype, type) and issubclass(ftype, C.Structure):
            continue
        if ftype in (f32p, f64p, i32p):
            key = prefix + name
            ctype = {f32p: C.c_float, f64p: C.c_double, i32p: C.c_int32}[ftype]
            setattr(struct, name, _ptr(arrays.get(key), ctype))
    return struct


class BatchDesc(C.Structure):           # packed networks (sbx_batch)
    _fields_ = [("nNet", C.c_int32)] + [(k, i32p) for k in ("segKey", "motKey", "bbKey", "linkKey", "seeds")] + [
        ("gridParams", f32p), ("gridDims", i32p), ("boxParams", f32p)]


class TurnoverBatchDesc(C.Structure):   # packed-network turnover tables (sbx_turnover_batch)
    _fields_ = [("nNet", C.c_int32), ("slotKey", i32p), ("slotBase", i32p), ("seeds", i32p), ("growParams", f32p),
                ("depolyParams", f32p), ("depolyRateParams", f32p), ("agingParams", f32p),
                ("cofilinParams", f32p), ("birthBox", f32p), ("onRate", f64p), ("pools", f64p),
                ("birthNet", i32p), ("birthBase", i32p)]


class DenseNoiseDesc(C.Structure):      # supplied Gaussians of the dense step (sbx_dense_noise)
    _fields_ = [("fil", f32p), ("mot", f32p), ("bb", f32p), ("t0", C.c_int32), ("nsteps", C.c_int32)]
