"""Generates the Java side of the drop-in boundary (java/src/...):

  * uk/ac/manchester/tornado/api/common/TornadoFunctions.java: the functional interfaces
    Task1 .. Task15 that TaskGraph.task method references bind to;
  * uk/ac/manchester/tornado/api/TaskGraph.java: the task recorder (one overload per arity);
  * softbox_b200/shim/<Class>Kernels.java: for every System method the dense contractile and
    diffusion harnesses call, a static method with the reference's Java signature whose body
    is a Foreign Function & Memory downcall into include/softbox_b200.h.

A maintainer splices each reference System method body into a one-line delegate, e.g.
`SpatialGrid.bodyCell(...) { SpatialGridKernels.bodyCell(...); }`; the harness sources stay
unchanged. The table below is the mapping: each Java argument list of the reference method
(file:line) and the C entry point with its arguments as Java expressions and FFM layouts.
tests/test_java_shim.py checks every generated FunctionDescriptor against the header.

    python java/gen_shim.py
"""
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "src")

A, I, D = "ADDRESS", "JAVA_INT", "JAVA_DOUBLE"

# (reference class, method, Java parameters, reference file:line, C function,
#  [(Java expression, layout)], note). An expression naming an array parameter passes
#  its device pointer; "CTX" is the shim's context; "NULL" a null pointer.
M = [
    ("SpatialGrid", "bodyCell",
     "FloatArray center, FloatArray gridParams, IntArray gridDims, IntArray counts, IntArray bodyCell",
     "SpatialGrid.java:51-75", "sbx_grid_body_cell",
     [("CTX", A), ("center.getSize() / 3", I), ("center", A), ("gridParams", A), ("gridDims", A), ("counts", A),
      ("bodyCell", A)], None),
    ("SpatialGrid", "gridScanAdd",
     "IntArray gridDims, IntArray gridCellOffsets, IntArray gridCellContents, IntArray cellCount, IntArray chunkSum",
     "SpatialGrid.java:137-160", "sbx_grid_build",
     [("CTX", A), ("GRID_BUILD.cap", I), ("GRID_BUILD.bodyCell", A), ("GRID_BUILD.counts", A),
      ("gridDims.get(3)", I), ("cellCount", A), ("chunkSum", A), ("gridCellOffsets", A), ("gridCellContents", A),
      ("gridCellContents.getSize()", I)],
     "the chunked build (gridChunkZero/Histogram/Reduce, gridScanLocal/Chunks/Add, gridChunkScatter) runs as "
     "one stable counting sort here, over the bodyCell / counts recorded by gridChunkHistogram; cellCount is "
     "then reset as the scan's write cursor"),
    ("BindingDetectionSystem", "gridReachable",
     "FloatArray head, FloatArray uVec, FloatArray rodUVec, FloatArray segEnd1, FloatArray segEnd2, "
     "FloatArray gridParams, IntArray gridDims, IntArray gridCellOffsets, IntArray gridCellContents, "
     "IntArray ownerStore, IntArray ownerSlot, IntArray motorReachSeg, IntArray motorReachCount, "
     "FloatArray kinParams, IntArray counts",
     "BindingDetectionSystem.java:143-228", "sbx_binding_grid_reachable",
     [("CTX", A), ("head", A), ("uVec", A), ("rodUVec", A), ("segEnd1.getSize() / 3", I), ("segEnd1", A),
      ("segEnd2", A), ("gridParams", A), ("gridDims", A), ("gridCellOffsets", A), ("gridCellContents", A),
      ("ownerStore", A), ("ownerSlot", A), ("motorReachSeg", A), ("motorReachCount", A), ("kinParams", A),
      ("counts.get(0)", I)], None),
    ("BindingDetectionSystem", "bindNearest",
     "FloatArray head, FloatArray uVec, FloatArray rodUVec, FloatArray segEnd1, FloatArray segEnd2, "
     "IntArray motorCandSeg, IntArray motorCandCount, IntArray boundSeg, FloatArray bindArc, FloatArray kinParams, "
     "IntArray counts",
     "BindingDetectionSystem.java:356-389", "sbx_binding_bind_nearest",
     [("CTX", A), ("head", A), ("uVec", A), ("rodUVec", A), ("segEnd1.getSize() / 3", I), ("segEnd1", A),
      ("segEnd2", A), ("motorCandSeg", A), ("motorCandCount", A), ("boundSeg", A), ("bindArc", A),
      ("kinParams", A), ("counts.get(0)", I)], None),
    ("NucleotideCycleSystem", "cycle",
     "IntArray nucleotideState, IntArray boundSeg, FloatArray forceDotHist, FloatArray nucParams, IntArray counts",
     "NucleotideCycleSystem.java:33-69", "sbx_nucleotide_cycle",
     [("CTX", A), ("nucleotideState.getSize()", I), ("nucleotideState", A), ("boundSeg", A), ("forceDotHist", A),
      ("nucParams", A), ("counts", A)], None),
    ("NucleotideCycleSystem", "catchSlipRelease",
     "IntArray boundSeg, FloatArray forceDotFil, FloatArray forceMag, IntArray cooldown, IntArray stats, "
     "IntArray capStats, FloatArray kinParams, IntArray counts",
     "NucleotideCycleSystem.java:77-134", "sbx_nucleotide_release",
     [("CTX", A), ("boundSeg.getSize()", I), ("boundSeg", A), ("forceDotFil", A), ("forceMag", A), ("cooldown", A),
      ("stats", A), ("capStats", A), ("kinParams", A), ("counts", A)], None),
    ("DragTensorSystem", "runFilament", "FloatArray segLength, IntArray monomerCount, IntArray end1NbrSlot, "
     "IntArray end2NbrSlot, FloatArray bTransGam, FloatArray bRotGam, FloatArray bTransDiff, FloatArray bRotDiff, "
     "double aeta",
     "DragTensorSystem.java:71-97", "sbx_drag_run_filament",
     [("CTX", A), ("segLength.getSize()", I), ("monomerCount", A), ("end1NbrSlot", A), ("end2NbrSlot", A),
      ("aeta", D), ("segLength", A), ("bTransGam", A), ("bRotGam", A), ("bTransDiff", A), ("bRotDiff", A)],
     "DragTensorSystem.run(FilamentStore s) delegates with s's arrays and Constants.aeta"),
    ("DragTensorSystem", "runMotor", "FloatArray segLength, FloatArray bTransGam, FloatArray bRotGam, "
     "FloatArray bTransDiff, FloatArray bRotDiff, double aeta",
     "DragTensorSystem.java:105-122", "sbx_drag_run_motor",
     [("CTX", A), ("segLength.getSize() / 3", I), ("aeta", D), ("segLength", A), ("bTransGam", A), ("bRotGam", A),
      ("bTransDiff", A), ("bRotDiff", A)],
     "DragTensorSystem.run(MotorStore mot) delegates with mot.body's arrays and Constants.aeta"),
    ("BrownianForceSystem", "brownianForce",
     "FloatArray randForce, FloatArray randTorque, FloatArray bTransGam, FloatArray bRotGam, "
     "FloatArray brownTransScale, FloatArray brownRotScale, FloatArray params, IntArray counts",
     "BrownianForceSystem.java:44-106", "sbx_brownian_force",
     [("CTX", A), ("randForce.getSize() / 3", I), ("randForce", A), ("randTorque", A), ("bTransGam", A),
      ("bRotGam", A), ("brownTransScale", A), ("brownRotScale", A), ("params", A), ("counts", A)], None),
    ("ChainBendingForceSystem", "zeroAccumulators", "FloatArray forceSum, FloatArray torqueSum, IntArray counts",
     "ChainBendingForceSystem.java:38-45", "sbx_zero_accumulators",
     [("CTX", A), ("forceSum.getSize() / 3", I), ("forceSum", A), ("torqueSum", A)], None),
    ("ChainBendingForceSystem", "chainForces",
     "FloatArray coord, FloatArray uVec, FloatArray segLength, IntArray end2NbrSlot, IntArray end2NbrSide, "
     "IntArray end1NbrSlot, IntArray end1NbrSide, FloatArray bTransGam, FloatArray bRotGam, FloatArray forceSum, "
     "FloatArray torqueSum, FloatArray chainParams, IntArray counts",
     "ChainBendingForceSystem.java:105-331", "sbx_chain_forces",
     [("CTX", A), ("coord.getSize() / 3", I), ("coord", A), ("uVec", A), ("segLength", A), ("end2NbrSlot", A),
      ("end2NbrSide", A), ("end1NbrSlot", A), ("end1NbrSide", A), ("bTransGam", A), ("bRotGam", A),
      ("forceSum", A), ("torqueSum", A), ("chainParams", A)], None),
    ("ContainmentSystem", "confine",
     "FloatArray coord, FloatArray uVec, FloatArray segLength, FloatArray bTransGam, FloatArray forceSum, "
     "FloatArray torqueSum, FloatArray boxParams, IntArray counts",
     "ContainmentSystem.java:58-126", "sbx_confine",
     [("CTX", A), ("coord.getSize() / 3", I), ("coord", A), ("uVec", A), ("segLength", A), ("bTransGam", A),
      ("forceSum", A), ("torqueSum", A), ("boxParams", A), ("counts", A)], None),
    ("RigidRodLangevinIntegrationSystem", "integrate",
     "FloatArray coord, FloatArray uVec, FloatArray yVec, FloatArray forceSum, FloatArray torqueSum, "
     "FloatArray randForce, FloatArray randTorque, FloatArray bTransGam, FloatArray bRotGam, FloatArray params, "
     "IntArray counts",
     "RigidRodLangevinIntegrationSystem.java:33-112", "sbx_integrate",
     [("CTX", A), ("coord.getSize() / 3", I), ("coord", A), ("NULL", A), ("uVec", A), ("yVec", A), ("forceSum", A),
      ("torqueSum", A), ("randForce", A), ("randTorque", A), ("bTransGam", A), ("bRotGam", A), ("params", A)],
     None),
    ("DerivedGeometrySystem", "derive",
     "FloatArray coord, FloatArray uVec, FloatArray yVec, FloatArray zVec, FloatArray end1, FloatArray end2, "
     "FloatArray segLength, IntArray counts",
     "DerivedGeometrySystem.java:27-73", "sbx_derive",
     [("CTX", A), ("coord.getSize() / 3", I), ("coord", A), ("uVec", A), ("yVec", A), ("zVec", A), ("end1", A),
      ("end2", A), ("segLength", A)], None),
    ("FilamentStore", "publishToBodyView",
     "FloatArray coord, FloatArray segLength, FloatArray center, FloatArray boundingRadius, IntArray ownerStore, "
     "IntArray ownerSlot, FloatArray viewParams, IntArray counts",
     "FilamentStore.java:275-295", "sbx_filament_publish",
     [("CTX", A), ("coord.getSize() / 3", I), ("coord", A), ("segLength", A), ("center.getSize() / 3", I),
      ("center", A), ("boundingRadius", A), ("ownerStore", A), ("ownerSlot", A), ("viewParams", A), ("NULL", A)],
     None),
    ("FilamentStore", "publishToBodyView",
     "FloatArray coord, FloatArray segLength, FloatArray center, FloatArray boundingRadius, IntArray ownerStore, "
     "IntArray ownerSlot, FloatArray viewParams, IntArray counts, IntArray filState",
     "FilamentStore.java:306-328", "sbx_filament_publish",
     [("CTX", A), ("coord.getSize() / 3", I), ("coord", A), ("segLength", A), ("center.getSize() / 3", I),
      ("center", A), ("boundingRadius", A), ("ownerStore", A), ("ownerSlot", A), ("viewParams", A),
      ("filState", A)], None),
    ("MotorStore", "publishHeadFromBody",
     "FloatArray bodyCoord, FloatArray bodyUVec, FloatArray bodySegLength, FloatArray head, FloatArray uVec, "
     "FloatArray rodUVec, IntArray counts",
     "MotorStore.java:300-314", "sbx_motor_publish_head",
     [("CTX", A), ("head.getSize() / 3", I), ("bodyCoord", A), ("bodyUVec", A), ("bodySegLength", A), ("head", A),
      ("uVec", A), ("rodUVec", A)], None),
    ("MotorStore", "publishToBodyView",
     "FloatArray head, FloatArray reach, FloatArray center, FloatArray boundingRadius, IntArray ownerStore, "
     "IntArray ownerSlot, IntArray publishParams, IntArray counts",
     "MotorStore.java:326-347", "sbx_motor_publish",
     [("CTX", A), ("head.getSize() / 3", I), ("head", A), ("reach", A), ("center.getSize() / 3", I), ("center", A),
      ("boundingRadius", A), ("ownerStore", A), ("ownerSlot", A), ("publishParams", A)], None),
    ("MotorJointSystem", "joints",
     "FloatArray coord, FloatArray uVec, FloatArray segLength, FloatArray bTransGam, FloatArray bRotGam, "
     "FloatArray forceSum, FloatArray torqueSum, IntArray nucleotideState, FloatArray jointParams, IntArray counts",
     "MotorJointSystem.java:72-197", "sbx_motor_joints",
     [("CTX", A), ("coord.getSize() / 3", I), ("coord", A), ("uVec", A), ("segLength", A), ("bTransGam", A),
      ("bRotGam", A), ("forceSum", A), ("torqueSum", A), ("nucleotideState", A), ("jointParams", A)], None),
    ("DimerCouplingSystem", "couple",
     "FloatArray coord, FloatArray uVec, FloatArray segLength, FloatArray bTransGam, FloatArray bRotGam, "
     "FloatArray forceSum, FloatArray torqueSum, IntArray motorA, IntArray motorB, IntArray parallel, "
     "FloatArray dimerParams, IntArray boundSeg",
     "DimerCouplingSystem.java:83-184", "sbx_dimer_couple",
     [("CTX", A), ("coord.getSize() / 3", I), ("coord", A), ("uVec", A), ("segLength", A), ("bTransGam", A),
      ("bRotGam", A), ("forceSum", A), ("torqueSum", A), ("motorA.getSize()", I), ("motorA", A), ("motorB", A),
      ("parallel", A), ("dimerParams", A), ("boundSeg", A)], None),
    ("MiniFilamentSystem", "tether",
     "FloatArray mCoord, FloatArray mUVec, FloatArray mSegLength, FloatArray mBTransGam, FloatArray mBRotGam, "
     "FloatArray mForceSum, FloatArray mTorqueSum, FloatArray bbCoord, FloatArray bbUVec, FloatArray bbInvDragY, "
     "IntArray headBackboneSlot, IntArray motorA, FloatArray attachAxial, FloatArray miniData, FloatArray miniParams",
     "MiniFilamentSystem.java:65-134", "sbx_mini_tether",
     [("CTX", A), ("mCoord.getSize() / 3", I), ("mCoord", A), ("mUVec", A), ("mSegLength", A), ("mBTransGam", A),
      ("mBRotGam", A), ("mForceSum", A), ("mTorqueSum", A), ("bbCoord.getSize() / 3", I), ("bbCoord", A),
      ("bbUVec", A), ("bbInvDragY", A), ("headBackboneSlot.getSize()", I), ("headBackboneSlot", A), ("motorA", A),
      ("attachAxial", A), ("miniData", A), ("miniParams", A)], None),
    ("MiniFilamentSystem", "backboneGather",
     "IntArray bbDimerOffsets, IntArray bbDimerList, FloatArray miniData, FloatArray bbForceSum, "
     "FloatArray bbTorqueSum, IntArray miniCounts",
     "MiniFilamentSystem.java:137-155", "sbx_mini_backbone_gather",
     [("CTX", A), ("miniCounts.get(3)", I), ("bbDimerOffsets", A), ("bbDimerList", A), ("miniData", A),
      ("bbForceSum", A), ("bbTorqueSum", A)], None),
    ("CrossBridgeSystem", "bondForces",
     "FloatArray motorCoord, FloatArray motorUVec, FloatArray motorYVec, FloatArray motorBRotGam, "
     "FloatArray filCoord, FloatArray filUVec, FloatArray filYVec, FloatArray filBRotGam, FloatArray filSegLength, "
     "IntArray boundSeg, FloatArray bindArc, IntArray nucleotideState, FloatArray bondData, FloatArray xbParams",
     "CrossBridgeSystem.java:58-142", "sbx_xbridge_bond_forces",
     [("CTX", A), ("motorCoord.getSize() / 3", I), ("motorCoord", A), ("motorUVec", A), ("motorYVec", A),
      ("motorBRotGam", A), ("filCoord.getSize() / 3", I), ("filCoord", A), ("filUVec", A), ("filYVec", A),
      ("filBRotGam", A), ("filSegLength", A), ("boundSeg", A), ("bindArc", A), ("nucleotideState", A),
      ("bondData", A), ("xbParams", A)], None),
    ("CrossBridgeSystem", "applyHeadForce",
     "FloatArray bondData, FloatArray bodyForceSum, FloatArray bodyTorqueSum, IntArray counts",
     "CrossBridgeSystem.java:145-157", "sbx_xbridge_apply_head_force",
     [("CTX", A), ("bodyForceSum.getSize() / 3", I), ("bondData", A), ("bodyForceSum", A), ("bodyTorqueSum", A)],
     None),
    ("CrossBridgeSystem", "registerForceDot",
     "FloatArray bondData, IntArray boundSeg, FloatArray forceDotFil, FloatArray forceMag, FloatArray forceDotHist, "
     "IntArray forceDotPlace, IntArray counts",
     "CrossBridgeSystem.java:166-187", "sbx_xbridge_register_force_dot",
     [("CTX", A), ("boundSeg.getSize()", I), ("bondData", A), ("boundSeg", A), ("forceDotFil", A), ("forceMag", A),
      ("forceDotHist", A), ("forceDotPlace", A)], None),
    ("CrossBridgeSystem", "csrScan", "IntArray counts, IntArray segMotorCount, IntArray segMotorOffsets",
     "CrossBridgeSystem.java:198-205", "sbx_csr_scan",
     [("CTX", A), ("counts.get(3)", I), ("segMotorCount", A), ("segMotorOffsets", A)], None),
    ("CrossBridgeSystem", "csrChunkReduce",
     "IntArray counts, IntArray csrChunkParams, IntArray csrMatrix, IntArray segMotorCount",
     "CrossBridgeSystem.java:260-276", "sbx_csr_build",
     [("CTX", A), ("CSR_BUILD.keys", A), ("CSR_BUILD.nItems", I), ("segMotorCount.getSize()", I),
      ("segMotorCount", A), ("CSR_BUILD.offsets", A), ("CSR_BUILD.list", A)],
     "the row counts (the histogram) of the keys recorded by csrChunkHistogram; csrScan then turns them into "
     "offsets"),
    ("CrossBridgeSystem", "csrChunkScatter",
     "IntArray boundSeg, IntArray counts, IntArray csrChunkParams, IntArray segMotorOffsets, IntArray segMotorMyo, "
     "IntArray csrMatrix",
     "CrossBridgeSystem.java:278-298", "sbx_csr_build",
     [("CTX", A), ("boundSeg", A), ("counts.get(0)", I), ("segMotorOffsets.getSize() - 1", I), ("CSR_BUILD.count", A),
      ("CSR_BUILD.offsets", A), ("segMotorMyo", A)],
     "the stable list: items in ascending index within each row, at the offsets csrScan wrote"),
    ("CrossBridgeSystem", "segGather",
     "IntArray segMotorOffsets, IntArray segMotorMyo, FloatArray bondData, FloatArray filForceSum, "
     "FloatArray filTorqueSum, IntArray counts",
     "CrossBridgeSystem.java:302-320", "sbx_xbridge_seg_gather",
     [("CTX", A), ("counts.get(3)", I), ("segMotorOffsets", A), ("segMotorMyo", A), ("bondData", A),
      ("filForceSum", A), ("filTorqueSum", A)], None),
    ("CrosslinkerSystem", "countActiveLinks",
     "IntArray linkState, IntArray linkFilA, IntArray linkFilB, IntArray activeLinkCount, IntArray formCounts",
     "CrosslinkerSystem.java:694-706", "sbx_xlink_count_active",
     [("CTX", A), ("linkState.getSize()", I), ("linkState", A), ("linkFilA", A), ("linkFilB", A),
      ("activeLinkCount.getSize()", I), ("activeLinkCount", A)], None),
    ("CrosslinkerSystem", "linkForces",
     "FloatArray filCoord, FloatArray filUVec, FloatArray filEnd1, FloatArray filBTransGam, IntArray linkFilA, "
     "IntArray linkFilB, FloatArray loc1, FloatArray loc2, IntArray filLinkCt, FloatArray xlinkData, "
     "FloatArray xlParams",
     "CrosslinkerSystem.java:51-124", "sbx_xlink_forces",
     [("CTX", A), ("filCoord.getSize() / 3", I), ("filCoord", A), ("filUVec", A), ("filEnd1", A),
      ("filBTransGam", A), ("linkFilA.getSize()", I), ("linkFilA", A), ("linkFilB", A), ("loc1", A), ("loc2", A),
      ("filLinkCt", A), ("xlinkData", A), ("xlParams", A)], None),
    ("CrosslinkerSystem", "linkTorsion",
     "FloatArray filUVec, IntArray linkFilA, IntArray linkFilB, IntArray linkState, IntArray linkOrientSame, "
     "FloatArray torqueMagHist, IntArray torqueMagPlace, FloatArray xlinkData, FloatArray torsionParams",
     "CrosslinkerSystem.java:767-808", "sbx_xlink_torsion",
     [("CTX", A), ("filUVec.getSize() / 3", I), ("filUVec", A), ("linkFilA.getSize()", I), ("linkFilA", A),
      ("linkFilB", A), ("linkState", A), ("linkOrientSame", A), ("torqueMagHist", A), ("torqueMagPlace", A),
      ("xlinkData", A), ("torsionParams", A)], None),
    ("CrosslinkerSystem", "segGatherA",
     "IntArray segOffsets, IntArray segLinkIdx, FloatArray xlinkData, IntArray linkState, FloatArray filForceSum, "
     "FloatArray filTorqueSum, IntArray counts",
     "CrosslinkerSystem.java:129-149", "sbx_xlink_seg_gather",
     [("CTX", A), ("0", I), ("counts.get(3)", I), ("segOffsets", A), ("segLinkIdx", A), ("xlinkData", A),
      ("linkState", A), ("filForceSum", A), ("filTorqueSum", A)], None),
    ("CrosslinkerSystem", "segGatherB",
     "IntArray segOffsets, IntArray segLinkIdx, FloatArray xlinkData, IntArray linkState, FloatArray filForceSum, "
     "FloatArray filTorqueSum, IntArray counts",
     "CrosslinkerSystem.java:153-173", "sbx_xlink_seg_gather",
     [("CTX", A), ("1", I), ("counts.get(3)", I), ("segOffsets", A), ("segLinkIdx", A), ("xlinkData", A),
      ("linkState", A), ("filForceSum", A), ("filTorqueSum", A)], None),
    ("CrosslinkerSystem", "unbind",
     "FloatArray filCoord, FloatArray filUVec, FloatArray filEnd1, IntArray linkFilA, IntArray linkFilB, "
     "FloatArray loc1, FloatArray loc2, IntArray linkState, FloatArray strainHist, IntArray strainPlace, "
     "FloatArray offParams, IntArray counts",
     "CrosslinkerSystem.java:231-281", "sbx_xlink_unbind",
     [("CTX", A), ("filCoord.getSize() / 3", I), ("filUVec", A), ("filEnd1", A), ("counts.get(0)", I),
      ("linkFilA", A), ("linkFilB", A), ("loc1", A), ("loc2", A), ("linkState", A), ("strainHist", A),
      ("strainPlace", A), ("offParams", A), ("counts", A)], None),
    ("DeflectionSupport", "seedAccumulators",
     "FloatArray forceSum, FloatArray torqueSum, FloatArray extForce, IntArray counts",
     "DeflectionSupport.java:24-33", "sbx_deflection_seed_accumulators",
     [("CTX", A), ("forceSum.getSize() / 3", I), ("forceSum", A), ("torqueSum", A), ("extForce", A), ("counts", A)],
     None),
    ("DeflectionSupport", "pinEndpoints",
     "FloatArray coord, FloatArray uVec, FloatArray segLength, IntArray pinSeg, IntArray pinEnd, "
     "FloatArray pinAnchor, IntArray counts",
     "DeflectionSupport.java:40-58", "sbx_deflection_pin_endpoints",
     [("CTX", A), ("coord.getSize() / 3", I), ("coord", A), ("uVec", A), ("segLength", A), ("pinSeg.getSize()", I),
      ("pinSeg", A), ("pinEnd", A), ("pinAnchor", A)], None),
]

# methods of the chunked builds whose work happens in a later call of the same build
NOOPS = [
    ("SpatialGrid", "gridChunkZero", "IntArray chunkParams, IntArray gridDims, IntArray chunkCellCount",
     "SpatialGrid.java:237-244", None),
    ("SpatialGrid", "gridChunkHistogram",
     "IntArray bodyCell, IntArray counts, IntArray chunkParams, IntArray gridDims, IntArray chunkCellCount",
     "SpatialGrid.java:248-273", "GRID_BUILD.record(bodyCell, counts);"),
    ("SpatialGrid", "gridChunkReduce",
     "IntArray gridDims, IntArray chunkParams, IntArray chunkCellCount, IntArray cellCount",
     "SpatialGrid.java:278-296", None),
    ("SpatialGrid", "gridScanLocal",
     "IntArray gridDims, IntArray cellCount, IntArray gridCellOffsets, IntArray chunkSum",
     "SpatialGrid.java:99-117", None),
    ("SpatialGrid", "gridScanChunks", "IntArray gridDims, IntArray chunkSum", "SpatialGrid.java:121-133", None),
    ("SpatialGrid", "gridChunkScatter",
     "IntArray bodyCell, IntArray counts, IntArray chunkParams, IntArray gridDims, IntArray gridCellOffsets, "
     "IntArray gridCellContents, IntArray chunkCellCount", "SpatialGrid.java:302-331", None),
    ("CrossBridgeSystem", "csrChunkZero", "IntArray csrChunkParams, IntArray counts, IntArray csrMatrix",
     "CrossBridgeSystem.java:232-237", None),
    ("CrossBridgeSystem", "csrChunkHistogram",
     "IntArray boundSeg, IntArray counts, IntArray csrChunkParams, IntArray csrMatrix",
     "CrossBridgeSystem.java:240-257", "CSR_BUILD.record(boundSeg, counts.get(0), csrMatrix);"),
]

HEADER = os.path.join(os.path.dirname(HERE), "include", "softbox_b200.h")


def header_args(c_fn):
    """The C parameter declarations of c_fn in the header."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    m = re.search(r"\b" + c_fn + r"\s*\(([^;]*?)\)\s*;", text, re.S)
    if not m:
        raise KeyError(c_fn)
    return [a.strip() for a in m.group(1).split(",")]


def params(plist):
    out = []
    for p in plist.split(","):
        t, n = p.strip().rsplit(" ", 1)
        out.append((t, n))
    return out


def java_arg(expr, layout, arrays):
    if expr == "CTX":
        return "Sbx.ctx()"
    if expr == "NULL":
        return "MemorySegment.NULL"
    if expr in arrays:
        return expr + ".dev()"
    if layout == A:
        return expr + ".dev()" if not expr.endswith(")") else expr
    return expr


def handle_name(c_fn, idx):
    return "H_" + c_fn[4:].upper() + ("" if idx == 0 else f"_{idx}")


def gen_kernels():
    by_class = {}
    for entry in M:
        by_class.setdefault(entry[0], []).append(("call", entry))
    for entry in NOOPS:
        by_class.setdefault(entry[0], []).append(("noop", entry))
    files = {}
    for cls, items in by_class.items():
        lines = [f"package softbox_b200.shim;", "",
                 "import java.lang.foreign.FunctionDescriptor;",
                 "import java.lang.foreign.MemorySegment;",
                 "import java.lang.invoke.MethodHandle;", "",
                 "import uk.ac.manchester.tornado.api.types.arrays.FloatArray;",
                 "import uk.ac.manchester.tornado.api.types.arrays.IntArray;", "",
                 "import static java.lang.foreign.ValueLayout.ADDRESS;",
                 "import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;",
                 "import static java.lang.foreign.ValueLayout.JAVA_INT;", "",
                 f"/** Downcall bodies of {cls}'s kernels (generated by java/gen_shim.py). Each method has the",
                 f" *  reference method's Java signature; its body moves the arguments' current contents to the",
                 f" *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */",
                 f"public final class {cls}Kernels {{", f"    private {cls}Kernels() {{}}", ""]
        seen = {}
        for kind, e in items:
            if kind == "noop":
                _, meth, plist, cite, body = e
                ps = params(plist)
                lines.append(f"    /** {cls}.{meth} ({cite}): {'records its inputs; ' if body else ''}its work runs"
                             f" in the build's last call. */")
                sig = ", ".join(f"{t} {n}" for t, n in ps)
                lines.append(f"    public static void {meth}({sig}) {{")
                if body:
                    lines.append(f"        {body}")
                lines.append("    }")
                lines.append("")
                continue
            _, meth, plist, cite, c_fn, cargs, note = e
            ps = params(plist)
            arrays = {n for t, n in ps if t in ("FloatArray", "IntArray")}
            idx = seen.get(c_fn, 0)
            seen[c_fn] = idx + 1
            hn = handle_name(c_fn, idx)
            layouts = ", ".join(l for _, l in cargs)
            lines.append(f"    private static final MethodHandle {hn} = Sbx.h(\"{c_fn}\",")
            lines.append(f"            FunctionDescriptor.of(JAVA_INT, {layouts}));")
            lines.append("")
            doc = f"    /** {cls}.{meth} ({cite}) -> {c_fn}."
            if note:
                doc += f" Note: {note}."
            lines.append(doc + " */")
            sig = ", ".join(f"{t} {n}" for t, n in ps)
            lines.append(f"    public static void {meth}({sig}) {{")
            # arrays the call reads (all of them) and writes (those at a non-const pointer)
            cdecl = header_args(c_fn)
            if len(cdecl) != len(cargs):
                raise ValueError(f"{c_fn}: {len(cargs)} arguments mapped, header has {len(cdecl)}")
            reads, writes = [], []
            for (x, l), decl in zip(cargs, cdecl):
                if l != A or x in ("CTX", "NULL"):
                    continue
                name = x if x in arrays or x.startswith(("GRID_BUILD", "CSR_BUILD")) else None
                if name is None:
                    continue
                reads.append(name)
                if "const" not in decl:
                    writes.append(name)
            if meth == "csrChunkReduce":
                lines.append("        CSR_BUILD.ensure(segMotorCount.getSize(), CSR_BUILD.nItems);")
            if meth == "csrChunkScatter":
                lines.append("        CSR_BUILD.ensure(segMotorOffsets.getSize() - 1, counts.get(0));")
            lines.append(f"        Sbx.toDevice({', '.join(reads)});")
            call = ", ".join(java_arg(x, l, arrays) if not x.startswith(("GRID_BUILD", "CSR_BUILD")) else
                             (x + ".dev()" if l == A else x) for x, l in cargs)
            lines.append("        try {")
            lines.append(f"            Sbx.check((int) {hn}.invokeExact({call}), \"{c_fn}\");")
            lines.append("        } catch (Throwable t) {")
            lines.append("            throw Sbx.rethrow(t);")
            lines.append("        }")
            if meth == "gridScanAdd":
                lines.append("        // the chunked reference leaves cellCount zero (its scan's write cursor, unused by")
                lines.append("        // the chunk scatter)")
                lines.append("        SbxAccess.memset(cellCount.dev(), 0, 4L * cellCount.getSize());")
            lines.append(f"        Sbx.written({', '.join(writes)});")
            lines.append("    }")
            lines.append("")
        if cls == "SpatialGrid":
            lines += ["    /** The inputs of the chunked grid build, recorded by gridChunkHistogram. */",
                      "    static final GridBuild GRID_BUILD = new GridBuild();", ""]
        if cls == "CrossBridgeSystem":
            lines += ["    /** The keys of the chunked CSR build, recorded by csrChunkHistogram, and its scratch. */",
                      "    static final CsrBuild CSR_BUILD = new CsrBuild();", ""]
        lines.append("}")
        files[f"{cls}Kernels.java"] = "\n".join(lines) + "\n"
    return files


def gen_functions(maxn=15):
    lines = ["package uk.ac.manchester.tornado.api.common;", "",
             "/** Stand-in: the functional interfaces TaskGraph.task method references bind to",
             " *  (generated by java/gen_shim.py). */",
             "public final class TornadoFunctions {", "    private TornadoFunctions() {}", ""]
    for n in range(1, maxn + 1):
        tp = ", ".join(f"T{i}" for i in range(1, n + 1))
        args = ", ".join(f"T{i} arg{i}" for i in range(1, n + 1))
        lines.append("    @FunctionalInterface")
        lines.append(f"    public interface Task{n}<{tp}> {{")
        lines.append(f"        void apply({args});")
        lines.append("    }")
        lines.append("")
    lines.append("}")
    return "\n".join(lines) + "\n"


def gen_taskgraph(maxn=15):
    lines = ["package uk.ac.manchester.tornado.api;", "",
             "import java.util.ArrayList;", "import java.util.List;", "",
             "import uk.ac.manchester.tornado.api.common.TornadoFunctions;",
             "import uk.ac.manchester.tornado.api.enums.DataTransferMode;", "",
             "/**",
             " * Stand-in for TornadoVM's TaskGraph (generated by java/gen_shim.py): records the",
             " * tasks, whose bodies are the System methods (now libsoftbox_b200 downcalls), and the",
             " * arrays to re-upload at every execute(); snapshot() freezes the list.",
             " */",
             "public final class TaskGraph {",
             "    private final String name;",
             "    private final List<Runnable> tasks = new ArrayList<>();",
             "    private final List<Object> everyExecution = new ArrayList<>();", "",
             "    public TaskGraph(String name) { this.name = name; }", "",
             "    public String getTaskGraphName() { return name; }", "",
             "    public TaskGraph transferToDevice(DataTransferMode mode, Object... arrays) {",
             "        if (mode == DataTransferMode.EVERY_EXECUTION) everyExecution.addAll(List.of(arrays));",
             "        return this;",
             "    }", "",
             "    public TaskGraph transferToHost(DataTransferMode mode, Object... arrays) { return this; }", "",
             "    public ImmutableTaskGraph snapshot() { return new ImmutableTaskGraph(tasks, everyExecution); }", ""]
    for n in range(1, maxn + 1):
        tp = ", ".join(f"T{i}" for i in range(1, n + 1))
        args = ", ".join(f"T{i} a{i}" for i in range(1, n + 1))
        call = ", ".join(f"a{i}" for i in range(1, n + 1))
        lines.append(f"    public <{tp}> TaskGraph task(String id, TornadoFunctions.Task{n}<{tp}> code, {args}) {{")
        lines.append(f"        tasks.add(() -> code.apply({call}));")
        lines.append("        return this;")
        lines.append("    }")
        lines.append("")
    lines.append("}")
    return "\n".join(lines) + "\n"


def write(path, text):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        f.write(text)


def main():
    for name, text in gen_kernels().items():
        write(os.path.join(SRC, "softbox_b200", "shim", name), text)
    write(os.path.join(SRC, "uk", "ac", "manchester", "tornado", "api", "common", "TornadoFunctions.java"),
          gen_functions())
    write(os.path.join(SRC, "uk", "ac", "manchester", "tornado", "api", "TaskGraph.java"), gen_taskgraph())


if __name__ == "__main__":
    main()
