"""The Java side of the drop-in boundary (java/): the generated sources are current, and every
Foreign Function & Memory downcall descriptor matches the C declaration in
include/softbox_b200.h (argument count, each argument's layout, the return layout). The Java
sources are not compiled here (no JDK on this image); this check is what guards them."""
import glob
import os
import re
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JAVA = os.path.join(ROOT, "java")
sys.path.insert(0, JAVA)


def _c_layout(decl):
    d = decl.replace("const", "").strip()
    if "*" in d or "[" in d:
        return "ADDRESS"
    base = d.split()[0]
    return {"int32_t": "JAVA_INT", "int": "JAVA_INT", "double": "JAVA_DOUBLE", "float": "JAVA_FLOAT",
            "int64_t": "JAVA_LONG", "uint64_t": "JAVA_LONG", "size_t": "JAVA_LONG"}[base]


def _header():
    text = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "softbox_b200.h")).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"^\s*([\w\s\*]+?)\s*\b(sbx_\w+)\s*\(([^;{]*?)\)\s*;", text, re.M | re.S):
        ret, name, args = m.group(1).strip(), m.group(2), m.group(3)
        if ret.startswith("typedef"):
            continue
        rl = "ADDRESS" if ret.endswith("*") else ("JAVA_LONG" if ret == "int64_t" else "JAVA_INT")
        argl = [a.strip() for a in args.split(",") if a.strip() and a.strip() != "void"]
        out[name] = (rl, [_c_layout(a) for a in argl])
    return out


def _downcalls():
    found = []
    for path in glob.glob(os.path.join(JAVA, "src", "**", "*.java"), recursive=True):
        src = open(path).read()
        for m in re.finditer(r'Sbx\.h\("(\w+)",\s*FunctionDescriptor\.of\(([^)]*)\)\)', src, re.S):
            layouts = [x.strip() for x in m.group(2).split(",")]
            found.append((os.path.relpath(path, JAVA), m.group(1), layouts[0], layouts[1:]))
    return found


def test_generated_sources_are_current(tmp_path):
    import gen_shim
    saved = gen_shim.SRC
    gen_shim.SRC = str(tmp_path)
    try:
        gen_shim.main()
    finally:
        gen_shim.SRC = saved
    for p in glob.glob(str(tmp_path / "**" / "*.java"), recursive=True):
        rel = os.path.relpath(p, tmp_path)
        committed = os.path.join(JAVA, "src", rel)
        assert os.path.exists(committed), rel
        assert open(p).read() == open(committed).read(), f"{rel} differs from java/gen_shim.py's output"


def test_every_downcall_descriptor_matches_the_header():
    hdr = _header()
    calls = _downcalls()
    assert len(calls) >= 35
    for path, name, ret, args in calls:
        assert name in hdr, f"{path}: {name} is not declared in the header"
        want_ret, want_args = hdr[name]
        assert ret == want_ret, (path, name, ret, want_ret)
        assert args == want_args, (path, name, args, want_args)


def test_shim_covers_the_harness_system_methods():
    """Every System method the dense contractile and diffusion harnesses call (their cpuStep
    and buildPlan task lists) has a body in the shim."""
    need = {"SpatialGrid": ["bodyCell", "gridChunkZero", "gridChunkHistogram", "gridChunkReduce", "gridScanLocal",
                            "gridScanChunks", "gridScanAdd", "gridChunkScatter"],
            "BindingDetectionSystem": ["gridReachable", "bindNearest"],
            "NucleotideCycleSystem": ["cycle", "catchSlipRelease"],
            "BrownianForceSystem": ["brownianForce"],
            "ChainBendingForceSystem": ["zeroAccumulators", "chainForces"],
            "ContainmentSystem": ["confine"],
            "RigidRodLangevinIntegrationSystem": ["integrate"],
            "DerivedGeometrySystem": ["derive"],
            "FilamentStore": ["publishToBodyView"],
            "MotorStore": ["publishHeadFromBody", "publishToBodyView"],
            "MotorJointSystem": ["joints"], "DimerCouplingSystem": ["couple"],
            "MiniFilamentSystem": ["tether", "backboneGather"],
            "CrossBridgeSystem": ["bondForces", "applyHeadForce", "registerForceDot", "csrScan", "csrChunkZero",
                                  "csrChunkHistogram", "csrChunkReduce", "csrChunkScatter", "segGather"],
            "CrosslinkerSystem": ["countActiveLinks", "linkForces", "linkTorsion", "segGatherA", "segGatherB",
                                  "unbind"],
            "DeflectionSupport": ["seedAccumulators", "pinEndpoints"],
            "DragTensorSystem": ["runFilament", "runMotor"]}
    for cls, methods in need.items():
        src = open(os.path.join(JAVA, "src", "softbox_b200", "shim", cls + "Kernels.java")).read()
        for m in methods:
            assert re.search(r"public static void " + m + r"\(", src), (cls, m)


def test_stand_ins_cover_the_tornado_api_surface():
    base = os.path.join(JAVA, "src", "uk", "ac", "manchester", "tornado", "api")
    for rel, names in {"TaskGraph.java": ["transferToDevice", "transferToHost", "snapshot", "task"],
                       "TornadoExecutionPlan.java": ["withGridScheduler", "execute"],
                       "TornadoExecutionResult.java": ["transferToHost"],
                       "GridScheduler.java": ["addWorkerGrid"], "WorkerGrid.java": ["setLocalWork"],
                       "types/arrays/FloatArray.java": ["get", "set", "getSize", "init", "fromElements"],
                       "types/arrays/IntArray.java": ["get", "set", "getSize", "init", "fromElements"]}.items():
        src = open(os.path.join(base, rel)).read()
        for n in names:
            assert re.search(r"\b" + n + r"\(", src), (rel, n)
    tg = open(os.path.join(base, "TaskGraph.java")).read()
    assert "Task15<" in tg
