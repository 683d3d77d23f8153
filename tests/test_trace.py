"""NVTX ranges of the host-side step sequence: a small injection tool (tests/nvtx_count_tool.c,
built here with gcc) counts the pushes and pops the library makes. The free-rod entry point
opens its range before its argument checks, so a call with a null context exercises the
mechanism without a GPU."""
import os
import shutil
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CUDA_INC = "/usr/local/cuda/include"


def test_range_names_in_library():
    from softbox_b200.runtime import LIB_PATH
    data = open(LIB_PATH, "rb").read()
    for name in (b"sbx.dense.step", b"sbx.dense.binding", b"sbx.dense.filament_forces", b"sbx.dense.myosin",
                 b"sbx.dense.integrate", b"sbx.dense.fused_launch", b"sbx.dense.graph_replay",
                 b"sbx.dense.unfused", b"sbx.dense.capture", b"sbx.free.run"):
        assert name in data, name


@pytest.mark.skipif(shutil.which("gcc") is None or not os.path.isdir(os.path.join(CUDA_INC, "nvtx3")),
                    reason="gcc or the NVTX headers missing")
def test_ranges_reach_an_injected_tool(tmp_path):
    tool = tmp_path / "libnvtxcount.so"
    subprocess.run(["gcc", "-shared", "-fPIC", "-O1", "-I" + CUDA_INC, "-o", str(tool),
                    os.path.join(HERE, "nvtx_count_tool.c")], check=True)
    out = tmp_path / "counts.txt"
    code = ("import ctypes as C, sys; sys.path.insert(0, %r)\n"
            "from softbox_b200.runtime import LIB\n"
            "st = LIB.sbx_free_rods_run(None, None, 0, 1, 0, 0, None)\n"
            "assert st != 0, st\n" % ROOT)
    env = dict(os.environ, NVTX_INJECTION64_PATH=str(tool), SBX_NVTX_COUNT_OUT=str(out))
    subprocess.run([sys.executable, "-c", code], check=True, env=env, cwd=ROOT)
    pushes, pops, names = out.read_text().split(" ", 2)
    assert int(pushes) == 1 and int(pops) == 1, (pushes, pops)
    assert names.strip().rstrip(",") == "sbx.free.run"


def test_check_build_library():
    """The index-checking debug twin is built beside the library, flags itself and exports
    the same C ABI (its counters read as zeros through the normal build)."""
    import ctypes as C
    from softbox_b200.runtime import LIB, LIB_PATH, parse_header
    check = os.path.join(os.path.dirname(LIB_PATH), "libsoftbox_b200_check.so")
    assert os.path.exists(check)
    lib = C.CDLL(check)
    for name in parse_header():
        getattr(lib, name)
    lib.sbx_check_build.restype = C.c_int32
    assert lib.sbx_check_build() == 1
    assert LIB.sbx_check_build() == 0
    c, s, i = C.c_int64(5), C.c_int32(5), C.c_int64(5)
    assert LIB.sbx_check_report(C.byref(c), C.byref(s), C.byref(i), 0) == 0
    assert (c.value, s.value, i.value) == (0, 0, 0)
