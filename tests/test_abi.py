"""The C-ABI library: it builds for sm_100a, loads, and exports every declared symbol.
No kernel is launched here (this runs on machines without a GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_builds_and_loads():
    from softbox_b200 import build
    lib = build.build()
    assert os.path.exists(lib)
    ctypes.CDLL(lib)


def test_every_declared_symbol_is_exported():
    from softbox_b200 import build, runtime
    lib = build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (sbx_\w+)", out))
    declared = set(runtime.SIGS)
    assert declared, "no declarations parsed"
    assert declared <= exported, sorted(declared - exported)


def test_binding_signatures_follow_header():
    from softbox_b200 import runtime
    import ctypes as C
    rt, args = runtime.SIGS["sbx_brownian_force_philox"]
    assert rt is C.c_int32 and args[-1] is C.c_uint64 and len(args) == 11
    rt, args = runtime.SIGS["sbx_ctx_last_error"]
    assert rt is C.c_char_p
