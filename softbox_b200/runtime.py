"""Loads libsoftbox_b200.so and exposes its C ABI to Python.

Argument and return types are read from include/softbox_b200.h, so the binding cannot
drift from the declared ABI. There is no fallback: if the library is missing or cannot
be loaded, importing this module raises, and on a machine without a CUDA device every
call fails with the CUDA runtime's error.
"""
import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
HEADER = os.path.join(ROOT, "include", "softbox_b200.h")
# SBX_LIB=check loads the index-checking debug build (python -m softbox_b200.build --check)
LIB_PATH = os.path.join(HERE, "_lib", "libsoftbox_b200_check.so" if os.environ.get("SBX_LIB") == "check"
                        else "libsoftbox_b200.so")

STATUS = {0: "SBX_OK", -1: "SBX_EINVAL", -2: "SBX_ECUDA", -3: "SBX_EOVERFLOW", -4: "SBX_ETIMEOUT",
          -5: "SBX_ENOMEM", -6: "SBX_ENONFINITE", -7: "SBX_ESTATE"}


class SbxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def _ctype(decl):
    d = decl.replace("const ", "").strip()
    if "*" in d:
        return C.c_void_p
    base = d.split()[0]
    return {"int32_t": C.c_int32, "int": C.c_int, "double": C.c_double, "float": C.c_float,
            "uint64_t": C.c_uint64, "int64_t": C.c_int64, "size_t": C.c_size_t}[base]


def parse_header(path=HEADER):
    """name -> (restype, [argtypes]) for every function declared in the header."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"^\s*([\w\s\*]+?)\s*\b(sbx_\w+)\s*\(([^;{]*?)\)\s*;", text, re.M | re.S):
        ret, name, args = m.group(1).strip(), m.group(2), m.group(3)
        if ret.startswith("typedef"):
            continue
        rt = {"sbx_status": C.c_int32, "const char*": C.c_char_p, "void*": C.c_void_p, "int64_t": C.c_int64,
              "int32_t": C.c_int32}.get(ret.replace(" *", "*").replace("char *", "char*"), C.c_int32)
        if "char" in ret:
            rt = C.c_char_p
        elif ret.endswith("*"):
            rt = C.c_void_p
        argl = [a.strip() for a in args.split(",") if a.strip() and a.strip() != "void"]
        out[name] = (rt, [_ctype(a.rsplit(" ", 1)[0] + (" *" if "*" in a else "")) for a in argl])
    return out


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m softbox_b200.build` "
                          "(there is no CPU fallback for the mechanics path)")
    lib = C.CDLL(LIB_PATH)
    sigs = parse_header()
    for name, (rt, at) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = rt
        fn.argtypes = at
    return lib, sigs


LIB, SIGS = _load()


def _arg(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    if isinstance(a, C.Structure):
        return C.addressof(a)
    return a


class Context:
    """One sbx_ctx bound to a CUDA device and stream (torch's current stream by default,
    so library launches and torch operations are ordered on the same queue)."""

    def __init__(self, device=0, stream=None):
        import torch
        if stream is None:
            # torch's legacy default stream (handle 0) cannot be captured into a graph:
            # the library then creates its own blocking stream, which stays ordered with it
            stream = torch.cuda.current_stream(device).cuda_stream or None
        self.device = device
        h = C.c_void_p()
        st = LIB.sbx_ctx_create(device, C.c_void_p(stream), C.byref(h))
        if st != 0:
            raise SbxError(st, "sbx_ctx_create failed")
        self.h = h

    def __call__(self, name, *args):
        fn = getattr(LIB, name)
        st = fn(self.h, *[_arg(a) for a in args])
        if fn.restype is C.c_int32 and st != 0:
            raise SbxError(st, f"{name}: {LIB.sbx_ctx_last_error(self.h).decode()}")
        return st

    def raw(self, name, *args):
        """Call without raising; returns the status code."""
        return getattr(LIB, name)(self.h, *[_arg(a) for a in args])

    def last_error(self):
        return LIB.sbx_ctx_last_error(self.h).decode()

    def launches(self):
        return LIB.sbx_ctx_launch_count(self.h)

    def scratch_bytes(self):
        return LIB.sbx_ctx_scratch_bytes(self.h)

    def sync(self):
        self("sbx_ctx_sync")

    def close(self):
        if self.h:
            LIB.sbx_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default = None


def default_context():
    global _default
    if _default is None:
        _default = Context(0)
    return _default
