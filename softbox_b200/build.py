"""Builds libsoftbox_b200.so in-tree (softbox_b200/_lib/) with nvcc for sm_100a.

Floating-point flags are part of the contract: -fmad=false (no FMA contraction),
IEEE division and square root, no flush-to-zero. With them every float/double
operation in the kernels is one IEEE round-to-nearest step, which is what lets the
kernels reproduce the reference's (and the CPU oracle's) bits.

    python -m softbox_b200.build [--force] [--verbose-ptxas] [--check]

--check builds the index-checking debug library (libsoftbox_b200_check.so, -DSBX_CHECK): its
kernels test every data-dependent index against the array it indexes, count and skip bad
ones (sbx_check_report). Select it at load time with SBX_LIB=check.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libsoftbox_b200.so")
LIB_CHECK = os.path.join(OUT_DIR, "libsoftbox_b200_check.so")
SOURCES = ["sbx_systems.cu", "sbx_sort.cu", "sbx_dense.cu", "sbx_free.cu", "sbx_fused.cu", "sbx_noalloc.cu", "sbx_form.cu", "sbx_turnover.cu", "sbx_batch.cu", "sbx_obs.cu", "sbx_mlp.cu", "sbx_turnover_batch.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FP_FLAGS = ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".h"))]
    files.append(os.path.join(ROOT, "include", "softbox_b200.h"))
    return files


def up_to_date(lib=LIB):
    if not os.path.exists(lib):
        return False
    t = os.path.getmtime(lib)
    return all(os.path.getmtime(f) <= t for f in _deps())


def build(force=False, verbose_ptxas=False, check=False):
    lib = LIB_CHECK if check else LIB
    if not force and up_to_date(lib):
        return lib
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = [nvcc_path(), "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-lineinfo"] + ARCH + FP_FLAGS
    if check:
        cmd += ["-DSBX_CHECK"]
    cmd += ["-I" + os.path.join(ROOT, "include"), "-o", lib + ".tmp"]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    # the host compiler must be the system g++ (an environment CXX wrapper may lack pieces)
    env = dict(os.environ)
    if os.path.exists("/usr/bin/g++"):
        cmd += ["-ccbin", "/usr/bin/g++"]
    r = subprocess.run(cmd, capture_output=True, text=True, env=env)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed")
    if verbose_ptxas:
        sys.stderr.write(r.stderr)
    os.replace(lib + ".tmp", lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="--verbose-ptxas" in sys.argv,
                check="--check" in sys.argv))
