"""softbox_b200 — B200-native per-step Brownian rigid-rod mechanics.

The compute path is hand-written sm_100a CUDA behind the C ABI declared in
include/softbox_b200.h (libsoftbox_b200.so, built in-tree by softbox_b200/build.py).
Python here only builds scenes on the host, moves arrays to the device with PyTorch,
and calls the library; there is no CPU fallback: importing the bindings fails loudly
when the library is missing.
"""
__all__ = ["scenes", "javarandom", "abi_types"]
