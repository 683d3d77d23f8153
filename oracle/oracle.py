"""ctypes wrapper of the CPU oracle (test infrastructure only).

Loads oracle/_build/liboracle.so (libm transcendentals, the reference's platform math),
liboracle_dm.so (the portable double functions the CUDA kernels evaluate) or
liboracle_f64.so (liboracle_dm.so with every float evaluated as double: its array
arguments are float64 where the others take float32). Only the tests, the smoke check and
bench.py's CPU-baseline leg use this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")

# argument codes: i int32, I uint64, d double, f float, p pointer, s struct pointer
_SIGS = {
    "orc_set_threads": "i", "orc_max_threads": "", "orc_accurate_acos": "d", "orc_angle_from_sin_cos": "dd",
    "orc_kT": "", "orc_rod_drag_si": "dddp", "orc_sphere_drag_si": "ddp",
    "orc_drag_run_filament": "ipppdppppp", "orc_drag_run_motor": "idppppp", "orc_backbone_drag": "iddpppppp",
    "orc_brownian_force": "ipppppppp", "orc_brownian_force_philox": "ippppppppI",
    "orc_brownian_force_supplied": "ipppppppp", "orc_gauss6_wang": "iiip", "orc_gauss6_philox": "iiIp",
    "orc_zero_accumulators": "ipp", "orc_integrate": "ippppppppppp", "orc_derive": "ippppppp",
    "orc_confine": "ipppppppp", "orc_force_build": "ipppppppppp", "orc_integ_derive": "ippppppppppppppp",
    "orc_integ_derive_confined": "ipppppppppppppppp", "orc_chain_forces": "ipppppppppppp",
    "orc_seed_accumulators": "ipppp", "orc_pin_endpoints": "ipppippp", "orc_fil_publish": "ippipppppp",
    "orc_mot_publish_head": "ipppppp", "orc_mot_publish": "ippippppi", "orc_body_cell": "ipppip",
    "orc_grid_zero": "ip", "orc_grid_histogram": "pip", "orc_grid_scan_local": "ippp",
    "orc_grid_scan_chunks": "ip", "orc_grid_scan_add": "ipipp", "orc_grid_scatter": "pippip",
    "orc_body_chunk_size": "ii", "orc_grid_chunk_zero": "iip", "orc_grid_chunk_histogram": "piiiip",
    "orc_grid_chunk_reduce": "iipp", "orc_grid_chunk_scatter": "piiiippip", "orc_broad_phase": "ipppppppipp",
    "orc_brute_force": "ipppipp", "orc_invert_candidates": "ppppiipp",
    "orc_grid_reachable": "ipppippppppppppp", "orc_compute_reachable": "ipppippppppp",
    "orc_brute_reachable": "ipppippppp", "orc_bind_nearest": "ipppippppppp",
    "orc_bind_kinetics": "ipppippppppppp", "orc_cycle": "ippppp", "orc_catch_slip_release": "ipppppppp",
    "orc_bond_forces": "ippppipppppppppp", "orc_apply_head_force": "ippp",
    "orc_register_force_dot": "ipppppp", "orc_csr_histogram": "piip", "orc_csr_scan": "ipp",
    "orc_csr_scatter": "pippp", "orc_csr_chunk_zero": "iip", "orc_csr_chunk_histogram": "piiiip",
    "orc_csr_chunk_reduce": "iipp", "orc_csr_chunk_scatter": "piiiippp", "orc_seg_gather": "ippppp",
    "orc_xb_brute_gather": "iipppp", "orc_link_forces": "ippppippppppp", "orc_seg_gather_a": "ipppppp",
    "orc_seg_gather_b": "ipppppp", "orc_xl_brute_gather": "iipppppp", "orc_xl_unbind": "ippippppppppp",
    "orc_count_active_links": "ipppip", "orc_link_torsion": "ipipppppppp",
    "orc_compute_fil_link_ct": "ipppip", "orc_joints": "ippppppppp", "orc_dimer_couple": "ipppppppippppp",
    "orc_mini_tether": "ipppppppipppippppp", "orc_backbone_gather": "ippppp",
    "orc_mini_brute_gather": "iipppp", "orc_torsional_restore": "ipppdd", "orc_dense_step": "si",
    "orc_dense_run": "sii", "orc_dense_run_supplied": "siippp", "orc_fdt_run": "sii", "orc_chain_run": "sii",
    "orc_m_log": "d", "orc_m_exp": "d", "orc_m_sin": "d", "orc_m_cos": "d", "orc_m_eval": "iipp",
    "orc_xl_fil_fil_candidates": "ipppipppp", "orc_xl_grid_form_count": "ippppppppp",
    "orc_xl_grid_form_scan": "ippippp", "orc_xl_grid_form_emit": "ipppppppppippp",
    "orc_xl_form_gates": "ippppipppppppp", "orc_xl_form_admit_reduce": "ipppip",
    "orc_xl_form_admit": "ipppppppippppppp", "orc_xl_free_flags": "ipp", "orc_xl_free_scatter": "ippp",
    "orc_xl_allocate": "ipppppppippppppp", "orc_xl_place_orient": "ippppippp",
    "orc_growth_grow": "ippppppp",
    "orc_growth_mark_splits": "ipppppppppipp",
    "orc_growth_split_wire": "iipppppppppppp",
    "orc_growth_recompute_drag": "ipppppppppp",
    "orc_depoly": "ippppppppp",
    "orc_depoly_proxy": "ippppppppppp",
    "orc_apply_death": "ipppppppppp",
    "orc_cofilin_accumulate": "ippppp",
    "orc_cofilin_dissolve": "ippppppp",
    "orc_nucleate_fresh_cofilin": "iipppp",
    "orc_birth_allocate": "iiippppppppppppp",
    "orc_aging_age": "ipppp",
    "orc_aging_growth_atp": "ippp",
    "orc_aging_split_inherit_nuc": "iipppp",
    "orc_aging_nucleate_fresh_atp": "iipppp",
    "orc_filid_init": "ippp",
    "orc_filid_jump": "ippp",
    "orc_pool_put_total": "ppi", "orc_pool_take_total": "ppi", "orc_turnover_begin": "iiiddpppppp",
    "orc_turnover_release_dead": "pipppip", "orc_birth_emit_constant_actin": "ippiipppp",
    "orc_birth_init_newborn": "iipppppp", "orc_birth_tag_seeds": "iipppp", "orc_pool_take_births": "ppipii",
    "orc_obs_extent": "ipipppp", "orc_obs_stress": "iipppppppppppippppppdpp",
    "orc_obs_clusters": "ipippipppippippp",
}
_CT = {"i": C.c_int32, "I": C.c_uint64, "d": C.c_double, "f": C.c_float, "p": C.c_void_p, "s": C.c_void_p}
_RET = {"orc_max_threads": C.c_int, "orc_accurate_acos": C.c_double, "orc_angle_from_sin_cos": C.c_double,
        "orc_kT": C.c_double, "orc_body_chunk_size": C.c_int32,
        "orc_m_log": C.c_double, "orc_m_exp": C.c_double, "orc_m_sin": C.c_double, "orc_m_cos": C.c_double}


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


class Oracle:
    """One loaded oracle library. Array arguments may be numpy arrays (passed by
    pointer), None (NULL) or ctypes structures (passed by reference)."""

    def __init__(self, devmath=False, fp64=False):
        name = "liboracle_f64.so" if fp64 else ("liboracle_dm.so" if devmath else "liboracle.so")
        path = os.path.join(_BUILD, name)
        if not os.path.exists(path):
            build()
        self.lib = C.CDLL(path)
        self.devmath = devmath or fp64
        self.fp64 = fp64
        for fn, sig in _SIGS.items():
            f = getattr(self.lib, fn)
            f.argtypes = [_CT[c] for c in sig]
            f.restype = _RET.get(fn, None)

    def __getattr__(self, name):
        fn = getattr(self.lib, "orc_" + name)
        sig = _SIGS["orc_" + name]

        def call(*args):
            if len(args) != len(sig):
                raise TypeError(f"orc_{name} takes {len(sig)} args, got {len(args)}")
            conv = []
            for a, c in zip(args, sig):
                if c in "ps":
                    if a is None:
                        conv.append(None)
                    elif isinstance(a, np.ndarray):
                        assert a.flags["C_CONTIGUOUS"]
                        conv.append(a.ctypes.data)
                    elif isinstance(a, C.Structure):
                        conv.append(C.addressof(a))
                    else:
                        raise TypeError(f"bad pointer arg {type(a)} for orc_{name}")
                else:
                    conv.append(a)
            return fn(*conv)
        return call


_cache = {}


def get(devmath=False, fp64=False):
    key = (devmath, fp64)
    if key not in _cache:
        _cache[key] = Oracle(devmath, fp64)
    return _cache[key]


def to_fp64(obj):
    """A copy of a (nested) host scene for the FP64 build: float32 arrays become float64,
    the separate FP64 centres are dropped (the centres themselves are double there)."""
    if isinstance(obj, dict):
        return {k: to_fp64(v) for k, v in obj.items() if k != "coord64"}
    if isinstance(obj, np.ndarray) and obj.dtype == np.float32:
        return obj.astype(np.float64)
    if isinstance(obj, np.ndarray):
        return obj.copy()
    return obj
