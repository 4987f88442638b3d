"""ctypes binding of libsfp.so (include/sfp.h).

The library is built in-tree by ``sfparticles_b200.build`` and is the only
compute path of this package: every call raises ``SFPError`` when the library
is missing or a CUDA device is unavailable -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import threading

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libsfp.so")


class SFPError(RuntimeError):
    """Raised when libsfp.so reports an error or cannot be used."""


c_d, c_i64, c_i32, c_u32, c_u64, c_sz, P = (ctypes.c_double, ctypes.c_int64, ctypes.c_int32, ctypes.c_uint32,
                                            ctypes.c_uint64, ctypes.c_size_t, ctypes.c_void_p)

# ---- data layouts of include/sfp_types.h -----------------------------------


class Segment(ctypes.Structure):
    _fields_ = [
        ("x", P), ("y", P), ("z", P), ("ux", P), ("uy", P), ("uz", P),
        ("sx", P), ("sy", P), ("sz", P), ("tau", P), ("delta", P), ("pruned", P),
        ("capacity", c_i64), ("q", c_d), ("ae", c_d),
        ("massless", c_i32), ("push", c_i32), ("rr", c_i32), ("spin", c_i32),
        ("radiating", c_i32), ("bw", c_i32), ("photon_dest", c_i32), ("ele_dest", c_i32), ("pos_dest", c_i32),
        ("channel", c_i32), ("instance", c_i32), ("stream", c_u32),
    ]


class Instance(ctypes.Structure):
    _fields_ = [("seed", c_u64), ("field_params", P), ("first_seg", c_i32), ("n_seg", c_i32)]


class ODTable(ctypes.Structure):
    _fields_ = [
        ("rate_total", P), ("cumulative", P), ("chi_N", c_i32), ("delta_N", c_i32),
        ("log_chi_min", c_d), ("log_chi_delta", c_d), ("log_chi_max", c_d),
        ("log_delta_min", c_d), ("log_delta_delta", c_d),
    ]


class RSTable(ctypes.Structure):
    _fields_ = [("int_Ai", P), ("Aip", P), ("z_N", c_i32), ("pad", c_i32), ("z_max", c_d)]


class RunState(ctypes.Structure):
    _fields_ = [("t", c_d), ("step", c_i64), ("halted", c_i32), ("error", c_i32), ("particle_steps", c_i64),
                ("appends_pending", c_i32), ("pad", c_i32)]


class RunConfig(ctypes.Structure):
    _fields_ = [("dt", c_d), ("photon_threshold", c_d), ("t0", c_d), ("step0", c_i64), ("qed", c_i32), ("form", c_i32),
                ("m_stages", c_i32), ("min_blocks", c_i32), ("p_stages", c_i32), ("p_min_blocks", c_i32), ("mlp_params", P),
                ("rs", RSTable), ("od_photon", ODTable),
                ("od_pair", ODTable)]


SFP_QED_REJECTION, SFP_QED_OPTICAL_DEPTH = 0, 1
SFP_FORM_FP64, SFP_FORM_FP32 = 0, 1
SFP_FIELD_PARAMS = 16
DEV_ERRORS = {2: "tile table too small", 3: "a long-tile step kernel met a step planned with shorter tiles"}

_SIGS = {
    "sfp_version": ([], ctypes.c_char_p),
    "sfp_last_error": ([], ctypes.c_char_p),
    "sfp_device_count": ([P], c_i32),
    "sfp_free": ([P], None),
    "sfp_nvrtc_compile": ([ctypes.c_char_p, ctypes.c_char_p, P, c_i32, P, P, P], c_i32),
    "sfp_module_load": ([P, c_sz, P], c_i32),
    "sfp_module_unload": ([P], c_i32),
    "sfp_field_eval": ([P, P, P, P, P, c_d, c_i64, P, P, P, P, P, P, P, P], c_i32),
    "sfp_push_position": ([P] * 7 + [c_i64, P, c_d, P], c_i32),
    "sfp_boris": ([P] * 10 + [c_d, c_i64, P, c_d, P], c_i32),
    "sfp_boris_tbmt": ([P] * 13 + [c_d, c_d, c_i64, P, c_d, P], c_i32),
    "sfp_LL_push": ([P] * 5 + [c_i64, P, c_d, P], c_i32),
    "sfp_CLL_push": ([P] * 5 + [c_i64, P, c_d, P], c_i32),
    "sfp_update_chi": ([P] * 11 + [c_i64, P, P], c_i32),
    "sfp_photon_recoil": ([P] * 6 + [c_i64, P, P], c_i32),
    "sfp_pick_hard_photon": ([P, P, P, c_d, c_i64, P], c_i32),
    "sfp_bool_sum": ([P, c_i64, P, P], c_i32),
    "sfp_find_event_index_workspace": ([c_i64], c_sz),
    "sfp_find_event_index": ([P, c_i64, c_i64, P, P, c_sz, P], c_i32),
    "sfp_find_event_index_noalloc": ([P, c_i64, c_i64, P, P], c_i32),
    "sfp_create_photon": ([P] * 16 + [c_i64, c_i64, P], c_i32),
    "sfp_create_pair": ([P] * 17 + [c_i64, c_i64, c_i32, P], c_i32),
    "sfp_photon_from_rejection_sampling": ([P, P, c_d, c_i64, P, P, P, P, c_u64, c_u32, c_u32, P], c_i32),
    "sfp_pair_from_rejection_sampling": ([P, P, c_d, c_i64, P, P, P, P, c_u64, c_u32, c_u32, P], c_i32),
    "sfp_update_tau": ([P, P, P, c_d, c_i64, P, P, P, P, c_u64, c_u32, c_u32, P], c_i32),
    "sfp_inv_gamma": ([P, P, P, P, c_i64, c_i32, P], c_i32),
    "sfp_run_create": ([P, P, c_i32, P, c_i32, P, P, P], c_i32),
    "sfp_run_update": ([P, c_i32, P, P], c_i32),
    "sfp_run_steps": ([P, c_i64, c_i32, P], c_i32),
    "sfp_run_steps_timed": ([P, c_i64, P, P], c_i32),
    "sfp_run_read_state": ([P, P, P, P], c_i32),
    "sfp_run_clear_halt": ([P, P], c_i32),
    "sfp_run_pending_need": ([P, P], c_i32),
    "sfp_run_resume": ([P, P], c_i32),
    "sfp_run_sync_positions": ([P, P], c_i32),
    "sfp_od_inverse_cdf": ([P, P, P, P, c_i64, P], c_i32),
    "sfp_mlp_make_samples": ([P, ctypes.c_uint64, ctypes.c_uint32, c_d, c_d, c_i64, P, P, P], c_i32),
    "sfp_mlp_grad": ([P, P, P, c_i64, P, P, P], c_i32),
    "sfp_mlp_adam": ([P, P, P, P, c_i64, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                      ctypes.c_float, P], c_i32),
    "sfp_mlp_infer": ([P, P, P, P, c_i64, P], c_i32),
    "sfp_mlp_infer_warp": ([P, P, P, P, c_i64, P], c_i32),
    "sfp_mlp_device_error": ([P], c_i32),
    "sfp_mlp_infer_withheld": ([P, P, P, P, c_i64, P], c_i32),
    "sfp_table_rs": ([P, c_i64, P, P, P], c_i32),
    "sfp_pair_rate_bound": ([P, P, c_i32, c_d, P, P], c_i32),
    "sfp_table_od": ([c_i32, c_d, P, c_i64, P, c_i64, P, P, P, P], c_i32),
    "sfp_run_destroy": ([P], c_i32),
}

_lib = None
_lock = threading.Lock()


def declared_symbols():
    return list(_SIGS)


def load(build_if_missing: bool = True):
    """Load libsfp.so (building it in-tree first when it is missing)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            if not build_if_missing:
                raise SFPError(f"{LIB_PATH} is missing; run sfparticles_b200.build.build()")
            from . import build as _build
            _build.build_library()
        try:
            L = ctypes.CDLL(LIB_PATH)
        except OSError as e:  # pragma: no cover - environment problem
            raise SFPError(f"cannot load {LIB_PATH}: {e}") from e
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
        return L


def check(rc: int, what: str = ""):
    if rc != 0:
        msg = load().sfp_last_error().decode(errors="replace")
        raise SFPError(f"{what}: {msg}" if what else msg)


def call(name: str, *args):
    """Call a status-returning entry point and raise on failure."""
    L = load()
    rc = getattr(L, name)(*args)
    check(rc, name)


def device_available() -> bool:
    L = load()
    n = c_i32(0)
    rc = L.sfp_device_count(ctypes.byref(n))
    return rc == 0 and n.value > 0
