"""ctypes binding of the C ABI declared in include/dgb.h (loads the in-tree libdgb.so)."""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libdgb.so"

# enum values (include/dgb.h)
OK, ERR_ARG, ERR_IO, ERR_MESH, ERR_UNSUPPORTED, ERR_CUDA, ERR_NONFINITE, ERR_DT_SMALL, ERR_TIMEOUT, ERR_NO_DEVICE = range(10)
FLUX = {"rusanov": 0, "rus": 0, "llf": 0, "hll": 1, "roe": 2}
LIMITER = {"none": 0, "hrl": 1, "m2l": 2, "hri": 3, "m2i": 4, "prl": 5, "pri": 6, "p0i": 7}
SSPRK3, RK4 = 3, 4
FORM = {"fp64": 0, "mixed": 1}
GAMMA_MODEL = {"gamncon": 0, "gamcons": 1}
BC = {"periodic": 1, "transmissive": 2, "reflective": 3, "frozen": 4}

# every exported entry point of include/dgb.h
EXPORTS = [
    "dgb_last_error", "dgb_abi_version", "dgb_problem_from_deck", "dgb_problem_structured",
    "dgb_mesh_write_msh", "dgb_problem_destroy", "dgb_problem_info", "dgb_problem_array_size",
    "dgb_problem_get_array", "dgb_problem_init_state", "dgb_write_pos", "dgb_read_pos", "dgb_create",
    "dgb_destroy", "dgb_set_state", "dgb_get_state", "dgb_set_state_device", "dgb_get_state_device",
    "dgb_residual", "dgb_solve", "dgb_limit", "dgb_dt_from_cfl", "dgb_advance", "dgb_last_dt",
    "dgb_conservation", "dgb_last_timing", "dgb_set_profiling", "dgb_kernel_timing", "dgb_limit_noalloc",
    "dgb_sensors", "dgb_set_form", "dgb_mlp_param_count", "dgb_indicator_features", "dgb_indicator_labels",
    "dgb_mlp_forward", "dgb_mlp_backward", "dgb_mlp_adam", "dgb_set_indicator", "dgb_indicator_scores",
    "dgb_cfl_dt", "dgb_batch_create", "dgb_batch_destroy", "dgb_batch_n_classes", "dgb_batch_class_info",
    "dgb_batch_autotune", "dgb_batch_set_tuning", "dgb_batch_advance", "dgb_problem_error_norms", "dgb_batch_case_stats",
    "dgb_batch_last_timing", "dgb_slab_ghost_rows", "dgb_step_begin", "dgb_step_wavespeed_word", "dgb_step_stage",
    "dgb_step_end", "dgb_halo_count", "dgb_halo_pack", "dgb_halo_unpack", "dgb_stream", "dgb_set_cfl_scale",
    "dgb_set_wait_limit", "dgb_set_indicator_interval", "dgb_slabs_advance_local", "dgb_advance_host",
]


class MeshSpec(C.Structure):
    _fields_ = [("dim", C.c_int), ("order", C.c_int), ("nx", C.c_int), ("ny", C.c_int),
                ("x0", C.c_double), ("x1", C.c_double), ("y0", C.c_double), ("y1", C.c_double),
                ("bc", C.c_int * 4)]


class Options(C.Structure):
    _fields_ = [("flux", C.c_int), ("limiter", C.c_int), ("cfl", C.c_double),
                ("thresholds", C.c_double * 3), ("n_thresholds", C.c_int), ("n_mass", C.c_int),
                ("gamma_model", C.c_int)]


class Info(C.Structure):
    _fields_ = [(n, C.c_int) for n in
                "dim order n_fields n_elem n_s n_g n_ifaces m_s m_g n_n n_reflective cartesian "
                "gpu_supported flux limiter nx ny".split()] + \
               [(n, C.c_double) for n in "cfl dx_min cfl_scaled final_time".split()] + \
               [("n_output_times", C.c_int), ("error_output", C.c_int), ("gamma_model", C.c_int),
                                            ("cons_output", C.c_int)]


class DGBError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dgb error {code}: {msg}")
        self.code = code


_lib = None


def lib() -> C.CDLL:
    """Loads libdgb.so; raises if it is missing (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("DGB_LIB", LIB_PATH))
    if not path.exists():
        raise ImportError(f"{path} is not built; run `python -m dg_b200.build`")
    L = C.CDLL(str(path))
    vp, ip, dp, cp = C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_char_p
    L.dgb_last_error.restype = cp
    L.dgb_abi_version.restype = ip
    sig = {
        "dgb_problem_from_deck": [cp, C.POINTER(vp)],
        "dgb_problem_structured": [C.POINTER(MeshSpec), C.POINTER(Options), C.POINTER(vp)],
        "dgb_mesh_write_msh": [C.POINTER(MeshSpec), cp],
        "dgb_problem_info": [vp, C.POINTER(Info)],
        "dgb_problem_array_size": [vp, cp, C.POINTER(C.c_size_t)],
        "dgb_problem_get_array": [vp, cp, vp, C.c_size_t],
        "dgb_problem_init_state": [vp, cp, dp, ip, C.c_uint64, dp],
        "dgb_write_pos": [vp, dp, ip, C.c_double, cp],
        "dgb_read_pos": [vp, ip, cp, dp, dp],
        "dgb_problem_error_norms": [vp, dp, dp, dp],
        "dgb_create": [vp, ip, C.POINTER(vp)],
        "dgb_set_state": [vp, dp],
        "dgb_get_state": [vp, dp],
        "dgb_set_state_device": [vp, vp],
        "dgb_get_state_device": [vp, vp],
        "dgb_residual": [vp, dp, dp],
        "dgb_solve": [vp, C.c_double, dp, dp],
        "dgb_limit": [vp, dp],
        "dgb_sensors": [vp, dp, C.POINTER(C.c_int)],
        "dgb_set_form": [vp, ip],
        "dgb_set_wait_limit": [vp, C.c_longlong],
        "dgb_set_indicator_interval": [vp, ip],
        "dgb_cfl_dt": [vp, dp],
        "dgb_indicator_features": [vp, vp],
        "dgb_indicator_labels": [vp, vp],
        "dgb_mlp_forward": [vp, vp, ip, vp, vp, vp],
        "dgb_mlp_backward": [vp, vp, vp, C.c_float, ip, vp, vp, vp, vp, vp, vp],
        "dgb_mlp_adam": [vp, vp, vp, vp, ip, C.c_float, vp],
        "dgb_set_indicator": [vp, vp, C.c_float],
        "dgb_indicator_scores": [vp, dp, C.POINTER(C.c_float), C.POINTER(C.c_int)],
        "dgb_dt_from_cfl": [vp, dp, dp],
        "dgb_advance": [vp, ip, ip, C.c_double, dp],
        "dgb_advance_host": [vp, dp, ip, ip, C.c_double, dp],
        "dgb_last_dt": [vp, dp],
        "dgb_conservation": [vp, dp],
        "dgb_last_timing": [vp, dp, C.POINTER(C.c_longlong)],
        "dgb_set_profiling": [vp, ip],
        "dgb_kernel_timing": [vp, cp, dp, C.POINTER(C.c_longlong)],
        "dgb_limit_noalloc": [vp, vp, vp, vp],
        "dgb_batch_create": [C.POINTER(vp), ip, C.POINTER(vp)],
        "dgb_batch_n_classes": [vp],
        "dgb_batch_class_info": [vp, ip, C.POINTER(C.c_int)],
        "dgb_batch_autotune": [vp, ip],
        "dgb_batch_set_tuning": [vp, ip, ip, ip, ip, ip],
        "dgb_batch_advance": [vp, ip, C.c_double, C.POINTER(C.c_int)],
        "dgb_batch_case_stats": [vp, dp, C.POINTER(C.c_int), dp],
        "dgb_batch_last_timing": [vp, dp, C.POINTER(C.c_longlong)],
        "dgb_slab_ghost_rows": [vp, ip, ip],
        "dgb_step_begin": [vp, ip, C.c_double],
        "dgb_step_wavespeed_word": [vp, C.POINTER(vp)],
        "dgb_step_stage": [vp, ip],
        "dgb_step_end": [vp, dp],
        "dgb_halo_count": [vp, ip, C.POINTER(C.c_size_t)],
        "dgb_halo_pack": [vp, ip, vp],
        "dgb_halo_unpack": [vp, ip, vp],
        "dgb_stream": [vp, C.POINTER(vp)],
        "dgb_set_cfl_scale": [vp, C.c_double],
        "dgb_slabs_advance_local": [C.POINTER(vp), ip, ip, ip, ip, C.c_double, dp],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ip
    L.dgb_mlp_param_count.argtypes = []
    L.dgb_mlp_param_count.restype = ip
    L.dgb_problem_destroy.argtypes = [vp]
    L.dgb_problem_destroy.restype = None
    L.dgb_destroy.argtypes = [vp]
    L.dgb_destroy.restype = None
    L.dgb_batch_destroy.argtypes = [vp]
    L.dgb_batch_destroy.restype = None
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != OK:
        raise DGBError(rc, lib().dgb_last_error().decode())


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))
