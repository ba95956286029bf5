"""ctypes binding of libnfgs_b200.so (declarations in include/nfgs_b200.h).

The library is the only compute path: if it cannot be loaded, importing
this module raises.  There is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("NFGS_B200_LIB", HERE / "libnfgs_b200.so"))

NFGS_OK = 0
NFGS_EINVAL = 1
NFGS_ECUDA = 2
NFGS_ENOMEM = 3
NFGS_ESTATE = 4
NFGS_EPOLICY = 5
NFGS_ETIMEDOUT = 6
NFGS_EUNSUPPORTED = 7

NFGS_F32, NFGS_F64 = 0, 1
NFGS_NDIAG = 40
NFGS_NSRCDIAG = 12
NFGS_HIST_COLS = 8
NFGS_NSTEPDIAG = 15
NFGS_MET_COUNT = 13

STOP_REASONS = {
    0: "running",
    1: "max_iter",
    2: "tol",
    3: "sigma_improvement_tol",
    4: "sigma_stall",
    5: "max_rollbacks",
    6: "source_zero_mode_error",
    7: "fixed_point",
}


class NfgsGeom(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("input_nx", C.c_int32), ("input_ny", C.c_int32), ("input_nz", C.c_int32),
                ("pad_x", C.c_int32), ("pad_y", C.c_int32), ("dtype", C.c_int32), ("device", C.c_int32)]


class NfgsParams(C.Structure):
    _fields_ = [("robin_weight", C.c_double), ("projection_weight", C.c_double),
                ("alpha_max", C.c_double), ("weak_field_floor_b2", C.c_double),
                ("mean_mode_tolerance", C.c_double), ("source_zero_mode_tolerance", C.c_double),
                ("user_open_bz", C.c_double),
                ("horizontal_zero_mode", C.c_int32), ("mean_bz_policy", C.c_int32),
                ("d0_policy", C.c_int32), ("source_policy", C.c_int32), ("harmonic_policy", C.c_int32),
                ("gaussian_spectral", C.c_int32), ("face_parallel_exact_jz", C.c_int32),
                ("buffer_thickness", C.c_int32), ("buffer_xy_only", C.c_int32),
                ("k0_smoothness", C.c_double), ("k0_update_mu", C.c_double),
                ("k0_spline_basis", C.c_int32), ("k0_legacy", C.c_int32),
                ("k0_face_target", C.c_int32), ("k0_reserved", C.c_int32)]


class NfgsBoundaryOpts(C.Structure):
    _fields_ = [("ny_obs", C.c_int32), ("nx_obs", C.c_int32), ("zero_net_current", C.c_int32),
                ("smooth_passes", C.c_int32), ("ijzbcor", C.c_int32), ("jz_mode", C.c_int32),
                ("nzo", C.c_int32), ("fov_y0", C.c_int32), ("fov_x0", C.c_int32),
                ("src_y0", C.c_int32), ("src_x0", C.c_int32), ("copy_ny", C.c_int32), ("copy_nx", C.c_int32)]


class NfgsStop(C.Structure):
    _fields_ = [("max_iter", C.c_int32), ("patience", C.c_int32), ("tol", C.c_double), ("mu", C.c_double),
                ("sigma_improvement_tol", C.c_double), ("polarity_mask", C.c_int32), ("adaptive_mu", C.c_int32),
                ("mu_min", C.c_double), ("mu_max", C.c_double), ("mu_backoff", C.c_double),
                ("mu_growth", C.c_double), ("growth_streak", C.c_int32), ("max_rollbacks", C.c_int32),
                ("divergence_factor", C.c_double), ("check_every", C.c_int32), ("use_graph", C.c_int32)]


class NfgsIterResult(C.Structure):
    _fields_ = [("n_hist", C.c_int32), ("best_iter", C.c_int32), ("final_iter", C.c_int32),
                ("stop_reason", C.c_int32), ("rollbacks", C.c_int32), ("kernel_launches", C.c_int32),
                ("best_sigma", C.c_double), ("final_sigma", C.c_double), ("final_vs_best_B_relative", C.c_double),
                ("sigma0", C.c_double), ("divB0", C.c_double), ("energy0", C.c_double),
                ("last_sigma_improvement", C.c_double), ("init_source_zero_mode_ratio", C.c_double),
                ("device_ms", C.c_double)]


_P = C.c_void_p
_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int32)

# name -> (restype, argtypes); every symbol declared in include/nfgs_b200.h
SIGNATURES = {
    "nfgs_create": (C.c_int, [C.POINTER(NfgsGeom), C.POINTER(NfgsParams), C.POINTER(C.c_void_p)]),
    "nfgs_set_boundary": (C.c_int, [_P, _DP, _DP, _DP, _DP, C.POINTER(NfgsBoundaryOpts), _DP]),
    "nfgs_iterate_begin": (C.c_int, [_P, C.POINTER(NfgsStop)]),
    "nfgs_iterate_initial": (C.c_int, [_P, _DP]),
    "nfgs_iterate_advance": (C.c_int, [_P, C.c_int32, _IP, _IP]),
    "nfgs_iterate_end": (C.c_int, [_P, C.POINTER(NfgsIterResult), _DP, C.c_int32]),
    "nfgs_get_history": (C.c_int, [_P, C.c_int32, C.c_int32, _DP, _IP]),
    "nfgs_iterate": (C.c_int, [_P, C.POINTER(NfgsStop), C.POINTER(NfgsIterResult), _DP, C.c_int32]),
    "nfgs_fields": (C.c_int, [_P, C.c_int32, C.c_int32, _DP, _IP]),
    "nfgs_fields_into": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_void_p, C.c_int32, _IP]),
    "nfgs_fields_device": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_void_p, C.c_int32, _IP]),
    "nfgs_field_metrics": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                     _DP, _IP, _DP, C.c_void_p]),
    "nfgs_get_scalars_state": (C.c_int, [_P, C.c_int32, _DP, _DP, _DP]),
    "nfgs_step": (C.c_int, [_P, C.c_double, C.c_int32]),
    "nfgs_gaussian_above": (C.c_int, [_P, _DP]),
    "nfgs_gaussian_above_noalloc": (C.c_int, [_P, C.c_void_p, C.c_void_p]),
    "nfgs_get_plane": (C.c_int, [_P, C.c_int32, _DP]),
    "nfgs_get_background": (C.c_int, [_P, _DP]),
    "nfgs_source_diagnostics": (C.c_int, [_P, _DP]),
    "nfgs_time_phases": (C.c_int, [_P, C.c_int32, _DP]),
    "nfgs_apply_transform": (C.c_int, [_P, C.c_int32, C.c_int32, _DP, _DP]),
    "nfgs_destroy": (C.c_int, [_P]),
    "nfgs_last_error": (C.c_char_p, []),
    "nfgs_version": (C.c_char_p, []),
    "nfgs_release_cached_memory": (C.c_int, [C.c_int32]),
    "nfgs_scan_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    "nfgs_scan_launch": (C.c_int, [_P, _IP]),
    "nfgs_scan_add": (C.c_int, [_P, C.POINTER(C.c_void_p), C.c_int32]),
    "nfgs_scan_destroy": (C.c_int, [_P]),
    "nfgs_iterate_start_state": (C.c_int, [_P, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "nfgs_iterate_restart_from": (C.c_int, [_P, _P, _P, C.c_int32, _DP]),
    "nfgs_iterate_soft_cfcf_start": (C.c_int, [_P, C.c_double, C.c_double, _DP]),
    "nfgs_iterate_cfcf_start": (C.c_int, [_P, C.c_int32, _DP, _DP]),
    "nfgs_step_diagnostics": (C.c_int, [_P, _DP]),
    "nfgs_iterate_fixed_point": (C.c_int, [_P, C.c_int32]),
    "nfgs_k0_state": (C.c_int, [_P, _DP, C.c_int32]),
    "nfgs_k0_operator": (C.c_int, [C.c_int32, C.c_double, C.c_int32, C.c_int32, C.c_int32, C.c_double, _DP, _DP,
                                   _DP]),
    "nfgs_trace_field_lines": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P, C.c_int64, _DP,
                                         C.c_double, C.c_int32, _P, _P, _P, _P, _P, _P]),
    "nfgs_qmap_plane": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, _P, _P, _P, _P, _P]),
    "nfgs_trace_fastqsl": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, _P, C.c_int64, _DP, C.c_double, C.c_double,
                                     C.c_int32, _P, _P, _P, _P, _P, _P, _P]),
    "nfgs_qcalc_plane": (C.c_int, [C.c_int32, C.c_int32, _P, _P, _P, _DP, C.c_double, _P, _P]),
    "nfgs_trace_qperp": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P, C.c_int64, C.c_double,
                                   C.c_double, C.c_int32, _P, _P, _P, _P, _P, _P, _P]),
    # learned warm start operator kernels (device pointers)
    "nfgs_nn_last_error": (C.c_char_p, []),
    "nfgs_nn_pointwise": (C.c_int, [_P, _P, _P, _P, C.c_int32, C.c_int32, C.c_int64, C.c_int32, _P]),
    "nfgs_nn_pointwise_bwd": (C.c_int, [_P, _P, _P, _P, _P, _P, C.c_int32, C.c_int32, C.c_int64, C.c_int32, _P,
                                        C.c_int64, _P]),
    "nfgs_nn_gelu": (C.c_int, [_P, _P, C.c_int64, _P]),
    "nfgs_nn_gelu_bwd": (C.c_int, [_P, _P, _P, C.c_int64, C.c_int32, _P]),
    "nfgs_nn_reduce3": (C.c_int, [_P, _P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P, _P, _P, C.c_int32,
                                  C.c_int32, C.c_int32, _P, _P, _P]),
    "nfgs_nn_expand3": (C.c_int, [_P, _P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P, _P, _P, C.c_int32,
                                  C.c_int32, C.c_int32, C.c_int32, _P, _P, _P]),
    "nfgs_nn_resample_linear": (C.c_int, [_P, _P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                          C.c_int32, _P]),
    "nfgs_nn_modemix": (C.c_int, [_P, _P, _P, C.c_int32, C.c_int32, C.c_int32, _P]),
    "nfgs_nn_modemix_bwd": (C.c_int, [_P, _P, _P, _P, _P, C.c_int32, C.c_int32, C.c_int32, _P]),
    "nfgs_nn_mse": (C.c_int, [_P, _P, _P, _P, C.c_int64, C.c_double, _P, _P, _P]),
    "nfgs_nn_adam": (C.c_int, [_P, _P, _P, _P, C.c_int64, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                               C.c_int32, _P]),
}


def load(path: Path | str = LIB_PATH) -> C.CDLL:
    path = Path(path)
    if not path.exists():
        raise ImportError(
            f"{path} is missing: build it with `python nfgs_b200/build.py` (nvcc, sm_100a). "
            "The NFGS B200 solver has no CPU path."
        )
    lib = C.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_LIB: C.CDLL | None = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = load()
    return _LIB


class NfgsError(RuntimeError):
    pass


def check(code: int) -> None:
    """Map an NFGS status to the reference's exception types."""
    if code == NFGS_OK:
        return
    msg = lib().nfgs_last_error().decode(errors="replace")
    if code in (NFGS_EINVAL, NFGS_EPOLICY):
        raise ValueError(msg)
    if code == NFGS_ESTATE:
        raise RuntimeError(msg)
    if code == NFGS_EUNSUPPORTED:
        raise NotImplementedError(msg)
    if code == NFGS_ENOMEM:
        raise MemoryError(msg)
    raise NfgsError(f"NFGS status {code}: {msg}")


def dptr(a):
    """Pointer to the data of a C-contiguous float64 numpy array."""
    return a.ctypes.data_as(_DP)
