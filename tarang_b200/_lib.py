"""ctypes binding of ``libtarang_b200.so`` (the C ABI in include/tarang_b200.h).

The library is the product: there is no Python or CPU fallback.  Loading
fails loudly when the shared object is missing.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "libtarang_b200.so"

TS_OK, TS_ERR_ARG, TS_ERR_CUDA, TS_ERR_NAN, TS_ERR_TIMEOUT, TS_ERR_UNSUPPORTED, TS_ERR_NOMEM = range(7)
TS_PR_LARGE, TS_PR_SMALL, TS_PR_ZERO, TS_PR_INFTY = range(4)
TS_U_LARGE, TS_U_SMALL = range(2)
STATUS_NAMES = {0: "TS_OK", 1: "TS_ERR_ARG", 2: "TS_ERR_CUDA", 3: "TS_ERR_NAN", 4: "TS_ERR_TIMEOUT",
                5: "TS_ERR_UNSUPPORTED", 6: "TS_ERR_NOMEM"}
TS_BASIS_FFF, TS_BASIS_SFF, TS_BASIS_SSF, TS_BASIS_SSS = 0, 1, 2, 3
TS_F64, TS_F32 = 0, 1
TS_NLIN_CONSERVATIVE, TS_NLIN_ROTATIONAL = 0, 1
TS_DEALIAS_NONE, TS_DEALIAS_REFERENCE_CORNER, TS_DEALIAS_TWO_THIRDS = 0, 1, 2
TS_FORCE_NONE, TS_FORCE_CARATI_ENERGY_SUPPLY, TS_FORCE_RBC = 0, 1, 51
KCLASS_NAMES = ["inv_x", "y_inv", "z_fused", "y_fwd", "fwd_x_update", "other"]


class TsMember(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int * 3), ("Ra", ctypes.c_double), ("Pr", ctypes.c_double)]


TUNE_CLASSES = ["x_inv", "y_inv", "z", "y_fwd", "x_fwd"]


class TsTuning(ctypes.Structure):
    _fields_ = [("variant", ctypes.c_int * 5), ("blocks_per_sm", ctypes.c_int * 5)]


class TsConfig(ctypes.Structure):
    _fields_ = [
        ("basis", ctypes.c_int),
        ("N", ctypes.c_int * 3),
        ("kfactor", ctypes.c_double * 3),
        ("precision", ctypes.c_int),
        ("nlin_form", ctypes.c_int),
        ("dealias_mode", ctypes.c_int),
        ("reality_fix", ctypes.c_int),
        ("nu", ctypes.c_double),
        ("kappa", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("force_type", ctypes.c_int),
        ("force_inner_radius", ctypes.c_double),
        ("force_outer_radius", ctypes.c_double),
        ("energy_supply", ctypes.POINTER(ctypes.c_double)),
        ("helicity_supply", ctypes.POINTER(ctypes.c_double)),
        ("n_supply", ctypes.c_int),
        ("Ra", ctypes.c_double),
        ("Pr", ctypes.c_double),
        ("Pr_option", ctypes.c_int),
        ("Uscaling", ctypes.c_int),
    ]


# exported symbols and their argument types (c_void_p for plan / field pointers)
_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
SIGNATURES = {
    "ts_config_default": (None, [ctypes.POINTER(TsConfig)]),
    "ts_plan_create": (ctypes.c_int, [ctypes.POINTER(TsConfig), ctypes.POINTER(ctypes.c_void_p)]),
    "ts_plan_destroy": (ctypes.c_int, [_P]),
    "ts_plan_set_stream": (ctypes.c_int, [_P, _P]),
    "ts_plan_sizes": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_int)]),
    "ts_plan_num_shells": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int)]),
    "ts_alloc_field": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "ts_free_field": (ctypes.c_int, [ctypes.c_void_p]),
    "ts_plan_set_dt": (ctypes.c_int, [_P, ctypes.c_double]),
    "ts_plan_status": (ctypes.c_int, [_P]),
    "ts_plan_clear_status": (ctypes.c_int, [_P]),
    "ts_plan_expire_wait": (ctypes.c_int, [_P, ctypes.c_int]),
    "ts_fft_forward": (ctypes.c_int, [_P, ctypes.c_char_p, _P, _P, ctypes.c_int]),
    "ts_fft_inverse": (ctypes.c_int, [_P, ctypes.c_char_p, _P, _P, ctypes.c_int]),
    "ts_nlin": (ctypes.c_int, [_P, _P, _P]),
    "ts_rk4_step": (ctypes.c_int, [_P, _P, ctypes.c_int]),
    "ts_rk4_step_rbc": (ctypes.c_int, [_P, _P, _P, ctypes.c_int]),
    "ts_energy": (ctypes.c_int, [_P, _P, ctypes.c_int, _D]),
    "ts_shell_spectrum": (ctypes.c_int, [_P, _P, ctypes.c_int, _D, ctypes.c_int]),
    "ts_flux": (ctypes.c_int, [_P, _P, _D, ctypes.c_int, _D]),
    "ts_dealias_field": (ctypes.c_int, [_P, _P, ctypes.c_int]),
    "ts_max_div": (ctypes.c_int, [_P, _P, _D]),
    "ts_shell_sums": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, _D, _D, ctypes.c_int]),
    "ts_force_field": (ctypes.c_int, [_P, _P, _P]),
    "ts_nusselt": (ctypes.c_int, [_P, _P, _P, _D]),
    "ts_rbc_slave": (ctypes.c_int, [_P, _P, _P]),
    "ts_init_energy_spectrum": (ctypes.c_int, [_P, _D, ctypes.c_int, ctypes.c_uint64, ctypes.c_double, _P]),
    "ts_init_temperature_perturbation": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, ctypes.c_uint64, _P]),
    "ts_ensemble_create": (ctypes.c_int, [ctypes.POINTER(TsConfig), _P, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "ts_ensemble_destroy": (ctypes.c_int, [_P]),
    "ts_ensemble_member": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                          ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p)]),
    "ts_ensemble_init_temperature": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, ctypes.c_uint64]),
    "ts_ensemble_run": (ctypes.c_int, [_P, ctypes.c_int]),
    "ts_ensemble_synchronize": (ctypes.c_int, [_P]),
    "ts_ensemble_nusselt": (ctypes.c_int, [_P, _D]),
    "ts_ensemble_health": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int), ctypes.c_int]),
    "ts_rk4_step_scalar": (ctypes.c_int, [_P, _P, _P, ctypes.c_int]),
    "ts_rk4_step_mhd": (ctypes.c_int, [_P, _P, _P, ctypes.c_int]),
    "ts_rk4_step_keep": (ctypes.c_int, [_P, _P, _P, _P]),
    "ts_adjoint_step": (ctypes.c_int, [_P, _P, _P, _P]),
    "ts_adjoint_work_bytes": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]),
    "ts_adjoint_window": (ctypes.c_int, [_P, _P, ctypes.c_int, _P, _P, ctypes.c_size_t]),
    "ts_tuning_candidates": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int)]),
    "ts_plan_get_tuning": (ctypes.c_int, [_P, ctypes.POINTER(TsTuning)]),
    "ts_plan_set_tuning": (ctypes.c_int, [_P, ctypes.POINTER(TsTuning)]),
    "ts_plan_autotune": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]),
    "ts_ensemble_get_tuning": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(TsTuning)]),
    "ts_ensemble_set_tuning": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(TsTuning)]),
    "ts_ensemble_autotune": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]),
    "ts_profile_enable": (ctypes.c_int, [_P, ctypes.c_int]),
    "ts_profile_reset": (ctypes.c_int, [_P]),
    "ts_profile_read": (ctypes.c_int, [_P, ctypes.c_int, _D, ctypes.POINTER(ctypes.c_longlong), _D]),
    "ts_shell_spectrum_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _D, _P,
                                                  ctypes.c_int, _P, ctypes.c_int, _P]),
    "ts_kernel_launch_count": (ctypes.c_longlong, []),
    "ts_last_error": (ctypes.c_char_p, []),
}

_lib = None


def lib_path() -> Path:
    return _LIB_PATH


def load() -> ctypes.CDLL:
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise RuntimeError(f"{_LIB_PATH} is missing: build it with `python -m tarang_b200.build_ext` "
                           "(the tarang_b200 path has no CPU fallback)")
    lib = ctypes.CDLL(str(_LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class TsError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = ""
        try:
            msg = load().ts_last_error().decode()
        except Exception:
            pass
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)} {msg}")
        self.status = status


def check(status: int, where: str):
    if status != TS_OK:
        raise TsError(status, where)
