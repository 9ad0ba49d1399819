"""ctypes mirror of the C ABI in include/optlab_b200.h, and the loader of liboptlab_b200.so.

The request structs keep the reference's field order (packages/native/cuda/include/optlab_cuda/requests.hpp:12-93),
so these definitions also bind the reference's own structs. The library is loaded from this directory only: there is
no fallback, and a missing library raises EngineError naming the build command.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

OB_OK, OB_EINVAL, OB_ENODEV, OB_ECUDA, OB_ETIMEOUT, OB_ENOMEM, OB_ESINGULAR = 0, 1, 2, 3, 4, 5, 6
OB_FP32, OB_FP64 = 0, 1
OB_MAX_NAMES, OB_MAX_WINDOWS, OB_MAX_OUT = 8, 2, 32
OB_BATCH_MAX_CARRY = 4
OB_MODEL_PATHS, OB_MODEL_HESTON_QE = 0, 1
OB_PRODUCT_LADDER, OB_PRODUCT_AUTOCALL = 0, 1
BARRIER = {"none": 0, "up-out": 1, "down-out": 2, "up-in": 3, "down-in": 4}
AUX_STREAM = 0x80000000

LIB_NAME = "liboptlab_b200.so"
LIB_PATH = Path(__file__).with_name(LIB_NAME)

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


try:  # where the reference's registry is importable, its callers catch its EngineError: be that class
    from optlab.core.engines import EngineError as _RegistryError
except ImportError:  # standalone
    _RegistryError = RuntimeError


class EngineError(_RegistryError):
    """The engine failed, or cannot run what was asked of it (optlab.core.engines.EngineError's role)."""


class ObRequest(C.Structure):
    _fields_ = [
        ("model", C.c_int),
        ("product", C.c_int),
        ("legs", C.c_int * 3),
        ("strikes", C.c_double * 3),
        ("H", C.c_double),
        ("n_steps", C.c_int),
        ("S0", C.c_double),
        ("r", C.c_double),
        ("q", C.c_double),
        ("T", C.c_double),
        ("sigma", C.c_double),
        ("v0", C.c_double),
        ("kappa", C.c_double),
        ("theta", C.c_double),
        ("xi", C.c_double),
        ("rho", C.c_double),
        ("n_paths", C.c_longlong),
        ("seed", C.c_ulonglong),
    ]


class ObResult(C.Structure):
    _fields_ = [
        ("price", C.c_double * 4),
        ("se", C.c_double * 4),
        ("n_paths", C.c_longlong),
        ("kernel_ms", C.c_double),
        ("total_ms", C.c_double),
    ]


class ObPathsRequest(C.Structure):
    _fields_ = [
        ("n_names", C.c_int),
        ("n_steps", C.c_int),
        ("n_obs", C.c_int),
        ("n_x", C.c_int),
        ("n_rows", C.c_int),
        ("n_pairs", C.c_longlong),
        ("first_pair", C.c_longlong),
        ("seed", C.c_ulonglong),
        ("dt", _dp),
        ("t0", _dp),
        ("obs_step", _ip),
        ("root", _dp),
        ("kind", _ip),
        ("cvar", _dp),
        ("heston", _dp),
        ("same", C.c_int),
        ("step_row", _ip),
        ("row_lo", _dp),
        ("row_inv_dx", _dp),
        ("table", _dp),
        ("fwd", _dp),
        ("mixer", C.c_int),
        ("mix", C.c_double * 8),
        ("low_root", _dp),
        ("n_cols", C.c_int),
        ("n_keep", C.c_int),
        ("col_of", _ip),
        ("n_windows", C.c_int),
        ("win_lo", _ip),
        ("win_hi", _ip),
        ("out", _dp),
        ("kernel_ms", C.c_double),
        ("total_ms", C.c_double),
    ]


class ObDevice(C.Structure):
    _fields_ = [
        ("name", C.c_char * 256),
        ("major", C.c_int),
        ("minor", C.c_int),
        ("sm_count", C.c_int),
        ("clock_mhz", C.c_int),
        ("total_mem", C.c_longlong),
        ("free_mem", C.c_longlong),
        ("integrated", C.c_int),
        ("kernel_timeout", C.c_int),
    ]


class ObLeverageRequest(C.Structure):
    _fields_ = [
        ("n_steps", C.c_int),
        ("dt", _dp),
        ("t0", _dp),
        ("n_pairs", C.c_longlong),
        ("seed", C.c_ulonglong),
        ("v0", C.c_double),
        ("kappa", C.c_double),
        ("theta", C.c_double),
        ("xi", C.c_double),
        ("rho", C.c_double),
        ("n_x", C.c_int),
        ("n_bins", C.c_int),
        ("n_fine", C.c_int),
        ("atm_vol", C.c_double),
        ("bandwidth_scale", C.c_double),
        ("l_min", C.c_double),
        ("l_max", C.c_double),
        ("q_lo", C.c_double),
        ("q_hi", C.c_double),
        ("local_linear", C.c_int),
        ("positive_part", C.c_int),
        ("n_lv", C.c_int),
        ("lv_lo", _dp),
        ("lv_inv_dx", _dp),
        ("lv_rows", _dp),
        ("x_grids", _dp),
        ("values", _dp),
        ("total_ms", C.c_double),
    ]


class ObMcRequest(C.Structure):
    _fields_ = [
        ("model", C.c_int),
        ("n_names", C.c_int),
        ("n_steps", C.c_int),
        ("n_pairs", C.c_longlong),
        ("first_pair", C.c_longlong),
        ("seed", C.c_ulonglong),
        ("dt", _dp),
        ("t0", _dp),
        ("root", _dp),
        ("kind", _ip),
        ("cvar", _dp),
        ("heston", _dp),
        ("same", C.c_int),
        ("n_x", C.c_int),
        ("n_rows", C.c_int),
        ("step_row", _ip),
        ("row_lo", _dp),
        ("row_inv_dx", _dp),
        ("table", _dp),
        ("spot", _dp),
        ("log_fwd", _dp),
        ("r", C.c_double),
        ("q", C.c_double),
        ("product", C.c_int),
        ("n_legs", C.c_int),
        ("leg_type", _ip),
        ("leg_strike", _dp),
        ("leg_barrier", _ip),
        ("leg_level", _dp),
        ("discount", C.c_double),
        ("n_obs", C.c_int),
        ("obs_step", _ip),
        ("obs_discount", _dp),
        ("trigger", _dp),
        ("coupon_barrier", C.c_double),
        ("coupon", C.c_double),
        ("ki_barrier", C.c_double),
        ("put_strike", C.c_double),
        ("memory", C.c_int),
        ("ki_daily", C.c_int),
        ("mixer", C.c_int),
        ("mix", C.c_double * 8),
        ("low_root", _dp),
    ]


class ObMcResult(C.Structure):
    _fields_ = [
        ("n_out", C.c_int),
        ("price", C.c_double * OB_MAX_OUT),
        ("se", C.c_double * OB_MAX_OUT),
        ("n_paths", C.c_longlong),
        ("kernel_ms", C.c_double),
        ("total_ms", C.c_double),
        ("sum_y", C.c_double * OB_MAX_OUT),
        ("sum_y2", C.c_double * OB_MAX_OUT),
    ]


OB_ADJ_BATCHES = 32


class ObAdjointRequest(C.Structure):
    _fields_ = [("base", ObMcRequest), ("smoothing", C.c_double), ("checkpoint", C.c_int)]


class ObAdjointResult(C.Structure):
    _fields_ = [
        ("price", C.c_double),
        ("price_se", C.c_double),
        ("delta", C.c_double * OB_MAX_NAMES),
        ("delta_se", C.c_double * OB_MAX_NAMES),
        ("n_paths", C.c_longlong),
        ("n_batches", C.c_int),
        ("forward_ms", C.c_double),
        ("backward_ms", C.c_double),
    ]


class ObBatchTrade(C.Structure):
    _fields_ = [
        ("model", C.c_int),
        ("product", C.c_int),
        ("n_names", C.c_int),
        ("n_steps", C.c_int),
        ("n_pairs", C.c_longlong),
        ("seed", C.c_ulonglong),
        ("table_row0", C.c_int),
        ("root0", C.c_int),
        ("heston", C.c_double * 5),
        ("r", C.c_double),
        ("q", C.c_double),
        ("n_legs", C.c_int),
        ("leg0", C.c_int),
        ("n_obs", C.c_int),
        ("obs0", C.c_int),
        ("coupon_barrier", C.c_double),
        ("coupon", C.c_double),
        ("ki_barrier", C.c_double),
        ("put_strike", C.c_double),
        ("memory", C.c_int),
        ("ki_daily", C.c_int),
        ("discount", C.c_double),
        ("corr_root0", C.c_int),
    ]


class ObBatchRequest(C.Structure):
    _fields_ = [
        ("n_trades", C.c_int),
        ("trades", C.POINTER(ObBatchTrade)),
        ("dt", C.c_double),
        ("horizon", C.c_double),
        ("n_exp", C.c_int),
        ("n_x", C.c_int),
        ("n_rows", C.c_int),
        ("table", _dp),
        ("row_lo", _dp),
        ("row_inv_dx", _dp),
        ("root", _dp),
        ("leg_type", _ip),
        ("leg_strike", _dp),
        ("leg_barrier", _ip),
        ("leg_level", _dp),
        ("obs_step", _ip),
        ("obs_trigger", _dp),
        ("obs_discount", _dp),
        ("n_spot", C.c_int),
        ("spot_shift", _dp),
        ("n_vol", C.c_int),
        ("vol_shift", _dp),
        ("vol_tilt", _dp),
        ("vol_table", _dp),
        ("n_carry", C.c_int),
        ("carry_rate", _dp),
        ("carry_div", _dp),
        ("n_corr", C.c_int),
    ]


class ObScriptRequest(C.Structure):
    _fields_ = [
        ("model", ObMcRequest),
        ("n_code", C.c_int),
        ("code", _ip),
        ("n_const", C.c_int),
        ("consts", _dp),
        ("n_regs", C.c_int),
        ("n_events", C.c_int),
        ("event_step", _ip),
        ("event_code", _ip),
        ("event_discount", _dp),
        ("n_windows", C.c_int),
        ("win_name", _ip),
        ("win_func", _ip),
        ("win_fix0", _ip),
        ("fix_step", _ip),
        ("win_lower", _dp),
        ("win_upper", _dp),
        ("smoothing", C.c_double),
        ("n_calls", C.c_int),
        ("call_state", _ip),
        ("n_state", C.c_int),
        ("call_mode", C.c_int),
        ("rules", _dp),
        ("record", _dp),
        ("branch", C.c_int),
        ("branch_step", C.c_int),
        ("branch_outer", C.c_longlong),
        ("branch_pairs", C.c_longlong),
        ("branch_seed", C.c_ulonglong),
        ("pair_value", _dp),
    ]


OB_RULE_STRIDE = 224


class ObScriptResult(C.Structure):
    _fields_ = [
        ("price", C.c_double),
        ("se", C.c_double),
        ("n_paths", C.c_longlong),
        ("bad_pay", C.c_longlong),
        ("bad_cond", C.c_longlong),
        ("bad_redemption", C.c_longlong),
        ("kernel_ms", C.c_double),
    ]


# Every symbol include/optlab_b200.h declares, with its ctypes signature (restype, argtypes).
SIGNATURES = {
    "ob_last_error": (C.c_char_p, []),
    "ob_version": (C.c_int, []),
    "ob_gpu_count": (C.c_int, []),
    "ob_has_cuda": (C.c_int, []),
    "ob_cpu_threads": (C.c_int, []),
    "ob_release_buffers": (C.c_int, []),
    "ob_set_wait_limit": (C.c_longlong, [C.c_longlong]),
    "ob_device_info": (C.c_int, [C.c_int, C.POINTER(ObDevice)]),
    "ob_philox_normals": (
        C.c_int,
        [
            C.c_ulonglong,
            C.c_longlong,
            C.c_longlong,
            C.c_uint,
            C.c_ulonglong,
            C.c_int,
            C.POINTER(C.c_uint),
            _dp,
            C.POINTER(C.c_float),
        ],
    ),
    "ob_paths": (C.c_int, [C.POINTER(ObPathsRequest), C.c_int]),
    "ob_leverage": (C.c_int, [C.POINTER(ObLeverageRequest), C.c_int]),
    "ob_price": (C.c_int, [C.POINTER(ObRequest), C.POINTER(ObResult), C.c_int]),
    "ob_price_noalloc": (C.c_int, [C.POINTER(ObRequest), C.POINTER(ObResult), C.c_int]),
    "ob_mc_price": (C.c_int, [C.POINTER(ObMcRequest), C.c_int, C.POINTER(ObMcResult)]),
    "ob_mc_plan_create": (C.c_int, [C.POINTER(ObMcRequest), C.c_int, C.POINTER(C.c_void_p)]),
    "ob_mc_run": (C.c_int, [C.c_void_p, C.c_longlong, C.c_longlong, C.c_ulonglong, C.c_void_p]),
    "ob_mc_result_get": (C.c_int, [C.c_void_p, C.POINTER(ObMcResult)]),
    "ob_mc_plan_destroy": (C.c_int, [C.c_void_p]),
    "ob_adjoint_plan_create": (C.c_int, [C.POINTER(ObAdjointRequest), C.c_int, C.POINTER(C.c_void_p)]),
    "ob_adjoint_run": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ob_adjoint_result_get": (C.c_int, [C.c_void_p, C.POINTER(ObAdjointResult), C.POINTER(C.c_longlong)]),
    "ob_adjoint_plan_destroy": (C.c_int, [C.c_void_p]),
    "ob_batch_create": (C.c_int, [C.POINTER(ObBatchRequest), C.c_int, C.POINTER(C.c_void_p)]),
    "ob_batch_tune": (C.c_int, [C.c_void_p, C.c_int]),
    "ob_batch_capture": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ob_batch_launch": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ob_batch_run_per_trade": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ob_batch_result": (C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    "ob_batch_classes": (C.c_int, [C.c_void_p, C.c_int, _ip, _ip]),
    "ob_batch_destroy": (C.c_int, [C.c_void_p]),
    "ob_script_price": (C.c_int, [C.POINTER(ObScriptRequest), C.c_int, C.POINTER(ObScriptResult)]),
    "ob_script_pilot_fit": (C.c_int, [C.POINTER(ObScriptRequest), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                      C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(ObScriptResult)]),
}

_lib: list = []


def load() -> C.CDLL:
    """The engine library, loaded once; EngineError when it is not built (there is no fallback)."""
    if _lib:
        return _lib[0]
    path = Path(os.environ.get("OPTLAB_B200_LIB", str(LIB_PATH)))
    if not path.exists():
        raise EngineError(f"{path.name} is not built: run `make -C option-pricing-lab_b200/csrc` (or build())")
    lib = C.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    _lib.append(lib)
    return lib


def check(status: int) -> None:
    """Raise EngineError with the engine's message for a failed call (ValueError for a bad request)."""
    if status == OB_OK:
        return
    msg = load().ob_last_error().decode(errors="replace")
    if status == OB_EINVAL:
        raise EngineError(f"invalid request: {msg}")
    raise EngineError(msg)


def ptr(a, ctype=C.c_double):
    """A ctypes pointer into a C-contiguous NumPy array (None for None or an empty array)."""
    if a is None or a.size == 0:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))
