"""Thin calls into the engine library: each builds nothing, converts nothing, and raises EngineError on failure.

These are the only functions that reach the device; the drop-in Engine module (optlab_b200) and the products layer
(optlab_b200.products) are written on top of them.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import EngineError, ObDevice, ObMcResult, check, load

PRECISION = {"fp32": _abi.OB_FP32, "fp64": _abi.OB_FP64, "float": _abi.OB_FP32, "double": _abi.OB_FP64}


def precision_code(precision) -> int:
    if isinstance(precision, int) and precision in (_abi.OB_FP32, _abi.OB_FP64):
        return precision
    try:
        return PRECISION[str(precision).lower()]
    except KeyError:
        raise ValueError(f"precision must be fp32 or fp64, not {precision!r}") from None


def gpu_count() -> int:
    return int(load().ob_gpu_count())


def device_info(device: int = 0) -> dict | None:
    d = ObDevice()
    if load().ob_device_info(int(device), C.byref(d)) != _abi.OB_OK:
        return None
    return {f: (getattr(d, f).decode() if f == "name" else getattr(d, f)) for f, _ in ObDevice._fields_}


def philox_normals(seed: int, first_pair: int, n_pairs: int, tag: int, first_block: int, n_blocks: int):
    """(u32, z64, z32) arrays of shape (n_pairs, n_blocks, 4): the engine's Philox outputs and normals."""
    u = np.empty((n_pairs, n_blocks, 4), np.uint32)
    z = np.empty((n_pairs, n_blocks, 4))
    f = np.empty((n_pairs, n_blocks, 4), np.float32)
    check(
        load().ob_philox_normals(
            int(seed) & (2**64 - 1),
            int(first_pair),
            int(n_pairs),
            int(tag),
            int(first_block),
            int(n_blocks),
            u.ctypes.data_as(C.POINTER(C.c_uint)),
            z.ctypes.data_as(C.POINTER(C.c_double)),
            f.ctypes.data_as(C.POINTER(C.c_float)),
        )
    )
    return u, z, f


def paths(held, precision="fp32") -> tuple[float, float]:
    """Fill the request's output columns on the device: (kernel_ms, total_ms)."""
    check(load().ob_paths(held.ref(), precision_code(precision)))
    return held.struct.kernel_ms, held.struct.total_ms


def leverage(held, precision="fp32") -> float:
    check(load().ob_leverage(held.ref(), precision_code(precision)))
    return held.struct.total_ms


def price_fixed(rq: _abi.ObRequest, precision="fp32") -> _abi.ObResult:
    res = _abi.ObResult()
    check(load().ob_price(C.byref(rq), C.byref(res), precision_code(precision)))
    return res


def mc_price(held, precision="fp32") -> ObMcResult:
    """Fused path + payoff + sums, end to end from host arrays."""
    res = ObMcResult()
    check(load().ob_mc_price(held.ref(), precision_code(precision), C.byref(res)))
    return res


class McPlan:
    """A fused request uploaded once and launched many times (inputs stay resident on the device)."""

    def __init__(self, held, precision="fp32"):
        self._held = held
        self._p = C.c_void_p()
        check(load().ob_mc_plan_create(held.ref(), precision_code(precision), C.byref(self._p)))

    def run(self, n_pairs: int, first_pair: int = 0, seed: int | None = None, stream: int = 0) -> None:
        s = self._held.struct.seed if seed is None else int(seed) & (2**64 - 1)
        check(load().ob_mc_run(self._p, int(n_pairs), int(first_pair), s, C.c_void_p(int(stream) or None)))

    def result(self) -> ObMcResult:
        res = ObMcResult()
        check(load().ob_mc_result_get(self._p, C.byref(res)))
        return res

    def close(self) -> None:
        if self._p:
            load().ob_mc_plan_destroy(self._p)
            self._p = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 (interpreter shutdown)
            pass


__all__ = [
    "EngineError",
    "McPlan",
    "device_info",
    "gpu_count",
    "leverage",
    "mc_price",
    "paths",
    "philox_normals",
    "precision_code",
    "price_fixed",
]
