"""The SLV leverage request (the reference's optlab_leverage_request, packages/native/cuda/include/optlab_cuda/
requests.hpp:76-93) built from NumPy arrays, with its two output tables attached."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from ._abi import ObLeverageRequest, ptr
from .requests import Held, f64


@dataclass
class LeverageHeld(Held):
    x_grids: np.ndarray = None
    values: np.ndarray = None


def leverage_request(
    *,
    dt,
    t0,
    n_pairs: int,
    seed: int,
    heston,
    n_x: int,
    lv_lo,
    lv_inv_dx,
    lv_rows,
    atm_vol: float,
    n_bins: int = 400,
    n_fine: int = 8192,
    bandwidth_scale: float = 1.0,
    l_bounds=(0.05, 8.0),
    quantiles=(0.0005, 0.9995),
    local_linear: int = 0,
    positive_part: int = 0,
) -> LeverageHeld:
    """heston = (v0, kappa, theta, xi, rho) with xi already scaled by the mixing fraction."""
    a = [f64(dt), f64(t0), f64(lv_lo), f64(lv_inv_dx), f64(lv_rows)]
    n_steps = len(a[0])
    rows = a[4].reshape(n_steps, -1)
    xg, vals = np.empty((n_steps, n_x)), np.empty((n_steps, n_x))
    s = ObLeverageRequest()
    s.n_steps, s.dt, s.t0 = n_steps, ptr(a[0]), ptr(a[1])
    s.n_pairs, s.seed = int(n_pairs), int(seed) & (2**64 - 1)
    s.v0, s.kappa, s.theta, s.xi, s.rho = (float(x) for x in heston)
    s.n_x, s.n_bins, s.n_fine = int(n_x), int(n_bins), int(n_fine)
    s.atm_vol, s.bandwidth_scale = float(atm_vol), float(bandwidth_scale)
    s.l_min, s.l_max = float(l_bounds[0]), float(l_bounds[1])
    s.q_lo, s.q_hi = float(quantiles[0]), float(quantiles[1])
    s.local_linear, s.positive_part = int(local_linear), int(positive_part)
    s.n_lv, s.lv_lo, s.lv_inv_dx, s.lv_rows = rows.shape[1], ptr(a[2]), ptr(a[3]), ptr(a[4])
    s.x_grids, s.values = ptr(xg), ptr(vals)
    return LeverageHeld(s, [*a, xg, vals], xg, vals)
