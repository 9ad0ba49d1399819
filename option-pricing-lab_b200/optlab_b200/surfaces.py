"""Implied-variance surfaces and the local-variance tables the kernels read.

`SSVI` restates the extended SSVI surface of the reference (packages/core/src/optlab/core/ssvi.py:26-115): theta(T) a
monotone cubic (scipy's PCHIP, as the reference) through the pillars, the wing slopes a = psi (1 + rho) and
b = psi (1 - rho) monotone cubics in theta, total variance
    w(k) = (theta + chi k + sqrt(psi^2 k^2 + 2 chi theta k + theta^2)) / 2,
analytic derivatives, and Dupire's local variance w_T / g clipped to [1e-4, 4] with g floored at 1e-6. The same
object also answers `local_var_rows`, the hook the reference's engine uses to tabulate a surface per step
(packages/native/src/optlab/native/__init__.py:129-144).

`LocalVarGrid` is the tabulated local variance of the benchmarks: one uniform log-moneyness row per expiry (the
40 expiries x 200 strikes of the local-vol configuration), each time step reading the row of the first expiry after
its start. Its rows are what the fused kernel stages into shared memory.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.interpolate import PchipInterpolator


class SSVI:
    def __init__(self, maturities, thetas, psis, rhos):
        self.maturities = np.asarray(maturities, dtype=float)
        self.thetas = np.asarray(thetas, dtype=float)
        self.psis = np.asarray(psis, dtype=float)
        self.rhos = np.asarray(rhos, dtype=float)
        t = np.concatenate([[0.0], self.maturities])
        th = np.concatenate([[0.0], self.thetas])
        a = np.concatenate([[0.0], self.psis * (1 + self.rhos)])
        b = np.concatenate([[0.0], self.psis * (1 - self.rhos)])
        self._theta_T = PchipInterpolator(t, th, extrapolate=False)
        self._dtheta_T = self._theta_T.derivative()
        self._a = PchipInterpolator(th, a, extrapolate=False)
        self._b = PchipInterpolator(th, b, extrapolate=False)
        self._da, self._db = self._a.derivative(), self._b.derivative()
        self._slope_last = (th[-1] - th[-2]) / (t[-1] - t[-2])

    @classmethod
    def power_law(cls, rho, eta, gamma, maturities, thetas) -> SSVI:
        """Plain SSVI with phi(theta) = eta / (theta^gamma (1 + theta)^(1 - gamma)) at the pillars (ssvi.py:43-48)."""
        th = np.asarray(thetas, dtype=float)
        psi = th * eta / (th**gamma * (1 + th) ** (1 - gamma))
        return cls(maturities, th, psi, np.full_like(th, rho))

    @classmethod
    def from_dict(cls, d: dict) -> SSVI:
        return cls(d["maturities"], d["thetas"], d["psis"], d["rhos"])

    def theta(self, T):
        T = np.asarray(T, dtype=float)
        last = self.maturities[-1]
        inside = self._theta_T(np.clip(T, 0.0, last))
        return np.where(T > last, self.thetas[-1] + self._slope_last * (T - last), inside)

    def dtheta(self, T):
        T = np.asarray(T, dtype=float)
        inside = self._dtheta_T(np.clip(T, 0.0, self.maturities[-1]))
        return np.where(T > self.maturities[-1], self._slope_last, inside)

    def _wings(self, theta):
        th = np.clip(theta, 0.0, self.thetas[-1])
        a, b = self._a(th), self._b(th)
        beyond = theta > self.thetas[-1]
        da = np.where(beyond, 0.0, self._da(th))
        db = np.where(beyond, 0.0, self._db(th))
        return a, b, da, db

    def w(self, k, T):
        k, T = np.broadcast_arrays(np.asarray(k, dtype=float), np.asarray(T, dtype=float))
        th = self.theta(T)
        a, b, _, _ = self._wings(th)
        psi, chi = 0.5 * (a + b), 0.5 * (a - b)
        return 0.5 * (th + chi * k + np.sqrt(psi**2 * k**2 + 2 * chi * th * k + th**2))

    def iv(self, k, T):
        return np.sqrt(self.w(k, T) / np.asarray(T, dtype=float))

    def derivatives(self, k, T):
        """w, dw/dk, d2w/dk2 and dw/dT (ssvi.py:88-103)."""
        k, T = np.broadcast_arrays(np.asarray(k, dtype=float), np.asarray(T, dtype=float))
        th = self.theta(T)
        a, b, da, db = self._wings(th)
        psi, chi = 0.5 * (a + b), 0.5 * (a - b)
        dpsi, dchi = 0.5 * (da + db), 0.5 * (da - db)
        R = np.sqrt(psi**2 * k**2 + 2 * chi * th * k + th**2)
        w = 0.5 * (th + chi * k + R)
        wk = 0.5 * (chi + (psi**2 * k + chi * th) / R)
        wkk = 0.5 * th**2 * (psi**2 - chi**2) / R**3
        dw_dtheta = 0.5 * (1 + (chi * k + th) / R)
        dw_dpsi = 0.5 * psi * k**2 / R
        dw_dchi = 0.5 * k * (1 + th / R)
        wT = (dw_dtheta + dw_dpsi * dpsi + dw_dchi * dchi) * self.dtheta(T)
        return w, wk, wkk, wT

    def local_var(self, k, T, floor=1e-4, cap=4.0):
        """Dupire local variance in total implied variance (ssvi.py:110-115), in FP64."""
        T = np.maximum(np.asarray(T, dtype=float), 1.0 / 365)
        w, wk, wkk, wT = self.derivatives(k, T)
        g = (1 - k * wk / (2 * w)) ** 2 - wk**2 / 4 * (1 / w + 0.25) + wkk / 2
        return np.clip(wT / np.maximum(g, 1e-6), floor, cap)


def local_var_rows(surface, t0, n_x: int, sd_range=(-8.0, 6.0)):
    """(lo, inv_dx, rows): the local variance at each step start on n_x uniform points over sd_range ATM standard
    deviations, the reference's per-step tabulation (packages/native/src/optlab/native/__init__.py:129-142)."""
    if hasattr(surface, "local_var_rows"):
        return surface.local_var_rows(np.asarray(t0, dtype=float), n_x, sd_range)
    t0 = np.asarray(t0, dtype=float)
    lo, inv, rows = np.empty(len(t0)), np.empty(len(t0)), np.empty((len(t0), n_x))
    for i, t in enumerate(t0):
        T = max(float(t), 1.0 / 365)
        sd = float(np.sqrt(surface.w(0.0, T)))
        a, b = sd_range[0] * sd, sd_range[1] * sd
        lo[i], inv[i] = a, (n_x - 1) / (b - a)
        rows[i] = surface.local_var(np.linspace(a, b, n_x), T)
    return lo, inv, rows


@dataclass
class LocalVarGrid:
    """Local variance tabulated per expiry: rows[j] on n_x uniform points from lo[j] with spacing 1 / inv_dx[j], used
    from the start of expiry j's bucket (the previous expiry) up to expiry j."""

    expiries: np.ndarray  # n_exp, increasing
    lo: np.ndarray  # n_exp
    inv_dx: np.ndarray  # n_exp
    rows: np.ndarray  # n_exp x n_x

    @classmethod
    def from_surface(cls, surface, expiries, n_x: int = 200, sd_range=(-8.0, 6.0)) -> LocalVarGrid:
        expiries = np.asarray(expiries, dtype=float)
        lo, inv, rows = local_var_rows(surface, expiries, n_x, sd_range)
        return cls(expiries, lo, inv, rows)

    @property
    def n_x(self) -> int:
        return self.rows.shape[1]

    def row_of(self, t0) -> np.ndarray:
        """Row read by a step starting at t0: the first expiry strictly after t0 (the last one beyond)."""
        j = np.searchsorted(self.expiries, np.asarray(t0, dtype=float) + 1e-12, side="right")
        return np.clip(j, 0, len(self.expiries) - 1).astype(np.int32)

    def local_var_rows(self, t0, n_x, sd_range=(-8.0, 6.0)):
        """The reference's per-step table hook: each step gets a copy of its expiry's row (resampled to n_x points
        when n_x differs from the grid's)."""
        rows_of = self.row_of(t0)
        if n_x == self.n_x:
            return self.lo[rows_of].copy(), self.inv_dx[rows_of].copy(), self.rows[rows_of].copy()
        lo, inv, out = np.empty(len(rows_of)), np.empty(len(rows_of)), np.empty((len(rows_of), n_x))
        for i, j in enumerate(rows_of):
            a = self.lo[j]
            b = a + (self.n_x - 1) / self.inv_dx[j]
            grid = np.linspace(a, b, n_x)
            lo[i], inv[i] = a, (n_x - 1) / (b - a)
            out[i] = np.interp(grid, np.linspace(a, b, self.n_x), self.rows[j])
        return lo, inv, out
