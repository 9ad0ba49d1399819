"""Implied-variance surfaces and the local-variance tables the kernels read.

`SSVI` is the extended SSVI surface the reference calibrates (packages/core/src/optlab/core/ssvi.py:1-17, Gatheral and
Jacquier 2014; Hendriks and Martini 2019), written here from its equations. A slice at expiry T has ATM total variance
theta and wing slopes a = psi (1 + rho), b = psi (1 - rho); with chi = (a - b) / 2 and u = theta + chi k, its total
implied variance at log-moneyness k is

    w(k) = (u + R) / 2,   R = sqrt(u^2 + a b k^2)

(the same as (theta + chi k + sqrt(psi^2 k^2 + 2 chi theta k + theta^2)) / 2, since psi^2 - chi^2 = a b). Between the
calibrated pillars theta is a monotone cubic in T, and a and b are monotone cubics in theta (`MonotoneCubic`); past
the last pillar theta continues along the last segment's slope and the wings stay at their last values. Dupire's local
variance in total variance is w_T / g with g = (1 - k w_k / 2w)^2 - (w_k^2 / 4)(1 / w + 1 / 4) + w_kk / 2 (Gatheral's
density factor), g floored at 1e-6 and the result clipped to [1e-4, 4]; expiries under a day are read at one day.
Everything is evaluated in FP64, vectorised over (k, T).

`local_var_rows` is the per-step tabulation of a surface that the reference's engine builds for its kernels
(packages/native/src/optlab/native/__init__.py:129-144): at each step start t, n_x uniform log-moneyness points over
[-8, 6] ATM standard deviations sqrt(w(0, max(t, 1/365))), all steps in one vectorised evaluation. A surface object
with its own `local_var_rows` (the reference's bumped surfaces) tabulates itself.

`LocalVarGrid` is the tabulated local variance of the benchmarks: one uniform log-moneyness row per expiry (the
40 expiries x 200 strikes of the local-vol configuration), each time step reading the row of the first expiry after
its start. Its rows are what the fused kernel stages into shared memory.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

MIN_EXPIRY = 1.0 / 365  # local variance is read at no earlier expiry than one day
G_FLOOR, LV_FLOOR, LV_CAP = 1e-6, 1e-4, 4.0


class MonotoneCubic:
    """The piecewise cubic Hermite interpolant of (x_i, y_i) whose knot slopes keep monotone data monotone: PCHIP
    (Fritsch and Carlson 1980) with interior slopes the weighted harmonic mean of the neighbouring secants where
    they agree in sign, zero otherwise (Fritsch and Butland 1984), and one-sided three-point end slopes limited to
    keep the shape (Moler, Numerical Computing with MATLAB, 2004, section 3.4), which is the rule of scipy's
    PchipInterpolator that the reference fits with. `at(t)` gives the value and the slope, for t inside
    [x_0, x_n] (callers clip)."""

    def __init__(self, x, y):
        self.x, self.y = np.asarray(x, dtype=float), np.asarray(y, dtype=float)
        h = np.diff(self.x)
        sec = np.diff(self.y) / h
        d = np.empty_like(self.y)
        if len(h) == 1:
            d[:] = sec[0]
        else:
            hl, hr, sl, sr = h[:-1], h[1:], sec[:-1], sec[1:]
            agree = (np.sign(sl) == np.sign(sr)) & (sl != 0) & (sr != 0)
            wl, wr = 2 * hr + hl, hr + 2 * hl
            with np.errstate(divide="ignore", invalid="ignore"):
                d[1:-1] = np.where(agree, (wl + wr) / (wl / sl + wr / sr), 0.0)
            d[0] = self._end_slope(h[0], h[1], sec[0], sec[1])
            d[-1] = self._end_slope(h[-1], h[-2], sec[-1], sec[-2])
        self.d, self.h = d, h

    @staticmethod
    def _end_slope(h0, h1, s0, s1):
        e = ((2 * h0 + h1) * s0 - h0 * s1) / (h0 + h1)
        if np.sign(e) != np.sign(s0):
            return 0.0
        if np.sign(s0) != np.sign(s1) and abs(e) > 3 * abs(s0):
            return 3 * s0
        return e

    def at(self, t):
        t = np.asarray(t, dtype=float)
        i = np.clip(np.searchsorted(self.x, t, side="right") - 1, 0, len(self.h) - 1)
        h = self.h[i]
        s = (t - self.x[i]) / h
        y0, y1, d0, d1 = self.y[i], self.y[i + 1], self.d[i], self.d[i + 1]
        sec = (y1 - y0) / h
        # the cubic's coefficients in powers of (t - x_i): y0 + d0 dx + c2 dx^2 + c3 dx^3
        c2 = (3 * sec - 2 * d0 - d1) / h
        c3 = (d0 + d1 - 2 * sec) / (h * h)
        dx = s * h
        value = y0 + dx * (d0 + dx * (c2 + dx * c3))
        slope = d0 + dx * (2 * c2 + 3 * dx * c3)
        return value, slope


class SSVI:
    """The eSSVI surface of pillars (maturities, thetas, psis, rhos) (see the module docstring). The hooks the
    engine and the reference's callers read are `w(k, T)`, `local_var(k, T)` and `theta(T)`."""

    def __init__(self, maturities, thetas, psis, rhos):
        self.maturities = np.asarray(maturities, dtype=float)
        self.thetas = np.asarray(thetas, dtype=float)
        self.psis = np.asarray(psis, dtype=float)
        self.rhos = np.asarray(rhos, dtype=float)
        theta_knots = np.append(0.0, self.thetas)
        self._term = MonotoneCubic(np.append(0.0, self.maturities), theta_knots)
        self._wing_a = MonotoneCubic(theta_knots, np.append(0.0, self.psis * (1 + self.rhos)))
        self._wing_b = MonotoneCubic(theta_knots, np.append(0.0, self.psis * (1 - self.rhos)))
        T_prev = self.maturities[-2] if len(self.maturities) > 1 else 0.0
        th_prev = self.thetas[-2] if len(self.thetas) > 1 else 0.0
        self._tail = (self.thetas[-1] - th_prev) / (self.maturities[-1] - T_prev)

    @classmethod
    def power_law(cls, rho, eta, gamma, maturities, thetas) -> SSVI:
        """Plain SSVI on the pillars: psi = theta phi(theta) with phi = eta / (theta^gamma (1 + theta)^(1 - gamma))
        (ssvi.py:43-48), the same rho on every slice."""
        th = np.asarray(thetas, dtype=float)
        return cls(maturities, th, eta * th / (th**gamma * (1 + th) ** (1 - gamma)), np.full_like(th, rho))

    @classmethod
    def from_dict(cls, d: dict) -> SSVI:
        return cls(d["maturities"], d["thetas"], d["psis"], d["rhos"])

    def _term_structure(self, T):
        """theta(T) and theta'(T)."""
        T = np.asarray(T, dtype=float)
        T_last = self.maturities[-1]
        val, slope = self._term.at(np.clip(T, 0.0, T_last))
        past = T > T_last
        return np.where(past, self.thetas[-1] + self._tail * (T - T_last), val), np.where(past, self._tail, slope)

    def _slice(self, T):
        """theta, theta'(T), the wings a and b and their slopes in theta, of the slices at T."""
        th, dth = self._term_structure(T)
        inside = np.clip(th, 0.0, self.thetas[-1])
        a, da = self._wing_a.at(inside)
        b, db = self._wing_b.at(inside)
        flat = th > self.thetas[-1]
        return th, dth, a, b, np.where(flat, 0.0, da), np.where(flat, 0.0, db)

    def theta(self, T):
        return self._term_structure(T)[0]

    def dtheta(self, T):
        return self._term_structure(T)[1]

    def w(self, k, T):
        k, T = np.broadcast_arrays(np.asarray(k, dtype=float), np.asarray(T, dtype=float))
        th, _, a, b, _, _ = self._slice(T)
        u = th + 0.5 * (a - b) * k
        return 0.5 * (u + np.sqrt(u * u + a * b * k * k))

    def iv(self, k, T):
        return np.sqrt(self.w(k, T) / np.asarray(T, dtype=float))

    def derivatives(self, k, T):
        """w, dw/dk, d2w/dk2 and dw/dT, analytic: the k-derivatives of the slice, and dw/dT through theta(T) and the
        wings' dependence on theta."""
        k, T = np.broadcast_arrays(np.asarray(k, dtype=float), np.asarray(T, dtype=float))
        th, dth, a, b, da, db = self._slice(T)
        chi, ab = 0.5 * (a - b), a * b
        u = th + chi * k
        R = np.sqrt(u * u + ab * k * k)
        w = 0.5 * (u + R)
        wk = 0.5 * (chi + (u * chi + ab * k) / R)
        wkk = 0.5 * th * th * ab / R**3
        # partial derivatives of w in theta, a and b at fixed k
        w_th = 0.5 * (1.0 + u / R)
        w_a = 0.25 * k * (1.0 + (u + b * k) / R)
        w_b = 0.25 * k * (-1.0 + (a * k - u) / R)
        return w, wk, wkk, (w_th + w_a * da + w_b * db) * dth

    def local_var(self, k, T, floor=LV_FLOOR, cap=LV_CAP):
        """Dupire local variance sigma_loc^2(T, k) from the total implied variance (ssvi.py:110-115), FP64."""
        w, wk, wkk, wT = self.derivatives(k, np.maximum(np.asarray(T, dtype=float), MIN_EXPIRY))
        g = (1.0 - k * wk / (2.0 * w)) ** 2 - 0.25 * wk * wk * (1.0 / w + 0.25) + 0.5 * wkk
        return np.clip(wT / np.maximum(g, G_FLOOR), floor, cap)


def local_var_rows(surface, t0, n_x: int, sd_range=(-8.0, 6.0)):
    """(lo, inv_dx, rows): the local variance at each step start on n_x uniform points over sd_range ATM standard
    deviations (see the module docstring), all steps at once."""
    if hasattr(surface, "local_var_rows"):
        return surface.local_var_rows(np.asarray(t0, dtype=float), n_x, sd_range)
    T = np.maximum(np.asarray(t0, dtype=float), MIN_EXPIRY)
    sd = np.sqrt(np.asarray(surface.w(np.zeros_like(T), T), dtype=float))
    lo, hi = sd_range[0] * sd, sd_range[1] * sd
    step = (hi - lo) / (n_x - 1)
    k = lo[:, None] + np.arange(n_x)[None, :] * step[:, None]
    k[:, -1] = hi
    rows = np.asarray(surface.local_var(k, np.broadcast_to(T[:, None], k.shape)), dtype=float)
    return lo, (n_x - 1) / (hi - lo), rows.reshape(len(T), n_x)


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
