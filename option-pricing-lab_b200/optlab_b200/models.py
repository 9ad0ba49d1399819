"""The model objects the engine accepts, restated so that the engine runs without the reference installed.

They carry the reference's class names and attributes (packages/core/src/optlab/core/models.py:46-116,
heston.py:19-27, market.py:37-55, packages/structured/src/optlab/structured/multiasset.py:30-74,
localcorr.py:33-95), and `plan()` reads them by name and attribute, so the reference's own objects are accepted too.
Also here: the time grid of the reference (models.py:117-135), its correlation root (multiasset.py:30-42) and the
local-correlation factors (localcorr.py:40-67, core/correlation.py:9-26).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class HestonParams:
    v0: float
    kappa: float
    theta: float
    xi: float
    rho: float

    def as_array(self) -> np.ndarray:
        return np.array([self.v0, self.kappa, self.theta, self.xi, self.rho])


@dataclass
class BlackScholesModel:
    vol: float
    has_variance = False


@dataclass
class HestonModel:
    params: HestonParams
    has_variance = True

    @property
    def heston(self) -> HestonParams:
        return self.params


@dataclass
class LocalVolModel:
    surface: object
    has_variance = False


class Leverage:
    """L(t, x) on a time grid: piecewise constant in t, linear in x, flat outside (models.py:74-97)."""

    def __init__(self, times, x_grids, values):
        self.times = np.asarray(times, dtype=float)
        self.x_grids = np.asarray(x_grids, dtype=float)
        self.values = np.asarray(values, dtype=float)

    def __call__(self, t, x):
        i = int(np.clip(np.searchsorted(self.times, t + 1e-12, side="right") - 1, 0, len(self.times) - 1))
        return np.interp(x, self.x_grids[i], self.values[i])


@dataclass
class SLVModel:
    params: HestonParams
    leverage: object
    mix: float = 1.0
    spot_driven: bool = False
    has_variance = True

    @property
    def heston(self) -> HestonParams:
        p = self.params
        return HestonParams(p.v0, p.kappa, p.theta, self.mix * p.xi, p.rho)


class Market:
    """Spot, discount factors and forwards, log-linear between pillars (market.py:20-55)."""

    def __init__(self, spot: float, t, discount, forward):
        self.spot = float(spot)
        self._t = np.concatenate([[0.0], np.asarray(t, dtype=float)])
        self._log_d = np.concatenate([[0.0], np.log(np.asarray(discount, dtype=float))])
        self._log_f = np.concatenate([[0.0], np.log(np.asarray(forward, dtype=float) / self.spot)])

    @classmethod
    def flat(cls, spot: float, r: float = 0.0, q: float = 0.0) -> Market:
        t = np.array([1.0])
        return cls(spot, t, np.exp(-r * t), spot * np.exp((r - q) * t))

    def _interp(self, values, T):
        T = np.asarray(T, dtype=float)
        slope = (values[-1] - values[-2]) / (self._t[-1] - self._t[-2])
        inside = np.interp(T, self._t, values)
        return np.where(T > self._t[-1], values[-1] + slope * (T - self._t[-1]), inside)

    def D(self, T):
        return np.exp(self._interp(self._log_d, T))

    def F(self, T):
        return self.spot * np.exp(self._interp(self._log_f, T))


def time_grid(times, dt_max, dt_min=None) -> np.ndarray:
    """Fine grid containing every observation time, steps no longer than dt_max; graded with dt_min: the step is
    dt_min + t / 60, capped at dt_max (models.py:117-135)."""
    times = np.asarray(times, dtype=float)
    grid = [0.0]
    for t in times:
        if dt_min is not None:
            while t - grid[-1] > 1e-12:
                h = min(dt_max, dt_min + grid[-1] / 60)
                remaining = t - grid[-1]
                grid.append(t if remaining < 1.5 * h else grid[-1] + h)
            continue
        n = max(1, int(np.ceil((t - grid[-1]) / dt_max - 1e-9)))
        grid.extend(np.linspace(grid[-1], t, n + 1)[1:])
    return np.array(grid)


def correlation_root(corr) -> np.ndarray:
    """L with L L^T = corr, by eigen-decomposition (multiasset.py:30-42)."""
    c = np.atleast_2d(np.asarray(corr, dtype=float))
    if c.shape[0] != c.shape[1] or not np.allclose(c, c.T, atol=1e-12):
        raise ValueError("the correlation matrix must be square and symmetric")
    if not np.allclose(np.diag(c), 1.0, atol=1e-12):
        raise ValueError("the correlation matrix must have ones on its diagonal")
    lam, vec = np.linalg.eigh(c)
    if lam.min() < -1e-10:
        raise ValueError(f"the correlation matrix is not positive semi-definite (eigenvalue {lam.min():.2e})")
    if c.shape[0] == 1:
        return np.ones((1, 1))
    return vec * np.sqrt(np.maximum(lam, 0.0))


def nearest_correlation(c, iterations: int = 50) -> np.ndarray:
    """The closest positive semi-definite matrix with a unit diagonal, by alternating projections (correlation.py)."""
    x = np.array(c, dtype=float)
    x = 0.5 * (x + x.T)
    for _ in range(iterations):
        lam, vec = np.linalg.eigh(x)
        if lam.min() >= -1e-12 and np.allclose(np.diag(x), 1.0, atol=1e-12):
            break
        x = (vec * np.maximum(lam, 0.0)) @ vec.T
        np.fill_diagonal(x, 1.0)
    lam, vec = np.linalg.eigh(x)
    if lam.min() < 0:
        x = (vec * np.maximum(lam, 1e-10)) @ vec.T
        d = np.sqrt(np.diag(x))
        x = x / np.outer(d, d)
    x = 0.5 * (x + x.T)
    np.fill_diagonal(x, 1.0)
    return x


def aligned_factors(corr, root, w0: float) -> tuple:
    """(factors of the low matrix with the signs of `root`, sign of the market factor, angle) of the local
    correlation (localcorr.py:40-67)."""
    c = np.asarray(corr, dtype=float)
    low = (c - w0) / (1.0 - w0)
    np.fill_diagonal(low, 1.0)
    low = correlation_root(nearest_correlation(np.clip(low, -0.999, 0.999))).copy()
    for j in range(low.shape[1] - 1):
        if np.dot(low[:, j], root[:, j]) < 0:
            low[:, j] = -low[:, j]
    if low[:, -1].mean() < 0:
        low[:, -1] = -low[:, -1]
    sign = 1.0 if root[:, -1].mean() >= 0 else -1.0
    return low, sign, float(np.arctan2(np.sqrt(1.0 - w0) * low[:, -1].mean(), np.sqrt(w0)))


@dataclass(frozen=True)
class LocalCorrelation:
    sigma: float
    level: float = 0.0
    down: float = 0.0
    up: float = 0.0
    w0: float = 0.3


@dataclass
class Basket:
    names: tuple
    models: dict
    markets: dict
    corr: np.ndarray
    vol_corr: str = "same"
    mixer: object = None
    root: np.ndarray = field(init=False)

    def __post_init__(self):
        if self.vol_corr not in ("same", "independent"):
            raise ValueError(f"unknown vol_corr {self.vol_corr!r}, expected same or independent")
        self.names = tuple(self.names)
        self.corr = np.atleast_2d(np.asarray(self.corr, dtype=float))
        self.root = correlation_root(self.corr)
