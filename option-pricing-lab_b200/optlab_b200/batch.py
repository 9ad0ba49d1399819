"""Batched risk revaluation: a seeded book of uneven trades, each revalued under spot, carry, parallel-vol, skew and
correlation scenarios, in one replay of a CUDA graph of persistent kernels (csrc/batch.cu through ob_batch_*).

The reference revalues a book group by group and scenario by scenario (packages/risk/src/optlab/risk/engine.py:382-425:
every shock that moves the model is its own simulation on the group's seed; :563-644: shocks that move only the spot,
the forwards or the discounting share the base simulation as factors on its paths, :8-11). `Batch` keeps that split:
per trade one base simulation carries the base, every spot move and every carry move (rates or dividends), and each
vol, skew or correlation move is one more simulation on the same random numbers; all of them are work items of the
same launch.

`sample_book` draws the benchmark's book: 512 trades of 1 to 5 names, 1 to 5 years of daily steps, 2^14 to 2^18 paths,
European, barrier or autocall payoffs (worst-of with several names), under Heston QE or local vol of per-name SSVI
surfaces, with 60 scenarios: 20 spot moves of +-1..20 %, 20 parallel moves of the implied vols of +-1..10 points and 20
skew moves of +-1..10 points (the rise of the 90 % vol against the 110 % one at one year). A vol scenario moves each
surface's implied vols as the reference's risk scenarios do (packages/risk/src/optlab/risk/shocks.py:63-108,
VolMove.apply -> bumped_surface, risk/surfaces.py:204) and re-tabulates Dupire's local variance on the base table's
points (optlab_b200.ivnodes.moved_local_var); the device reads those tables. Carry moves (CARRY_MOVES: rates +-1 %,
dividend yield +-1 %) and correlation moves (CORR_MOVES: every pair +-0.10) are added on request.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np
import torch

from ._abi import (
    BARRIER,
    OB_MODEL_HESTON_QE,
    OB_MODEL_PATHS,
    OB_PRODUCT_AUTOCALL,
    OB_PRODUCT_LADDER,
    ObBatchRequest,
    ObBatchTrade,
    check,
    load,
)
from .engine import precision_code
from .models import correlation_root, nearest_correlation
from .ivnodes import grid_points, moved_local_var
from .surfaces import SSVI, LocalVarGrid

_STEPS = np.array([0.01, 0.02, 0.03, 0.04, 0.05, 0.075, 0.10, 0.125, 0.15, 0.20])
SPOT_MOVES = np.concatenate([-_STEPS[::-1], _STEPS])
VOL_SHIFTS = np.concatenate([-np.arange(10, 0, -1), np.arange(1, 11)]) / 100.0  # parallel implied-vol moves
SKEW_TILTS = VOL_SHIFTS.copy()  # skew moves: the 90 % - 110 % implied-vol gap at one year
CARRY_MOVES = ((0.01, 0.0), (-0.01, 0.0), (0.0, 0.01), (0.0, -0.01))  # (rate, dividend yield)
CORR_MOVES = (-0.10, 0.10)
MAX_OBS = 64
MAX_SPOT = 31

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _arr(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


@dataclass
class Book:
    """Trades, their pools and the scenarios, held for the C ABI (the arrays stay alive with the book)."""

    trades: list
    labels: list
    dt: float
    horizon: float
    n_exp: int
    n_x: int
    table: np.ndarray
    row_lo: np.ndarray
    row_inv_dx: np.ndarray
    root: np.ndarray
    leg_type: np.ndarray
    leg_strike: np.ndarray
    leg_barrier: np.ndarray
    leg_level: np.ndarray
    obs_step: np.ndarray
    obs_trigger: np.ndarray
    obs_discount: np.ndarray
    spot_shift: np.ndarray
    vol_shift: np.ndarray
    vol_tilt: np.ndarray
    vol_table: np.ndarray = field(default_factory=lambda: np.zeros(0))  # n_vol x pool rows x n_x
    carry_rate: np.ndarray = field(default_factory=lambda: np.zeros(0))
    carry_div: np.ndarray = field(default_factory=lambda: np.zeros(0))
    corr_move: np.ndarray = field(default_factory=lambda: np.zeros(0))  # each trade's moved roots at corr_root0
    struct: ObBatchRequest = field(init=False)

    _DOUBLES = ("table", "row_lo", "row_inv_dx", "root", "leg_strike", "leg_level", "obs_trigger", "obs_discount",
                "spot_shift", "vol_shift", "vol_tilt", "vol_table", "carry_rate", "carry_div", "corr_move")

    def __post_init__(self):
        for k in self._DOUBLES:
            setattr(self, k, _arr(getattr(self, k), np.float64).ravel())
        for k in ("leg_type", "leg_barrier", "obs_step"):
            setattr(self, k, _arr(getattr(self, k), np.int32).ravel())
        self._trades = (ObBatchTrade * len(self.trades))(*self.trades)
        s = ObBatchRequest()
        s.n_trades = len(self.trades)
        s.trades = self._trades
        s.dt, s.horizon, s.n_exp, s.n_x = self.dt, self.horizon, self.n_exp, self.n_x
        s.n_rows = len(self.row_lo)
        if len(self.vol_shift) and self.vol_table.size != len(self.vol_shift) * len(self.row_lo) * self.n_x:
            raise ValueError("vol_table must hold every pool row under every vol scenario")
        for k in self._DOUBLES[:-1]:
            a = getattr(self, k)
            setattr(s, k, a.ctypes.data_as(_dp) if a.size else None)
        for k in ("leg_type", "leg_barrier", "obs_step"):
            a = getattr(self, k)
            setattr(s, k, a.ctypes.data_as(_ip) if a.size else None)
        s.n_spot, s.n_vol, s.n_carry, s.n_corr = self.n_spot, self.n_vol, self.n_carry, self.n_corr
        self.struct = s

    @property
    def n_trades(self) -> int:
        return len(self.trades)

    @property
    def n_spot(self) -> int:
        return len(self.spot_shift)

    @property
    def n_vol(self) -> int:
        return len(self.vol_shift)

    @property
    def n_carry(self) -> int:
        return len(self.carry_rate)

    @property
    def n_corr(self) -> int:
        return len(self.corr_move)

    @property
    def n_scenarios(self) -> int:
        """Values per trade: base, spot moves, carry moves, vol moves, correlation moves."""
        return 1 + self.n_spot + self.n_carry + self.n_vol + self.n_corr

    def sims_of(self, t) -> int:
        """A trade's simulations: the base, and under local vol one per vol move and (2 names or more) one per
        correlation move."""
        if t.model != OB_MODEL_PATHS:
            return 1
        return 1 + self.n_vol + (self.n_corr if t.n_names > 1 else 0)

    def simulations(self) -> int:
        """Simulations of one revaluation."""
        return sum(self.sims_of(t) for t in self.trades)

    def path_steps(self) -> int:
        """Name-path-steps of one revaluation: 2 paths per pair x steps x names over every simulation."""
        return sum(2 * t.n_pairs * t.n_steps * t.n_names * self.sims_of(t) for t in self.trades)

    def revaluations(self) -> int:
        """(trade, scenario) values of one revaluation."""
        return self.n_trades * self.n_scenarios


def _surfaces(rng, n_names, horizon, n_exp, n_x):
    """Per-name SSVI power-law surfaces (theta_t = c t, c in 0.03..0.06, rho in -0.7..-0.4, eta 1, gamma 0.5) and
    their local variance tabulated on n_exp expiries x n_x log-strikes over the horizon."""
    T = horizon * np.arange(1, n_exp + 1) / n_exp
    surfaces, grids = [], []
    for _ in range(n_names):
        c, rho = rng.uniform(0.03, 0.06), rng.uniform(-0.7, -0.4)
        surfaces.append(SSVI.power_law(rho, 1.0, 0.5, T, c * T))
        grids.append(LocalVarGrid.from_surface(surfaces[-1], T, n_x))
    return surfaces, grids


def scenario_tables(surfaces, grids, vol_shifts, skew_moves) -> np.ndarray:
    """(n_vol, pool rows, n_x): each grid's local variance on its own points with the surface's implied vols moved by
    each scenario's (parallel shift, skew move)."""
    out = []
    for p, k in zip(vol_shifts, skew_moves):
        rows = []
        for surf, g in zip(surfaces, grids):
            kk = grid_points(g.lo, g.inv_dx, g.n_x)
            TT = np.broadcast_to(g.expiries[:, None], kk.shape)
            rows.append(moved_local_var(surf, kk, TT, parallel=float(p), skew=float(k)))
        out.append(np.vstack(rows))
    return np.asarray(out).reshape(len(out), -1, grids[0].n_x if grids else 0)


def moved_corr(corr, move: float) -> np.ndarray:
    """The correlation matrix with every pair moved by `move`, clipped to +-0.999, repaired to the nearest correlation
    matrix when it is no longer positive definite (packages/risk/src/optlab/risk/shocks.py:337-359)."""
    c = np.array(corr, dtype=float)
    if not move:
        return c
    c = np.clip(c + move * (1.0 - np.eye(len(c))), -0.999, 0.999)
    np.fill_diagonal(c, 1.0)
    try:
        np.linalg.cholesky(c)
        return c
    except np.linalg.LinAlgError:
        return nearest_correlation(c)


def sample_book(n_trades: int = 512, seed: int = 2024, paths_log2=(14, 18), years=(1, 5), steps_per_year: int = 252,
                max_names: int = 5, heston_share: float = 0.25, n_surfaces: int = 16, n_exp: int = 40, n_x: int = 200,
                spot_moves=SPOT_MOVES, vol_shifts=VOL_SHIFTS, skew_tilts=SKEW_TILTS, carry_moves=(),
                corr_moves=()) -> Book:
    """A seeded book of uneven trades. Each trade: Heston QE (one name, heston_share of the book) or local vol of
    1..max_names consecutive names of a pool of per-name surfaces; maturity a whole number of years in `years`, one
    step a day; 2^k paths with k uniform in paths_log2; a European ladder (1 to 3 calls or puts), a barrier option
    (up-and-out or up-and-in call, down-and-in or down-and-out put), or a Phoenix autocall (quarterly or monthly),
    each on the worst performance of its names. Scenarios: the spot moves, the carry moves ((rate, dividend yield)
    pairs), the parallel implied-vol shifts, then the skew moves (a vol scenario is a (shift, skew) pair: (s, 0) or
    (0, k), its tables re-tabulated from the moved implied vols),
    then the correlation moves (every pair of a multi-name trade; its moved roots follow its root in the pool)."""
    rng = np.random.default_rng(seed)
    horizon = float(years[1])
    dt = 1.0 / steps_per_year
    surfaces, grids = _surfaces(rng, n_surfaces, horizon, n_exp, n_x)
    table = np.vstack([g.rows for g in grids])
    row_lo = np.concatenate([g.lo for g in grids])
    row_inv = np.concatenate([g.inv_dx for g in grids])
    root, legs, obs = [], [], []
    trades, labels = [], []
    r = 0.02
    for _ in range(n_trades):
        heston = rng.random() < heston_share
        n = 1 if heston else int(rng.integers(1, max_names + 1))
        T = int(rng.integers(years[0], years[1] + 1))
        k = int(rng.integers(paths_log2[0], paths_log2[1] + 1))
        product = ("european", "barrier", "autocall")[int(rng.integers(0, 3))]
        t = ObBatchTrade()
        t.model = OB_MODEL_HESTON_QE if heston else OB_MODEL_PATHS
        t.n_names, t.n_steps, t.n_pairs = n, T * steps_per_year, 2 ** (k - 1)
        t.seed = int(rng.integers(1, 2**62))
        t.r, t.q = r, float(rng.uniform(0.0, 0.02))
        if heston:
            t.heston[:] = [rng.uniform(0.02, 0.06), rng.uniform(1.0, 3.0), rng.uniform(0.02, 0.06),
                           rng.uniform(0.3, 0.7), rng.uniform(-0.8, -0.4)]
        else:
            first = int(rng.integers(0, n_surfaces - n + 1))
            t.table_row0 = first * n_exp
            rho = rng.uniform(0.3, 0.8)
            corr = np.full((n, n), rho) + (1.0 - rho) * np.eye(n)
            t.root0 = sum(len(x) for x in root)
            root.append(np.asarray(correlation_root(corr), dtype=float).ravel())
            t.corr_root0 = sum(len(x) for x in root)
            if n > 1:
                for m in corr_moves:
                    root.append(np.asarray(correlation_root(moved_corr(corr, m)), dtype=float).ravel())
            t.heston[:] = [0.04, 1.0, 0.04, 0.5, 0.0]
        if product in ("european", "barrier"):
            t.product = OB_PRODUCT_LADDER
            t.discount = float(np.exp(-r * T))
            if product == "european":
                m = int(rng.integers(1, 4))
                rows = [(int(rng.integers(1, 3)), rng.uniform(0.8, 1.2), 0, 0.0) for _ in range(m)]
            else:
                kind = int(rng.integers(0, 4))
                K = rng.uniform(0.9, 1.1)
                if kind == 0:
                    rows = [(1, K, BARRIER["up-out"], rng.uniform(1.2, 1.5))]
                elif kind == 1:
                    rows = [(1, K, BARRIER["up-in"], rng.uniform(1.2, 1.5))]
                elif kind == 2:
                    rows = [(2, K, BARRIER["down-in"], rng.uniform(0.6, 0.8))]
                else:
                    rows = [(2, K, BARRIER["down-out"], rng.uniform(0.6, 0.8))]
            t.n_legs, t.leg0 = len(rows), sum(len(x) for x in legs)
            legs.append(rows)
        else:
            t.product = OB_PRODUCT_AUTOCALL
            per_year = 4 if rng.random() < 0.6 else 12
            n_obs = T * per_year
            steps = (np.arange(1, n_obs + 1) * steps_per_year) // per_year
            times = np.arange(1, n_obs + 1) / per_year
            trig = np.full(n_obs, 1.0)
            trig[-1] = 0.0
            t.n_obs, t.obs0 = n_obs, sum(len(x) for x in obs)
            obs.append(list(zip(steps, trig, np.exp(-r * times))))
            t.coupon_barrier = rng.uniform(0.6, 0.8)
            t.coupon = rng.uniform(0.02, 0.10) / per_year
            t.ki_barrier, t.put_strike = rng.uniform(0.5, 0.7), 1.0
            t.memory, t.ki_daily = int(rng.random() < 0.5), int(rng.random() < 0.7)
        trades.append(t)
        labels.append(f"{'heston' if heston else 'lv'}-{n}-{product}-{T}y-2^{k}")
    legs_flat = [x for rows in legs for x in rows] or [(0, 0.0, 0, 0.0)]
    obs_flat = [x for rows in obs for x in rows] or [(1, 0.0, 1.0)]
    carry = np.asarray(carry_moves, float).reshape(-1, 2)
    vs = np.concatenate([np.asarray(vol_shifts, float), np.zeros(len(skew_tilts))])
    vt = np.concatenate([np.zeros(len(vol_shifts)), np.asarray(skew_tilts, float)])
    vol_table = scenario_tables(surfaces, grids, vs, vt) if len(vs) else np.zeros(0)
    return Book(
        trades=trades,
        labels=labels,
        dt=dt,
        horizon=horizon,
        n_exp=n_exp,
        n_x=n_x,
        table=table,
        row_lo=row_lo,
        row_inv_dx=row_inv,
        root=np.concatenate(root) if root else np.ones(1),
        leg_type=[x[0] for x in legs_flat],
        leg_strike=[x[1] for x in legs_flat],
        leg_barrier=[x[2] for x in legs_flat],
        leg_level=[x[3] for x in legs_flat],
        obs_step=[x[0] for x in obs_flat],
        obs_trigger=[x[1] for x in obs_flat],
        obs_discount=[x[2] for x in obs_flat],
        spot_shift=np.asarray(spot_moves, float),
        vol_shift=vs,
        vol_tilt=vt,
        vol_table=vol_table,
        carry_rate=carry[:, 0],
        carry_div=carry[:, 1],
        corr_move=np.asarray(corr_moves, float),
    )


class Batch:
    """A book uploaded for revaluation: tune picks tiles and block sizes per trade class, capture records the whole
    revaluation as one CUDA graph, launch replays it (or runs it directly before a capture); run_per_trade runs the
    same simulations as one launch each, the comparison."""

    def __init__(self, book: Book, precision="fp32"):
        self.book = book
        self._p = C.c_void_p()
        check(load().ob_batch_create(C.byref(book.struct), precision_code(precision), C.byref(self._p)))

    def tune(self, budget_ms: int = 0) -> None:
        check(load().ob_batch_tune(self._p, int(budget_ms)))

    def capture(self, stream=None) -> None:
        check(load().ob_batch_capture(self._p, _stream(stream)))

    def launch(self, stream=None) -> None:
        check(load().ob_batch_launch(self._p, _stream(stream)))

    def run_per_trade(self, stream=None) -> None:
        check(load().ob_batch_run_per_trade(self._p, _stream(stream)))

    def result(self):
        """(price, se) as (n_trades, n_scenarios) arrays (base, spot, carry, vol, correlation moves), and the last
        run's device time in ms."""
        b = self.book
        price = np.empty((b.n_trades, b.n_scenarios))
        se = np.empty_like(price)
        ms = C.c_double()
        check(load().ob_batch_result(self._p, price.ctypes.data_as(_dp), se.ctypes.data_as(_dp), C.byref(ms)))
        return price, se, ms.value

    def classes(self) -> list[dict]:
        """The trade classes (one persistent kernel each) with their trades, current tile and block, and after tune()
        the tuner's sample time at the shape before tuning and at the kept one (microseconds)."""
        n = C.c_int()
        check(load().ob_batch_classes(self._p, 0, C.byref(n), None))
        info = np.zeros(8 * max(n.value, 1), np.int32)
        check(load().ob_batch_classes(self._p, n.value, C.byref(n), info.ctypes.data_as(_ip)))
        keys = ("model", "names", "product", "trades", "tile", "block", "untuned_us", "tuned_us")
        return [dict(zip(keys, map(int, info[8 * k:8 * k + 8]))) for k in range(n.value)]

    def close(self) -> None:
        if self._p:
            load().ob_batch_destroy(self._p)
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


def _stream(stream):
    if stream is None:
        return C.c_void_p(torch.cuda.current_stream().cuda_stream) if torch.cuda.is_available() else None
    return C.c_void_p(stream.cuda_stream)
