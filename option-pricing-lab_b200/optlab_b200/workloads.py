"""The benchmark workloads as seeded synthetic requests (no market data is read: every input is generated here).

- `heston_qe_ladder`: Heston by Andersen's QE-M, S0 100, v0 .04, kappa 1.5, theta .04, xi .5, rho -.7, r .02, q .01,
  one year of 252 daily steps, 2^16 paths; eleven European calls K = 80, 84, ..., 120 and a daily up-and-out call
  K 100, B 130; prices with standard errors.
- `lv_phoenix`: Dupire local vol of the SSVI power-law surface theta_t = 0.04 t, rho -0.6, eta 1, gamma 0.5, tabulated
  on 200 log-strikes x 40 expiries (T_j = 3 j / 40); a 3-year single-name Phoenix, quarterly observations,
  autocall at 100 %, coupon 2 % at 70 % with memory, knock-in at 60 % on daily closes into a put struck at 100 %;
  756 daily steps, 2^20 paths; flat market r .02, q .01.
- `slv_leverage`: the SLV leverage by particles, Heston of `heston_qe_ladder` (xi unscaled, mix 1) on the surface of
  `lv_phoenix`; 2^18 particles, 504 uniform steps over two years; regression on 128 points, 400 bins, 8192 fine bins,
  Nadaraya-Watson with the reference's bandwidth; the local variance on rows of 801 points per step.
- `worst_of`: three names, each its own SSVI power-law surface (theta_t = c t with c = 0.03, 0.045, 0.06; rho = -0.7,
  -0.55, -0.4; eta 1, gamma 0.5) tabulated on 40 expiries x 200 log-strikes over four years, pairwise correlation 0.6;
  a worst-of Phoenix, quarterly over four years (16 observations), 1008 daily steps, 2^19 paths. Its Greeks: delta per
  name and vega per node of each local-vol surface on 10 expiries x 15 log-strikes.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from ._abi import BARRIER, OB_MODEL_HESTON_QE, OB_MODEL_PATHS, OB_PRODUCT_AUTOCALL, OB_PRODUCT_LADDER
from .models import correlation_root
from .requests import Held, mc_request
from .surfaces import SSVI, LocalVarGrid

HESTON_CFG0 = (0.04, 1.5, 0.04, 0.5, -0.7)  # v0, kappa, theta, xi, rho


@dataclass(frozen=True)
class FlatMarket:
    spot: float
    r: float
    q: float

    def F(self, t):
        return self.spot * np.exp((self.r - self.q) * np.asarray(t, dtype=float))

    def D(self, t):
        return np.exp(-self.r * np.asarray(t, dtype=float))

    def log_fwd(self, t):
        """ln(F(t) / spot)."""
        return (self.r - self.q) * np.asarray(t, dtype=float)


def uniform_grid(T: float, n_steps: int):
    """(dt, t0) of n_steps equal steps to T."""
    h = T / n_steps
    return np.full(n_steps, h), np.arange(n_steps) * h


def heston_qe_ladder(n_paths: int = 2**16, seed: int = 1, n_steps: int = 252, T: float = 1.0) -> Held:
    m = FlatMarket(100.0, 0.02, 0.01)
    dt, t0 = uniform_grid(T, n_steps)
    strikes = np.append(np.arange(80.0, 120.0 + 1e-9, 4.0), 100.0)
    n_legs = len(strikes)
    barrier = np.zeros(n_legs, np.int32)
    barrier[-1] = BARRIER["up-out"]
    level = np.zeros(n_legs)
    level[-1] = 130.0
    return mc_request(
        model=OB_MODEL_HESTON_QE,
        dt=dt,
        t0=t0,
        spot=[m.spot],
        n_pairs=n_paths // 2,
        seed=seed,
        heston=HESTON_CFG0,
        r=m.r,
        q=m.q,
        product=OB_PRODUCT_LADDER,
        leg_type=np.ones(n_legs, np.int32),
        leg_strike=strikes,
        leg_barrier=barrier,
        leg_level=level,
        discount=float(m.D(T)),
    )


def lv_surface(rho=-0.6, eta=1.0, gamma=0.5, theta_rate=0.04, horizon=3.0, n_exp=40) -> SSVI:
    T = horizon * np.arange(1, n_exp + 1) / n_exp
    return SSVI.power_law(rho, eta, gamma, T, theta_rate * T)


def lv_grid(surface: SSVI | None = None, horizon=3.0, n_exp=40, n_x=200) -> LocalVarGrid:
    surface = surface or lv_surface(horizon=horizon, n_exp=n_exp)
    return LocalVarGrid.from_surface(surface, horizon * np.arange(1, n_exp + 1) / n_exp, n_x)


@dataclass(frozen=True)
class Phoenix:
    """A Phoenix autocall on one name or the worst of several (notional 1)."""

    years: float = 3.0
    obs_per_year: int = 4
    trigger: float = 1.0
    coupon_barrier: float = 0.7
    coupon: float = 0.02
    ki_barrier: float = 0.6
    put_strike: float = 1.0
    memory: bool = True
    ki_daily: bool = True

    def schedule(self, steps_per_year: int):
        """(obs_step, obs_time) of the observation dates on a grid of steps_per_year uniform steps a year."""
        n_obs = int(round(self.years * self.obs_per_year))
        steps = (np.arange(1, n_obs + 1) * steps_per_year) // self.obs_per_year
        return steps.astype(np.int32), np.arange(1, n_obs + 1) / self.obs_per_year


def autocall_fields(ph: Phoenix, market: FlatMarket, steps_per_year: int) -> dict:
    obs_step, obs_t = ph.schedule(steps_per_year)
    trig = np.full(len(obs_step), ph.trigger)
    trig[-1] = 0.0  # no call on the final date: the redemption decides there
    return dict(
        product=OB_PRODUCT_AUTOCALL,
        obs_step=obs_step,
        obs_discount=market.D(obs_t),
        trigger=trig,
        coupon_barrier=ph.coupon_barrier,
        coupon=ph.coupon,
        ki_barrier=ph.ki_barrier,
        put_strike=ph.put_strike,
        memory=int(ph.memory),
        ki_daily=int(ph.ki_daily),
    )


def lv_phoenix(n_paths: int = 2**20, seed: int = 7, steps_per_year: int = 252, phoenix: Phoenix | None = None,
               grid: LocalVarGrid | None = None) -> Held:
    ph = phoenix or Phoenix()
    m = FlatMarket(100.0, 0.02, 0.01)
    n_steps = int(round(ph.years * steps_per_year))
    dt, t0 = uniform_grid(ph.years, n_steps)
    g = grid or lv_grid(horizon=ph.years)
    t_end = np.concatenate([[0.0], t0 + dt])
    return mc_request(
        model=OB_MODEL_PATHS,
        dt=dt,
        t0=t0,
        spot=[m.spot],
        n_pairs=n_paths // 2,
        seed=seed,
        kind=[1],
        cvar=[0.0],
        log_fwd=m.log_fwd(t_end)[None, :],
        step_row=g.row_of(t0)[None, :],
        lo=g.lo,
        inv_dx=g.inv_dx,
        table=g.rows,
        n_x=g.n_x,
        **autocall_fields(ph, m, steps_per_year),
    )


def slv_leverage(n_particles: int = 2**18, seed: int = 5, n_steps: int = 504, T: float = 2.0, n_x: int = 128,
                 n_lv: int = 801, local_linear: int = 0):
    from .leverage import leverage_request
    from .surfaces import local_var_rows

    surface = lv_surface(horizon=3.0)
    dt, t0 = uniform_grid(T, n_steps)
    lo, inv, rows = local_var_rows(surface, t0, n_lv)
    atm_vol = float(np.sqrt(surface.theta(1.0) / 1.0))
    return leverage_request(
        dt=dt, t0=t0, n_pairs=n_particles // 2, seed=seed, heston=HESTON_CFG0, n_x=n_x, lv_lo=lo, lv_inv_dx=inv,
        lv_rows=rows, atm_vol=atm_vol, local_linear=local_linear, positive_part=local_linear,
    )


def path_steps(held: Held) -> int:
    """Path-steps of one run of a fused request: 2 n_pairs paths x n_steps steps x n_names names."""
    s = held.struct
    return 2 * s.n_pairs * s.n_steps * s.n_names


@dataclass
class WorstOf:
    """The worst-of request with what its node vegas need: each table row's name, expiry and log-strike grid."""

    held: Held
    row_name: np.ndarray
    row_T: np.ndarray
    row_lo: np.ndarray
    row_inv_dx: np.ndarray
    n_x: int
    node_T: np.ndarray
    node_k: np.ndarray
    spots: np.ndarray


def worst_of(n_paths: int = 2**19, seed: int = 11, years: float = 4.0, steps_per_year: int = 252, n_names: int = 3,
             c=(0.03, 0.045, 0.06), rho=(-0.7, -0.55, -0.4), corr: float = 0.6, n_exp: int = 40, n_x: int = 200,
             n_node_T: int = 10, n_node_k: int = 15, phoenix: Phoenix | None = None) -> WorstOf:
    ph = phoenix or Phoenix(years=years)
    m = FlatMarket(100.0, 0.02, 0.01)
    n_steps = int(round(years * steps_per_year))
    dt, t0 = uniform_grid(years, n_steps)
    t_end = np.concatenate([[0.0], t0 + dt])
    T = years * np.arange(1, n_exp + 1) / n_exp
    grids = [lv_grid(SSVI.power_law(rho[a], 1.0, 0.5, T, c[a] * T), horizon=years, n_exp=n_exp, n_x=n_x)
             for a in range(n_names)]
    step_row = np.stack([g.row_of(t0) + a * n_exp for a, g in enumerate(grids)])
    C = np.full((n_names, n_names), corr) + (1.0 - corr) * np.eye(n_names)
    spots = np.full(n_names, m.spot)
    held = mc_request(
        model=OB_MODEL_PATHS,
        dt=dt,
        t0=t0,
        spot=spots,
        n_pairs=n_paths // 2,
        seed=seed,
        root=correlation_root(C),
        kind=np.ones(n_names, np.int32),
        cvar=np.zeros(n_names),
        log_fwd=np.tile(m.log_fwd(t_end), (n_names, 1)),
        step_row=step_row,
        lo=np.concatenate([g.lo for g in grids]),
        inv_dx=np.concatenate([g.inv_dx for g in grids]),
        table=np.vstack([g.rows for g in grids]),
        n_x=n_x,
        **autocall_fields(ph, m, steps_per_year),
    )
    return WorstOf(
        held,
        np.repeat(np.arange(n_names), n_exp),
        np.tile(T, n_names),
        np.concatenate([g.lo for g in grids]),
        np.concatenate([g.inv_dx for g in grids]),
        n_x,
        years * np.arange(1, n_node_T + 1) / n_node_T,
        np.linspace(-1.0, 0.5, n_node_k),
        spots,
    )
