"""The oracle's fused pricing of a local-correlation basket (or_mc_price with the mixer) against its own path engine
(or_paths, pinned to the reference's compiled engine's local-correlation paths in test_oracle): the same request's
terminal spots, priced by a call ladder on the worst performance in NumPy, give the same price to rounding."""

import numpy as np

from optlab_b200 import workloads
from optlab_b200.models import LocalCorrelation, aligned_factors, correlation_root
from optlab_b200.requests import mc_request, paths_request


def test_the_oracles_mixer_pricing_is_its_mixer_paths(oracle):
    n, n_steps, years, n_pairs = 3, 60, 0.5, 2**11
    corr = np.full((n, n), 0.55) + 0.45 * np.eye(n)
    root = correlation_root(corr)
    lc = LocalCorrelation(0.15, 0.0, 0.3, 0.1)
    low, sign, turn = aligned_factors(corr, root, lc.w0)
    mix = (lc.w0, lc.level, lc.down, lc.up, lc.sigma, sign, np.cos(turn), np.sin(turn))
    g = workloads.lv_grid(horizon=years, n_exp=6, n_x=80)
    dt, t0 = workloads.uniform_grid(years, n_steps)
    t_end = np.concatenate([[0.0], t0 + dt])
    m = workloads.FlatMarket(100.0, 0.02, 0.01)
    common = dict(dt=dt, t0=t0, root=root, kind=np.ones(n, np.int32), cvar=np.zeros(n), n_pairs=n_pairs, seed=77,
                  step_row=np.tile(g.row_of(t0), (n, 1)), lo=g.lo, inv_dx=g.inv_dx, table=g.rows, n_x=g.n_x,
                  mixer=1, mix=mix, low_root=low)
    strikes = [0.9, 1.0, 1.1]
    fused = oracle.mc_price(mc_request(model=0, spot=np.full(n, 100.0), log_fwd=np.tile(m.log_fwd(t_end), (n, 1)),
                                       product=0, leg_type=[1, 1, 2], leg_strike=[100.0 * k for k in strikes],
                                       discount=float(m.D(years)), **common))
    held = paths_request(obs_step=[n_steps], heston=np.tile([0.0, 1.0, 1.0, 0.0, 0.0], n), same=1,
                         fwd=np.full((n, 1), m.F(years)), **common)
    oracle.paths(held)
    out = next(a for a in held.keep if isinstance(a, np.ndarray) and a.ndim == 3)  # names x 1 x 2 pairs
    worst = (out[:, 0, :] / 100.0).min(axis=0)
    pays = [np.maximum(worst - strikes[0], 0), np.maximum(worst - strikes[1], 0), np.maximum(strikes[2] - worst, 0)]
    for k, pay in enumerate(pays):
        y = 0.5 * (pay[:n_pairs] + pay[n_pairs:]) * 100.0 * float(m.D(years))
        assert abs(fused.price[k] - y.mean()) <= 1e-12 * max(1.0, abs(y.mean())), (k, fused.price[k], y.mean())
