"""The calibration and the Greeks at the sizes of the benchmark's own configurations, not only at small test sizes.

- SLV leverage by particles at 2^18 particles x 504 daily steps over two years, a 128-point regression grid, 400
  bins and 8192 fine bins, Heston (v0 .04, kappa 1.5, theta .04, xi .5, rho -.7) under the SSVI surface of the
  local-vol Phoenix (801-point local-variance rows): FP64 equals the oracle, which follows the reference's
  `calibrate_leverage` (RC/src/leverage.cpp:42-97) and is pinned to it on one thread, within 1e-8 relative; FP32
  particles (FP64 bins and regression) stay within the stated float noise of it.
- Adjoint Greeks of the 3-name worst-of autocall over its full 4 years of daily steps (1008 steps, 2^16 paths):
  the three deltas and 30 node vegas spread over expiries, strikes and names against central finite differences of
  the FP64 revaluation on common random numbers.
"""

import numpy as np
import pytest
import torch

from optlab_b200 import engine, workloads
from optlab_b200.adjoint import AdjointPlan, VegaNodes, autocall_greeks

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def leverage_oracle(oracle):
    o = workloads.slv_leverage()
    oracle.leverage(o)
    return o


def test_fp64_leverage_at_the_calibration_size_matches_the_oracle(leverage_oracle):
    o = leverage_oracle
    g = workloads.slv_leverage()
    assert (g.struct.n_pairs * 2, g.struct.n_steps, g.struct.n_x) == (2**18, 504, 128)
    engine.leverage(g, "fp64")
    assert np.abs(g.x_grids - o.x_grids).max() <= 1e-9 * np.abs(o.x_grids).max()
    rel = np.abs(g.values / o.values - 1)
    assert rel.max() < 1e-8, (np.median(rel), rel.max())


def test_fp32_leverage_at_the_calibration_size_stays_within_float_noise(leverage_oracle):
    """Float particles (FP64 bins and regression) move the bins' contents and the quantiles by float rounding, and the
    fit feeds back into the particles for 504 steps. Measured against the FP64 oracle: median 1.0e-3, 90th percentile
    6.2e-3, largest 5.1e-2, the largest on the grid's ends (the distribution's tails, a few particles a bin) and in
    the later steps; the central half of the grid median 7.7e-4, largest 2.1e-2. Bounds: about twice those."""
    o = leverage_oracle
    g = workloads.slv_leverage()
    engine.leverage(g, "fp32")
    rel = np.abs(g.values / o.values - 1)
    assert np.median(rel) < 2e-3 and np.quantile(rel, 0.9) < 1.2e-2 and rel.max() < 0.1, \
        (np.median(rel), np.quantile(rel, 0.9), rel.max())
    mid = rel[:, 32:96]
    assert np.median(mid) < 1.5e-3 and mid.max() < 4e-2, (np.median(mid), mid.max())
    assert np.abs(g.x_grids - o.x_grids).max() < 2e-2


# ---------------------------------------------------------------------------------------------------- adjoint

EPS = 0.005
H = 1e-6  # a bump well inside the smoothed digitals' ramps (relative width 0.005)
# The bumps over the full horizon: across 1008 steps, 3 names and 16 dates the worst-of's kinks (which name is worst,
# which step is lowest) lie closer together than 1e-6 of spot, so the central difference of the oracle's revaluation
# only settles at smaller bumps: name 1's from 1.8947e-3 (h = 1e-5) and 1.88568e-3 (1e-6) to 1.884610e-3 (1e-7), name
# 2's from 2.34116e-3 (1e-6) and 2.33338e-3 (1e-7) to 2.3284445e-3 (3e-8 and 1e-8), each the adjoint's value to 1e-9.
H_SPOT = 1e-8
H_VOL = 1e-7


def _shifted_log_fwd(held, name, h):
    """The same request with name's log-forwards after t = 0 moved by log(1 + h): its spot moved by the factor
    1 + h, the local vol read in moneyness."""
    s = held.struct
    lf = np.ctypeslib.as_array(s.log_fwd, shape=(s.n_names * (s.n_steps + 1),)).reshape(s.n_names, -1)
    saved = lf[name, 1:].copy()
    lf[name, 1:] += np.log1p(h)
    return saved


def test_adjoint_greeks_over_the_full_worst_of_horizon_match_central_differences():
    w = workloads.worst_of(n_paths=2**16, years=4.0, seed=31)
    s = w.held.struct
    assert (s.n_steps, s.n_names) == (1008, 3)
    nodes = VegaNodes(w.row_name, w.row_T, w.row_lo, w.row_inv_dx, w.n_x, w.node_T, w.node_k)
    g = autocall_greeks(w.held, nodes, EPS, "fp64")
    vega = g["vega"]
    scale = np.abs(vega).max()
    # deltas: each name's forwards moved by 1 +- h on the same draws
    lf = np.ctypeslib.as_array(s.log_fwd, shape=(s.n_names * (s.n_steps + 1),)).reshape(s.n_names, -1)
    for a in range(3):
        v = []
        for sgn in (1, -1):
            saved = _shifted_log_fwd(w.held, a, sgn * H_SPOT)
            try:
                with AdjointPlan(w.held, EPS, "fp64") as p:
                    v.append(p.run(grad=False).price)
            finally:
                lf[a, 1:] = saved
        fd = (v[0] - v[1]) / (np.log1p(H_SPOT) - np.log1p(-H_SPOT)) / w.spots[a]
        assert abs(g["delta"][a] - fd) <= 1e-4 * abs(fd) + 1e-9, (a, g["delta"][a], fd)
    # 30 node vegas: per name the two largest, and eight on a spread of expiries x strikes
    picks = []
    for a in range(3):
        order = np.argsort(-np.abs(vega[a]).ravel())
        picks += [(a, *np.unravel_index(f, vega[a].shape)) for f in order[:2]]
        picks += [(a, e, k) for e, k in ((0, 7), (1, 10), (2, 4), (3, 12), (5, 7), (6, 2), (8, 9), (9, 13))]
    assert len(set(picks)) == 30
    base = torch.tensor(np.ctypeslib.as_array(s.table, shape=(s.n_rows * s.n_x,)).reshape(s.n_rows, s.n_x),
                        dtype=torch.float64, device="cuda")
    with AdjointPlan(w.held, EPS, "fp64") as plan:
        for idx in picks:
            v = []
            for sgn in (1, -1):
                b = torch.zeros(nodes.shape, dtype=torch.float64, device="cuda")
                b[idx] = sgn * H_VOL
                v.append(plan.run(nodes.table(base, b), grad=False).price)
            fd = (v[0] - v[1]) / (2 * H_VOL)
            assert abs(vega[idx] - fd) <= 1e-4 * abs(fd) + 1e-6 * scale, (idx, vega[idx], fd)
