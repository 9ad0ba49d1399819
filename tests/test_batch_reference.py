"""The batch's scenarios against the reference's own risk engine (tests/golden/reference_scenarios.json, made by
tests/golden/make_scenario_fixtures.py from packages/risk/src/optlab/risk/engine.py:382-425 and surfaces.py:204).

- The vol scenarios' tables: this package's implied-vol moves (parallel shift and skew rotation, Dupire re-read) equal
  the reference's bumped surfaces' local variance at sampled points.
- A four-trade book (a call-and-put ladder, a daily down-and-in put, a Phoenix with a daily knock-in, a 2-name
  worst-of autocall; one year) under spot moves of +-5 %, parallel moves of +-2 implied-vol points and skew moves of
  +-2 points, valued by the oracle's batch semantics (or_batch_trade: spot moves on the base simulation, each vol move
  a simulation of the moved tables on the same random numbers; the GPU batch equals it within 1e-10), against the
  reference's run_group values and P&Ls. The two simulations differ in their grids (the reference grades its first
  steps and tabulates 801 points a step; the batch steps daily on 40 expiries x 200 points), so they agree in
  distribution: every value within 4 combined standard errors, every scenario P&L within 4 of its combined standard
  error."""

import json
from pathlib import Path

import numpy as np
import pytest

from optlab_b200 import ivnodes
from optlab_b200._abi import BARRIER, OB_MODEL_PATHS, OB_PRODUCT_AUTOCALL, OB_PRODUCT_LADDER, ObBatchTrade
from optlab_b200.batch import Book, scenario_tables
from optlab_b200.models import correlation_root
from optlab_b200.surfaces import SSVI, LocalVarGrid

FIX = json.loads((Path(__file__).resolve().parent / "golden" / "reference_scenarios.json").read_text())
N_EXP, N_X = 40, 200
ORDER = ["spot+", "spot-", "vol+", "vol-", "skew+", "skew-"]  # the batch's outputs after the base


def _surface(name):
    c, rho = FIX["surfaces"][name]
    T = 3.0 * np.arange(1, 41) / 40
    return SSVI.power_law(rho, 1.0, 0.5, T, c * T)


def test_moved_surfaces_are_the_references():
    m = FIX["moved_local_var"]
    surf = _surface(m["surface"])
    k, T = np.array(m["k"]), np.array(m["T"])
    assert np.max(np.abs(ivnodes.moved_local_var(surf, k, T) / np.array(m["base"]) - 1)) < 1e-12
    for key, want in m["moved"].items():
        kind, h = FIX["moves"][key]
        got = ivnodes.moved_local_var(surf, k, T, parallel=h if kind == "parallel" else 0.0,
                                      skew=h if kind == "skew" else 0.0)
        assert np.max(np.abs(got / np.array(want) - 1)) < 1e-12, key


def _book():
    """The fixture's trades as a batch book: pool [A, B, A, C] (a trade's names are consecutive pool surfaces)."""
    r, q = FIX["r"], FIX["q"]
    pool = ["A", "B", "A", "C"]
    first = {"ladder-A": 0, "down-in-put-B": 1, "phoenix-A": 2, "worst-of-A-C": 2}
    expiries = 1.0 * np.arange(1, N_EXP + 1) / N_EXP
    surfaces = [_surface(n) for n in pool]
    grids = [LocalVarGrid.from_surface(s, expiries, N_X) for s in surfaces]
    trades, roots, legs, obs = [], [], [], []
    obs_t = np.array([0.25, 0.5, 0.75, 1.0])
    for tr in FIX["trades"]:
        t = ObBatchTrade()
        n = len(tr["names"])
        t.model, t.n_names, t.n_steps, t.n_pairs = OB_MODEL_PATHS, n, 252, FIX["n_paths"] // 2
        t.seed, t.r, t.q = tr["key"], r, q
        t.table_row0 = first[tr["label"]] * N_EXP
        c = float(tr.get("corr", 0.0))
        t.root0 = sum(len(x) for x in roots)
        roots.append(np.asarray(correlation_root(np.full((n, n), c) + (1 - c) * np.eye(n)), float).ravel())
        t.corr_root0 = t.root0
        t.heston[:] = [0.04, 1.0, 0.04, 0.5, 0.0]
        if tr["product"] == "ladder":
            t.product, t.discount = OB_PRODUCT_LADDER, float(np.exp(-r))
            t.n_legs, t.leg0 = len(tr["legs"]), sum(len(x) for x in legs)
            legs.append([tuple(x) for x in tr["legs"]])
        else:
            t.product = OB_PRODUCT_AUTOCALL
            t.n_obs, t.obs0 = 4, sum(len(x) for x in obs)
            obs.append(list(zip([63, 126, 189, 252], [1.0, 1.0, 1.0, 0.0], np.exp(-r * obs_t))))
            t.coupon_barrier, t.coupon, t.ki_barrier, t.put_strike = 0.7, 0.02, 0.6, 1.0
            t.memory, t.ki_daily = 1, int(tr["ki_daily"])
        trades.append(t)
    assert BARRIER["down-in"] == 4
    legs_flat = [x for rows in legs for x in rows]
    obs_flat = [x for rows in obs for x in rows]
    vs = np.array([0.02, -0.02, 0.0, 0.0])
    vt = np.array([0.0, 0.0, 0.02, -0.02])
    return Book(
        trades=trades, labels=[tr["label"] for tr in FIX["trades"]], dt=1.0 / 252, horizon=1.0, n_exp=N_EXP, n_x=N_X,
        table=np.vstack([g.rows for g in grids]), row_lo=np.concatenate([g.lo for g in grids]),
        row_inv_dx=np.concatenate([g.inv_dx for g in grids]), root=np.concatenate(roots),
        leg_type=[x[0] for x in legs_flat], leg_strike=[x[1] for x in legs_flat], leg_barrier=[x[2] for x in legs_flat],
        leg_level=[x[3] for x in legs_flat], obs_step=[x[0] for x in obs_flat], obs_trigger=[x[1] for x in obs_flat],
        obs_discount=[x[2] for x in obs_flat], spot_shift=np.array([0.05, -0.05]), vol_shift=vs, vol_tilt=vt,
        vol_table=scenario_tables(surfaces, grids, vs, vt),
    )


@pytest.fixture(scope="module")
def valued(oracle):
    b = _book()
    return b, [oracle.batch_trade(b, i) for i in range(b.n_trades)]


@pytest.mark.parametrize("i", range(4))
def test_scenario_values_agree_with_the_references_risk_engine(valued, i):
    b, vals = valued
    price, se = vals[i]
    tr = FIX["trades"][i]
    ref_base, ref_se = tr["base"]
    assert abs(price[0] - ref_base) <= 4 * np.hypot(se[0], ref_se), (tr["label"], price[0], ref_base, ref_se)
    for s, key in enumerate(ORDER, start=1):
        want = tr["values"][key]
        assert abs(price[s] - want) <= 4 * np.hypot(se[s], ref_se), (tr["label"], key, price[s], want)


@pytest.mark.parametrize("i", range(4))
def test_scenario_pnls_agree_with_the_references_and_the_vol_moves_are_felt(valued, i):
    """P&L against the base on each side's own random numbers; the two sides' P&L noise is of the reference's size
    (same paths a side), so the combined standard error is sqrt(2) times the reference's."""
    b, vals = valued
    price, _ = vals[i]
    tr = FIX["trades"][i]
    for s, key in enumerate(ORDER, start=1):
        mine = price[s] - price[0]
        want, want_se = tr["pnl"][key]
        assert abs(mine - want) <= 4 * np.sqrt(2) * want_se + 2e-3 * abs(want), (tr["label"], key, mine, want, want_se)
    # the vol and skew moves are measured, not noise, on the reference's side: the comparison has teeth
    assert abs(tr["pnl"]["vol+"][0]) > 4 * tr["pnl"]["vol+"][1]
