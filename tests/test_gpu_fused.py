"""The fused pricing kernels (the specialised one of fused.cu and the generic one of mc.cu) against the oracle, for every
model kind, basket size and product they cover: FP64 within 1e-10 relative, FP32 within 4 standard errors."""

import numpy as np
import pytest

from optlab_b200 import engine, workloads
from optlab_b200.requests import mc_request

pytestmark = pytest.mark.gpu


def _request(kinds, product, n_pairs=2**12, seed=17, n_steps=126, years=0.5):
    n = len(kinds)
    corr = np.full((n, n), 0.6) + 0.4 * np.eye(n)
    g = workloads.lv_grid(horizon=years, n_exp=8, n_x=120)
    dt, t0 = workloads.uniform_grid(years, n_steps)
    t_end = np.concatenate([[0.0], t0 + dt])
    m = workloads.FlatMarket(100.0, 0.02, 0.01)
    hes = np.tile([0.04, 1.5, 0.04, 0.5, -0.7], n).reshape(n, 5)
    hes[:, 3] = np.linspace(0.3, 0.6, n)
    kw = dict(
        model=0, dt=dt, t0=t0, spot=100.0 + 10 * np.arange(n), n_pairs=n_pairs, seed=seed,
        root=np.linalg.cholesky(corr), kind=kinds, cvar=np.full(n, 0.04), heston=hes,
        log_fwd=np.tile(m.log_fwd(t_end), (n, 1)), step_row=np.tile(g.row_of(t0), (n, 1)), lo=g.lo,
        inv_dx=g.inv_dx, table=g.rows * (0.5 if any(k == 3 for k in kinds) else 1.0) + (1.0 if 3 in kinds else 0.0),
        n_x=g.n_x,
    )
    if product == "autocall":
        ph = workloads.Phoenix(years=years, obs_per_year=8)
        kw.update(workloads.autocall_fields(ph, m, int(round(n_steps / years))))
    else:
        strikes = [80.0, 100.0, 120.0, 100.0, 100.0]
        kw.update(product=0, leg_type=[1, 1, 1, 2, 1], leg_strike=strikes, leg_barrier=[0, 0, 0, 4, 1],
                  leg_level=[0, 0, 0, 85.0, 125.0], discount=float(m.D(years)))
    return kw


CASES = [
    ([1], "autocall"), ([1], "ladder"), ([2], "ladder"), ([3], "autocall"), ([3], "ladder"), ([1, 1], "autocall"),
    ([1, 1, 1], "autocall"), ([1, 1, 1], "ladder"), ([1, 1, 1, 1, 1], "autocall"), ([2, 2, 2], "autocall"),
    ([3, 3], "ladder"), ([1, 2], "autocall"), ([1] * 7, "ladder"), ([0], "autocall"), ([0, 0, 0], "ladder"),
    ([0] * 5, "autocall"),
]


@pytest.mark.parametrize("generic", [False, True], ids=["specialised", "generic"])
@pytest.mark.parametrize("kinds,product", CASES, ids=[f"{k}-{p}" for k, p in CASES])
def test_fp64_fused_prices_match_the_oracle(oracle, monkeypatch, kinds, product, generic):
    if generic:
        monkeypatch.setenv("OPTLAB_B200_GENERIC", "1")
    kw = _request(kinds, product)
    g = engine.mc_price(mc_request(**kw), "fp64")
    o = oracle.mc_price(mc_request(**kw))
    n = o.n_out
    pg, po = np.array(g.price[:n]), np.array(o.price[:n])
    nz = po != 0
    assert np.all(pg[~nz] == 0)
    assert np.abs(pg[nz] / po[nz] - 1).max() < 1e-10, (pg, po)


@pytest.mark.parametrize("kinds,product", CASES, ids=[f"{k}-{p}" for k, p in CASES])
def test_fp32_fused_prices_are_within_4_se_of_the_fp64_oracle(oracle, kinds, product):
    kw = _request(kinds, product, n_pairs=2**14)
    g = engine.mc_price(mc_request(**kw), "fp32")
    o = oracle.mc_price(mc_request(**kw))
    n = o.n_out
    pg, po, so = np.array(g.price[:n]), np.array(o.price[:n]), np.array(o.se[:n])
    assert np.all(np.abs(pg - po) <= 4 * so + 1e-12), (pg - po, so)


@pytest.mark.parametrize("kind", [1, 0])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_observations_on_the_edges_of_step_batches_are_all_taken(oracle, kind, prec):
    """Observation dates at the first step, either side of an eight-step batch's edge, on consecutive steps and at the
    last step. The single-name kernel runs a batch whose first step's record says the next date is at least eight
    steps away without testing each step for one; every one of these dates must still be observed."""
    n_steps, years = 126, 0.5
    kw = _request([kind], "autocall", n_pairs=2**13, n_steps=n_steps, years=years)
    steps = np.array([1, 8, 9, 16, 17, 40, 41, 42, 64, 100, 125, 126], dtype=np.int32)
    m = workloads.FlatMarket(100.0, 0.02, 0.01)
    trig = np.full(len(steps), kw["trigger"][0])
    trig[-1] = 0.0
    kw.update(obs_step=steps, obs_discount=m.D(steps * (years / n_steps)), trigger=trig)
    g = engine.mc_price(mc_request(**kw), prec)
    o = oracle.mc_price(mc_request(**kw))
    n = o.n_out
    pg, po, so = np.array(g.price[:n]), np.array(o.price[:n]), np.array(o.se[:n])
    if prec == "fp64":
        nz = po != 0
        assert np.abs(pg[nz] / po[nz] - 1).max() < 1e-10, (pg, po)
    else:
        assert np.all(np.abs(pg - po) <= 4 * so + 1e-12), (pg - po, so)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_heston_qe_autocall_matches_the_oracle(oracle, prec):
    h = workloads.heston_qe_ladder(n_paths=2**13, seed=5)
    s = h.struct
    m = workloads.FlatMarket(100.0, 0.02, 0.01)
    fields = workloads.autocall_fields(workloads.Phoenix(years=1.0), m, 252)
    kw = dict(model=1, dt=np.full(252, 1 / 252), t0=np.arange(252) / 252, spot=[100.0], n_pairs=s.n_pairs, seed=5,
              heston=workloads.HESTON_CFG0, r=0.02, q=0.01, **fields)
    g = engine.mc_price(mc_request(**kw), prec)
    o = oracle.mc_price(mc_request(**kw))
    if prec == "fp64":
        assert np.abs(np.array(g.price[:4]) / np.array(o.price[:4]) - 1).max() < 1e-10
    else:
        assert abs(g.price[0] - o.price[0]) < 4 * o.se[0]


def test_the_specialised_and_generic_kernels_agree(monkeypatch):
    kw = _request([1, 1, 1], "autocall", n_pairs=2**13)
    a = engine.mc_price(mc_request(**kw), "fp64")
    monkeypatch.setenv("OPTLAB_B200_GENERIC", "1")
    b = engine.mc_price(mc_request(**kw), "fp64")
    assert np.abs(np.array(a.price[:4]) / np.array(b.price[:4]) - 1).max() < 1e-12
