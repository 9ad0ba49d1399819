"""Local correlation (the reference's mixer, RC/include/optlab_cuda/paths.hpp:219-237, localcorr.py:47-83) in the fused
pricing kernels and the payoff-script interpreter: local-vol baskets of 2 to 5 names whose names' normals mix a common
factor with a weight that moves with the level of the basket. The specialised fused kernel (MIX) and the generic one
against the oracle (FP64 within 1e-10 relative), FP32 within 4 standard errors of FP64, and a worst-of Phoenix written
as a script against the fused kernel on the same basket."""

import numpy as np
import pytest

from optlab_b200 import _abi, engine, workloads
from optlab_b200 import script as sc
from optlab_b200.models import LocalCorrelation, aligned_factors, correlation_root
from optlab_b200.requests import mc_request

pytestmark = pytest.mark.gpu


def _request(n, product, n_pairs=2**12, seed=29, n_steps=126, years=0.5, mixer=LocalCorrelation(0.15, 0.0, 0.3, 0.1)):
    corr = np.full((n, n), 0.55) + 0.45 * np.eye(n)
    root = correlation_root(corr)
    low, sign, turn = aligned_factors(corr, root, mixer.w0)
    mix = (mixer.w0, mixer.level, mixer.down, mixer.up, mixer.sigma, sign, np.cos(turn), np.sin(turn))
    g = workloads.lv_grid(horizon=years, n_exp=8, n_x=120)
    dt, t0 = workloads.uniform_grid(years, n_steps)
    t_end = np.concatenate([[0.0], t0 + dt])
    m = workloads.FlatMarket(100.0, 0.02, 0.01)
    kw = dict(
        model=0, dt=dt, t0=t0, spot=np.full(n, 100.0), n_pairs=n_pairs, seed=seed, root=root,
        kind=np.ones(n, np.int32), cvar=np.zeros(n), log_fwd=np.tile(m.log_fwd(t_end), (n, 1)),
        step_row=np.tile(g.row_of(t0), (n, 1)), lo=g.lo, inv_dx=g.inv_dx, table=g.rows, n_x=g.n_x,
        mixer=1, mix=mix, low_root=low,
    )
    if product == "autocall":
        ph = workloads.Phoenix(years=years, obs_per_year=4)
        kw.update(workloads.autocall_fields(ph, m, int(round(n_steps / years))))
    else:
        kw.update(product=0, leg_type=[1, 2, 1], leg_strike=[100.0, 95.0, 105.0], leg_barrier=[0, 4, 1],
                  leg_level=[0.0, 80.0, 120.0], discount=float(m.D(years)))
    return kw


CASES = [(2, "autocall"), (3, "ladder"), (3, "autocall"), (5, "autocall"), (5, "ladder")]


@pytest.mark.parametrize("generic", [False, True], ids=["specialised", "generic"])
@pytest.mark.parametrize("n,product", CASES, ids=[f"{n}-{p}" for n, p in CASES])
def test_fp64_local_correlation_prices_match_the_oracle(oracle, monkeypatch, n, product, generic):
    if generic:
        monkeypatch.setenv("OPTLAB_B200_GENERIC", "1")
    kw = _request(n, product)
    g = engine.mc_price(mc_request(**kw), "fp64")
    o = oracle.mc_price(mc_request(**kw))
    k = o.n_out
    pg, po = np.array(g.price[:k]), np.array(o.price[:k])
    nz = po != 0
    assert np.all(pg[~nz] == 0)
    assert np.abs(pg[nz] / po[nz] - 1).max() < 1e-10, (pg, po)


def test_the_mixer_moves_the_price():
    """The same basket without the mixer (its plain correlation) prices differently: the mixer is not ignored."""
    kw = _request(3, "autocall", n_pairs=2**14)
    with_mix = engine.mc_price(mc_request(**kw), "fp64")
    kw.update(mixer=0)
    plain = engine.mc_price(mc_request(**kw), "fp64")
    assert abs(with_mix.price[0] - plain.price[0]) > 4 * with_mix.se[0]


@pytest.mark.parametrize("n,product", [(3, "autocall"), (5, "ladder")])
def test_fp32_local_correlation_is_within_4_standard_errors_of_fp64(n, product):
    kw = _request(n, product, n_pairs=2**15)
    g32 = engine.mc_price(mc_request(**kw), "fp32")
    g64 = engine.mc_price(mc_request(**kw), "fp64")
    k = g64.n_out
    for j in range(k):
        assert abs(g32.price[j] - g64.price[j]) <= 4 * g64.se[j] + 1e-12, (j, g32.price[j], g64.price[j])


def test_a_worst_of_phoenix_script_on_a_local_correlation_basket_equals_the_fused_kernel():
    """The interpreter's generic path carries the mixer: a worst-of Phoenix written as a script prices like the fused
    kernel on the same basket and the same normals (FP64, to rounding)."""
    n, years = 3, 0.5
    kw = _request(n, "autocall", n_pairs=2**13, years=years)
    ph = workloads.Phoenix(years=years, obs_per_year=4)
    held = mc_request(**kw)
    worst = "X0 / S0"
    for a in range(1, n):
        worst = f"min({worst}, X{a} / S0)"
    lines = [f"underlying X{a}" for a in range(n)] + [
        "param S0 = 100", f"param cb = {ph.coupon_barrier!r}", f"param cpn = {ph.coupon!r}",
        f"param call = {ph.trigger!r}", f"param ki = {ph.ki_barrier!r}", f"param K = {ph.put_strike!r}"]
    n_obs = int(round(years * ph.obs_per_year))
    for j in range(1, n_obs + 1):
        t = j / ph.obs_per_year
        lines.append(f"event t={t!r} pay t={t!r}")
        if j == 1:
            lines.append("  missed = 0")
        lines += [f"  perf = {worst}", "  if perf >= cb then", "    pay cpn * (1 + missed) as coupon",
                  "    missed = 0", "  else", "    missed = missed + 1", "  end"]
        if j < n_obs:
            lines += ["  if perf >= call then", "    pay 1 as redemption", "    terminate", "  end"]
        else:
            n_fix = 126
            lows = [f"lowest(X{a}, t=0, t={t!r}, n={n_fix})" for a in range(n)]
            low = lows[0]
            for w in lows[1:]:
                low = f"min({low}, {w})"
            lines += [f"  knocked = {low} < ki * S0", "  if knocked then",
                      "    pay 1 - max(K - perf, 0) as redemption", "  else", "    pay 1 as redemption", "  end"]
        lines.append("end")
    comp = sc.compile_script("\n".join(lines) + "\n")
    fused = engine.mc_price(held, "fp64")
    res = sc.run(sc.script_request(comp, held, lambda t: np.exp(-0.02 * t)), "fp64")
    assert abs(res.price - fused.price[0]) <= 1e-10 * abs(fused.price[0]), (res.price, fused.price[0])


def test_the_adjoint_refuses_a_local_correlation_basket():
    from optlab_b200.adjoint import AdjointPlan

    kw = _request(3, "autocall")
    with pytest.raises(_abi.EngineError, match="no local correlation"):
        AdjointPlan(mc_request(**kw), 0.005, "fp64")
