"""Adjoint Greeks of the worst-of autocall on the GPU: the smoothed price against the oracle, deltas and node vegas
against central finite differences on common random numbers (the engine's FP64 revaluation and the CPU oracle), and
FP32 against FP64 within 4 standard errors (the target's check: every Greek within 4 SE and 1e-4 relative of FP64)."""

import numpy as np
import pytest
import torch

from optlab_b200 import engine, workloads
from optlab_b200.adjoint import AdjointPlan, VegaNodes, autocall_greeks
from optlab_b200.requests import mc_request

pytestmark = pytest.mark.gpu

EPS = 0.005


def _wo(n_paths=2**14, years=1.0, seed=21, **kw):
    return workloads.worst_of(n_paths=n_paths, years=years, seed=seed, **kw)


def _nodes(w):
    return VegaNodes(w.row_name, w.row_T, w.row_lo, w.row_inv_dx, w.n_x, w.node_T, w.node_k)


def _base(w):
    s = w.held.struct
    return torch.tensor(np.ctypeslib.as_array(s.table, shape=(s.n_rows * s.n_x,)).reshape(s.n_rows, s.n_x),
                        dtype=torch.float64, device="cuda")


def test_the_smoothed_price_matches_the_oracle(oracle):
    w = _wo()
    with AdjointPlan(w.held, EPS, "fp64") as plan:
        r0 = plan.run(grad=False)
        r1 = plan.run(grad=True)
    p, se = oracle.autocall_smooth(w.held, EPS)
    assert abs(r0.price / p - 1) < 1e-10 and abs(r1.price / p - 1) < 1e-10
    assert abs(r0.price_se / se - 1) < 1e-6


def test_without_smoothing_the_adjoint_prices_the_exact_autocall():
    w = _wo(n_paths=2**13)
    exact = engine.mc_price(w.held, "fp64")
    with AdjointPlan(w.held, 0.0, "fp64") as plan:
        r = plan.run(grad=False)
    assert abs(r.price / exact.price[0] - 1) < 1e-10


def _shifted(w, name, h):
    """The request with name's spot moved by the factor 1 + h (its log-forward shifted; local vol in moneyness)."""
    s = w.held.struct
    arrays = {k: np.ctypeslib.as_array(getattr(s, k), shape=(n,)).copy() for k, n in (
        ("dt", s.n_steps), ("t0", s.n_steps), ("spot", s.n_names), ("root", s.n_names**2),
        ("log_fwd", s.n_names * (s.n_steps + 1)), ("step_row", s.n_names * s.n_steps), ("row_lo", s.n_rows),
        ("row_inv_dx", s.n_rows), ("table", s.n_rows * s.n_x), ("obs_step", s.n_obs), ("obs_discount", s.n_obs),
        ("trigger", s.n_obs))}
    lf = arrays["log_fwd"].reshape(s.n_names, -1)
    lf[name, 1:] += np.log1p(h)
    return mc_request(
        model=0, dt=arrays["dt"], t0=arrays["t0"], spot=arrays["spot"], n_pairs=s.n_pairs, seed=s.seed,
        root=arrays["root"].reshape(s.n_names, -1), kind=np.ones(s.n_names, np.int32), cvar=np.zeros(s.n_names),
        log_fwd=lf, step_row=arrays["step_row"].reshape(s.n_names, -1), lo=arrays["row_lo"], inv_dx=arrays["row_inv_dx"],
        table=arrays["table"].reshape(s.n_rows, -1), n_x=s.n_x, product=1, obs_step=arrays["obs_step"],
        obs_discount=arrays["obs_discount"], trigger=arrays["trigger"], coupon_barrier=s.coupon_barrier,
        coupon=s.coupon, ki_barrier=s.ki_barrier, put_strike=s.put_strike, memory=s.memory, ki_daily=s.ki_daily,
    )


# The smoothed digitals are ramps of relative width 0.005: a bump must stay well inside one (h = 1e-6 relative) for
# the central difference to converge to the derivative; at 1e-4 its bias is ~2 %, measured. FP64 keeps such a
# difference accurate to ~1e-8 relative.
H = 1e-6


def test_deltas_match_central_differences_on_common_random_numbers():
    w = _wo()
    with AdjointPlan(w.held, EPS, "fp64") as plan:
        r = plan.run(grad=True)
    h = H
    for a in range(3):
        v = []
        for sgn in (1, -1):
            with AdjointPlan(_shifted(w, a, sgn * h), EPS, "fp64") as p:
                v.append(p.run(grad=False).price)
        fd = (v[0] - v[1]) / (np.log1p(h) - np.log1p(-h)) / w.spots[a]
        assert abs(r.delta[a] - fd) <= 1e-4 * abs(fd) + 1e-9, (a, r.delta[a], fd)


def test_node_vegas_match_central_differences_on_common_random_numbers(oracle):
    w = _wo()
    nodes = _nodes(w)
    g = autocall_greeks(w.held, nodes, EPS, "fp64")
    vega = g["vega"]
    base = _base(w)
    flat = np.argsort(-np.abs(vega).ravel())
    picks = list(flat[:4]) + list(flat[[len(flat) // 3, len(flat) // 2]])
    h = H
    scale = np.abs(vega).max()
    with AdjointPlan(w.held, EPS, "fp64") as plan:
        for f in picks:
            idx = np.unravel_index(f, vega.shape)
            v = []
            for sgn in (1, -1):
                b = torch.zeros(nodes.shape, dtype=torch.float64, device="cuda")
                b[idx] = sgn * h
                v.append(plan.run(nodes.table(base, b), grad=False).price)
            fd = (v[0] - v[1]) / (2 * h)
            assert abs(vega[idx] - fd) <= 1e-4 * abs(fd) + 1e-6 * scale, (idx, vega[idx], fd)
    # one node again against the CPU oracle's FP64 revaluation of the bumped table
    idx = np.unravel_index(flat[0], vega.shape)
    s = w.held.struct
    v = []
    for sgn in (1, -1):
        b = torch.zeros(nodes.shape, dtype=torch.float64, device="cuda")
        b[idx] = sgn * h
        tab = nodes.table(base, b).cpu().numpy()
        orig = np.ctypeslib.as_array(s.table, shape=(s.n_rows * s.n_x,))
        saved = orig.copy()
        orig[:] = tab.ravel()
        try:
            v.append(oracle.autocall_smooth(w.held, EPS)[0])
        finally:
            orig[:] = saved
    fd = (v[0] - v[1]) / (2 * h)
    assert abs(vega[idx] - fd) <= 1e-4 * abs(fd) + 1e-6 * scale, (vega[idx], fd)


def test_fp32_greeks_agree_with_fp64_within_4_standard_errors():
    w = _wo(n_paths=2**15)
    nodes = _nodes(w)
    g64 = autocall_greeks(w.held, nodes, EPS, "fp64")
    g32 = autocall_greeks(w.held, nodes, EPS, "fp32")
    assert abs(g32["price"] - g64["price"]) <= 4 * g64["price_se"]
    assert np.all(np.abs(g32["delta"] - g64["delta"]) <= 4 * g64["delta_se"])
    assert np.all(np.abs(g32["vega"] - g64["vega"]) <= 4 * g64["vega_se"] + 1e-9)
    # the float paths move the Greeks by far less than their noise: 1e-3 of the largest vega
    assert np.abs(g32["vega"] - g64["vega"]).max() <= 1e-3 * np.abs(g64["vega"]).max()


def test_autograd_vegas_are_the_contracted_table_gradient():
    w = _wo(n_paths=2**12)
    nodes = _nodes(w)
    with AdjointPlan(w.held, EPS, "fp64") as plan:
        g = autocall_greeks(w.held, nodes, EPS, plan=plan)
        direct = nodes.contract(plan.gradient, _base(w)).cpu().numpy()
    assert np.allclose(g["vega"], direct, rtol=1e-12, atol=1e-15)
    assert g["vega"].shape == (3, 10, 15)


@pytest.mark.parametrize("precision,rel", [("fp64", 1e-9), ("fp32", 2e-4)])
def test_stored_states_and_recomputed_segments_give_the_same_greeks(precision, rel):
    """checkpoint=1 stores every step and the backward recovers each step's noise from the stored states;
    checkpoint=4 recomputes 4-step segments from their checkpoints and redraws the normals: the same gradient."""
    w = _wo(n_paths=2**13)
    nodes = _nodes(w)
    with AdjointPlan(w.held, EPS, precision, checkpoint=1) as dense, \
            AdjointPlan(w.held, EPS, precision, checkpoint=4) as sparse:
        gd = autocall_greeks(w.held, nodes, EPS, plan=dense)
        gs = autocall_greeks(w.held, nodes, EPS, plan=sparse)
        bd, bs = dense.batch_pairs, sparse.batch_pairs
    assert gd["price"] == gs["price"] and np.array_equal(gd["delta"], gs["delta"])
    # the two backwards split the pairs into the 32 standard-error batches differently; neither loses a pair
    assert float(bd.sum()) == float(bs.sum()) == w.held.struct.n_pairs
    scale = np.abs(gs["vega"]).max()
    assert np.abs(gd["vega"] - gs["vega"]).max() <= rel * scale, np.abs(gd["vega"] - gs["vega"]).max() / scale

