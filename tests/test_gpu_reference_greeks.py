"""The adjoint's Greeks against the reference's own bump-and-revalue Greeks (tests/golden/reference_greeks.json: its
risk package's `compute` on a 3-name worst-of autocall under local vol, revalued on its compiled CPU engine).

This engine builds the same plan from the same model (this package's SSVI and plan(), which equal the reference's to
1e-14), with the same Philox key and pairs, so the adjoint runs on the very paths the reference revalued. Its delta per
name (dV/dS, sticky moneyness) is the reference's delta per 1 % of spot divided by 1 % of spot; its vegas on the
reference's implied-vol nodes are the table gradient contracted with the derivative of the per-step Dupire table in each
node's tent (optlab_b200.ivnodes), per vol point. The reference's Greeks are differences of revaluations: with small
bumps (1e-4) they converge to these derivatives, so the adjoint must match them within 4 of their standard errors and a
part in a thousand; with its default bumps (1 % of spot, one vol point, the node vegas one-sided) they carry their own
finite-difference bias: the deltas still agree, the node vegas in sign where the reference measures them clearly."""

import json
from pathlib import Path

import numpy as np
import pytest

from optlab_b200 import ivnodes, plan
from optlab_b200 import models as M
from optlab_b200._abi import OB_MODEL_PATHS, OB_PRODUCT_AUTOCALL
from optlab_b200.adjoint import AdjointPlan
from optlab_b200.requests import mc_request
from optlab_b200.surfaces import SSVI

pytestmark = pytest.mark.gpu

FIX = json.loads((Path(__file__).resolve().parent / "golden" / "reference_greeks.json").read_text())
NAMES = tuple(FIX["names"])


def _surfaces():
    T = 3.0 * np.arange(1, 41) / 40
    return [SSVI.power_law(FIX["rho"][a], 1.0, 0.5, T, FIX["c_rate"][a] * T) for a in range(len(NAMES))]


def _request(p, surfaces):
    """The worst-of autocall of the fixture as this engine's adjoint request, on plan p."""
    r, q, s0 = FIX["r"], FIX["q"], FIX["spot"]
    times = np.asarray(FIX["sim_times"])
    t_end = np.concatenate([[0.0], np.cumsum(p.dt)])
    obs_t = np.array([0.25, 0.5, 0.75, 1.0])
    obs_step = np.searchsorted(t_end, obs_t - 1e-12).astype(np.int32)
    assert np.allclose(t_end[obs_step], obs_t, atol=1e-12)
    assert np.allclose(t_end[p.obs_step], times, atol=1e-12)
    n = len(NAMES)
    return mc_request(
        model=OB_MODEL_PATHS, dt=p.dt, t0=p.t0, spot=np.full(n, s0), n_pairs=FIX["n_paths"] // 2, seed=FIX["key"],
        root=p.root, kind=np.ones(n, np.int32), cvar=np.zeros(n), same=p.same,
        log_fwd=np.tile((r - q) * t_end, (n, 1)), step_row=p.step_row, lo=p.lo, inv_dx=p.inv_dx, table=p.table,
        n_x=p.n_x, product=OB_PRODUCT_AUTOCALL, obs_step=obs_step, obs_discount=np.exp(-r * obs_t),
        trigger=np.array([1.0, 1.0, 1.0, 0.0]), coupon_barrier=0.7, coupon=0.02, ki_barrier=0.6, put_strike=1.0,
        memory=1, ki_daily=0,
    )


@pytest.fixture(scope="module")
def adjoint():
    surfaces = _surfaces()
    corr = np.full((3, 3), FIX["corr"]) + (1 - FIX["corr"]) * np.eye(3)
    market = M.Market.flat(FIX["spot"], FIX["r"], FIX["q"])
    basket = M.Basket(NAMES, {n: M.LocalVolModel(s) for n, s in zip(NAMES, surfaces)}, {n: market for n in NAMES},
                      corr)
    p = plan(basket, None, np.asarray(FIX["sim_times"]))
    held = _request(p, surfaces)
    with AdjointPlan(held, FIX["smoothing"], "fp64") as ap:
        res = ap.run(grad=True)
        grad = ap.gradient.cpu().numpy()
        batch = (ap.batch_grad / ap.batch_pairs.clamp(min=1.0)[:, None, None]).cpu().numpy()
        w = (ap.batch_pairs / ap.batch_pairs.sum()).cpu().numpy()
    S = p.step_row.shape[1]
    vega, vega_se = [], []
    for a, surf in enumerate(surfaces):
        rows = slice(a * S, (a + 1) * S)
        vega.append(ivnodes.node_jacobian_contract(grad[rows], surf, p.t0, p.n_x))
        per_batch = np.stack([ivnodes.node_jacobian_contract(b[rows], surf, p.t0, p.n_x) for b in batch])
        mean = np.tensordot(w, per_batch, axes=1)
        var = np.tensordot(w, (per_batch - mean) ** 2, axes=1) * len(w) / (len(w) - 1) / len(w)
        vega_se.append(np.sqrt(var))
    return {"price": res.price, "price_se": res.price_se, "delta": np.array(res.delta[:3]),
            "delta_se": np.array(res.delta_se[:3]), "vega": np.array(vega), "vega_se": np.array(vega_se)}


def _ref(label):
    g = FIX["greeks"][label]
    delta = np.array([g["delta"][n] for n in NAMES])  # (names, 2): value, se
    vega = np.array([g["vega_node"][n] for n in NAMES])  # (names, strikes, tenors, 2)
    return delta, vega


def test_deltas_match_the_references_small_bump_deltas(adjoint):
    delta, _ = _ref("small")
    mine = adjoint["delta"] * 0.01 * FIX["spot"]  # per 1 % of spot
    assert np.all(np.abs(mine - delta[:, 0]) <= 4 * delta[:, 1] + 1e-3 * np.abs(delta[:, 0])), (mine, delta)


def test_node_vegas_match_the_references_small_bump_vegas(adjoint):
    _, vega = _ref("small")
    ref, se = vega[..., 0], vega[..., 1]
    mine = adjoint["vega"]
    scale = np.abs(ref).max()
    assert scale > 0
    assert np.all(np.abs(mine - ref) <= 4 * se + 1e-3 * np.abs(ref) + 1e-9 * scale), \
        np.max(np.abs(mine - ref) / (se + 1e-300))
    # nodes the product cannot feel (tenors after its last date) have no vega in either
    assert np.all(np.abs(mine[:, :, 5:]) <= 1e-12 * scale) and np.all(np.abs(ref[:, :, 5:]) <= 1e-12 * scale)


def test_the_references_default_bumps_agree_where_they_measure_something(adjoint):
    """One vol point one-sided and 1 % of spot central: the reference's desk Greeks. A central 1 % spot move is close
    to the derivative (its error is third order), so the deltas agree within 4 SE and 5 %. A one-sided vol point is
    not: at short tenors it moves the paths across the smoothed autocall and coupon ramps (width 0.5 % of spot), so a
    node's one-sided difference and its derivative can part by much of the node's size. There the nodes that the
    reference measures clearly (4 SE and a tenth of the largest) must have the adjoint's sign, and the deviations are
    printed."""
    delta, vega = _ref("default")
    mine_d = adjoint["delta"] * 0.01 * FIX["spot"]
    assert np.all(np.abs(mine_d - delta[:, 0]) <= 4 * delta[:, 1] + 0.05 * np.abs(delta[:, 0]))
    ref, se = vega[..., 0], vega[..., 1]
    scale = np.abs(ref).max()
    clear = (np.abs(ref) > 4 * se) & (np.abs(ref) > 0.1 * scale)
    assert clear.sum() >= 5
    assert np.all(np.sign(adjoint["vega"][clear]) == np.sign(ref[clear]))
    dev = np.abs(adjoint["vega"] - ref)
    print(f"default-bump node vegas: max |adjoint - reference| = {dev.max() / scale:.3f} of the largest vega, "
          f"median over the clear nodes {np.median(dev[clear] / np.abs(ref[clear])):.3f} of the node")
