"""The issuer's dual bound on the GPU: branched continuations follow their outer path exactly up to the branch and
draw their own after it, and the device's Andersen-Broadie bound of a callable reverse convertible under
Black-Scholes brackets the reference's PDE value as the reference's own test asks (the bound below the PDE within 4 SE,
the gap to the policy's price under 10 bp), beside the reference's own bound at the same sizes."""

import json
from pathlib import Path

import numpy as np
import pytest

from optlab_b200 import exercise
from optlab_b200 import script as sc
from optlab_b200._abi import OB_MODEL_PATHS, OB_PRODUCT_LADDER
from optlab_b200.models import time_grid
from optlab_b200.requests import mc_request

pytestmark = pytest.mark.gpu

DUAL = json.loads((Path(__file__).resolve().parent / "golden" / "script_dual.json").read_text())
R, Q, VOL = DUAL["r"], DUAL["q"], DUAL["vol"]


def _disc(t):
    return float(np.exp(-R * t))


def _bs(comp, n_pairs, seed, dt_max=1 / 12):
    """Black-Scholes as a flat local-variance table (vol^2 at every node: the interpolation is exact, and so is the
    log-Euler step), forward drift r - q."""
    grid = time_grid(comp.timeline.sim_times, dt_max)
    dt, t0 = np.diff(grid), grid[:-1]
    n_x = 11
    return mc_request(model=OB_MODEL_PATHS, dt=dt, t0=t0, spot=[100.0], n_pairs=n_pairs, seed=seed, root=[[1.0]],
                      kind=np.ones(1, np.int32), cvar=[VOL**2], log_fwd=(R - Q) * grid[None, :],
                      step_row=np.zeros((1, len(dt)), np.int32), lo=[-5.0], inv_dx=[(n_x - 1) / 10.0],
                      table=np.full((1, n_x), VOL**2), n_x=n_x, r=R, q=Q, product=OB_PRODUCT_LADDER, leg_type=[1],
                      leg_strike=[1.0])


@pytest.fixture(scope="module")
def comp():
    return sc.compile_script(DUAL["script"])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_continuations_follow_their_outer_path_up_to_the_branch(comp, precision):
    """Recorded runs: every event up to the branch step has, on both legs of every continuation, the flows of the
    outer path it continues (bit for bit: the same normals through the same arithmetic); later events part."""
    P, per = 8, 3
    outer_seed = 12345
    outer = sc.script_request(comp, _bs(comp, P, outer_seed), _disc, call_mode=1)
    sc.run(outer, precision)
    ev_step = outer.keep[1]["event_step"]
    n_ev = len(ev_step)
    k = 1  # branch at the second event
    inner = sc.script_request(comp, _bs(comp, 2 * P * per, 777), _disc, call_mode=1,
                              branch=(int(ev_step[k]), P, per, outer_seed))
    sc.run(inner, precision)
    ro, ri = outer.keep[1]["record"], inner.keep[1]["record"]
    n_in = 2 * P * per
    for p in range(n_in):
        o = p // per
        for leg in (p, n_in + p):
            assert np.array_equal(ri[leg, : 2 * (k + 1)], ro[o, : 2 * (k + 1)]), (p, leg)
    later = ri[:, 2 * (k + 1): 2 * n_ev]
    assert not np.array_equal(later[:n_in], later[n_in:])  # the legs part after the branch


def test_a_branch_at_the_start_is_an_ordinary_run(comp):
    P, per = 4, 4
    plain = sc.script_request(comp, _bs(comp, 2 * P * per, 99), _disc, pair_values=True)
    branched = sc.script_request(comp, _bs(comp, 2 * P * per, 99), _disc, branch=(0, P, per, 5))
    a, b = sc.run(plain, "fp64"), sc.run(branched, "fp64")
    assert a.price == b.price
    assert np.array_equal(plain.keep[1]["pair_value"], branched.keep[1]["pair_value"])


def test_a_branched_run_refuses_what_it_cannot_continue(comp):
    from optlab_b200._abi import EngineError

    sim = _bs(comp, 10, 1)
    with pytest.raises(EngineError, match="branch_pairs pairs for each"):
        sc.run(sc.script_request(comp, sim, _disc, branch=(3, 2, 3, 5)), "fp64")


def test_the_dual_bound_and_the_policy_bracket_the_pde(comp):
    """The reference's test_issuer_call criteria on the device: a policy from a device pilot, its price within 4 SE
    (plus the 10 bp policy bias allowance) of the PDE, the dual bound from 1000 outer paths x 200 continuations below
    the PDE within 4 SE, and a gap between -4 SE and 10 bp; the gap agrees with the reference's bound at the same
    sizes within 4 SE of their difference."""
    pde = DUAL["pde"]
    res, policy = exercise.price(comp, lambda n, seed: _bs(comp, n, seed), 2**17, 11, _disc, "fp64")
    assert pde - 4 * res.se < res.price < pde + 4 * res.se + 0.001
    bound = exercise.dual_bound(comp, lambda n, seed: _bs(comp, n, seed), policy, res.price, res.se, 11, _disc,
                                n_outer=1000, n_inner=200, precision="fp64")
    assert bound["outer"] == 1000 and bound["inner"] == 200
    assert bound["lower"] < pde + 4 * bound["lower_se"]
    assert -4 * bound["gap_se"] < bound["gap"] < 0.001
    ref = DUAL["big"]
    assert abs(bound["gap"] - ref["gap"]) < 4 * np.hypot(bound["gap_se"], ref["gap_se"]) + 2e-4


def test_fp32_dual_bound_agrees_with_fp64(comp):
    res, policy = exercise.price(comp, lambda n, seed: _bs(comp, n, seed), 2**15, 3, _disc, "fp64")
    b64 = exercise.dual_bound(comp, lambda n, seed: _bs(comp, n, seed), policy, res.price, res.se, 3, _disc,
                              n_outer=400, n_inner=100, precision="fp64")
    b32 = exercise.dual_bound(comp, lambda n, seed: _bs(comp, n, seed), policy, res.price, res.se, 3, _disc,
                              n_outer=400, n_inner=100, precision="fp32")
    assert abs(b32["gap"] - b64["gap"]) < 4 * b64["gap_se"] + 1e-5
