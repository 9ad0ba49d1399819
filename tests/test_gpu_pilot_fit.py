"""The issuer's Longstaff-Schwartz fit on the device (ob_script_pilot_fit, optlab_b200.exercise.pilot_fit) against
the same regression on the host (optlab_b200.exercise.fit, pinned to the reference's own fit on its recorded case by
tests/test_exercise.py). On the same pilot (the same draws: the device's record is the one the host reads) the rules'
normalisation, basis and hinges equal the host's, the coefficients agree to the regression's conditioning, the
decisions and the in-sample value agree, and the policy prices as the host's. Nearly collinear terms are left to the
host."""

import numpy as np
import pytest

from optlab_b200 import exercise
from optlab_b200 import script as sc
from test_gpu_dual import DUAL, _bs
from test_gpu_dual import _disc as _disc_bs
from test_gpu_script import CALLABLE, _disc, _simulation

pytestmark = pytest.mark.gpu


def _case(name):
    """(compiled script, make_sim(n_pairs, seed), discount) of the reference's recorded callable (two state
    variables, local vol) or of the dual bound's callable reverse convertible (one, Black-Scholes)."""
    if name == "callable":
        comp = sc.compile_script(CALLABLE)
        return comp, lambda n, seed: _simulation(comp, {"SPX": 100.0}, n_pairs=n, seed=seed)[0], _disc
    comp = sc.compile_script(DUAL["script"])
    return comp, lambda n, seed: _bs(comp, n, seed), _disc_bs


def _inputs(comp, disc):
    pay_d = [float(disc(t)) if t is not None and t > 0 else 0.0 for t in comp.pay_times]
    return [k for k, _ in comp.calls], pay_d


def _host_fit(comp, make_sim, disc, n_pairs, seed, precision):
    pilot = sc.script_request(comp, make_sim(n_pairs, seed), disc, call_mode=1)
    res = sc.run(pilot, precision)
    rec = exercise.PilotRecord.from_device(pilot.keep[1]["record"], len(comp.event_times), len(comp.calls),
                                           len(comp.calls[0][1]))
    events, pay_d = _inputs(comp, disc)
    return exercise.fit(rec, events, pay_d), rec, res


CASES = [("callable", "fp64"), ("callable", "fp32"), ("dual", "fp64")]


@pytest.mark.parametrize("name,precision", CASES, ids=[f"{n}-{p}" for n, p in CASES])
def test_the_device_fit_equals_the_host_fit_on_the_same_pilot(name, precision):
    comp, make_sim, disc = _case(name)
    n_pairs, seed = 10000, 4242
    host, rec, res_h = _host_fit(comp, make_sim, disc, n_pairs, seed, precision)
    events, pay_d = _inputs(comp, disc)
    fitted = exercise.pilot_fit(sc.script_request(comp, make_sim(n_pairs, seed), disc, call_mode=1), events, pay_d,
                                precision)
    assert fitted is not None
    dev, res_d = fitted
    assert res_d.price == res_h.price and res_d.se == res_h.se  # the same pilot
    assert dev.pilot_paths == host.pilot_paths == 2 * n_pairs
    worst = 0.0
    for c, (rd, rh) in enumerate(zip(dev.rules, host.rules)):
        assert (rd is None) == (rh is None), c
        if rd is None:
            continue
        assert rd.powers == rh.powers, c
        assert [v for v, _ in rd.knots] == [v for v, _ in rh.knots], c
        assert np.allclose([k for _, k in rd.knots], [k for _, k in rh.knots], rtol=1e-12, atol=1e-14), c
        assert np.allclose(rd.mean, rh.mean, rtol=1e-12, atol=1e-15) and np.allclose(rd.scale, rh.scale, rtol=1e-12)
        cd, ch = np.array(rd.coef), np.array(rh.coef)
        gap = np.abs(cd - ch).max() / np.abs(ch).max()
        worst = max(worst, gap)
        assert gap < 1e-8, (c, gap)
    print(f"\n{name} {precision}: largest coefficient gap to the host's least squares {worst:.2e} of the largest")
    assert abs(dev.in_sample - host.in_sample) <= 1e-9 * abs(host.in_sample)
    flips = np.mean(exercise.decisions(dev, rec) != exercise.decisions(host, rec))
    assert flips <= 1e-4, flips


def test_a_callable_prices_the_same_with_the_device_fit():
    """exercise.price (pilot and fit on the device) against a pricing run applying the host-fitted policy of the
    same pilot: the FP64 prices agree to 1e-9 (a decision whose continuation sits on the amount may flip)."""
    comp, make_sim, disc = _case("callable")
    n_pairs, seed = 2**14, 77
    res, policy = exercise.price(comp, make_sim, n_pairs, seed, disc, "fp64")
    host, _, _ = _host_fit(comp, make_sim, disc, exercise.pilot_paths(2 * n_pairs) // 2, seed ^ exercise.PILOT_KEY,
                           "fp64")
    n_state = len(comp.calls[0][1])
    held = sc.script_request(comp, make_sim(n_pairs, seed), disc, call_mode=2, rules=host.pack(n_state))
    want = sc.run(held, "fp64")
    assert abs(res.price - want.price) <= 1e-9 * abs(want.price), (res.price, want.price)
    assert all(r is not None for r in policy.rules)


def test_collinear_terms_are_left_to_the_host():
    """A call state of two equal variables makes the regression's terms collinear (the same normalised state twice):
    the device refuses the fit (OB_ESINGULAR) and exercise.price fits that pilot on the host, the reference's way."""
    text = CALLABLE.replace("  low = lowest(SPX, t=0, t=0.25, n=12) / S0\n", "  low = SPX / S0\n").replace(
        "  low = min(low, lowest(SPX, t=0.25, t=0.5, n=12) / S0)\n", "  low = SPX / S0\n")
    assert text != CALLABLE
    comp = sc.compile_script(text)
    make_sim = lambda n, seed: _simulation(comp, {"SPX": 100.0}, n_pairs=n, seed=seed)[0]  # noqa: E731
    events, pay_d = _inputs(comp, _disc)
    pilot = sc.script_request(comp, make_sim(10000, 5), _disc, call_mode=1)
    assert exercise.pilot_fit(pilot, events, pay_d, "fp64") is None
    res, policy = exercise.price(comp, make_sim, 2**12, 5, _disc, "fp64")
    assert np.isfinite(res.price) and all(r is not None for r in policy.rules)
