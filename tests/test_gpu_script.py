"""Payoff scripts on the GPU: the device's simulation + interpreter against the oracle's paths (C restatement of the
path engine) evaluated by the NumPy oracle evaluator, in FP64 within 1e-10 relative and FP32 within 4 SE; a Phoenix
written as a script against the fused Phoenix kernel on the same random numbers (local vol and Heston QE); undefined
scripts reported as the reference reports them."""

import json
from pathlib import Path

import numpy as np
import pytest

from optlab_b200 import engine, workloads
from optlab_b200 import script as sc
from optlab_b200._abi import OB_MODEL_HESTON_QE, OB_MODEL_PATHS, OB_PRODUCT_LADDER
from optlab_b200.models import correlation_root, time_grid
from optlab_b200.requests import mc_request, paths_request

pytestmark = pytest.mark.gpu

CASES = {c["name"]: c for c in json.loads((Path(__file__).resolve().parent / "golden" / "script_cases.json")
                                         .read_text())["cases"]}
R = 0.02


def _disc(t):
    return np.exp(-R * t)


def _simulation(comp, spot0, n_pairs=2**11, seed=17, local_vol=True, dt_max=1 / 48):
    """Local vol (one surface a name, the benchmark's SSVI family) or constant vol (0.2^2), correlation 0.5, flat
    r = 2 %; the grid holds every observation time."""
    grid = time_grid(comp.timeline.sim_times, dt_max)
    dt, t0 = np.diff(grid), grid[:-1]
    n = len(comp.names)
    spot = np.array([spot0[k] for k in comp.names])
    lf = np.tile(R * grid, (n, 1))
    root = correlation_root(np.full((n, n), 0.5) + 0.5 * np.eye(n))
    kw = dict(model=OB_MODEL_PATHS, dt=dt, t0=t0, spot=spot, n_pairs=n_pairs, seed=seed, root=root,
              cvar=np.full(n, 0.04), log_fwd=lf, r=R, product=OB_PRODUCT_LADDER, leg_type=[1], leg_strike=[1.0])
    if local_vol:
        horizon = float(grid[-1])
        grids = [workloads.lv_grid(workloads.lv_surface(rho=-0.5 - 0.05 * a, theta_rate=0.04 + 0.005 * a,
                                                         horizon=horizon, n_exp=10), horizon=horizon, n_exp=10,
                                   n_x=101) for a in range(n)]
        kw.update(kind=np.ones(n, np.int32), step_row=np.stack([g.row_of(t0) + 10 * a for a, g in enumerate(grids)]),
                  lo=np.concatenate([g.lo for g in grids]), inv_dx=np.concatenate([g.inv_dx for g in grids]),
                  table=np.vstack([g.rows for g in grids]), n_x=101)
    else:
        kw.update(kind=np.zeros(n, np.int32))
    return mc_request(**kw), grid


def _oracle_price(case, comp, sim, grid, oracle):
    """The oracle's paths at every observation step, the oracle evaluator on them, mean of the pair averages."""
    from script_oracle import ScriptOracle

    s = sim.struct
    arrays = {k: np.ctypeslib.as_array(getattr(s, k), shape=(m,)).copy() for k, m in (
        ("dt", s.n_steps), ("t0", s.n_steps), ("root", s.n_names**2), ("kind", s.n_names), ("cvar", s.n_names),
        ("heston", 5 * s.n_names), ("log_fwd", s.n_names * (s.n_steps + 1)), ("spot", s.n_names))}
    steps = np.searchsorted(grid, comp.timeline.sim_times - 1e-12)
    lf = arrays["log_fwd"].reshape(s.n_names, -1)
    fwd = arrays["spot"][:, None] * np.exp(lf[:, steps])
    kw = dict(dt=arrays["dt"], t0=arrays["t0"], obs_step=steps, root=arrays["root"].reshape(s.n_names, -1),
              kind=arrays["kind"], cvar=arrays["cvar"], heston=arrays["heston"], same=1, fwd=fwd, n_pairs=s.n_pairs,
              seed=s.seed)
    if s.n_rows:
        kw.update(step_row=np.ctypeslib.as_array(s.step_row, shape=(s.n_names * s.n_steps,)).copy(),
                  lo=np.ctypeslib.as_array(s.row_lo, shape=(s.n_rows,)).copy(),
                  inv_dx=np.ctypeslib.as_array(s.row_inv_dx, shape=(s.n_rows,)).copy(),
                  table=np.ctypeslib.as_array(s.table, shape=(s.n_rows * s.n_x,)).copy(), n_x=s.n_x)
    held = paths_request(**kw)
    oracle.paths(held)
    out = np.ctypeslib.as_array(held.struct.out, shape=(s.n_names, len(steps), 2 * s.n_pairs))
    times = comp.timeline.sim_times
    spot0 = dict(zip(comp.names, arrays["spot"]))

    def col(name, t):
        if t <= 0:
            return np.full(2 * s.n_pairs, spot0[name])
        k = int(np.argmin(np.abs(times - t)))
        assert abs(times[k] - t) < 1e-9
        return out[comp.names.index(name), k]

    o = ScriptOracle(case["script"], case["params"], case["smoothing"], case["valuation"], _disc)
    res = o.run(2 * s.n_pairs, col, lambda name, ts: np.stack([col(name, t) for t in ts], axis=1))
    y = 0.5 * (res["pv"][: s.n_pairs] + res["pv"][s.n_pairs:])
    return y.mean(), y.std(ddof=1) / np.sqrt(len(y)), res


CHECKED = ["phoenix", "phoenix_smooth", "worst_of", "worst_of_smooth", "variance", "cliquet", "dated"]


@pytest.mark.parametrize("name", CHECKED)
@pytest.mark.parametrize("local_vol", [True, False])
def test_fp64_scripts_match_the_oracle(name, local_vol, oracle):
    case = CASES[name]
    comp = sc.compile_script(case["script"], case["params"], case["smoothing"], case["valuation"])
    sim, grid = _simulation(comp, case["spot0"], local_vol=local_vol)
    res = sc.run(sc.script_request(comp, sim, _disc), "fp64")
    want, se, _ = _oracle_price(case, comp, sim, grid, oracle)
    assert abs(res.price - want) <= 1e-10 * max(abs(want), 1e-3), (res.price, want)
    assert abs(res.se - se) <= 1e-6 * se + 1e-15
    assert res.n_paths == 2 * sim.struct.n_pairs


@pytest.mark.parametrize("name", ["phoenix", "worst_of_smooth", "variance", "cliquet"])
def test_fp32_scripts_are_within_4_standard_errors_of_fp64(name):
    case = CASES[name]
    comp = sc.compile_script(case["script"], case["params"], case["smoothing"], case["valuation"])
    sim, _ = _simulation(comp, case["spot0"], n_pairs=2**13)
    r64 = sc.run(sc.script_request(comp, sim, _disc), "fp64")
    r32 = sc.run(sc.script_request(comp, sim, _disc), "fp32")
    assert abs(r32.price - r64.price) <= 4 * r64.se + 1e-7, (r32.price, r64.price, r64.se)


def _phoenix_script(ph: workloads.Phoenix, steps_per_year: int) -> str:
    """The Phoenix of the fused kernel written in the payoff language (coupon with memory, call before the last date,
    daily knock-in from the strike date into a put at the last)."""
    n_obs = int(round(ph.years * ph.obs_per_year))
    lines = ["underlying X", "param S0 = 1", f"param cb = {ph.coupon_barrier!r}", f"param cpn = {ph.coupon!r}",
             f"param call = {ph.trigger!r}", f"param ki = {ph.ki_barrier!r}", f"param K = {ph.put_strike!r}"]
    for j in range(1, n_obs + 1):
        t = j / ph.obs_per_year
        lines.append(f"event t={t!r} pay t={t!r}")
        if j == 1:
            lines.append("  missed = 0")
        lines += ["  perf = X / S0", "  if perf >= cb then", "    pay cpn * (1 + missed) as coupon", "    missed = 0",
                  "  else", "    missed = missed + 1", "  end"]
        if j < n_obs:
            lines += ["  if perf >= call then", "    pay 1 as redemption", "    terminate", "  end"]
        else:
            n_fix = int(round(ph.years * steps_per_year))
            lines += [f"  knocked = lowest(X, t=0, t={t!r}, n={n_fix}) < ki * S0", "  if knocked then",
                      "    pay 1 - max(K - perf, 0) as redemption", "  else", "    pay 1 as redemption", "  end"]
        lines.append("end")
    return "\n".join(lines) + "\n"


def test_a_phoenix_script_equals_the_fused_phoenix_kernel():
    """Local vol, 2^14 paths x 756 daily steps: the script on the device and the fused kernel read the same normals;
    their FP64 prices agree to rounding."""
    ph = workloads.Phoenix()
    held = workloads.lv_phoenix(n_paths=2**14, phoenix=ph)
    text = _phoenix_script(ph, 252)
    s = held.struct
    grid = np.concatenate([[0.0], np.ctypeslib.as_array(s.t0, shape=(s.n_steps,))
                           + np.ctypeslib.as_array(s.dt, shape=(s.n_steps,))])
    # the fused request's spot is 100 with strikes as fractions: the script reads S / S0 with S0 = 100
    comp = sc.compile_script(text, params={"S0": float(s.spot[0])})
    fused = engine.mc_price(held, "fp64")
    res = sc.run(sc.script_request(comp, held, lambda t: np.exp(-0.02 * t)), "fp64")
    assert abs(res.price - fused.price[0]) <= 1e-10 * abs(fused.price[0]), (res.price, fused.price[0])
    assert abs(res.se - fused.se[0]) <= 1e-8 * fused.se[0]
    assert len(grid) == s.n_steps + 1


def _dated_phoenix_script(times, n_fix: int) -> str:
    """The Phoenix of the fused kernel's defaults with its observations at the given times."""
    ph = workloads.Phoenix()
    lines = ["underlying X", "param S0 = 1", f"param cb = {ph.coupon_barrier!r}", f"param cpn = {ph.coupon!r}",
             f"param call = {ph.trigger!r}", f"param ki = {ph.ki_barrier!r}", f"param K = {ph.put_strike!r}"]
    for j, t in enumerate(times):
        lines.append(f"event t={t!r} pay t={t!r}")
        if j == 0:
            lines.append("  missed = 0")
        lines += ["  perf = X / S0", "  if perf >= cb then", "    pay cpn * (1 + missed) as coupon", "    missed = 0",
                  "  else", "    missed = missed + 1", "  end"]
        if j < len(times) - 1:
            lines += ["  if perf >= call then", "    pay 1 as redemption", "    terminate", "  end"]
        else:
            lines += [f"  knocked = lowest(X, t=0, t={t!r}, n={n_fix}) < ki * S0", "  if knocked then",
                      "    pay 1 - max(K - perf, 0) as redemption", "  else", "    pay 1 as redemption", "  end"]
        lines.append("end")
    return "\n".join(lines) + "\n"


def test_events_on_the_edges_of_step_batches_price_as_the_fused_kernel():
    """Observation dates at the first step, either side of an eight-step batch's edge, on consecutive steps and at the
    last step: the script kernel runs a batch without an event without testing its steps for one, and so does the
    fused kernel for observations; on the same request and normals their FP64 prices agree to rounding."""
    n_steps, years = 126, 0.5
    ph = workloads.Phoenix(years=years, obs_per_year=8)
    m = workloads.FlatMarket(100.0, 0.02, 0.01)
    g = workloads.lv_grid(horizon=years, n_exp=8, n_x=120)
    dt, t0 = workloads.uniform_grid(years, n_steps)
    t_end = np.concatenate([[0.0], t0 + dt])
    steps = np.array([1, 8, 9, 16, 17, 40, 41, 42, 64, 100, 125, 126], dtype=np.int32)
    fields = workloads.autocall_fields(ph, m, int(round(n_steps / years)))
    trig = np.full(len(steps), ph.trigger)
    trig[-1] = 0.0
    fields.update(obs_step=steps, obs_discount=m.D(t_end[steps]), trigger=trig)
    held = mc_request(model=OB_MODEL_PATHS, dt=dt, t0=t0, spot=[100.0], n_pairs=2**13, seed=29, root=[[1.0]],
                      kind=[1], cvar=[0.04], heston=[[0.04, 1.5, 0.04, 0.5, -0.7]], log_fwd=m.log_fwd(t_end)[None, :],
                      step_row=g.row_of(t0)[None, :], lo=g.lo, inv_dx=g.inv_dx, table=g.rows, n_x=g.n_x, **fields)
    comp = sc.compile_script(_dated_phoenix_script([float(t) for t in t_end[steps]], n_steps), params={"S0": 100.0})
    fused = engine.mc_price(held, "fp64")
    res = sc.run(sc.script_request(comp, held, lambda t: np.exp(-0.02 * t)), "fp64")
    assert abs(res.price - fused.price[0]) <= 1e-10 * abs(fused.price[0]), (res.price, fused.price[0])


def test_a_heston_qe_phoenix_script_equals_the_fused_qe_kernel():
    ph = workloads.Phoenix(years=1.0, obs_per_year=4)
    base = workloads.heston_qe_ladder(n_paths=2**13, n_steps=252)
    s = base.struct
    dt = np.full(252, 1 / 252)
    fields = workloads.autocall_fields(ph, workloads.FlatMarket(100.0, 0.02, 0.01), 252)
    held = mc_request(model=OB_MODEL_HESTON_QE, dt=dt, t0=np.arange(252) / 252, spot=[100.0], n_pairs=s.n_pairs,
                      seed=s.seed, heston=workloads.HESTON_CFG0, r=0.02, q=0.01, **fields)
    comp = sc.compile_script(_phoenix_script(ph, 252), params={"S0": 100.0})
    fused = engine.mc_price(held, "fp64")
    res = sc.run(sc.script_request(comp, held, lambda t: np.exp(-0.02 * t)), "fp64")
    assert abs(res.price - fused.price[0]) <= 1e-10 * abs(fused.price[0]), (res.price, fused.price[0])


def test_an_undefined_payment_is_reported_as_the_reference_reports_it():
    case = CASES["undefined"]
    comp = sc.compile_script(case["script"])
    sim, _ = _simulation(comp, case["spot0"], local_vol=False)
    with pytest.raises(sc.ScriptError, match="not finite"):
        sc.run(sc.script_request(comp, sim, _disc), "fp64")


CALLABLE = json.loads((Path(__file__).resolve().parent / "golden" / "script_callable.json").read_text())["script"]


def _oracle_run(text, comp, sim, grid, oracle, **kw):
    """The oracle evaluator on the C oracle's paths of `sim` (as _oracle_price), any mode."""
    case = {"script": text, "params": {}, "smoothing": 0.0, "valuation": None}
    _, _, res = _oracle_price_mode(case, comp, sim, grid, oracle, **kw)
    return res


def _oracle_price_mode(case, comp, sim, grid, oracle, **kw):
    from script_oracle import ScriptOracle

    s = sim.struct
    arrays = {k: np.ctypeslib.as_array(getattr(s, k), shape=(m,)).copy() for k, m in (
        ("dt", s.n_steps), ("t0", s.n_steps), ("root", s.n_names**2), ("kind", s.n_names), ("cvar", s.n_names),
        ("heston", 5 * s.n_names), ("log_fwd", s.n_names * (s.n_steps + 1)), ("spot", s.n_names))}
    steps = np.searchsorted(grid, comp.timeline.sim_times - 1e-12)
    fwd = arrays["spot"][:, None] * np.exp(arrays["log_fwd"].reshape(s.n_names, -1)[:, steps])
    kw_p = dict(dt=arrays["dt"], t0=arrays["t0"], obs_step=steps, root=arrays["root"].reshape(s.n_names, -1),
                kind=arrays["kind"], cvar=arrays["cvar"], heston=arrays["heston"], same=1, fwd=fwd,
                n_pairs=s.n_pairs, seed=s.seed)
    if s.n_rows:
        kw_p.update(step_row=np.ctypeslib.as_array(s.step_row, shape=(s.n_names * s.n_steps,)).copy(),
                    lo=np.ctypeslib.as_array(s.row_lo, shape=(s.n_rows,)).copy(),
                    inv_dx=np.ctypeslib.as_array(s.row_inv_dx, shape=(s.n_rows,)).copy(),
                    table=np.ctypeslib.as_array(s.table, shape=(s.n_rows * s.n_x,)).copy(), n_x=s.n_x)
    held = paths_request(**kw_p)
    oracle.paths(held)
    out = np.ctypeslib.as_array(held.struct.out, shape=(s.n_names, len(steps), 2 * s.n_pairs))
    times = comp.timeline.sim_times
    spot0 = dict(zip(comp.names, arrays["spot"]))

    def col(name, t):
        if t <= 0:
            return np.full(2 * s.n_pairs, spot0[name])
        return out[comp.names.index(name), int(np.argmin(np.abs(times - t)))]

    o = ScriptOracle(case["script"], case["params"], case["smoothing"], case["valuation"], _disc)
    res = o.run(2 * s.n_pairs, col, lambda name, ts: np.stack([col(name, t) for t in ts], axis=1), **kw)
    y = 0.5 * (res["pv"][: s.n_pairs] + res["pv"][s.n_pairs:])
    return y.mean(), y.std(ddof=1) / np.sqrt(len(y)), res


def _callable_sim(comp, n_pairs, seed):
    return _simulation(comp, {"SPX": 100.0}, n_pairs=n_pairs, seed=seed)


def test_the_device_pilot_record_is_the_oracles(oracle):
    from optlab_b200 import exercise

    comp = sc.compile_script(CALLABLE)
    sim, grid = _callable_sim(comp, 2**11, 29)
    held = sc.script_request(comp, sim, _disc, call_mode=1)
    sc.run(held, "fp64")
    rec = exercise.PilotRecord.from_device(held.keep[1]["record"], len(comp.event_times), len(comp.calls), 2)
    want = _oracle_run(CALLABLE, comp, sim, grid, oracle, mode="record")
    for k in ("pre", "post", "mask", "alive", "amount", "state"):
        assert np.allclose(getattr(rec, k), want[k], rtol=1e-10, atol=1e-13), k


def test_an_issuer_call_policy_prices_as_the_oracle_applies_it(oracle):
    """The policy fitted on the device's pilot, applied by the device on other pairs and by the oracle evaluator on
    the oracle's paths of those pairs: FP64 prices within 1e-9 (a decision on the boundary may flip in the last
    bits of the continuation)."""
    from optlab_b200 import exercise

    comp = sc.compile_script(CALLABLE)
    sim, grid = _callable_sim(comp, 2**12, 31)
    result, policy = exercise.price(comp, lambda n, seed: _callable_sim(comp, n, seed)[0], 2**12, 31, _disc, "fp64")
    assert all(r is not None for r in policy.rules) and policy.pilot_paths == 20000
    want, se, res = _oracle_price_mode({"script": CALLABLE, "params": {}, "smoothing": 0.0, "valuation": None}, comp,
                                       sim, grid, oracle, mode="apply", rules=policy.rules)
    assert abs(result.price - want) <= 1e-9 * abs(want), (result.price, want)
    never = sc.run(sc.script_request(comp, sim, _disc), "fp64")
    assert result.price < never.price  # the issuer's option is worth something to the issuer
    assert result.bad_redemption == 0
