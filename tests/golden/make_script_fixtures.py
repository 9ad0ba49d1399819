"""Writes tests/golden/script_cases.json: payoff scripts of this repository's tests, evaluated by the reference's own
script pipeline (optlab.structured.script: parse, validate, build_timeline, Evaluator) on seeded synthetic fixings,
with each path's present value (cashflows.py:30-41, flat discount exp(-r t)); and tests/golden/script_callable.json:
a callable note's pilot record, the policy the reference fits on it (optlab.structured.exercise.fit) and that policy
applied to other paths; and tests/golden/script_dual.json: the reference's dual bound of a callable reverse convertible
under Black-Scholes (optlab.structured.exercise.dual_bound) on 40 outer paths with 16 continuations each, with the
outer paths and continuations it drew, the policy it used and its result, plus the reference's PDE value of the note
(tests/helpers/_callable_refs.py: callable_note) and the reference's bound at 1000 x 200.

The fixings are lognormal paths of every underlying on the script's simulation times (the valuation date is the
spot); the fake scenario answers `spot(name, t)` and `fixings(name, times)` from them. A case whose evaluation the
reference refuses (an undefined payment or condition) records the refusal instead of values.

Run where the reference tree is present:  python tests/golden/make_script_fixtures.py [reference root; default $OPTLAB_REFERENCE, else /root/reference]
"""

from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
R = 0.02

PHOENIX = """
underlying SPX
param N = 1
param cpn = 0.02
param coupon_barrier = 0.7
param call = 1
param ki = 0.6
param S0 = 100
event t=0.25 pay t=0.25
  missed = 0
  perf = SPX / S0
  if perf >= coupon_barrier then
    pay N * cpn as coupon
  else
    missed = missed + 1
  end
  if perf >= call then
    pay N as redemption
    terminate
  end
end
event t=0.5 pay t=0.5
  perf = SPX / S0
  if perf >= coupon_barrier then
    pay N * cpn * (1 + missed) as coupon
    missed = 0
  else
    missed = missed + 1
  end
  if perf >= call then
    pay N as redemption
    terminate
  end
end
event t=0.75 pay t=0.75
  perf = SPX / S0
  if perf >= coupon_barrier then
    pay N * cpn * (1 + missed) as coupon
    missed = 0
  else
    missed = missed + 1
  end
  if perf >= call then
    pay N as redemption
    terminate
  end
end
event t=1 pay t=1
  perf = SPX / S0
  if perf >= coupon_barrier then
    pay N * cpn * (1 + missed) as coupon
  end
  knocked = lowest(SPX, t=0, t=1, n=48) < ki * S0
  if knocked then
    pay N - N * max(1 - perf, 0) as redemption
  else
    pay N as redemption
  end
end
"""

WORST_OF = """
underlying A
underlying B
underlying C
param A0 = 100
param B0 = 50
param C0 = 20
param strike = 0.95
param digital = 0.04
event t=0.5 pay t=0.52
  w = worst(A / A0, B / B0, C / C0)
  b = best(A / A0, B / B0, C / C0)
  if w >= 1 and not (b > 1.3) then
    pay digital as coupon
  end
end
event t=1 pay t=1.02
  w = worst(A / A0, B / B0, C / C0)
  if w < strike or w == 0.5 then
    pay 1 - max(strike - w, 0) / strike as redemption
  else
    pay 1 as redemption
  end
  pay 0.5 * max(w - 1, 0) as upside
end
"""

VARIANCE = """
underlying SPX
param kvar = 0.04
param lo = 80
param hi = 130
event t=1 pay t=1
  v = variance(SPX, t=0, t=1, n=48)
  vc = variance(SPX, t=0.5, t=1, n=24, lo, hi)
  pay 100 * (v - kvar) / 0.4 as upside
  pay abs(vc - kvar) + sqrt(v) - exp(-v) + log(1 + v) as coupon
  pay 1 as redemption
end
"""

CLIQUET = """
underlying SPX
param cap = 0.05
param floor = -0.03
event t=0.25
  last = SPX
  total = 0
end
event t=0.5
  r = SPX / last - 1
  total = total + min(max(r, floor), cap)
  last = SPX
end
event t=0.75
  r = SPX / last - 1
  total = total + min(max(r, floor), cap)
  last = SPX
end
event t=1 pay t=1.05
  r = SPX / last - 1
  total = total + min(max(r, floor), cap)
  hit = highest(SPX, t=0.5, t=1, n=24) >= 115
  if hit then
    pay max(total, 0) as upside
  else
    pay 0.5 * max(total, 0) - (-0.01) as upside
  end
  pay 1 as redemption
end
"""

DATED = """
underlying SX5E
param S0 = 4000
param barrier = 0.75
event 2025-03-21 pay 2025-03-28
  perf = SX5E / S0
  if perf >= 1 then
    pay 1.03 as redemption
    terminate
  end
end
event 2025-06-20 pay 2025-06-27
  perf = SX5E / S0
  low = lowest(SX5E, 2025-01-02, 2025-06-20) / S0
  if low < barrier then
    pay perf as redemption
  else
    pay max(perf, 1) as redemption
  end
end
"""

UNDEFINED = """
underlying SPX
event t=1 pay t=1
  x = log(SPX / 100 - 0.9)
  pay x as upside
  pay 1 as redemption
end
"""

CALLABLE = """
underlying SPX
param S0 = 100
param cpn = 0.015
state perf, low
event t=0.25 pay t=0.25
  perf = SPX / S0
  low = lowest(SPX, t=0, t=0.25, n=12) / S0
  pay cpn as coupon
  call pay 1
end
event t=0.5 pay t=0.5
  perf = SPX / S0
  low = min(low, lowest(SPX, t=0.25, t=0.5, n=12) / S0)
  pay cpn as coupon
  call pay 1
end
event t=0.75 pay t=0.75
  perf = SPX / S0
  pay cpn as coupon
  call pay 1 + cpn
end
event t=1 pay t=1
  perf = SPX / S0
  pay cpn as coupon
  if perf < 0.7 then
    pay perf as redemption
  else
    pay 1 as redemption
  end
end
"""

CASES = [
    ("phoenix", PHOENIX, {}, 0.0, None, {"SPX": 100.0}),
    ("phoenix_smooth", PHOENIX, {"cpn": 0.025}, 0.01, None, {"SPX": 100.0}),
    ("worst_of", WORST_OF, {}, 0.0, None, {"A": 100.0, "B": 50.0, "C": 20.0}),
    ("worst_of_smooth", WORST_OF, {"strike": 0.9}, 0.02, None, {"A": 100.0, "B": 50.0, "C": 20.0}),
    ("variance", VARIANCE, {}, 0.0, None, {"SPX": 100.0}),
    ("cliquet", CLIQUET, {}, 0.0, None, {"SPX": 100.0}),
    ("dated", DATED, {}, 0.0, "2025-01-02", {"SX5E": 4000.0}),
    ("undefined", UNDEFINED, {}, 0.0, None, {"SPX": 100.0}),
]


class Scenario:
    """The evaluator's view of a batch of paths: spots at the simulation times (t = 0: the spot)."""

    def __init__(self, times, paths, spot0):
        self.times, self.paths, self.spot0 = np.asarray(times), paths, spot0
        self.n_paths = next(iter(paths.values())).shape[0]

    def col(self, name, t):
        if t <= 0:
            return np.full(self.n_paths, self.spot0[name])
        k = int(np.argmin(np.abs(self.times - t)))
        assert abs(self.times[k] - t) < 1e-12
        return self.paths[name][:, k]

    def spot(self, name, t):
        return self.col(name, t)

    def fixings(self, name, times):
        return np.stack([self.col(name, t) for t in times], axis=1)


def main(ref_root: str = os.environ.get("OPTLAB_REFERENCE", "/root/reference")) -> None:
    ref = Path(ref_root)
    sys.path[:0] = [str(ref / "packages/structured/src"), str(ref / "packages/core/src")]
    from optlab.structured.script.evaluator import Evaluator
    from optlab.structured.script.lexer import ScriptError
    from optlab.structured.script.parser import parse
    from optlab.structured.script.timeline import Clock, build_timeline
    from optlab.structured.script.validate import validate

    rng = np.random.default_rng(20260301)
    n_paths = 64
    out = {"source": "the reference's optlab.structured.script pipeline on seeded lognormal fixings", "r": R,
           "cases": []}
    for name, text, params, eps, valuation, spot0 in CASES:
        program = validate(parse(text))
        tl = build_timeline(program, Clock(valuation))
        times = np.asarray(tl.sim_times, float)
        dts = np.diff(np.concatenate([[0.0], times]))
        paths = {}
        for und, s0 in spot0.items():
            z = rng.standard_normal((n_paths, len(times)))
            paths[und] = s0 * np.exp(np.cumsum(-0.5 * 0.25**2 * dts + 0.25 * np.sqrt(dts) * z, axis=1))
        scen = Scenario(times, paths, spot0)
        case = {"name": name, "script": text, "params": params, "smoothing": eps, "valuation": valuation,
                "spot0": spot0, "times": times.tolist(), "paths": {k: v.tolist() for k, v in paths.items()}}
        try:
            flows = Evaluator(program, tl, params, eps).run(scen)
            pv = np.zeros(n_paths)
            for (t, _tag), f in flows.flows.items():
                if t is not None and t > 0:
                    pv = pv + np.exp(-R * t) * f
            case["pv"] = np.broadcast_to(pv, (n_paths,)).tolist()
        except ScriptError as exc:
            case["refused"] = str(exc)
        out["cases"].append(case)
    (HERE / "script_cases.json").write_text(json.dumps(out))
    print("wrote", HERE / "script_cases.json", [c["name"] + ("*" if "refused" in c else "") for c in out["cases"]])
    callable_case(rng)


def callable_case(rng) -> None:
    """tests/golden/script_callable.json: the reference's pilot record and fitted policy (exercise.fit) of a
    callable note on 600 pilot paths, and its policy applied to 300 other paths (Policy.apply)."""
    from optlab.structured import exercise
    from optlab.structured.script.evaluator import Evaluator
    from optlab.structured.script.parser import parse
    from optlab.structured.script.timeline import Clock, build_timeline
    from optlab.structured.script.validate import validate

    program = validate(parse(CALLABLE))
    tl = build_timeline(program, Clock(None))
    times = np.asarray(tl.sim_times, float)
    dts = np.diff(np.concatenate([[0.0], times]))

    def paths(n):
        z = rng.standard_normal((n, len(times)))
        return {"SPX": 100.0 * np.exp(np.cumsum(-0.5 * 0.3**2 * dts + 0.3 * np.sqrt(dts) * z, axis=1))}

    pilot, pricing = paths(600), paths(300)
    disc = lambda t: float(np.exp(-R * t))  # noqa: E731
    out = Evaluator(program, tl, {}, 0.0).run(Scenario(times, pilot, {"SPX": 100.0}))
    ex = out.exercise
    n = 600
    pre = [disc(ev.t_pay) * sum((np.broadcast_to(f, (n,)) for f in ev.pre.values()), np.zeros(n)) for ev in ex.events]
    post = [disc(ev.t_pay) * sum((np.broadcast_to(f, (n,)) for f in ev.post.values()), np.zeros(n))
            for ev in ex.events]
    calls = [ex.calls[k] for k in sorted(ex.calls)]
    policy = exercise.fit(out, disc)
    priced = Evaluator(program, tl, {}, 0.0).run(Scenario(times, pricing, {"SPX": 100.0}))
    priced = policy.apply(priced)
    pv = np.zeros(300)
    for (t, _tag), f in priced.flows.items():
        if t is not None and t > 0:
            pv = pv + disc(t) * f
    rules = []
    for k in sorted(ex.calls):
        r = policy.rules[k]
        rules.append(None if r is None else {"mean": r.mean, "scale": r.scale, "powers": r.powers,
                                             "knots": r.knots, "coef": r.coef})
    case = {
        "script": CALLABLE, "times": times.tolist(), "spot0": {"SPX": 100.0},
        "pilot": {k: v.tolist() for k, v in pilot.items()}, "pricing": {k: v.tolist() for k, v in pricing.items()},
        "record": {"pre": np.array(pre).tolist(), "post": np.array(post).tolist(),
                   "mask": [np.broadcast_to(c.mask, (n,)).tolist() for c in calls],
                   "alive": [np.broadcast_to(c.alive, (n,)).tolist() for c in calls],
                   "amount": [np.broadcast_to(c.amount, (n,)).tolist() for c in calls],
                   "state": [np.asarray(c.state).tolist() for c in calls]},
        "rules": rules, "in_sample": policy.in_sample, "pv": np.broadcast_to(pv, (300,)).tolist(),
    }
    (HERE / "script_callable.json").write_text(json.dumps(case))
    print("wrote", HERE / "script_callable.json", "in-sample", policy.in_sample, "priced", pv.mean())
    dual_case(rng)


CALLABLE_RC = """
underlying SPX
param c = 0.06
event t=0.5 pay t=0.5
  pay c * 0.5 as coupon
  call pay 1
end
event t=1 pay t=1
  pay c * 0.5 as coupon
  call pay 1
end
event t=1.5 pay t=1.5
  pay c * 0.5 as coupon
  call pay 1
end
event t=2 pay t=2
  pay c * 0.5 as coupon
  pay min(SPX / 100, 1) as redemption
end
"""
DUAL_R, DUAL_Q, DUAL_VOL = 0.04, 0.01, 0.2


def dual_case(rng) -> None:
    """tests/golden/script_dual.json (see the module docstring)."""
    import optlab.core.models as core_models
    from optlab.core import BlackScholesModel, Market
    from optlab.structured import exercise
    from optlab.structured.script.evaluator import Evaluator
    from optlab.structured.script.parser import parse
    from optlab.structured.script.timeline import Clock, build_timeline
    from optlab.structured.script.validate import validate

    sys.path.insert(0, str(Path(exercise.__file__).resolve().parents[5] / "tests" / "helpers"))
    from _callable_refs import callable_note

    program = validate(parse(CALLABLE_RC))
    tl = build_timeline(program, Clock(None))
    times = np.asarray(tl.sim_times, float)
    dts = np.diff(np.concatenate([[0.0], times]))
    model, market = BlackScholesModel(DUAL_VOL), Market.flat(100.0, DUAL_R, DUAL_Q)
    disc = lambda t: float(np.exp(-DUAL_R * t))  # noqa: E731

    def paths(n):
        z = rng.standard_normal((n, len(times)))
        drift = (DUAL_R - DUAL_Q - 0.5 * DUAL_VOL**2) * dts
        return 100.0 * np.exp(np.cumsum(drift + DUAL_VOL * np.sqrt(dts) * z, axis=1))

    def pvs(out):
        pv = np.zeros(out.n_paths)
        for (t, _tag), f in out.flows.items():
            if t is not None and t > 0:
                pv = pv + disc(t) * f
        return pv

    from optlab.structured.scenario import Scenario as RefScenario

    pilot = Evaluator(program, tl, {}, 0.0, True).run(RefScenario("SPX", times, paths(4000), 100.0))
    policy = exercise.fit(pilot, disc)
    priced = policy.apply(Evaluator(program, tl, {}, 0.0, True).run(RefScenario("SPX", times, paths(4000), 100.0)))
    pv = pvs(priced)
    price0, price_se = float(pv.mean()), float(pv.std(ddof=1) / np.sqrt(len(pv)))
    drawn = {"outer": None, "tails": []}
    simulate, continued = core_models.simulate, exercise._continued

    def keep_outer(*a, **k):
        drawn["outer"] = simulate(*a, **k)
        return drawn["outer"]

    def keep_tail(*a, **k):
        tail = continued(*a, **k)
        drawn["tails"].append(tail)
        return tail

    core_models.simulate, exercise._continued = keep_outer, keep_tail
    try:
        small = exercise.dual_bound(model, market, "SPX", tl, program, {}, 100.0, None, policy, disc, price0,
                                    price_se, 11, n_outer=40, n_inner=16)
    finally:
        core_models.simulate, exercise._continued = simulate, continued
    big = exercise.dual_bound(model, market, "SPX", tl, program, {}, 100.0, None, policy, disc, price0, price_se, 11,
                              n_outer=1000, n_inner=200)
    pde = callable_note(lambda p: np.minimum(p, 1.0), 2.0, [(t, 0.03) for t in (0.5, 1.0, 1.5, 2.0)],
                        [(0.5, 1.0), (1.0, 1.0), (1.5, 1.0)], r=DUAL_R, q=DUAL_Q, vol=DUAL_VOL)
    rules = []
    for k in sorted(pilot.exercise.calls):
        r = policy.rules[k]
        rules.append(None if r is None else {"mean": r.mean, "scale": r.scale, "powers": r.powers,
                                             "knots": r.knots, "coef": r.coef})
    case = {
        "script": CALLABLE_RC, "times": times.tolist(), "spot0": {"SPX": 100.0}, "r": DUAL_R, "q": DUAL_Q,
        "vol": DUAL_VOL, "rules": rules, "price0": price0, "price_se": price_se,
        "outer": drawn["outer"].tolist(), "tails": [t.tolist() for t in drawn["tails"]], "n_inner": 16,
        "small": small, "big": big, "pde": float(pde),
    }
    (HERE / "script_dual.json").write_text(json.dumps(case))
    print("wrote", HERE / "script_dual.json", "price0", price0, "small", small, "big", big, "pde", pde)


if __name__ == "__main__":
    main(*sys.argv[1:])
