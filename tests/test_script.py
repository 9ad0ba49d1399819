"""Payoff scripts without a GPU: the parser and validator refuse what the reference refuses, the NumPy oracle equals the
reference's own evaluator on its recorded cases (tests/golden/script_cases.json), and the compiled bytecode, run by a
NumPy model of the device's interpreter, equals the oracle on the same paths."""

import json
import re
from pathlib import Path

import numpy as np
import pytest

from optlab_b200 import script as sc

GOLDEN = Path(__file__).resolve().parent / "golden" / "script_cases.json"
CASES = json.loads(GOLDEN.read_text())
R = CASES["r"]


class Paths:
    def __init__(self, case):
        self.times = np.asarray(case["times"])
        self.paths = {k: np.asarray(v) for k, v in case["paths"].items()}
        self.spot0 = case["spot0"]
        self.n = next(iter(self.paths.values())).shape[0]

    def col(self, name, t):
        if t <= 0:
            return np.full(self.n, self.spot0[name])
        k = int(np.argmin(np.abs(self.times - t)))
        assert abs(self.times[k] - t) < 1e-12
        return self.paths[name][:, k]

    def spot(self, name, t):
        return self.col(name, t)

    def fixings(self, name, times):
        return np.stack([self.col(name, t) for t in times], axis=1)


def _oracle(case):
    from script_oracle import ScriptOracle

    o = ScriptOracle(case["script"], case["params"], case["smoothing"], case["valuation"], lambda t: np.exp(-R * t))
    p = Paths(case)
    return o.run(p.n, p.spot, p.fixings), p


@pytest.mark.parametrize("case", CASES["cases"], ids=[c["name"] for c in CASES["cases"]])
def test_the_oracle_equals_the_references_evaluator(case):
    res, _ = _oracle(case)
    if "refused" in case:
        assert res["bad_pay"].any() or res["bad_cond"].any(), case["refused"]
        return
    want = np.asarray(case["pv"])
    assert not (res["bad_pay"].any() or res["bad_cond"].any())
    assert np.allclose(res["pv"], want, rtol=1e-12, atol=1e-14), np.abs(res["pv"] - want).max()


def interpret(compiled, paths, eps, discount):
    """The device's interpreter, restated over arrays of paths (csrc/script.cu run_event and fix_windows)."""
    n = paths.n
    reg = np.zeros((compiled.n_regs, n))
    reg[: len(compiled.consts)] = compiled.consts[:, None]
    alive, pv, red = np.ones(n), np.zeros(n), np.zeros(n)
    bad_pay, bad_cond = np.zeros(n, bool), np.zeros(n, bool)
    names = compiled.names
    ops = {v: k for k, v in sc.OP.items()}
    for k, t in enumerate(compiled.event_times):
        t_pay = compiled.pay_times[k]
        disc = discount(t_pay) if t_pay is not None and t_pay > 0 else 0.0
        for op, d, a, b in compiled.code[compiled.event_code[k]:compiled.event_code[k + 1]]:
            name = ops[int(op)]
            with np.errstate(all="ignore"):
                if name == "spot":
                    reg[d] = paths.spot(names[a], t)
                elif name == "win":
                    i, f, times, lo, hi = compiled.windows[a]
                    fix = paths.fixings(names[i], times)
                    if f == 0:
                        reg[d] = fix.min(axis=1)
                    elif f == 1:
                        reg[d] = fix.max(axis=1)
                    else:
                        r2 = np.log(fix[:, 1:] / fix[:, :-1]) ** 2
                        prev = fix[:, :-1]
                        inside = (np.isnan(lo) | (prev >= lo)) & (np.isnan(hi) | (prev <= hi))
                        reg[d] = sc.ANNUAL / (fix.shape[1] - 1) * np.where(inside, r2, 0.0).sum(axis=1)
                elif name == "mov":
                    reg[d] = reg[a]
                elif name in ("add", "sub", "mul", "div", "min", "max"):
                    f = {"add": np.add, "sub": np.subtract, "mul": np.multiply, "div": np.divide,
                         "min": np.minimum, "max": np.maximum}[name]
                    reg[d] = f(reg[a], reg[b])
                elif name in ("neg", "abs", "exp", "log", "sqrt", "not"):
                    f = {"neg": np.negative, "abs": np.abs, "exp": np.exp, "log": np.log, "sqrt": np.sqrt,
                         "not": lambda x: 1.0 - x}[name]
                    reg[d] = f(reg[a])
                elif name in ("ge", "gt", "le", "lt", "eq"):
                    x, y = reg[a], reg[b]
                    h = {"ge": x >= y, "gt": x > y, "le": x <= y, "lt": x < y, "eq": x == y}[name].astype(float)
                    out = h
                    if eps != 0 and name != "eq":
                        scale = eps * np.abs(y)
                        dd = x - y if name in ("ge", "gt") else y - x
                        out = np.where(scale > 0, np.clip(dd / scale + 0.5, 0, 1), h)
                    reg[d] = np.where(np.isnan(x) | np.isnan(y), np.nan, out)
                elif name == "and":
                    reg[d] = np.where((reg[a] == 0) | (reg[b] == 0), 0.0, reg[a] * reg[b])
                elif name == "or":
                    reg[d] = np.where((reg[a] == 1) | (reg[b] == 1), 1.0, reg[a] + reg[b] - reg[a] * reg[b])
                elif name == "assign":
                    m, e, old = reg[b], reg[a], reg[d].copy()
                    reg[d] = np.where(m == 1, e, np.where(m == 0, old, m * e + (1 - m) * old))
                elif name == "pay":
                    w, e = reg[b] * alive, reg[a]
                    live = w != 0
                    bad_pay |= live & ~np.isfinite(e)
                    pv = pv + np.where(live & np.isfinite(e), disc * (w * e), 0.0)
                    if d == 2:
                        red = red + w
                elif name == "term":
                    alive = alive * (1 - reg[a])
                elif name == "cond":
                    c = reg[a]
                    bad_cond |= np.isnan(c) & (reg[b] * alive != 0)
                    reg[d] = np.where(np.isnan(c), 0.0, c)
    return pv, bad_pay, bad_cond, red


@pytest.mark.parametrize("case", CASES["cases"], ids=[c["name"] for c in CASES["cases"]])
def test_the_compiled_bytecode_equals_the_oracle(case):
    comp = sc.compile_script(case["script"], case["params"], case["smoothing"], case["valuation"])
    assert comp.n_regs <= sc.MAX_REGS and comp.code.shape[1] == 4
    res, paths = _oracle(case)
    pv, bad_pay, bad_cond, red = interpret(comp, paths, case["smoothing"], lambda t: np.exp(-R * t))
    assert np.array_equal(bad_pay, res["bad_pay"]) and np.array_equal(bad_cond, res["bad_cond"])
    ok = ~(bad_pay | bad_cond)
    assert np.allclose(pv[ok], res["pv"][ok], rtol=1e-12, atol=1e-14), np.abs(pv - res["pv"])[ok].max()
    if "refused" not in case and case["smoothing"] == 0.0:
        assert np.all(np.abs(red - 1.0) <= 1e-12)


@pytest.mark.parametrize(
    "text,message",
    [
        ("event t=1\nend\n", "no underlying declared"),
        ("underlying A\n", "the script has no event"),
        ("underlying A\nevent t=1\n  pay 1 as redemption\nend\n", "'pay' in an event without a payment date"),
        ("underlying A\nevent t=1 pay t=1\n  pay 1 as bonus\nend\n", "unknown flow tag 'bonus'"),
        ("underlying A\nevent t=1 pay t=1\n  pay x as redemption\nend\n", "'x' is used before it is assigned"),
        ("underlying A\nevent t=2\nend\nevent t=1\nend\n", "event dates must be strictly increasing"),
        ("underlying A\nevent t=1 pay t=1\n  x = lowest(A, t=0, t=2, n=4)\nend\n", "window ends after the event"),
        ("underlying A\nevent t=1\n  x = 1 < 2 < 3\nend\n", "chained comparisons are not allowed"),
        ("underlying A\nevent t=1\n  x = foo(1)\nend\n", "unknown function 'foo'"),
        ("underlying A\nevent t=1\n  x = min(1)\nend\n", "min takes 2 argument(s), got 1"),
        ("underlying A\nevent t=1\n  x = 1 $ 2\nend\n", "unexpected character '$'"),
        ("underlying A\nevent 2025-01-02\nend\nevent t=2\nend\n", "dates and times (t=...) cannot be mixed"),
    ],
)
def test_bad_scripts_are_refused_with_the_references_messages(text, message):
    with pytest.raises(sc.ScriptError, match=re.escape(message)):
        sc.compile_script(text)


def test_what_the_device_does_not_evaluate_is_refused():
    call = ("underlying A\nstate a, b, c, d, e\nevent t=1 pay t=1\n  a = 1\n  b = 1\n  c = 1\n  d = 1\n  e = 1\n"
            "  call pay 1\n  pay 1 as redemption\nend\n")
    with pytest.raises(sc.ScriptError, match="at most 4 state variables"):
        sc.compile_script(call)
    corridor = ("underlying A\nevent t=1 pay t=1\n  x = A\n  v = variance(A, t=0, t=1, n=4, x, 200)\n"
                "  pay v as upside\n  pay 1 as redemption\nend\n")
    with pytest.raises(sc.ScriptError, match="corridor on the device"):
        sc.compile_script(corridor)
    with pytest.raises(KeyError, match="unknown parameter"):
        sc.compile_script("underlying A\nevent t=1\nend\n", params={"zz": 1})


def test_parameters_override_and_the_timeline_holds_every_observation():
    comp = sc.compile_script(CASES["cases"][0]["script"], params={"cpn": 0.03})
    assert 0.03 in comp.consts and 0.02 not in comp.consts
    tl = comp.timeline
    assert np.allclose(tl.event_times, [0.25, 0.5, 0.75, 1.0])
    assert len(tl.windows) == 1 and np.allclose(tl.window_times[0], np.arange(1, 49) / 48)
    assert set(np.round(tl.sim_times, 12)) >= set(np.round(tl.window_times[0], 12))


def _sim(comp, n_steps=48):
    from optlab_b200._abi import OB_MODEL_PATHS, OB_PRODUCT_LADDER
    from optlab_b200.models import time_grid
    from optlab_b200.requests import mc_request

    grid = time_grid(comp.timeline.sim_times, 1.0 / n_steps)
    n = len(comp.names)
    return mc_request(model=OB_MODEL_PATHS, dt=np.diff(grid), t0=grid[:-1], spot=np.full(n, 100.0), n_pairs=64,
                      seed=3, kind=np.zeros(n, np.int32), cvar=np.full(n, 0.04), log_fwd=np.zeros((n, len(grid))),
                      product=OB_PRODUCT_LADDER, leg_type=[1], leg_strike=[1.0])


def test_requests_the_device_could_misread_are_refused_before_any_launch():
    """Every register, name, window and step index the kernel follows is checked on the host."""
    from optlab_b200 import _abi

    comp = sc.compile_script(CASES["cases"][0]["script"])
    held = sc.script_request(comp, _sim(comp), lambda t: 1.0)
    code = held.keep[1]["code"]
    saved = code.copy()
    for k, bad, message in [(1, comp.n_regs, "register beyond n_regs"), (0, 99, "unknown instruction")]:
        code[k] = bad
        with pytest.raises(_abi.EngineError, match=message):
            sc.run(held, "fp64")
        code[:] = saved
    steps = held.keep[1]["event_step"]
    steps[1] = steps[0]
    with pytest.raises(_abi.EngineError, match="event steps must increase"):
        sc.run(held, "fp64")


def test_observations_off_the_grid_are_refused():
    comp = sc.compile_script(CASES["cases"][0]["script"])
    sim = _sim(sc.compile_script("underlying A\nevent t=1\nend\n"), n_steps=10)
    with pytest.raises(ValueError, match="no step ending"):
        sc.script_request(comp, sim, lambda t: 1.0)
