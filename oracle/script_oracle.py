"""ORACLE — test infrastructure only: the reference's payoff-script evaluation restated in NumPy over arrays of paths.

It follows packages/structured/src/optlab/structured/script/evaluator.py:123-231 (block, expressions, masks, pays,
terminate, undefined values) and cashflows.py:30-41 (present value of the flows: the discount factor of each payment
date after the valuation date), on a program parsed by optlab_b200.script (whose parsing and evaluation are pinned
against the reference's own evaluator by tests/golden/script_cases.json). The spots come from `spot(name, t)` and the
window fixings from `fixings(name, times)`, arrays over paths: the tests fill them from the C oracle's paths.

Only tests import this module; the engine never does.
"""

from __future__ import annotations

import functools

import numpy as np

from optlab_b200.script import (
    ANNUAL,
    Assign,
    Binary,
    Call,
    If,
    IssuerCall,
    Name,
    Num,
    Pay,
    Terminate,
    Unary,
    Window,
    build_timeline,
    parse,
    validate,
)

_FUNCS = {"min": np.minimum, "max": np.maximum, "abs": np.abs, "exp": np.exp, "log": np.log, "sqrt": np.sqrt}
_ARITH = {"+": np.add, "-": np.subtract, "*": np.multiply, "/": np.divide}
_HARD = {"<": np.less, "<=": np.less_equal, ">": np.greater, ">=": np.greater_equal, "==": np.equal}


def _compare(op, a, b, eps):
    hard = np.asarray(_HARD[op](a, b), dtype=float)
    nan = np.isnan(a) | np.isnan(b)
    hard = np.where(nan, np.nan, hard)
    if eps == 0 or op == "==":
        return hard
    scale = eps * np.abs(b)
    d = np.subtract(a, b) if op in (">", ">=") else np.subtract(b, a)
    with np.errstate(divide="ignore", invalid="ignore"):
        ramp = np.clip(d / scale + 0.5, 0.0, 1.0)
    return np.where(scale > 0, ramp, hard)


def realised_variance(f, lower=None, upper=None):
    """Annualised realised variance of (n_paths, n) fixings, returns counted where the fixing before them is in
    [lower, upper] (varswap.py:27-44)."""
    r2 = np.log(f[:, 1:] / f[:, :-1]) ** 2
    if lower is not None or upper is not None:
        prev = f[:, :-1]
        inside = np.ones_like(prev, dtype=bool)
        if lower is not None:
            inside &= prev >= lower
        if upper is not None:
            inside &= prev <= upper
        r2 = np.where(inside, r2, 0.0)
    return ANNUAL / r2.shape[1] * r2.sum(axis=1)


class ScriptOracle:
    """Evaluate a script on n_paths paths: `run()` gives each path's present value and its undefined-value counts."""

    def __init__(self, text, params=None, smoothing=0.0, valuation=None, discount=None):
        self.program = validate(parse(text))
        self.timeline = build_timeline(self.program, valuation)
        self.params = {k: v[0] for k, v in self.program.params.items()}
        self.params.update({k: float(v) for k, v in (params or {}).items()})
        self.eps = float(smoothing)
        self.discount = discount or (lambda t: 1.0)

    def run(self, n_paths, spot, fixings, mode="never", rules=None):
        """mode: "never" (the issuer never calls), "record" (the pilot's record of every call: the result's "pre",
        "post", "mask", "alive", "amount", "state"), or "apply" (the issuer calls where rules[c] (a Rule, or None:
        never) continues above the amount, paying the amount as redemption and terminating; exercise.py:71-122)."""
        self.n, self.spot, self.fixings = n_paths, spot, fixings
        self.mode, self.rules = mode, rules
        self.vars = {}
        self.alive = np.ones(n_paths)
        self.pv = np.zeros(n_paths)
        self.red = np.zeros(n_paths)
        self.bad_pay = np.zeros(n_paths, bool)
        self.bad_cond = np.zeros(n_paths, bool)
        n_ev = len(self.program.events)
        self.pre, self.post = np.zeros((n_ev, n_paths)), np.zeros((n_ev, n_paths))
        self.calls = []  # (mask, alive, amount, state) of each call, in order
        with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
            for k, ev in enumerate(self.program.events):
                self.k, self.after = k, False
                self.t_obs = float(self.timeline.event_times[k])
                t_pay = self.timeline.pay_times[k]
                self.disc = float(self.discount(t_pay)) if t_pay is not None and t_pay > 0 else 0.0
                self.block(ev.body, 1.0)
        tol = 1e-12 if self.eps == 0 else 1e-9
        bad_red = ~(np.abs(self.red - 1.0) <= tol)
        out = {"pv": self.pv, "bad_pay": self.bad_pay, "bad_cond": self.bad_cond, "bad_redemption": bad_red,
               "pre": self.pre, "post": self.post}
        if self.calls:
            out.update(mask=np.array([c[0] for c in self.calls]), alive=np.array([c[1] for c in self.calls]),
                       amount=np.array([c[2] for c in self.calls]), state=np.array([c[3] for c in self.calls]))
        return out

    def block(self, body, m):
        for s in body:
            if isinstance(s, Assign):
                e = self.expr(s.expr)
                if isinstance(m, float) and m == 1.0:
                    self.vars[s.name] = np.broadcast_to(np.asarray(e, float), (self.n,)).copy()
                else:
                    old = self.vars.get(s.name, 0.0)
                    self.vars[s.name] = np.where(m == 1.0, e, np.where(m == 0.0, old, m * e + (1 - m) * old))
            elif isinstance(s, Pay):
                w = m * self.alive
                e = np.broadcast_to(np.asarray(self.expr(s.expr), float), (self.n,))
                live = np.broadcast_to(w != 0, (self.n,))
                self.bad_pay |= live & ~np.isfinite(e)
                paid = np.where(live & np.isfinite(e), w * e, 0.0)
                self.pv = self.pv + self.disc * paid
                if self.after:
                    self.post[self.k] += self.disc * paid
                else:
                    self.pre[self.k] += self.disc * paid
                if s.tag == "redemption":
                    self.red = self.red + w
            elif isinstance(s, Terminate):
                self.alive = self.alive * (1.0 - m)
            elif isinstance(s, IssuerCall):
                self.issuer_call(s, m)
            elif isinstance(s, If):
                c = np.broadcast_to(np.asarray(self.expr(s.cond), float), (self.n,))
                undefined = np.isnan(c)
                self.bad_cond |= undefined & (np.asarray(m * self.alive) != 0)
                c = np.where(undefined, 0.0, c)
                self.block(s.body, m * c)
                if s.orelse:
                    self.block(s.orelse, m * (1.0 - c))
            else:
                raise TypeError(f"not evaluated by the oracle: {s!r}")

    def issuer_call(self, s, m):
        names = self.program.states or [u[0] for u in self.program.underlyings]
        amount = np.broadcast_to(np.asarray(self.expr(s.expr), float), (self.n,))
        state = np.stack([np.broadcast_to(np.asarray(self.expr(Name(x)), float), (self.n,)) for x in names], axis=1)
        mask = np.broadcast_to(np.asarray(m, float), (self.n,))
        c = len(self.calls)
        self.calls.append((mask.copy(), self.alive.copy(), amount.copy(), state.copy()))
        if self.mode == "record":
            self.after = True
        elif self.mode == "apply":
            rule = self.rules[c]
            decide = np.zeros(self.n) if rule is None else (rule.continuation(state) > amount).astype(float)
            md = mask * decide
            w = md * self.alive
            self.bad_pay |= (w != 0) & ~np.isfinite(amount)
            self.pv = self.pv + self.disc * np.where((w != 0) & np.isfinite(amount), w * amount, 0.0)
            self.red = self.red + w
            self.alive = self.alive * (1.0 - md)

    def expr(self, e):
        if isinstance(e, Num):
            return e.value
        if isinstance(e, Name):
            if e.id in self.vars:
                return self.vars[e.id]
            if e.id in self.params:
                return self.params[e.id]
            return self.spot(e.id, self.t_obs)
        if isinstance(e, Binary):
            a, b = self.expr(e.left), self.expr(e.right)
            if e.op in _ARITH:
                return _ARITH[e.op](a, b)
            if e.op == "and":
                return np.where((np.asarray(a) == 0) | (np.asarray(b) == 0), 0.0, np.multiply(a, b))
            if e.op == "or":
                return np.where((np.asarray(a) == 1) | (np.asarray(b) == 1), 1.0, np.add(a, b) - np.multiply(a, b))
            return _compare(e.op, a, b, self.eps)
        if isinstance(e, Unary):
            v = self.expr(e.operand)
            return -v if e.op == "-" else 1.0 - v
        if isinstance(e, Call):
            args = [self.expr(a) for a in e.args]
            if e.func in ("worst", "best"):
                return functools.reduce(np.minimum if e.func == "worst" else np.maximum, args)
            return _FUNCS[e.func](*args)
        if isinstance(e, Window):
            k = next(i for i, w in enumerate(self.timeline.windows) if w is e)
            fix = self.fixings(e.underlying, self.timeline.window_times[k])
            if e.func == "variance":
                lo = None if e.lower is None else self.expr(e.lower)
                hi = None if e.upper is None else self.expr(e.upper)
                return realised_variance(fix, lo, hi)
            return fix.min(axis=1) if e.func == "lowest" else fix.max(axis=1)
        raise TypeError(f"cannot evaluate {e!r}")
