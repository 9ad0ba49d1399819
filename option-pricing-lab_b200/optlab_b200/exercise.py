"""The issuer's call of a payoff script on the device: a Longstaff-Schwartz policy fitted on a pilot simulation, then
applied out of sample by the pricing run.

The method is the reference's (packages/structured/src/optlab/structured/exercise.py:1-17, fit at :212-252, the basis
at :125-140): the script runs on the pilot as if the issuer never called, recording per path each event's discounted
flows before and after its call statement and, at each call, its mask, the alive mass, the amount and the state;
backward from the last call date, the note's continuation per unit reached, in money of the call date, is regressed on
polynomials and hinges of the normalised state over the paths the call reaches, and the issuer calls where the fitted
continuation is above the amount. Here the pilot runs on the device and the fit too (ob_script_pilot_fit: the record
stays in device memory, every pass over the paths is a kernel, the at most 25 x 25 normal equations are solved and
refined on the host), and the pricing run applies the rules on the device (call mode 2): a call there pays the amount
as redemption and terminates, which is what the reference's `survival_and_flows` rebuilds from the uncalled record.
`fit` is the same regression on a record brought to the host, with the reference's own least-squares solve: the
device hands a pilot to it when a regression's terms are nearly collinear.
"""

from __future__ import annotations

import ctypes as C
import itertools
from dataclasses import dataclass

import numpy as np

from ._abi import OB_ESINGULAR, OB_RULE_STRIDE, ObScriptResult, check, load, ptr
from . import script as sc

MAX_TERMS = 25  # regression terms, the constant included
MAX_KNOTS = 9  # hinges per state variable, at its deciles
MIN_PATHS_PER_TERM = 20  # fewer paths reaching a call than this per term: fewer hinges, a lower degree


def powers(d: int, degree: int) -> list:
    """Exponents of the monomials of total degree <= degree in d variables: the constant first, then by degree, each
    degree in the order of the variables' multisets."""
    out = []
    for total in range(degree + 1):
        for combo in itertools.combinations_with_replacement(range(d), total):
            p = [0] * d
            for i in combo:
                p[i] += 1
            out.append(tuple(p))
    return out


def basis(z: np.ndarray):
    """(powers, knots) of the regression on the normalised state z (paths x variables): polynomials (degree 3 in one
    variable, 2 in up to four, 1 beyond, lower when the paths are few) and hinges max(z_i - k, 0) at each variable's
    deciles, as many as MIN_PATHS_PER_TERM paths a term allow, at most MAX_TERMS terms."""
    n, d = z.shape
    room = min(MAX_TERMS, n // MIN_PATHS_PER_TERM)
    for degree in (3 if d == 1 else 2 if d <= 4 else 1, 1, 0):
        pw = powers(d, degree)
        if len(pw) <= room:
            break
    per = max(0, min(MAX_KNOTS, (room - len(pw)) // d))
    knots = []
    for i in range(d):
        levels = np.unique(np.quantile(z[:, i], np.linspace(0.0, 1.0, per + 2)[1:-1])) if per else []
        lo, hi = z[:, i].min(), z[:, i].max()
        knots += [(i, float(k)) for k in levels if lo < k < hi]
    return pw, knots


@dataclass(frozen=True)
class Rule:
    """One call date's rule: the fitted continuation of the state, against the call amount."""

    mean: tuple
    scale: tuple
    powers: tuple
    knots: tuple
    coef: tuple = ()

    def features(self, state: np.ndarray) -> np.ndarray:
        """(paths, terms): the monomials of z, then the hinges, z the normalised state; written column by column
        into one array (one variable: z ** e itself, the product of a single factor)."""
        z = (state - np.asarray(self.mean)) / np.asarray(self.scale)
        out = np.empty((z.shape[0], len(self.powers) + len(self.knots)))
        for j, p in enumerate(self.powers):
            out[:, j] = z[:, 0] ** p[0] if z.shape[1] == 1 else np.prod(z ** np.asarray(p), axis=1)
        for j, (i, k) in enumerate(self.knots):
            np.maximum(z[:, i] - k, 0.0, out=out[:, len(self.powers) + j])
        return out

    def continuation(self, state: np.ndarray) -> np.ndarray:
        return self.features(state) @ np.asarray(self.coef)


@dataclass(frozen=True)
class Policy:
    """The issuer's rule at each call (by call index; None: the pilot reached no path there, never called)."""

    rules: tuple
    pilot_paths: int
    in_sample: float = float("nan")  # the pilot's value under its own policy

    def pack(self, n_state: int) -> np.ndarray:
        """The device's rules: (n_calls, OB_RULE_STRIDE) rows of valid, n_poly, n_knots, mean[4], scale[4],
        powers[25][4], knot variable[25], knot[25], coefficients[50]."""
        out = np.zeros((len(self.rules), OB_RULE_STRIDE))
        for c, r in enumerate(self.rules):
            if r is None:
                continue
            row = out[c]
            row[0], row[1], row[2] = 1.0, len(r.powers), len(r.knots)
            row[3:3 + n_state] = r.mean
            row[7:7 + n_state] = r.scale
            for t, p in enumerate(r.powers):
                row[11 + 4 * t:11 + 4 * t + n_state] = p
            for q, (v, k) in enumerate(r.knots):
                row[111 + q], row[136 + q] = v, k
            row[161:161 + len(r.coef)] = r.coef
        return out

    @classmethod
    def unpack(cls, rows: np.ndarray, n_state: int, pilot_paths: int, in_sample: float = float("nan")) -> Policy:
        """The policy of packed rules (the layout of pack; a row whose first value is 0: no rule)."""
        rules = []
        for row in np.asarray(rows, dtype=np.float64):
            if row[0] == 0.0:
                rules.append(None)
                continue
            n_poly, n_knots = int(row[1]), int(row[2])
            rules.append(Rule(
                tuple(float(v) for v in row[3:3 + n_state]), tuple(float(v) for v in row[7:7 + n_state]),
                tuple(tuple(int(v) for v in row[11 + 4 * t:11 + 4 * t + n_state]) for t in range(n_poly)),
                tuple((int(row[111 + q]), float(row[136 + q])) for q in range(n_knots)),
                tuple(float(v) for v in row[161:161 + n_poly + n_knots])))
        return cls(tuple(rules), pilot_paths, in_sample)


@dataclass
class PilotRecord:
    """The pilot's record, per path: each event's discounted flows before and after its call statement, and per call
    its mask, alive mass, amount and state."""

    pre: np.ndarray  # (events, paths)
    post: np.ndarray
    mask: np.ndarray  # (calls, paths)
    alive: np.ndarray
    amount: np.ndarray
    state: np.ndarray  # (calls, paths, n_state)

    @classmethod
    def from_device(cls, record: np.ndarray, n_events: int, n_calls: int, n_state: int) -> PilotRecord:
        ev = record[:, : 2 * n_events].reshape(-1, n_events, 2)
        calls = record[:, 2 * n_events:].reshape(-1, n_calls, 3 + n_state)
        return cls(ev[:, :, 0].T.copy(), ev[:, :, 1].T.copy(), calls[:, :, 0].T.copy(), calls[:, :, 1].T.copy(),
                   calls[:, :, 2].T.copy(), np.transpose(calls[:, :, 3:], (1, 0, 2)).copy())


def fit(rec: PilotRecord, call_events: list, pay_discount: list) -> Policy:
    """Backward regression on a pilot record (exercise.py:212-252): call_events[c] is the event of call c,
    pay_discount[k] the discount factor of event k's payment (0 where it pays nothing counted)."""
    n = rec.pre.shape[1]
    call_of = {k: c for c, k in enumerate(call_events)}
    rules: list = [None] * len(call_events)
    future = np.zeros(n)
    for k in range(rec.pre.shape[0] - 1, -1, -1):
        c = call_of.get(k)
        if c is None:
            future = rec.pre[k] + rec.post[k] + future
            continue
        after = rec.post[k] + future
        reach = rec.mask[c] * rec.alive[c]
        on = reach > 0
        d = pay_discount[k] if pay_discount[k] > 0 else 1.0
        decide = np.zeros(n)
        if on.any():
            y = after[on] / (d * reach[on])
            x = rec.state[c][on]
            mean, scale = x.mean(axis=0), x.std(axis=0)
            scale = np.where(scale > 0, scale, 1.0)
            pw, knots = basis((x - mean) / scale)
            shape = Rule(tuple(float(v) for v in mean), tuple(float(v) for v in scale), tuple(pw), tuple(knots))
            feats = shape.features(rec.state[c])  # every path's terms: the regression's rows, then the decisions
            coef = np.linalg.lstsq(feats[on], y, rcond=None)[0]
            rule = Rule(shape.mean, shape.scale, shape.powers, shape.knots, tuple(float(v) for v in coef))
            rules[c] = rule
            decide = (feats @ np.asarray(rule.coef) > rec.amount[c]).astype(float)
        called = rec.mask[c] * decide
        paid = d * called * rec.alive[c] * rec.amount[c]
        future = rec.pre[k] + (1.0 - called) * after + paid
    return Policy(tuple(rules), n, float(np.mean(future)))


def pilot_fit(pilot: sc.ScriptHeld, call_events: list, pay_discount: list, precision="fp32"):
    """Run the pilot (a call_mode 1 request) and fit the policy on the device (ob_script_pilot_fit): the record stays
    in device memory. Returns (policy, the pilot's result), or None where a regression's terms are nearly collinear
    (the device then leaves the fit to `fit` and the reference's own least squares)."""
    from .engine import precision_code

    s = pilot.struct
    rules = np.zeros((s.n_calls, OB_RULE_STRIDE))
    events = np.ascontiguousarray(call_events, dtype=np.int32)
    disc = np.ascontiguousarray(pay_discount, dtype=np.float64)
    res, ins = ObScriptResult(), C.c_double()
    kept = C.cast(s.record, C.c_void_p).value  # (a pointer field read from a Structure shares its memory)
    s.record = None  # the record stays on the device
    try:
        status = load().ob_script_pilot_fit(C.byref(s), precision_code(precision), ptr(events, C.c_int), ptr(disc),
                                            ptr(rules), C.byref(ins), C.byref(res))
    finally:
        s.record = C.cast(kept, C.POINTER(C.c_double))
    if status == OB_ESINGULAR:
        return None
    check(status)
    sc.check_result(pilot, res)
    return Policy.unpack(rules, s.n_state, 2 * s.model.n_pairs, ins.value), res


def pilot_paths(n_paths: int) -> int:
    """The pilot's size: half the pricing paths, between 20,000 and 100,000, even (exercise.py:256-259)."""
    n = max(20_000, min(n_paths // 2, 100_000))
    return n + n % 2


PILOT_KEY = 0x5EEDCA11  # the pilot's Philox key is the pricing seed xor this: no pricing pair shares its draws


def price(compiled, make_sim, n_pairs: int, seed: int, discount, precision="fp32"):
    """The price of a callable script: a pilot of pilot_paths(2 n_pairs) paths on seed ^ PILOT_KEY, the policy fitted
    on its record on the device (the host's `fit` where the device refuses a regression), then the pricing run of
    n_pairs pairs on `seed` applying it. make_sim(n_pairs, seed) builds the
    simulation request. Returns (result, policy)."""
    if not compiled.calls:
        return sc.run(sc.script_request(compiled, make_sim(n_pairs, seed), discount), precision), None
    n_state = len(compiled.calls[0][1])
    pilot = sc.script_request(compiled, make_sim(pilot_paths(2 * n_pairs) // 2, seed ^ PILOT_KEY), discount,
                              call_mode=1)
    pay_d = [float(discount(t)) if t is not None and t > 0 else 0.0 for t in compiled.pay_times]
    call_events = [k for k, _ in compiled.calls]
    fitted = pilot_fit(pilot, call_events, pay_d, precision)
    if fitted is not None:
        policy = fitted[0]
    else:
        sc.run(pilot, precision)
        rec = PilotRecord.from_device(pilot.keep[1]["record"], len(compiled.event_times), len(compiled.calls), n_state)
        policy = fit(rec, call_events, pay_d)
    held = sc.script_request(compiled, make_sim(n_pairs, seed), discount, call_mode=2, rules=policy.pack(n_state))
    return sc.run(held, precision), policy


DUAL_OUTER_KEY = 0xD0A1B0D5  # the dual bound's outer paths draw on seed ^ this
DUAL_INNER_KEY = 0x1A2B3C4D  # the continuations from call c draw on seed ^ this ^ (c + 1)


def decisions(policy: Policy, rec: PilotRecord) -> np.ndarray:
    """(calls, paths): 1 where the policy calls at a call the path reaches, the rule's continuation of the state
    above the amount (exercise.py: Policy.decisions); 0 at calls without a rule."""
    out = np.zeros_like(rec.amount)
    for c, rule in enumerate(policy.rules):
        if rule is not None:
            out[c] = (rule.continuation(rec.state[c]) > rec.amount[c]).astype(float)
    return out


def dual_recursion(pre, post, mask, alive, amount, decide, call_events, call_discount, H, price0):
    """The martingale dual of the issuer's (minimising) problem, exercise.py:353-372. pre, post: (events, paths)
    discounted flows of the uncalled outer paths before and after each event's call statement; mask, alive, amount,
    decide: (calls, paths); call_events[c]: the event of call c, call_discount[c] the discount factor of its
    payment; H[c]: (paths,) the policy's value from call c on, not called at c or before (mean of the
    continuations). Returns per path min_j (G_j - M_j), G_j the note's flows if called at call j (never: the last
    H), M the martingale of the policy's value started at price0."""
    pv = pre + post
    n = pv.shape[1]
    M = np.zeros(n)
    best = np.full(n, np.inf)
    previous = np.full(n, float(price0))
    for c, k in enumerate(call_events):
        reach = mask[c] * alive[c]
        g = np.where(reach > 0, pv[:k].sum(axis=0) + pre[k] + call_discount[c] * reach * amount[c], np.inf)
        called = decide[c] * (reach > 0)
        level = np.where(called > 0, g, H[c])
        M = M + level - previous
        best = np.minimum(best, g - M)
        previous = H[c]
    return np.minimum(best, previous - M)


def dual_bound(compiled, make_sim, policy: Policy, price0: float, price_se: float, seed: int, discount,
               n_outer: int = 1000, n_inner: int = 200, precision="fp64") -> dict:
    """Andersen-Broadie for the issuer, who minimises (exercise.py:294-380): the note's value is at least
    E[min_j (G_j - M_j)], G_j the note's flows if called at call date j, M the martingale of the policy's own value,
    whose conditional expectations come from n_inner continuations of each of n_outer outer paths branched at each
    call date. On the device: the outer paths are a recorded uncalled run (call mode 1, n_outer / 2 antithetic
    pairs on seed ^ DUAL_OUTER_KEY); the continuations from call c are one branched run (n_outer x n_inner / 2
    pairs, each following its outer path's draws up to the call's step end, its own after it) that applies the
    policy after c and never at c or before, and returns each pair's value. price0 and price_se are the policy's
    price and SE (the pricing run's). A single local-vol name (the reference's bound needs a model without a
    variance process and a single name); returns lower, lower_se, gap, gap_se, outer, inner (the SE of the gap on
    the outer pairs' averages)."""
    if not compiled.calls:
        raise ValueError("no dual bound without an issuer call")
    if len(compiled.names) != 1:
        raise ValueError("no dual bound for a basket")
    n_outer += n_outer % 2
    n_inner += n_inner % 2
    P, per = n_outer // 2, n_inner // 2
    n_state = len(compiled.calls[0][1])
    n_ev = len(compiled.event_times)
    outer_seed = (seed ^ DUAL_OUTER_KEY) & (2**64 - 1)
    outer = sc.script_request(compiled, make_sim(P, outer_seed), discount, call_mode=1)
    s = outer.struct.model
    if s.model != 0 or s.kind[0] != 1:
        raise ValueError("no dual bound for a model with a variance process (local vol only)")
    sc.run(outer, precision)
    rec = PilotRecord.from_device(outer.keep[1]["record"], n_ev, len(compiled.calls), n_state)
    ev_step = outer.keep[1]["event_step"]
    pay_d = [float(discount(t)) if t is not None and t > 0 else 0.0 for t in compiled.pay_times]
    call_events = [k for k, _ in compiled.calls]
    call_disc = [pay_d[k] if pay_d[k] > 0 else 1.0 for k in call_events]
    packed = policy.pack(n_state)
    H = []
    for c, k in enumerate(call_events):
        rules = packed.copy()
        rules[: c + 1] = 0.0  # not called at c nor before
        inner_seed = (seed ^ DUAL_INNER_KEY ^ (c + 1)) & (2**64 - 1)
        inner = sc.script_request(compiled, make_sim(n_outer * per, inner_seed), discount, call_mode=2, rules=rules,
                                  branch=(int(ev_step[k]), P, per, outer_seed))
        sc.run(inner, precision)
        H.append(inner.keep[1]["pair_value"].reshape(n_outer, per).mean(axis=1))
    best = dual_recursion(rec.pre, rec.post, rec.mask, rec.alive, rec.amount, decisions(policy, rec), call_events,
                          call_disc, H, price0)
    pairs = 0.5 * (best[:P] + best[P:])
    gap = float(price0 - pairs.mean())
    gap_se = float(pairs.std(ddof=1) / np.sqrt(P))
    return {"lower": float(price0) - gap, "lower_se": float(np.hypot(price_se, gap_se)), "gap": gap,
            "gap_se": gap_se, "outer": n_outer, "inner": n_inner}
