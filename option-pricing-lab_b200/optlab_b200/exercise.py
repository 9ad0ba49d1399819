"""The issuer's call of a payoff script on the device: a Longstaff-Schwartz policy fitted on a pilot simulation, then
applied out of sample by the pricing run.

The method is the reference's (packages/structured/src/optlab/structured/exercise.py:1-17, fit at :212-252, the basis
at :125-140): the script runs on the pilot as if the issuer never called, recording per path each event's discounted
flows before and after its call statement and, at each call, its mask, the alive mass, the amount and the state;
backward from the last call date, the note's continuation per unit reached, in money of the call date, is regressed on
polynomials and hinges of the normalised state over the paths the call reaches, and the issuer calls where the fitted
continuation is above the amount. Here the pilot's record comes from the device (call mode 1 of ob_script_price), the
regressions (a few tens of thousands of paths, at most 25 terms) run on the host, and the pricing run applies the rules
on the device (call mode 2): a call there pays the amount as redemption and terminates, which is what the reference's
`survival_and_flows` rebuilds from the uncalled record.
"""

from __future__ import annotations

import itertools
from dataclasses import dataclass

import numpy as np

from ._abi import OB_RULE_STRIDE
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
        z = (state - np.asarray(self.mean)) / np.asarray(self.scale)
        cols = [np.prod(z ** np.asarray(p), axis=1) for p in self.powers]
        cols += [np.maximum(z[:, i] - k, 0.0) for i, k in self.knots]
        return np.stack(cols, axis=1)

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
            coef = np.linalg.lstsq(shape.features(x), y, rcond=None)[0]
            rule = Rule(shape.mean, shape.scale, shape.powers, shape.knots, tuple(float(v) for v in coef))
            rules[c] = rule
            decide = (rule.continuation(rec.state[c]) > rec.amount[c]).astype(float)
        called = rec.mask[c] * decide
        paid = d * called * rec.alive[c] * rec.amount[c]
        future = rec.pre[k] + (1.0 - called) * after + paid
    return Policy(tuple(rules), n, float(np.mean(future)))


def pilot_paths(n_paths: int) -> int:
    """The pilot's size: half the pricing paths, between 20,000 and 100,000, even (exercise.py:256-259)."""
    n = max(20_000, min(n_paths // 2, 100_000))
    return n + n % 2


PILOT_KEY = 0x5EEDCA11  # the pilot's Philox key is the pricing seed xor this: no pricing pair shares its draws


def price(compiled, make_sim, n_pairs: int, seed: int, discount, precision="fp32"):
    """The price of a callable script: a pilot of pilot_paths(2 n_pairs) paths on seed ^ PILOT_KEY, the policy fitted
    on its record, then the pricing run of n_pairs pairs on `seed` applying it. make_sim(n_pairs, seed) builds the
    simulation request. Returns (result, policy)."""
    if not compiled.calls:
        return sc.run(sc.script_request(compiled, make_sim(n_pairs, seed), discount), precision), None
    n_state = len(compiled.calls[0][1])
    pilot = sc.script_request(compiled, make_sim(pilot_paths(2 * n_pairs) // 2, seed ^ PILOT_KEY), discount,
                              call_mode=1)
    sc.run(pilot, precision)
    rec = PilotRecord.from_device(pilot.keep[1]["record"], len(compiled.event_times), len(compiled.calls), n_state)
    pay_d = [float(discount(t)) if t is not None and t > 0 else 0.0 for t in compiled.pay_times]
    policy = fit(rec, [k for k, _ in compiled.calls], pay_d)
    held = sc.script_request(compiled, make_sim(n_pairs, seed), discount, call_mode=2, rules=policy.pack(n_state))
    return sc.run(held, precision), policy
