"""The issuer's call without a GPU: the oracle's pilot record, the Longstaff-Schwartz fit of optlab_b200.exercise and
the policy applied out of sample equal the reference's (optlab.structured.exercise) on its recorded case
(tests/golden/script_callable.json)."""

import json
from pathlib import Path

import numpy as np
import pytest

from optlab_b200 import exercise
from optlab_b200 import script as sc

CASE = json.loads((Path(__file__).resolve().parent / "golden" / "script_callable.json").read_text())
R = 0.02


def _disc(t):
    return float(np.exp(-R * t))


class Paths:
    def __init__(self, paths):
        self.times = np.asarray(CASE["times"])
        self.paths = {k: np.asarray(v) for k, v in paths.items()}
        self.n = next(iter(self.paths.values())).shape[0]

    def col(self, name, t):
        if t <= 0:
            return np.full(self.n, CASE["spot0"][name])
        k = int(np.argmin(np.abs(self.times - t)))
        return self.paths[name][:, k]

    def spot(self, name, t):
        return self.col(name, t)

    def fixings(self, name, times):
        return np.stack([self.col(name, t) for t in times], axis=1)


def _oracle():
    from script_oracle import ScriptOracle

    return ScriptOracle(CASE["script"], discount=_disc)


def _record():
    p = Paths(CASE["pilot"])
    res = _oracle().run(p.n, p.spot, p.fixings, mode="record")
    return exercise.PilotRecord(res["pre"], res["post"], res["mask"], res["alive"], res["amount"], res["state"])


def test_the_oracles_pilot_record_is_the_references():
    rec, want = _record(), CASE["record"]
    for k in ("pre", "post", "mask", "alive", "amount", "state"):
        assert np.allclose(getattr(rec, k), np.asarray(want[k]), rtol=1e-12, atol=1e-14), k


def test_the_fit_is_the_references():
    comp = sc.compile_script(CASE["script"])
    pay_d = [_disc(t) if t is not None and t > 0 else 0.0 for t in comp.pay_times]
    policy = exercise.fit(_record(), [k for k, _ in comp.calls], pay_d)
    assert policy.in_sample == pytest.approx(CASE["in_sample"], rel=1e-12)
    assert len(policy.rules) == len(CASE["rules"]) == 3
    for mine, ref in zip(policy.rules, CASE["rules"]):
        assert mine.powers == tuple(tuple(p) for p in ref["powers"])
        assert len(mine.knots) == len(ref["knots"])
        assert np.allclose([k for _, k in mine.knots], [k for _, k in ref["knots"]], rtol=1e-12)
        assert np.allclose(mine.mean, ref["mean"], rtol=1e-13) and np.allclose(mine.scale, ref["scale"], rtol=1e-13)
        assert np.allclose(mine.coef, ref["coef"], rtol=1e-7, atol=1e-9)


def test_the_policy_applied_out_of_sample_is_the_references():
    comp = sc.compile_script(CASE["script"])
    pay_d = [_disc(t) if t is not None and t > 0 else 0.0 for t in comp.pay_times]
    policy = exercise.fit(_record(), [k for k, _ in comp.calls], pay_d)
    p = Paths(CASE["pricing"])
    res = _oracle().run(p.n, p.spot, p.fixings, mode="apply", rules=policy.rules)
    assert np.allclose(res["pv"], CASE["pv"], rtol=1e-12, atol=1e-14)
    assert not res["bad_redemption"].any()


def test_the_packed_rules_hold_every_term():
    comp = sc.compile_script(CASE["script"])
    pay_d = [_disc(t) if t is not None and t > 0 else 0.0 for t in comp.pay_times]
    policy = exercise.fit(_record(), [k for k, _ in comp.calls], pay_d)
    packed = policy.pack(2)
    assert packed.shape == (3, 224)
    for c, r in enumerate(policy.rules):
        row = packed[c]
        assert row[0] == 1 and row[1] == len(r.powers) and row[2] == len(r.knots)
        assert np.array_equal(row[161:161 + len(r.coef)], r.coef)
        assert np.array_equal(row[11:11 + 4 * len(r.powers)].reshape(-1, 4)[:, :2], np.array(r.powers))
    assert comp.calls[0][0] == 0 and [k for k, _ in comp.calls] == [0, 1, 2]
    assert exercise.pilot_paths(2**15) == 20000 and exercise.pilot_paths(2**20) == 100000


def test_packed_rules_unpack_to_the_same_policy():
    """The device fit returns packed rules (the layout call mode 2 reads): unpacking them gives the rules back, a row
    of zeros a call without a rule."""
    comp = sc.compile_script(CASE["script"])
    pay_d = [_disc(t) if t is not None and t > 0 else 0.0 for t in comp.pay_times]
    policy = exercise.fit(_record(), [k for k, _ in comp.calls], pay_d)
    packed = policy.pack(2)
    back = exercise.Policy.unpack(packed, 2, policy.pilot_paths, policy.in_sample)
    assert back == policy
    packed[1] = 0.0
    assert exercise.Policy.unpack(packed, 2, 0).rules[1] is None


DUAL = json.loads((Path(__file__).resolve().parent / "golden" / "script_dual.json").read_text())


def _columns(paths, times, spot0):
    def col(name, t):
        if t <= 0:
            return np.full(paths.shape[0], spot0)
        return paths[:, int(np.argmin(np.abs(times - t)))]

    return col, lambda name, ts: np.stack([col(name, t) for t in ts], axis=1)


def _rule(r):
    if r is None:
        return None
    return exercise.Rule(tuple(r["mean"]), tuple(r["scale"]), tuple(tuple(p) for p in r["powers"]),
                         tuple(tuple(k) for k in r["knots"]), tuple(r["coef"]))


def test_the_dual_recursion_on_the_references_draws_gives_the_references_bound():
    """The reference's dual bound (exercise.py:294-380) on 40 outer paths x 16 continuations, redone here on the
    same draws: the oracle evaluator records the outer paths and values the continuations under the forced policy,
    exercise.dual_recursion takes the martingale dual; the gap and its SE equal the reference's."""
    from script_oracle import ScriptOracle

    times = np.asarray(DUAL["times"])
    outer = np.asarray(DUAL["outer"])
    n_outer, n_inner = outer.shape[0], DUAL["n_inner"]
    r = DUAL["r"]
    disc = lambda t: float(np.exp(-r * t))  # noqa: E731
    o = ScriptOracle(DUAL["script"], {}, 0.0, None, disc)
    rec = o.run(n_outer, *_columns(outer, times, 100.0), mode="record")
    rules = [_rule(x) for x in DUAL["rules"]]
    policy = exercise.Policy(tuple(rules), 0)
    comp = sc.compile_script(DUAL["script"])
    call_events = [k for k, _ in comp.calls]
    pay_d = [disc(t) if t is not None and t > 0 else 0.0 for t in comp.pay_times]
    H = []
    for c, k in enumerate(call_events):
        col = int(np.searchsorted(times, comp.event_times[k], side="right")) - 1
        tail = np.asarray(DUAL["tails"][c])
        paths = np.concatenate([np.repeat(outer[:, : col + 1], n_inner, axis=0), tail], axis=1)
        forced = [None if j <= c else rules[j] for j in range(len(rules))]
        res = o.run(paths.shape[0], *_columns(paths, times, 100.0), mode="apply", rules=forced)
        H.append(res["pv"].reshape(n_outer, n_inner).mean(axis=1))
    pilot = exercise.PilotRecord(rec["pre"], rec["post"], rec["mask"], rec["alive"], rec["amount"], rec["state"])
    best = exercise.dual_recursion(rec["pre"], rec["post"], rec["mask"], rec["alive"], rec["amount"],
                                   exercise.decisions(policy, pilot), call_events,
                                   [pay_d[k] if pay_d[k] > 0 else 1.0 for k in call_events], H, DUAL["price0"])
    gap = DUAL["price0"] - best.mean()
    assert gap == pytest.approx(DUAL["small"]["gap"], rel=1e-10, abs=1e-14)
    assert best.std(ddof=1) / np.sqrt(n_outer) == pytest.approx(DUAL["small"]["gap_se"], rel=1e-10)


def test_the_references_bound_brackets_its_pde_value():
    """The fixture's own sanity: the reference's bound at 1000 x 200 is below the PDE value within 4 SE, and the
    policy's price above it within 4 SE plus the policy's 10 bp bias allowance."""
    big, pde = DUAL["big"], DUAL["pde"]
    assert big["lower"] < pde + 4 * big["lower_se"]
    assert DUAL["price0"] > pde - 4 * DUAL["price_se"]
    assert -4 * big["gap_se"] < big["gap"] < 0.001
