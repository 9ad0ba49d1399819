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
