"""The implied-vol node vegas' restatement against the reference's own risk grid (tests/golden/reference_greeks.json,
made by tests/golden/make_greeks_fixtures.py from packages/risk/src/optlab/risk/grid.py and surfaces.py): the strike
and tenor tents, the tent-bumped local-variance tables the reference's engine reads, and the analytic derivative of
those tables in a node's amplitude against the reference's own central difference."""

import json
from pathlib import Path

import numpy as np
import pytest

from optlab_b200 import ivnodes
from optlab_b200.surfaces import SSVI

FIX = json.loads((Path(__file__).resolve().parent / "golden" / "reference_greeks.json").read_text())


def _surface(name):
    a = FIX["names"].index(name)
    T = 3.0 * np.arange(1, 41) / 40
    return SSVI.power_law(FIX["rho"][a], 1.0, 0.5, T, FIX["c_rate"][a] * T)


def test_the_tents_are_the_reference_grids():
    t = FIX["tents"]
    k, T = np.meshgrid(np.array(t["k"]), np.array(t["T"]), indexing="ij")
    for mine, theirs in zip(ivnodes.strike_tents(k, T), t["strike"]):
        assert np.max(np.abs(mine - np.array(theirs))) < 1e-13
    for mine, theirs in zip(ivnodes.tenor_tents(np.array(t["T"])), t["tenor"]):
        assert np.max(np.abs(mine - np.array(theirs))) < 1e-13
    # both families are partitions of unity: every node bumped by h is the parallel bump h
    phi = ivnodes.strike_tents(k, T)[0]
    assert np.allclose(phi.sum(0), 1.0, atol=1e-13)


def test_tent_bumped_tables_are_the_references():
    tb = FIX["tables"]
    surf = _surface(tb["name"])
    t0 = np.arange(252) / 252.0
    steps, pts = np.array(tb["steps"]), np.array(tb["points"])
    lo, inv, base = ivnodes.bumped_table(surf, t0, 801, np.zeros((10, 8)))
    assert np.allclose(lo[steps], tb["lo"], rtol=1e-14) and np.allclose(inv[steps], tb["inv_dx"], rtol=1e-14)
    assert np.max(np.abs(base[np.ix_(steps, pts)] / np.array(tb["base"]) - 1)) < 1e-12
    for nd in tb["nodes"]:
        i, j = nd["node"]
        for sgn, key in ((1.0, "plus"), (-1.0, "minus")):
            H = np.zeros((10, 8))
            H[i, j] = sgn * tb["h"]
            _, _, rows = ivnodes.bumped_table(surf, t0, 801, H)
            ref = np.array(nd[key])
            assert np.max(np.abs(rows[np.ix_(steps, pts)] / ref - 1)) < 1e-11, (i, j, key)


@pytest.mark.parametrize("which", [0, 1, 2])
def test_the_table_derivative_in_a_node_is_the_references_central_difference(which):
    tb = FIX["tables"]
    nd = tb["nodes"][which]
    i, j = nd["node"]
    surf = _surface(tb["name"])
    t0 = np.arange(252) / 252.0
    steps, pts = np.array(tb["steps"]), np.array(tb["points"])
    J_all = ivnodes.node_table_derivative(surf, t0, 801, i, j)
    J = J_all[np.ix_(steps, pts)]
    # the reference's central difference at h = 1e-4 carries its O(h^2) truncation: at most 3e-5 of the largest entry
    fd = (np.array(nd["plus"]) - np.array(nd["minus"])) / (2 * tb["h"])
    scale = np.abs(fd).max()
    assert scale > 0
    assert np.max(np.abs(J - fd)) <= 1e-4 * scale, np.max(np.abs(J - fd)) / scale
    # and the whole table against the exact bumped tables (pinned to the reference's above) at h = 1e-6
    H = np.zeros((10, 8))
    H[i, j] = 1e-6
    fd6 = (ivnodes.bumped_table(surf, t0, 801, H)[2] - ivnodes.bumped_table(surf, t0, 801, -H)[2]) / 2e-6
    assert np.max(np.abs(J_all - fd6)) <= 1e-7 * np.abs(fd6).max()


def test_contracting_a_gradient_sums_the_node_derivatives():
    surf = _surface("A")
    t0 = np.arange(60) / 252.0
    rng = np.random.default_rng(2)
    G = rng.normal(size=(60, 101))
    vega = ivnodes.node_jacobian_contract(G, surf, t0, 101)
    for i, j in ((5, 1), (3, 0), (9, 2)):
        direct = 0.01 * np.sum(G * ivnodes.node_table_derivative(surf, t0, 101, i, j))
        assert abs(vega[i, j] - direct) <= 1e-12 * max(abs(direct), 1e-300)
