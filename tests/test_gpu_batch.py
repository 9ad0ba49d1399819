"""Batched revaluation on the GPU: every (trade, scenario) of a seeded book (spot, carry, vol, skew and correlation
moves) against the oracle's own simulation of it (FP64 within 1e-10 relative, FP32 within 4 standard errors), the
graph replay deterministic and equal to a direct run, the autotuned and per-trade launches equal up to the order of
the sums."""

import numpy as np
import pytest

from optlab_b200._abi import OB_MODEL_HESTON_QE, OB_MODEL_PATHS
from optlab_b200.batch import CARRY_MOVES, CORR_MOVES, Batch, sample_book

pytestmark = pytest.mark.gpu


def _book(seed=3, n=20, **kw):
    args = dict(n_trades=n, seed=seed, paths_log2=(10, 12), years=(1, 2), steps_per_year=52, n_surfaces=8,
                spot_moves=[-0.2, -0.05, 0.05, 0.2], vol_shifts=[-0.05, 0.05], skew_tilts=[-0.1, 0.1],
                carry_moves=CARRY_MOVES, corr_moves=CORR_MOVES)
    args.update(kw)
    return sample_book(**args)


@pytest.fixture(scope="module")
def book():
    return _book()


@pytest.fixture(scope="module")
def want(book, oracle):
    out = [oracle.batch_trade(book, i) for i in range(book.n_trades)]
    return np.array([p for p, _ in out]), np.array([s for _, s in out])


def _close(a, b, rel):
    return np.abs(a - b) <= rel * np.maximum(np.abs(b), 1e-3)


def test_fp64_graph_matches_the_oracle_on_every_scenario(book, want):
    p_ref, se_ref = want
    with Batch(book, "fp64") as b:
        b.capture()
        b.launch()
        price, se, ms = b.result()
    assert ms > 0
    ok = _close(price, p_ref, 1e-10)
    bad = np.argwhere(~ok)
    assert ok.all(), [(book.labels[i], j, price[i, j], p_ref[i, j]) for i, j in bad[:8]]
    assert np.all(_close(se, se_ref, 1e-6))


def test_fp32_is_within_4_standard_errors_of_fp64(book, want):
    p_ref, se_ref = want
    with Batch(book, "fp32") as b:
        b.capture()
        b.launch()
        price, _, _ = b.result()
    gap = np.abs(price - p_ref)
    assert np.all(gap <= 4 * se_ref + 1e-7), gap.max()
    # the float paths move a value by far less than its noise
    assert np.median(gap / np.maximum(se_ref, 1e-12)) < 0.2


def test_replays_are_bit_identical_and_equal_a_direct_run(book):
    with Batch(book, "fp64") as b:
        b.launch()
        direct = b.result()[0]
        b.capture()
        b.launch()
        first = b.result()[0]
        b.launch()
        second = b.result()[0]
    assert np.array_equal(first, second) and np.array_equal(first, direct)


def test_tuned_and_per_trade_runs_agree_with_the_default_shapes(book):
    with Batch(book, "fp64") as b:
        b.launch()
        base = b.result()[0]
        b.run_per_trade()
        per_trade = b.result()[0]
        b.tune()
        b.capture()
        b.launch()
        tuned = b.result()[0]
    assert np.all(_close(per_trade, base, 1e-12)) and np.all(_close(tuned, base, 1e-12))


def test_heston_trades_do_not_move_under_vol_scenarios_and_local_vol_trades_do(book):
    with Batch(book, "fp64") as b:
        b.launch()
        price = b.result()[0]
    v0 = 1 + book.n_spot + book.n_carry
    vol, corr = slice(v0, v0 + book.n_vol), slice(v0 + book.n_vol, None)
    carry = slice(1 + book.n_spot, v0)
    assert book.n_carry == 4 and book.n_corr == 2
    for i, t in enumerate(book.trades):
        if t.model == OB_MODEL_HESTON_QE:
            assert np.all(price[i, vol] == price[i, 0])
        if t.model == OB_MODEL_HESTON_QE or t.n_names == 1:
            assert np.all(price[i, corr] == price[i, 0])
        elif price[i, 0] != 0:
            assert np.all(price[i, corr] != price[i, 0])
        if price[i, 0] != 0:
            assert np.all(price[i, carry] != price[i, 0])  # every trade's forwards and discounting move
    lv = [i for i, t in enumerate(book.trades) if t.model == OB_MODEL_PATHS]
    assert lv and any(np.any(price[i, vol] != price[i, 0]) for i in lv)


def test_rate_up_lowers_a_call_ladder_less_than_its_discount_and_dividends_move_the_other_way(book):
    """Under a 1 % rate rise a call gains forward and loses discount; a 1 % dividend rise only lowers the forward:
    the carry outputs keep the signs of rho and dividend sensitivity on the calls of the book."""
    with Batch(book, "fp64") as b:
        b.launch()
        price = b.result()[0]
    c0 = 1 + book.n_spot
    for i, t in enumerate(book.trades):
        if t.product != 0 or t.n_legs != 1 or book.leg_type[t.leg0] != 1 or book.leg_barrier[t.leg0] != 0:
            continue
        assert price[i, c0 + 2] < price[i, 0] < price[i, c0 + 3]  # dividends up / down
        assert price[i, c0 + 1] < price[i, 0] < price[i, c0]  # rates down / up


def test_a_book_of_every_name_count_and_long_schedules_matches_the_oracle(oracle):
    """Five names, monthly autocalls over five years (60 observations), daily steps, on the oracle in FP64."""
    b = _book(seed=11, n=12, paths_log2=(9, 10), years=(4, 5), steps_per_year=252, heston_share=0.1,
              spot_moves=[-0.1], vol_shifts=[0.02], skew_tilts=[])
    assert max(t.n_names for t in b.trades) >= 4
    with Batch(b, "fp64") as g:
        g.capture()
        g.launch()
        price, se, _ = g.result()
    for i in range(b.n_trades):
        p, s = oracle.batch_trade(b, i)
        assert np.all(_close(price[i], p, 1e-10)), (b.labels[i], price[i], p)
