"""The batched revaluation without a GPU: the seeded book has the benchmark's mix, the oracle's per-trade scenarios
agree with its pinned single-request pricer, and bad batches are refused before any device work."""

import numpy as np
import pytest

from optlab_b200 import _abi
from optlab_b200._abi import OB_MODEL_HESTON_QE, OB_MODEL_PATHS, OB_PRODUCT_AUTOCALL, OB_PRODUCT_LADDER
from optlab_b200.batch import CARRY_MOVES, CORR_MOVES, Batch, moved_corr, sample_book
from optlab_b200.models import correlation_root
from optlab_b200.requests import mc_request


def test_the_benchmark_book_has_the_stated_mix():
    b = sample_book()
    assert b.n_trades == 512 and b.n_spot == 20 and b.n_vol == 40 and b.n_carry == 0 and b.n_corr == 0
    assert b.n_scenarios == 61
    wide = sample_book(n_trades=8, carry_moves=CARRY_MOVES, corr_moves=CORR_MOVES)
    assert wide.n_carry == 4 and wide.n_corr == 2 and wide.n_scenarios == 67
    t = b.trades
    names = np.array([x.n_names for x in t])
    paths = np.array([2 * x.n_pairs for x in t])
    steps = np.array([x.n_steps for x in t])
    assert set(names) == {1, 2, 3, 4, 5}
    assert paths.min() == 2**14 and paths.max() == 2**18
    assert set(steps) == {252 * y for y in range(1, 6)}
    models = {x.model for x in t}
    products = {x.product for x in t}
    assert models == {OB_MODEL_PATHS, OB_MODEL_HESTON_QE} and products == {OB_PRODUCT_LADDER, OB_PRODUCT_AUTOCALL}
    assert all(x.n_names == 1 for x in t if x.model == OB_MODEL_HESTON_QE)
    assert max(x.n_obs for x in t) <= 64
    assert any("barrier" in lab for lab in b.labels) and any("european" in lab for lab in b.labels)
    assert np.allclose(sorted(b.spot_shift), sorted(np.concatenate([-b.spot_shift[10:], b.spot_shift[10:]])))
    assert abs(b.spot_shift).max() == pytest.approx(0.20) and abs(b.spot_shift).min() == pytest.approx(0.01)
    again = sample_book()
    assert [x.seed for x in again.trades] == [x.seed for x in t] and again.labels == b.labels


def _trade_request(book, i, shift=0.0, dr=0.0, dq=0.0, root=None):
    """The trade as an independent ob_mc_request (spot 1), log-forwards moved by ln(1 + shift), the rate by dr (in
    the forwards and the discounting) and the dividend yield by dq, on `root` (default: its own)."""
    t = book.trades[i]
    S, N, E = t.n_steps, t.n_names, book.n_exp
    dt = np.full(S, book.dt)
    t0 = np.arange(S) * book.dt
    T = book.horizon * np.arange(1, E + 1) / E
    rows = np.clip(np.searchsorted(T, t0 + 1e-12, side="right"), 0, E - 1)
    lf = (t.r + dr - t.q - dq) * (np.arange(S + 1) * book.dt) + np.log1p(shift)
    lf[0] = 0.0
    kw = dict(dt=dt, t0=t0, spot=np.ones(N), n_pairs=t.n_pairs, seed=t.seed, r=t.r + dr, q=t.q + dq)
    if t.model == OB_MODEL_PATHS:
        r0 = t.table_row0
        root = book.root[t.root0:t.root0 + N * N].reshape(N, N) if root is None else root
        kw.update(model=OB_MODEL_PATHS, root=root,
                  kind=np.ones(N, np.int32), cvar=np.zeros(N), log_fwd=np.tile(lf, (N, 1)),
                  step_row=np.stack([rows + a * E for a in range(N)]), lo=book.row_lo[r0:r0 + N * E],
                  inv_dx=book.row_inv_dx[r0:r0 + N * E], table=book.table.reshape(-1, book.n_x)[r0:r0 + N * E],
                  n_x=book.n_x)
    else:  # the QE ladder reads the spot: S = spot exp(y)
        kw.update(model=OB_MODEL_HESTON_QE, heston=list(t.heston), spot=[1.0 + shift])
    if t.product == OB_PRODUCT_LADDER:
        sl = slice(t.leg0, t.leg0 + t.n_legs)
        kw.update(product=OB_PRODUCT_LADDER, leg_type=book.leg_type[sl], leg_strike=book.leg_strike[sl],
                  leg_barrier=book.leg_barrier[sl], leg_level=book.leg_level[sl],
                  discount=t.discount * np.exp(-dr * S * book.dt))
    else:
        sl = slice(t.obs0, t.obs0 + t.n_obs)
        disc = book.obs_discount[sl] * np.exp(-dr * book.obs_step[sl] * book.dt)
        kw.update(product=OB_PRODUCT_AUTOCALL, obs_step=book.obs_step[sl], obs_discount=disc,
                  trigger=book.obs_trigger[sl], coupon_barrier=t.coupon_barrier, coupon=t.coupon,
                  ki_barrier=t.ki_barrier, put_strike=t.put_strike, memory=t.memory, ki_daily=t.ki_daily)
    return mc_request(**kw)


def _small(seed=5, n=24, **kw):
    args = dict(n_trades=n, seed=seed, paths_log2=(9, 10), years=(1, 2), steps_per_year=26, n_surfaces=8,
                spot_moves=[-0.2, 0.05], vol_shifts=[0.03], skew_tilts=[-0.05], carry_moves=[], corr_moves=[])
    args.update(kw)
    return sample_book(**args)


def test_the_oracles_batch_scenarios_agree_with_its_single_request_pricer(oracle):
    """or_batch_trade composes the pinned or_mc_price: the base and a spot move (log-forwards moved, which is the
    same path factor wherever the start of the path does not decide the payoff)."""
    b = _small()
    seen = set()
    for i, t in enumerate(b.trades):
        key = (t.model, t.product, t.n_names > 1)
        if key in seen:
            continue
        seen.add(key)
        price, se = oracle.batch_trade(b, i)
        base = oracle.mc_price(_trade_request(b, i))
        want = sum(base.price[:t.n_legs]) if t.product == OB_PRODUCT_LADDER else base.price[0]
        assert abs(price[0] - want) <= 1e-12 * max(1.0, abs(want)), (b.labels[i], price[0], want)
        if t.product == OB_PRODUCT_AUTOCALL:
            assert se[0] == pytest.approx(base.se[0], rel=1e-12)
        if t.model == OB_MODEL_PATHS or t.product == OB_PRODUCT_LADDER:
            up = oracle.mc_price(_trade_request(b, i, 0.05))
            want = sum(up.price[:t.n_legs]) if t.product == OB_PRODUCT_LADDER else up.price[0]
            assert abs(price[2] - want) <= 1e-12 * max(1.0, abs(want)), (b.labels[i], price[2], want)
        if t.model == OB_MODEL_HESTON_QE:
            assert price[3] == price[0] and price[4] == price[0]  # the Heston model ignores the surface
    assert len(seen) >= 5


def test_vol_scenarios_move_local_vol_trades(oracle):
    b = _small()
    i = next(k for k, t in enumerate(b.trades) if t.model == OB_MODEL_PATHS and t.product == OB_PRODUCT_LADDER)
    price, se = oracle.batch_trade(b, i)
    assert price[3] != price[0] and price[4] != price[0]
    assert np.all(np.isfinite(price)) and np.all(se >= 0)


def _break(book, **over):
    for k, v in over.items():
        setattr(book.trades[0], k, v)
    book.__post_init__()
    return book


@pytest.mark.parametrize(
    "over,message",
    [
        (dict(model=3), "trade model must be 0 or 1"),
        (dict(n_names=6), "a trade has 1 to 5 names"),
        (dict(n_steps=0), "a trade needs steps and pairs"),
        (dict(product=7), "product must be 0 or 1"),
    ],
)
def test_bad_batches_are_refused_before_device_work(over, message):
    b = _break(_small(), **over)
    with pytest.raises(_abi.EngineError, match=message):
        Batch(b, "fp64")


def test_too_many_spot_scenarios_are_refused():
    b = sample_book(n_trades=2, seed=1, paths_log2=(9, 9), years=(1, 1), steps_per_year=12, n_surfaces=6,
                    spot_moves=np.linspace(-0.3, 0.3, 32))
    with pytest.raises(_abi.EngineError, match="n_spot must be 0 to 31"):
        Batch(b, "fp32")


def _value(res, t):
    return sum(res.price[:t.n_legs]) if t.product == OB_PRODUCT_LADDER else res.price[0]


def test_the_oracles_carry_and_correlation_scenarios_are_the_moved_trades(oracle):
    """A carry move is the trade priced with the moved rate and dividend yield (forwards and discounting), a
    correlation move the trade on its moved root; single-name and Heston trades keep their base under the latter."""
    carry = [(0.01, 0.0), (0.0, -0.02)]
    b = _small(seed=8, spot_moves=[0.05], vol_shifts=[], skew_tilts=[], carry_moves=carry, corr_moves=[-0.2, 0.15])
    assert b.n_scenarios == 1 + 1 + 2 + 0 + 2
    seen = set()
    for i, t in enumerate(b.trades):
        key = (t.model, t.product, t.n_names > 1)
        if key in seen:
            continue
        seen.add(key)
        price, _ = oracle.batch_trade(b, i)
        for c, (dr, dq) in enumerate(carry):
            want = _value(oracle.mc_price(_trade_request(b, i, dr=dr, dq=dq)), t)
            assert abs(price[2 + c] - want) <= 1e-12 * max(1.0, abs(want)), (b.labels[i], c, price[2 + c], want)
        N = t.n_names
        for k in range(2):
            if t.model == OB_MODEL_PATHS and N > 1:
                root = b.root[t.corr_root0 + k * N * N:t.corr_root0 + (k + 1) * N * N].reshape(N, N)
                want = _value(oracle.mc_price(_trade_request(b, i, root=root)), t)
                assert abs(price[4 + k] - want) <= 1e-12 * max(1.0, abs(want))
                assert price[4 + k] != price[0]
            else:
                assert price[4 + k] == price[0]
    assert len(seen) >= 5


def test_the_books_moved_roots_are_the_moved_correlations():
    b = _small(seed=9, corr_moves=[-0.1, 0.1])
    multi = [t for t in b.trades if t.model == OB_MODEL_PATHS and t.n_names > 1]
    assert multi
    for t in multi:
        N = t.n_names
        base = b.root[t.root0:t.root0 + N * N].reshape(N, N)
        corr = base @ base.T
        for k, m in enumerate((-0.1, 0.1)):
            r = b.root[t.corr_root0 + k * N * N:t.corr_root0 + (k + 1) * N * N].reshape(N, N)
            assert np.allclose(r @ r.T, moved_corr(corr, m), atol=1e-12)
            assert np.allclose(np.diag(r @ r.T), 1.0) and np.allclose((r @ r.T - corr)[~np.eye(N, dtype=bool)], m)


def test_a_move_past_positive_definite_is_clipped_and_repaired():
    c = np.array([[1.0, 0.9, -0.9], [0.9, 1.0, -0.9], [-0.9, -0.9, 1.0]])
    m = moved_corr(c, 0.5)
    assert np.allclose(np.diag(m), 1.0) and np.linalg.eigvalsh(m).min() >= -1e-10
    assert np.abs(m[~np.eye(3, dtype=bool)]).max() <= 0.999
    np.testing.assert_allclose(correlation_root(m) @ correlation_root(m).T, m, atol=1e-10)
    assert np.array_equal(moved_corr(c, 0.0), c)


@pytest.mark.parametrize(
    "kw,message",
    [
        (dict(carry_moves=[(0.01, 0.0)] * 5), "n_carry must be 0 to 4"),
        (dict(spot_moves=np.linspace(-0.3, 0.3, 30), carry_moves=[(0.01, 0.0)] * 2), "1 \\+ n_spot \\+ n_carry"),
        (dict(carry_moves=[(float("nan"), 0.0)]), "carry moves must be finite"),
    ],
)
def test_bad_carry_scenarios_are_refused(kw, message):
    with pytest.raises(_abi.EngineError, match=message):
        Batch(_small(n=3, **kw), "fp32")
