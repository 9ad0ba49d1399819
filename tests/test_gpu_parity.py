"""The engine on the GPU against the oracle (the C restatement of the reference's algorithms), on the same random
numbers: Philox integer streams bit for bit, FP64 results within 1e-10 relative, FP32 results within the reference's
own float-against-double criteria (packages/native/tests/test_native.py:95-111, RC/tests/test_paths.cpp:141-168)."""

import numpy as np
import pytest

from optlab_b200 import engine, workloads
from optlab_b200._abi import AUX_STREAM
from optlab_b200.requests import mc_request, paths_request

pytestmark = pytest.mark.gpu


def out_of(held):
    return next(a for a in held.keep if isinstance(a, np.ndarray) and a.ndim == 3)


# ------------------------------------------------------------------------------------------------------ Philox


@pytest.mark.parametrize(
    "seed,first_pair,tag,first_block",
    [(20261105, 0, 0, 0), (2**63 + 12345, 2**33 + 7, AUX_STREAM, 2**32 - 2), (1, 123456, 0, 500)],
)
def test_philox_integer_streams_are_bit_exact(oracle, seed, first_pair, tag, first_block):
    u, z64, z32 = engine.philox_normals(seed, first_pair, 64, tag, first_block, 8)
    ou, oz = oracle.philox_normals(seed, first_pair, 64, tag, first_block, 8)
    assert np.array_equal(u, ou)
    assert np.max(np.abs(z64 - oz)) < 1e-13  # sincospi against cos/sin(2 pi v): libm rounding only
    assert np.max(np.abs(z32 - oz)) < 2e-5  # float Box-Muller (|z| <= 6.7)


def test_float_normals_over_four_million_draws(oracle):
    """The float normals against the double ones over 2^14 pairs x 64 blocks: where the radius r = sqrt(-2 ln u) is
    at least 0.1 they stay within 1e-5 of r (the angle's hardware sine and cosine, measured 3e-6); below it the float
    u near 1 (spaced 2^-24, as the reference's float definition has it) sets the error, within 1e-4 absolute
    (measured 1.6e-5)."""
    u, _, z32 = engine.philox_normals(20261105, 0, 16384, 0, 0, 64)
    _, oz = oracle.philox_normals(20261105, 0, 16384, 0, 0, 64)
    err = np.abs(z32 - oz).reshape(-1, 2).max(axis=1)  # the two normals of one Box-Muller draw
    r = np.sqrt(-2.0 * np.log((u.reshape(-1, 2)[:, 0].astype(np.float64) + 0.5) * 2.0**-32))
    big = r >= 0.1
    assert np.max(err[big] / r[big]) < 1e-5, np.max(err[big] / r[big])
    assert np.max(err) < 1e-4, np.max(err)


# ------------------------------------------------------------------------------------------------------ paths


def _paths_case(kinds, n_steps=60, n_pairs=4096, mixer=0, same=1, n_x=101, seed=987654321, first_pair=11):
    n = len(kinds)
    rng = np.random.default_rng(0)
    dt, t0 = np.full(n_steps, 1 / 252), np.arange(n_steps) / 252
    corr = np.full((n, n), 0.5) + 0.5 * np.eye(n)
    root = np.linalg.cholesky(corr)
    table = (0.04 + 0.02 * np.sin(np.linspace(0, 3, n_x)))[None, :] * (1 + 0.1 * rng.random((n_steps, n_x)))
    kw = dict(
        dt=dt,
        t0=t0,
        obs_step=[0, 10, 25, n_steps],
        root=root,
        kind=kinds,
        cvar=np.full(n, 0.04),
        heston=np.tile([0.04, 1.5, 0.04, 0.5, -0.7], n),
        same=same,
        fwd=np.tile([100.0, 101.0, 102.0, 103.0], n).reshape(n, 4),
        n_pairs=n_pairs,
        seed=seed,
        first_pair=first_pair,
        step_row=np.tile(np.arange(n_steps), n),
        lo=np.full(n_steps, -1.0),
        inv_dx=np.full(n_steps, (n_x - 1) / 2.0),
        table=table,
        n_x=n_x,
        win_lo=[1],
        win_hi=[3],
    )
    if mixer:
        kw.update(mixer=1, mix=(0.3, 0.0, 0.3, 0.1, 0.15, 1.0, np.cos(0.2), np.sin(0.2)), low_root=root)
    return kw


CASES = {
    "bs": dict(kinds=[0]),
    "lv": dict(kinds=[1]),
    "heston": dict(kinds=[2]),
    "slv": dict(kinds=[3]),
    "lv+heston": dict(kinds=[1, 2]),
    "slv,slv,lv": dict(kinds=[3, 3, 1]),
    "five lv": dict(kinds=[1, 1, 1, 1, 1]),
    "local correlation": dict(kinds=[1, 1, 1], mixer=1),
    "black-scholes basket, local correlation": dict(kinds=[0, 0, 0, 0], mixer=1),
    "five lv, local correlation": dict(kinds=[1, 1, 1, 1, 1], mixer=1),
    "independent residuals": dict(kinds=[3, 2, 1, 0], same=0),
    "eight names, local correlation": dict(kinds=[1, 1, 3, 1, 0, 1, 3, 1], mixer=1),
    "eight names, independent residuals": dict(kinds=[3, 2, 1, 0, 3, 2, 1, 1], same=0),
}


@pytest.mark.parametrize("name", list(CASES))
def test_fp64_paths_match_the_oracle(oracle, name):
    kw = _paths_case(**CASES[name])
    g, o = paths_request(**kw), paths_request(**kw)
    engine.paths(g, "fp64")
    oracle.paths(o)
    rel = np.abs(out_of(g) / out_of(o) - 1.0)
    if any(k in (2, 3) for k in CASES[name]["kinds"]):
        # a variance within rounding of zero may be truncated on one side only: the paths then part by ~1e-10
        assert np.median(rel) < 1e-13 and np.quantile(rel, 0.999) < 1e-9, (np.median(rel), rel.max())
    else:
        assert rel.max() < 1e-12, rel.max()


@pytest.mark.parametrize("name", list(CASES))
def test_fp32_paths_match_the_oracle_within_the_references_float_criteria(oracle, name):
    kw = _paths_case(**CASES[name])
    g, o = paths_request(**kw), paths_request(**kw)
    engine.paths(g, "fp32")
    oracle.paths(o)
    rel = np.abs(out_of(g) / out_of(o) - 1.0)
    if any(k in (2, 3) for k in CASES[name]["kinds"]):
        assert np.median(rel) < 1e-5 and np.mean(rel > 1e-3) < 0.06, (np.median(rel), np.mean(rel > 1e-3))
    else:
        assert np.median(rel) < 1e-6 and rel.max() < 1e-4, (np.median(rel), rel.max())


def test_a_daily_window_gives_the_extremes_of_the_full_columns():
    """RC/tests/test_paths.cpp:114-139 on the GPU: lowest, highest and last spot of a reduced daily window equal those
    of the full columns, bit for bit."""
    n_steps, pairs = 252, 4000
    base = dict(
        dt=np.full(n_steps, 1 / 252),
        t0=np.arange(n_steps) / 252,
        obs_step=np.arange(1, n_steps + 1),
        root=[[1.0]],
        kind=[2],
        cvar=[0.0],
        heston=[0.0228, 3.09, 0.0537, 1.31, -0.69],
        same=1,
        fwd=np.full((1, n_steps), 100.0),
        n_pairs=pairs,
        seed=20261105,
    )
    for prec in ("fp32", "fp64"):
        full = paths_request(**base)
        col_of = np.full(n_steps, -1)
        col_of[-1] = 0
        red = paths_request(**base, col_of=col_of, n_keep=1, win_lo=[0], win_hi=[n_steps - 1])
        engine.paths(full, prec)
        engine.paths(red, prec)
        F, Rd = out_of(full)[0], out_of(red)[0]
        assert np.array_equal(Rd[1], F.min(axis=0)) and np.array_equal(Rd[2], F.max(axis=0))
        assert np.array_equal(Rd[0], F[-1])


def test_paths_depend_on_the_seed_and_the_global_pair_only():
    kw = _paths_case([3, 1], n_pairs=2000, first_pair=0)
    whole = paths_request(**kw)
    engine.paths(whole, "fp32")
    kw2 = dict(kw, n_pairs=1000, first_pair=1000)
    tail = paths_request(**kw2)
    engine.paths(tail, "fp32")
    W, T = out_of(whole), out_of(tail)
    # pair 1000 + i of the whole run is pair i of the tail, in both legs
    assert np.array_equal(W[:, :, 1000:2000], T[:, :, :1000])
    assert np.array_equal(W[:, :, 3000:4000], T[:, :, 1000:2000])


@pytest.mark.parametrize("kinds", [[1], [3, 1]])
def test_a_large_output_read_back_in_chunks_equals_the_same_pairs_in_two_calls(kinds):
    """Outputs of 32 MB and more come back in four chunks on two streams (one chunk's kernel running while the
    previous chunk is copied); each half of the pairs, asked for alone, is one chunk: the same columns bit for bit
    (the local-vol kernel and the generic one)."""
    n = 2**19
    kw = _paths_case(kinds, n_pairs=n, first_pair=0)
    whole = paths_request(**kw)
    engine.paths(whole, "fp32")
    W = out_of(whole)
    assert W.nbytes >= 32 << 20
    for f in (0, n // 2):
        part = paths_request(**dict(kw, n_pairs=n // 2, first_pair=f))
        engine.paths(part, "fp32")
        P = out_of(part)
        assert np.array_equal(W[:, :, f:f + n // 2], P[:, :, : n // 2])
        assert np.array_equal(W[:, :, n + f:n + f + n // 2], P[:, :, n // 2:])


# ------------------------------------------------------------------------------------------------------ fused


def _rel(a, b):
    return np.abs(np.asarray(a) / np.asarray(b) - 1.0)


def test_heston_qe_ladder_fp64_matches_the_oracle(oracle):
    g = workloads.heston_qe_ladder(n_paths=2**15, seed=3)
    o = workloads.heston_qe_ladder(n_paths=2**15, seed=3)
    rg, ro = engine.mc_price(g, "fp64"), oracle.mc_price(o)
    pg, po = np.array(rg.price[: rg.n_out]), np.array(ro.price[: ro.n_out])
    sg, so = np.array(rg.se[: rg.n_out]), np.array(ro.se[: ro.n_out])
    assert rg.n_out == 13 and rg.n_paths == 2**15
    assert _rel(pg, po).max() < 1e-10, _rel(pg, po)
    assert _rel(sg, so).max() < 1e-8, _rel(sg, so)


def test_heston_qe_ladder_fp32_is_within_4_se_and_1e4_of_fp64(oracle):
    g = workloads.heston_qe_ladder(n_paths=2**16, seed=1)
    o = workloads.heston_qe_ladder(n_paths=2**16, seed=1)
    rg, ro = engine.mc_price(g, "fp32"), oracle.mc_price(o)
    n = ro.n_out
    pg, po, so = np.array(rg.price[:n]), np.array(ro.price[:n]), np.array(ro.se[:n])
    assert np.all(np.abs(pg - po) < 4 * so)
    big = po > 1.0  # relative gaps on prices above 1 (the deep out-of-the-money call is 0.78)
    assert _rel(pg[big], po[big]).max() < 1e-4, _rel(pg, po)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("fp32", 1e-4)])
def test_local_vol_phoenix_matches_the_oracle(oracle, prec, tol):
    g = workloads.lv_phoenix(n_paths=2**14, seed=11)
    o = workloads.lv_phoenix(n_paths=2**14, seed=11)
    rg, ro = engine.mc_price(g, prec), oracle.mc_price(o)
    pg, po, so = np.array(rg.price[:4]), np.array(ro.price[:4]), np.array(ro.se[:4])
    assert abs(pg[0] - po[0]) < 4 * so[0]
    assert _rel(pg[0], po[0]) < tol, (pg, po)
    if prec == "fp64":
        assert _rel(pg, po).max() < 1e-10, (pg, po)


def test_worst_of_phoenix_on_three_correlated_names_fp64_matches_the_oracle(oracle):
    n_steps, n = 252, 3
    corr = np.full((n, n), 0.6) + 0.4 * np.eye(n)
    grid = workloads.lv_grid(horizon=1.0, n_exp=10, n_x=200)
    dt, t0 = workloads.uniform_grid(1.0, n_steps)
    t_end = np.concatenate([[0.0], t0 + dt])
    m = workloads.FlatMarket(100.0, 0.02, 0.01)
    ph = workloads.Phoenix(years=1.0)
    kw = dict(
        model=0,
        dt=dt,
        t0=t0,
        spot=[100.0, 50.0, 20.0],
        n_pairs=2**12,
        seed=5,
        root=np.linalg.cholesky(corr),
        kind=[1, 1, 1],
        cvar=np.zeros(n),
        log_fwd=np.tile(m.log_fwd(t_end), (n, 1)),
        step_row=np.tile(grid.row_of(t0), (n, 1)),
        lo=grid.lo,
        inv_dx=grid.inv_dx,
        table=grid.rows,
        n_x=grid.n_x,
        **workloads.autocall_fields(ph, m, 252),
    )
    rg, ro = engine.mc_price(mc_request(**kw), "fp64"), oracle.mc_price(mc_request(**kw))
    assert _rel(rg.price[:4], ro.price[:4]).max() < 1e-10


def test_a_plan_runs_in_pieces_like_one_call():
    """Prices depend on (seed, pairs) only: two runs of half the pairs (first_pair offset) give the one-call numbers."""
    h = workloads.lv_phoenix(n_paths=2**14, seed=2)
    one = engine.mc_price(h, "fp64")
    with engine.McPlan(h, "fp64") as plan:
        plan.run(2**12, 0)
        plan.run(2**12, 2**12)
        two = plan.result()
    assert two.n_paths == one.n_paths
    assert _rel(two.price[:4], one.price[:4]).max() < 1e-12


def test_a_result_starts_the_next_accumulation():
    """A plan's result reads the runs since the previous result: the first run after it replaces the sums (no
    clearing between calls), later runs add to them, and a result with no run since is empty."""
    h = workloads.lv_phoenix(n_paths=2**13, seed=4)
    one = engine.mc_price(h, "fp64")
    with engine.McPlan(h, "fp64") as plan:
        plan.run(2**12, 0, seed=99)
        plan.result()
        plan.run(2**11, 0)
        plan.run(2**11, 2**11)
        again = plan.result()
        empty = plan.result()
    assert again.n_paths == one.n_paths
    assert _rel(again.price[:4], one.price[:4]).max() < 1e-12  # nothing of the seed-99 run is left in the sums
    assert empty.n_paths == 0 and all(v == 0.0 for v in empty.sum_y[:4])
