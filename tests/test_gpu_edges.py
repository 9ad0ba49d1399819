"""Edge sizes on the GPU against the oracle: pair counts that fill no warp or leave the last one ragged, a single time
step, the first pair far into the stream, and a local-variance table as large as the reference's own rows (801
points for each of 756 steps, RN/src/optlab/native/__init__.py:129-144): more than the kernels' shared-memory stage
holds, so the path, fused and script kernels read the rows from global memory. FP64 within the tolerances of the
parity tests, FP32 within 4 standard errors of the FP64 oracle."""

import numpy as np
import pytest

from optlab_b200 import engine, workloads
from optlab_b200 import script as sc
from optlab_b200.requests import paths_request

pytestmark = pytest.mark.gpu


def _paths(kinds, n_pairs, n_steps=40, first_pair=0, n_x=101, seed=4242):
    n = len(kinds)
    rng = np.random.default_rng(1)
    corr = np.full((n, n), 0.4) + 0.6 * np.eye(n)
    table = (0.04 + 0.02 * np.cos(np.linspace(0, 2, n_x)))[None, :] * (1 + 0.2 * rng.random((n_steps, n_x)))
    obs = sorted({0, n_steps // 2, n_steps})
    return dict(dt=np.full(n_steps, 1 / 252), t0=np.arange(n_steps) / 252, obs_step=obs,
                root=np.linalg.cholesky(corr), kind=kinds, cvar=np.full(n, 0.04),
                heston=np.tile([0.04, 1.5, 0.04, 0.5, -0.7], n), same=1,
                fwd=np.tile(100.0 + np.arange(len(obs)), n).reshape(n, len(obs)), n_pairs=n_pairs, seed=seed,
                first_pair=first_pair, step_row=np.tile(np.arange(n_steps), n), lo=np.full(n_steps, -1.0),
                inv_dx=np.full(n_steps, (n_x - 1) / 2.0), table=table, n_x=n_x, win_lo=[0], win_hi=[len(obs) - 1])


def _out(held):
    return next(a for a in held.keep if isinstance(a, np.ndarray) and a.ndim == 3)


def _match(g, o, kinds):
    rel = np.abs(_out(g) / _out(o) - 1.0)
    if any(k in (2, 3) for k in kinds):
        # a variance within rounding of zero may be truncated on one side only
        assert np.median(rel) < 1e-13 and np.quantile(rel, 0.999) < 1e-9, rel.max()
    else:
        assert rel.max() < 1e-12, rel.max()


@pytest.mark.parametrize("n_pairs", [1, 33, 4097])
@pytest.mark.parametrize("kinds", [[1], [3, 3, 1]], ids=["lv", "slv,slv,lv"])
def test_paths_at_ragged_pair_counts_match_the_oracle(oracle, kinds, n_pairs):
    kw = _paths(kinds, n_pairs, first_pair=2**31 + 5)
    g, o = paths_request(**kw), paths_request(**kw)
    engine.paths(g, "fp64")
    oracle.paths(o)
    assert _out(g).shape[-1] == 2 * n_pairs
    _match(g, o, kinds)


@pytest.mark.parametrize("kinds", [[1], [2, 1]], ids=["lv", "heston,lv"])
def test_paths_of_a_single_step_match_the_oracle(oracle, kinds):
    kw = _paths(kinds, 100, n_steps=1)
    g, o = paths_request(**kw), paths_request(**kw)
    engine.paths(g, "fp64")
    oracle.paths(o)
    _match(g, o, kinds)


def _phoenix(n_pairs, grid=None, seed=5):
    return workloads.lv_phoenix(n_paths=2 * n_pairs, seed=seed, grid=grid)


@pytest.mark.parametrize("n_pairs", [2, 31, 1025])
def test_fused_phoenix_at_ragged_pair_counts_matches_the_oracle(oracle, n_pairs):
    g = engine.mc_price(_phoenix(n_pairs), "fp64")
    o = oracle.mc_price(_phoenix(n_pairs))
    for k in range(o.n_out):  # value, called, knocked in, coupons: a fraction of 0 is exactly 0 on both
        assert abs(g.price[k] - o.price[k]) <= 1e-10 * abs(o.price[k]), (k, g.price[k], o.price[k])
    # the value's SE (the indicator outputs may have none: a variance of rounding residuals is not compared)
    assert abs(g.se[0] - o.se[0]) <= 1e-8 * o.se[0], (g.se[0], o.se[0])


@pytest.fixture(scope="module")
def reference_size_grid():
    """The benchmark surface tabulated as the reference does: one 801-point row for each of the 756 daily steps."""
    return workloads.LocalVarGrid.from_surface(workloads.lv_surface(horizon=3.0), 3.0 * np.arange(1, 757) / 756, 801)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_paths_on_a_reference_size_table_match_the_oracle(oracle, reference_size_grid, prec):
    """The drop-in path kernel with the rows left in global memory: quarterly columns and a window over them."""
    g = reference_size_grid
    n_steps = 756
    dt, t0 = workloads.uniform_grid(3.0, n_steps)
    t_end = np.concatenate([[0.0], t0 + dt])
    obs = np.arange(0, n_steps + 1, 63)
    m = workloads.FlatMarket(100.0, 0.02, 0.01)
    kw = dict(dt=dt, t0=t0, obs_step=obs, root=[[1.0]], kind=[1], cvar=[0.0], heston=[0.0, 1, 1, 0, 0], same=1,
              fwd=m.F(t_end[obs])[None, :], n_pairs=2**12, seed=9, step_row=g.row_of(t0), lo=g.lo, inv_dx=g.inv_dx,
              table=g.rows, n_x=g.n_x, win_lo=[0], win_hi=[len(obs) - 1])
    assert len(np.unique(g.row_of(t0))) > 700  # a row for (nearly) every step
    gh, oh = paths_request(**kw), paths_request(**kw)
    engine.paths(gh, prec)
    oracle.paths(oh)
    rel = np.abs(_out(gh) / _out(oh) - 1.0)
    if prec == "fp64":
        assert rel.max() < 1e-12, rel.max()
    else:
        assert np.median(rel) < 1e-6 and rel.max() < 1e-4, (np.median(rel), rel.max())


def test_a_table_larger_than_the_shared_memory_stage_prices_like_the_oracle(oracle, reference_size_grid):
    held = _phoenix(2**12, reference_size_grid)
    assert held.struct.n_rows == 756 and held.struct.n_x == 801  # 4.8 MB of float (value, slope) pairs: global
    g64 = engine.mc_price(held, "fp64")
    o = oracle.mc_price(_phoenix(2**12, reference_size_grid))
    assert abs(g64.price[0] / o.price[0] - 1) < 1e-10, (g64.price[0], o.price[0])
    g32 = engine.mc_price(_phoenix(2**12, reference_size_grid), "fp32")
    assert abs(g32.price[0] - o.price[0]) < 4 * o.se[0], (g32.price[0], o.price[0], o.se[0])


def test_a_script_at_a_ragged_pair_count_matches_the_oracle(oracle):
    from test_gpu_script import CASES, _disc, _oracle_price, _simulation

    case = CASES["phoenix"]
    comp = sc.compile_script(case["script"], case["params"], case["smoothing"], case["valuation"])
    sim, grid = _simulation(comp, case["spot0"], n_pairs=45)
    res = sc.run(sc.script_request(comp, sim, _disc), "fp64")
    want, se, _ = _oracle_price(case, comp, sim, grid, oracle)
    assert res.n_paths == 90
    assert abs(res.price - want) <= 1e-10 * max(abs(want), 1e-3), (res.price, want)
    assert abs(res.se - se) <= 1e-6 * se + 1e-15


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_a_script_on_a_reference_size_table_equals_the_fused_kernel(reference_size_grid, prec):
    """The Phoenix as a payoff script with the rows left in global memory, against the fused kernel on the same rows
    (itself checked against the oracle above): FP64 to rounding, FP32 within 4 standard errors."""
    from test_gpu_script import _phoenix_script

    ph = workloads.Phoenix()
    held = _phoenix(2**12, reference_size_grid)
    comp = sc.compile_script(_phoenix_script(ph, 252), params={"S0": float(held.struct.spot[0])})
    fused = engine.mc_price(_phoenix(2**12, reference_size_grid), "fp64")
    res = sc.run(sc.script_request(comp, held, lambda t: np.exp(-0.02 * t)), prec)
    if prec == "fp64":
        assert abs(res.price - fused.price[0]) <= 1e-10 * abs(fused.price[0]), (res.price, fused.price[0])
    else:
        assert abs(res.price - fused.price[0]) < 4 * fused.se[0], (res.price, fused.price[0], fused.se[0])


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("kinds,same", [([2, 2], 1), ([2, 2, 2], 0), ([3, 3], 1), ([3, 3, 3], 0), ([0] * 5, 1)],
                         ids=["heston x2", "heston x3 independent", "slv x2", "slv x3 independent", "bs x5"])
def test_baskets_of_one_kind_on_the_staged_path_kernel_match_the_oracle(oracle, kinds, same, prec):
    """Names of one kind run the staged path kernel (Heston residuals from stream 0, SLV residuals from the aux
    stream, correlated through the root when `same`; Black-Scholes at its constant variance): FP64 to the Heston
    criterion of the parity tests, FP32 to the reference's float criterion
    (packages/native/tests/test_native.py:95-111)."""
    kw = dict(_paths(kinds, 2048, n_steps=60), same=same)
    g, o = paths_request(**kw), paths_request(**kw)
    engine.paths(g, prec)
    oracle.paths(o)
    rel = np.abs(_out(g) / _out(o) - 1.0)
    if prec == "fp64":
        assert np.median(rel) < 1e-13 and np.quantile(rel, 0.999) < 1e-9, (np.median(rel), rel.max())
    else:
        assert np.median(rel) < 1e-5 and np.mean(rel > 1e-3) < 0.06, (np.median(rel), np.mean(rel > 1e-3))


def test_one_shot_calls_reuse_device_buffers_without_changing_their_results():
    """One-shot calls hand their device buffers to the next call; interleaved calls of other sizes and kinds (which
    take and return those buffers) leave every result bit-identical to its first run."""
    kw = _paths([1, 1], 3000, n_steps=30)
    first = paths_request(**kw)
    engine.paths(first, "fp64")
    m1 = engine.mc_price(_phoenix(1500), "fp64")
    for n_pairs in (50, 5000, 3000):
        engine.paths(paths_request(**_paths([3], n_pairs, n_steps=20)), "fp32")
        engine.mc_price(_phoenix(n_pairs), "fp32")
        again = paths_request(**kw)
        engine.paths(again, "fp64")
        assert np.array_equal(_out(again), _out(first))
        m2 = engine.mc_price(_phoenix(1500), "fp64")
        assert list(m2.price[: m2.n_out]) == list(m1.price[: m1.n_out])
        assert list(m2.se[: m2.n_out]) == list(m1.se[: m1.n_out])


def test_calls_after_the_buffer_cache_is_released_price_as_before():
    """ob_release_buffers empties the one-shot calls' buffer cache (what a caller does before resetting a device);
    the next call allocates again and gives the same prices."""
    from optlab_b200 import _abi

    lib = _abi.load()
    first = engine.mc_price(workloads.lv_phoenix(n_paths=2**14, seed=5), "fp64")
    _abi.check(lib.ob_release_buffers())
    _abi.check(lib.ob_release_buffers())  # an empty cache is fine too
    again = engine.mc_price(workloads.lv_phoenix(n_paths=2**14, seed=5), "fp64")
    assert list(first.price[: first.n_out]) == list(again.price[: again.n_out])
