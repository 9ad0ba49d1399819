"""GPU parity of the SLV leverage calibration and of the fixed products (ob_leverage, ob_price) against the oracle,
and of the path engine against the reference's recorded golden vectors."""

import json
from pathlib import Path

import numpy as np
import pytest

from optlab_b200 import _abi, engine
from optlab_b200.leverage import leverage_request
from optlab_b200.requests import paths_request

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "reference_paths.json"


def _lev_kw(local_linear=0, n_pairs=2**14, n_steps=60):
    n_lv = 201
    x = np.linspace(-1, 1, n_lv)
    t0 = np.arange(n_steps) / 100
    return dict(
        dt=np.full(n_steps, 1 / 100),
        t0=t0,
        n_pairs=n_pairs,
        seed=42,
        heston=(0.04, 1.5, 0.04, 0.25, -0.7),
        n_x=64,
        lv_lo=np.full(n_steps, -1.0),
        lv_inv_dx=np.full(n_steps, (n_lv - 1) / 2.0),
        lv_rows=np.array([0.04 * (1 + 0.5 * x**2 - 0.3 * x) * (1 + 0.1 * t) for t in t0]),
        atm_vol=0.2,
        local_linear=local_linear,
        positive_part=local_linear,
    )


@pytest.mark.parametrize("local_linear", [0, 1])
def test_fp64_leverage_matches_the_oracle(oracle, local_linear):
    g, o = leverage_request(**_lev_kw(local_linear)), leverage_request(**_lev_kw(local_linear))
    engine.leverage(g, "fp64")
    oracle.leverage(o)
    assert np.abs(g.x_grids - o.x_grids).max() < 1e-9
    rel = np.abs(g.values / o.values - 1)
    assert rel.max() < 1e-8, (np.median(rel), rel.max())


def test_fp32_particles_give_the_fp64_leverage_within_float_noise(oracle):
    g, o = leverage_request(**_lev_kw()), leverage_request(**_lev_kw())
    engine.leverage(g, "fp32")
    oracle.leverage(o)
    rel = np.abs(g.values / o.values - 1)
    # float particles move bins and quantiles by float rounding; the leverage follows within 1e-3 (median 1e-5)
    assert np.median(rel) < 1e-4 and rel.max() < 2e-2, (np.median(rel), rel.max())
    assert np.abs(g.x_grids - o.x_grids).max() < 1e-3


def test_leverage_refuses_more_bins_than_shared_memory_holds():
    kw = _lev_kw()
    h = leverage_request(**kw, n_bins=600)
    with pytest.raises(_abi.EngineError, match="n_bins must be <= 512"):
        engine.leverage(h, "fp32")


# ------------------------------------------------------------------------------------------------- fixed products


def _req(model, product, legs=(1, 2, 3), strikes=(100.0, 100.0, 100.0), H=80.0, n_steps=52, n_paths=2**15):
    rq = _abi.ObRequest()
    rq.model, rq.product = model, product
    for k in range(3):
        rq.legs[k], rq.strikes[k] = legs[k], strikes[k]
    rq.H, rq.n_steps, rq.S0, rq.r, rq.q, rq.T, rq.sigma = H, n_steps, 100.0, 0.04, 0.01, 1.0, 0.2
    rq.v0, rq.kappa, rq.theta, rq.xi, rq.rho = 0.0228, 3.09, 0.0537, 1.31, -0.69
    rq.n_paths, rq.seed = n_paths, 20261029
    return rq


CASES = {
    "bs european": (0, 0, (1, 2, 3)),
    "bs asian": (0, 1, (1, 0, 0)),
    "bs down-and-out": (0, 2, (1, 0, 0)),
    "heston european": (1, 0, (1, 1, 2)),
    "heston asian": (1, 1, (1, 0, 0)),
    "heston down-and-out": (1, 2, (1, 0, 0)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_fixed_products_match_the_oracle(oracle, name):
    model, product, legs = CASES[name]
    strikes = (100.0, 119.0, 80.0) if model == 1 and product == 0 else (100.0, 100.0, 100.0)
    rq = _req(model, product, legs, strikes)
    ro = oracle.price(rq)
    r64 = engine.price_fixed(rq, "fp64")
    r32 = engine.price_fixed(rq, "fp32")
    for k in range(4):
        if ro.price[k] == 0.0:
            assert r64.price[k] == 0.0
            continue
        assert abs(r64.price[k] / ro.price[k] - 1) < 1e-10, (k, r64.price[k], ro.price[k])
        assert abs(r64.se[k] / ro.se[k] - 1) < 1e-8
        assert abs(r32.price[k] - ro.price[k]) < 0.5 * ro.se[k]  # RC/tests/test_prices.cpp:125-145


def test_fixed_heston_call_is_near_fourier():
    """RC/tests/test_prices.cpp:64-71: Heston QE call K 100 against Fourier 8.403656 within 4 SE + 0.02."""
    rq = _req(1, 0, (1, 1, 2), (100.0, 119.0, 80.0), n_steps=252, n_paths=2**21)
    r = engine.price_fixed(rq, "fp32")
    for k, ref in enumerate((8.403656, 1.010290, 1.737996)):
        assert abs(r.price[k] - ref) < 4 * r.se[k] + 0.02, (k, r.price[k], ref)
    assert abs(r.price[3] - 100.0 * np.exp(0.03)) < 4 * r.se[3]


# ------------------------------------------------------------------------------------------------- golden


@pytest.mark.parametrize("name", ["bs", "heston"])
def test_fp64_paths_reproduce_the_references_golden_vectors(name):
    fx = json.loads(GOLDEN.read_text())
    case = fx["cases"][name]
    grid = np.asarray(case["grid"])
    obs = np.searchsorted(grid, np.asarray(fx["times"])).astype(np.int32)
    h = paths_request(
        dt=np.diff(grid), t0=grid[:-1], obs_step=obs, root=[[1.0]], kind=[case["kind"]], cvar=[case["cvar"]],
        heston=case["heston"], same=1, fwd=np.asarray(fx["fwd"])[None, :], n_pairs=fx["n_paths"] // 2,
        seed=fx["seed"],
    )
    engine.paths(h, "fp64")
    out = next(a for a in h.keep if isinstance(a, np.ndarray) and a.ndim == 3)
    S = np.ascontiguousarray(out[0].T).ravel()
    idx = np.linspace(0, S.size - 1, 32).astype(int)
    exp = case["expected"]
    assert np.max(np.abs(S[idx] / np.asarray(exp["samples"]) - 1)) < 1e-12
    assert abs(S.sum() / exp["sum"] - 1) < 1e-12


def test_the_persistent_calibration_equals_the_three_kernel_schedule(monkeypatch):
    """The calibration runs as one persistent kernel with grid barriers; OPTLAB_B200_LEVERAGE=graphs runs the same
    phases as three kernels a step replayed as graphs. The counts and v sums are integers and the regression the same
    arithmetic, so the two give the same tables (FP64 to the last bits of the regression's block sums)."""
    a, b = leverage_request(**_lev_kw()), leverage_request(**_lev_kw())
    engine.leverage(a, "fp64")
    monkeypatch.setenv("OPTLAB_B200_LEVERAGE", "graphs")
    engine.leverage(b, "fp64")
    assert np.abs(a.x_grids - b.x_grids).max() <= 1e-12 * np.abs(b.x_grids).max()
    assert np.abs(a.values / b.values - 1).max() < 1e-12


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_the_packed_fine_histogram_equals_the_unpacked_one(monkeypatch, precision):
    """The persistent kernel packs the fine histogram two 16-bit counts to a word; OPTLAB_B200_LEVERAGE=unpacked keeps
    32-bit counts. Counts are integers and the regression the same arithmetic: the tables are identical."""
    a, b = leverage_request(**_lev_kw()), leverage_request(**_lev_kw())
    engine.leverage(a, precision)
    monkeypatch.setenv("OPTLAB_B200_LEVERAGE", "unpacked")
    engine.leverage(b, precision)
    assert np.array_equal(a.x_grids, b.x_grids)
    assert np.array_equal(a.values, b.values)


def test_a_fine_bin_past_the_packed_counts_reruns_unpacked(monkeypatch):
    """With 16 fine bins and 2^19 particles the middle bins hold over 2^16 particles each, more than a packed count
    holds: the kernel sees the histogram's total fall short, and the call runs the calibration again unpacked, so the
    tables equal the unpacked run's and the three-kernel schedule's."""
    kw = dict(_lev_kw(n_pairs=2**18, n_steps=12), n_fine=16)
    a, b, c = (leverage_request(**kw) for _ in range(3))
    engine.leverage(a, "fp64")
    monkeypatch.setenv("OPTLAB_B200_LEVERAGE", "unpacked")
    engine.leverage(b, "fp64")
    monkeypatch.setenv("OPTLAB_B200_LEVERAGE", "graphs")
    engine.leverage(c, "fp64")
    assert np.array_equal(a.values, b.values) and np.array_equal(a.x_grids, b.x_grids)
    assert np.abs(a.values / c.values - 1).max() < 1e-12


def test_a_grid_barrier_that_gives_up_returns_a_timeout_and_the_device_stays_usable():
    """With a wait limit of zero polls every block gives up at its first wait on a grid barrier (a count that, as far
    as it may wait, nobody completes); the call returns OB_ETIMEOUT, every block leaves the kernel, and the next
    calibration, with the default limit, runs as before."""
    lib = _abi.load()
    h = leverage_request(**_lev_kw(n_pairs=2**12, n_steps=8))
    prev = lib.ob_set_wait_limit(0)
    try:
        with pytest.raises(_abi.EngineError, match="gave up waiting"):
            engine.leverage(h, "fp32")
    finally:
        lib.ob_set_wait_limit(-1)
    assert lib.ob_set_wait_limit(-1) == prev  # the default was restored
    g, o = leverage_request(**_lev_kw()), leverage_request(**_lev_kw())
    engine.leverage(g, "fp64")
    engine.leverage(o, "fp64")
    assert np.array_equal(g.values, o.values)
