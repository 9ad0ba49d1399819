"""The oracle pinned before it is trusted: against the reference's recorded golden vectors, against published Philox
known-answer vectors, and against the reference's own CPU engine compiled from its sources (where the reference tree
is present: `make -C oracle ref`)."""

import json
from pathlib import Path

import numpy as np
import pytest

from optlab_b200 import workloads
from optlab_b200.requests import mc_request, paths_request

GOLDEN = Path(__file__).resolve().parent / "golden" / "reference_paths.json"


def out_of(held):
    return next(a for a in held.keep if isinstance(a, np.ndarray) and a.ndim == 3)


# ------------------------------------------------------------------------------------------------- Philox KAT


def test_philox_matches_the_published_known_answers(oracle):
    """Random123's known-answer vectors for Philox4x32-10 (Salmon et al., SC 2011): the algorithm the reference names
    (packages/native/cuda/include/optlab_cuda/philox.hpp:1-4)."""
    kat = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        (
            (0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344),
            (0xA4093822, 0x299F31D0),
            (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1),
        ),
    ]
    for ctr, key, want in kat:
        assert oracle.philox(ctr, *key) == list(want)


# ------------------------------------------------------------------------------------------------- golden vectors


def _golden_run(oracle, case: dict, fx: dict) -> np.ndarray:
    grid = np.asarray(case["grid"])
    times = np.asarray(fx["times"])
    obs = np.searchsorted(grid, times).astype(np.int32)
    h = paths_request(
        dt=np.diff(grid),
        t0=grid[:-1],
        obs_step=obs,
        root=[[1.0]],
        kind=[case["kind"]],
        cvar=[case["cvar"]],
        heston=case["heston"],
        same=1,
        fwd=np.asarray(fx["fwd"])[None, :],
        n_pairs=fx["n_paths"] // 2,
        seed=fx["seed"],
    )
    oracle.paths(h)
    return np.ascontiguousarray(out_of(h)[0].T)  # (paths, dates) as the reference's simulate() returns


@pytest.mark.parametrize("name", ["bs", "heston"])
def test_oracle_reproduces_the_references_golden_paths(oracle, name):
    """tests/golden/native_cpu.json of the reference (its CPU engine, recorded on another machine and libm): the
    oracle's paths give the same 32 samples and the same sum, to libm rounding."""
    fx = json.loads(GOLDEN.read_text())
    case = fx["cases"][name]
    S = _golden_run(oracle, case, fx)
    exp = case["expected"]
    flat = S.ravel()
    idx = np.linspace(0, flat.size - 1, 32).astype(int)
    assert list(S.shape) == exp["shape"]
    assert np.max(np.abs(flat[idx] / np.asarray(exp["samples"]) - 1)) < 1e-12
    assert abs(flat.sum() / exp["sum"] - 1) < 1e-12


# ------------------------------------------------------------------------------------------------- live reference


def _paths_kw(kinds, n_steps=40, n_pairs=1500, mixer=0, same=1, n_x=81):
    n = len(kinds)
    rng = np.random.default_rng(1)
    corr = np.full((n, n), 0.4) + 0.6 * np.eye(n)
    root = np.linalg.cholesky(corr)
    kw = dict(
        dt=np.full(n_steps, 1 / 100),
        t0=np.arange(n_steps) / 100,
        obs_step=[0, 7, 20, n_steps],
        root=root,
        kind=kinds,
        cvar=np.full(n, 0.05),
        heston=np.tile([0.03, 2.0, 0.05, 0.6, -0.6], n),
        same=same,
        fwd=np.tile([100.0, 100.5, 101.0, 102.0], n).reshape(n, 4),
        n_pairs=n_pairs,
        seed=2**40 + 3,
        first_pair=2**33,
        step_row=np.tile(np.arange(n_steps), n),
        lo=np.full(n_steps, -1.2),
        inv_dx=np.full(n_steps, (n_x - 1) / 2.2),
        table=0.03 + 0.03 * rng.random((n_steps, n_x)),
        n_x=n_x,
        win_lo=[0, 1],
        win_hi=[3, 2],
    )
    if mixer:
        kw.update(mixer=1, mix=(0.2, 0.1, 0.4, 0.05, 0.2, -1.0, np.cos(0.4), np.sin(0.4)), low_root=root)
    return kw


@pytest.mark.parametrize(
    "kinds,mixer,same",
    [([0], 0, 1), ([1], 0, 1), ([2], 0, 1), ([3], 0, 1), ([3, 1, 2], 0, 1), ([2, 3], 0, 0), ([1] * 8, 0, 1),
     ([1, 1, 1], 1, 1)],
)
def test_oracle_paths_match_the_references_cpu_engine(oracle, reference, kinds, mixer, same):
    kw = _paths_kw(kinds, mixer=mixer, same=same)
    a, b = paths_request(**kw), paths_request(**kw)
    oracle.paths(a, 4)
    reference.paths(b, 4)
    assert np.abs(out_of(a) / out_of(b) - 1).max() < 1e-13


def test_oracle_philox_matches_the_reference(oracle, reference):
    for args in [(20261105, 0, 16, 0, 0, 5), (2**64 - 1, 2**40, 8, 0x80000000, 2**32 - 3, 6)]:
        ua, za = oracle.philox_normals(*args)
        ub, zb = reference.philox_normals(*args)
        assert np.array_equal(ua, ub) and np.array_equal(za, zb)


def test_oracle_qe_ladder_matches_the_references_qe_step(oracle, reference):
    """The composed QE oracle (reference make_consts<double> + qe_step<double> on its NormalStream<double>)."""
    h = workloads.heston_qe_ladder(n_paths=2**13, seed=4)
    r = oracle.mc_price(h)
    n = r.n_out
    lt = np.ones(12, np.int32)
    ks = np.append(np.arange(80.0, 121.0, 4.0), 100.0)
    up = np.zeros(12, np.int32)
    up[-1] = 1
    lv = np.zeros(12)
    lv[-1] = 130.0
    p, se = reference.qe_ladder(100.0, 0.02, 0.01, 1.0, 252, workloads.HESTON_CFG0, 2**12, 4, lt, ks, up, lv)
    assert np.abs(np.array(r.price[:n]) / p - 1).max() < 1e-12
    assert np.abs(np.array(r.se[:n]) / se - 1).max() < 1e-9


def test_oracle_leverage_matches_the_reference_on_one_thread(oracle, reference):
    from optlab_b200.leverage import leverage_request

    for ll in (0, 1):
        a = leverage_request(**_lev_kw(ll))
        b = leverage_request(**_lev_kw(ll))
        oracle.leverage(a)
        reference.leverage(b, 1)
        assert np.abs(a.x_grids - b.x_grids).max() < 1e-12
        assert np.abs(a.values / b.values - 1).max() < 1e-10


def _lev_kw(local_linear):
    n_steps, n_lv = 30, 201
    x = np.linspace(-1, 1, n_lv)
    t0 = np.arange(n_steps) / 100
    return dict(
        dt=np.full(n_steps, 1 / 100),
        t0=t0,
        n_pairs=8000,
        seed=42,
        heston=(0.04, 1.5, 0.04, 0.25, -0.7),
        n_x=41,
        lv_lo=np.full(n_steps, -1.0),
        lv_inv_dx=np.full(n_steps, (n_lv - 1) / 2.0),
        lv_rows=np.array([0.04 * (1 + 0.5 * x**2 - 0.3 * x) * (1 + 0.1 * t) for t in t0]),
        atm_vol=0.2,
        local_linear=local_linear,
        positive_part=local_linear,
    )


def test_oracle_worst_of_autocall_is_the_pair_average_of_its_columns(oracle):
    """The fused oracle's autocall equals the Phoenix evaluated on the oracle's own spot columns (the reference's
    split: paths to columns, then the payoff), on one name with a daily knock-in window."""
    import bench

    ph = workloads.Phoenix(years=1.0)
    m = workloads.FlatMarket(100.0, 0.02, 0.01)
    g = workloads.lv_grid(horizon=1.0, n_exp=8, n_x=120)
    n_steps = 252
    dt, t0 = workloads.uniform_grid(1.0, n_steps)
    t_end = np.concatenate([[0.0], t0 + dt])
    fused = mc_request(
        model=0, dt=dt, t0=t0, spot=[100.0], n_pairs=3000, seed=9, kind=[1], cvar=[0.0],
        log_fwd=m.log_fwd(t_end)[None, :], step_row=g.row_of(t0)[None, :], lo=g.lo, inv_dx=g.inv_dx, table=g.rows,
        n_x=g.n_x, **workloads.autocall_fields(ph, m, 252),
    )
    r = oracle.mc_price(fused)
    obs_step, _ = ph.schedule(252)
    all_obs = np.arange(0, n_steps + 1, dtype=np.int32)
    col_of = np.full(len(all_obs), -1, np.int32)
    col_of[obs_step] = np.arange(len(obs_step), dtype=np.int32)
    cols = paths_request(
        dt=dt, t0=t0, obs_step=all_obs, root=[[1.0]], kind=[1], cvar=[0.0], heston=[0, 1, 1, 0, 0], same=1,
        fwd=m.F(t_end)[None, :], n_pairs=3000, seed=9, step_row=g.row_of(t0), lo=g.lo, inv_dx=g.inv_dx,
        table=g.rows, n_x=g.n_x, col_of=col_of, n_keep=len(obs_step), win_lo=[0], win_hi=[n_steps],
    )
    oracle.paths(cols)
    out = out_of(cols)[0]
    price, se = bench.phoenix_payoff(out[: len(obs_step)].T / 100.0, out[len(obs_step)] / 100.0, ph, m)
    assert abs(r.price[0] / price - 1) < 1e-12 and abs(r.se[0] / se - 1) < 1e-9
