"""The drop-in Engine module on the GPU: simulate/run against the oracle on the same plan, and the reference's own
end-to-end checks (packages/native/tests/test_native.py:54-82,228-243): local vol reprices its surface, and an SLV
model whose leverage this engine calibrated reprices it too."""

import numpy as np
import pytest
from scipy.stats import norm

import optlab_b200 as eng
from optlab_b200 import models as M
from optlab_b200 import workloads
from optlab_b200.requests import paths_request

pytestmark = pytest.mark.gpu

K = np.array([80.0, 90.0, 100.0, 110.0, 120.0])


def calls(S, D, strikes=K):
    h = len(S) // 2
    pay = D * np.maximum(S[:, None] - strikes, 0.0)
    pay = 0.5 * (pay[:h] + pay[h:])
    return pay.mean(axis=0), pay.std(axis=0, ddof=1) / np.sqrt(h)


def black(F, K, T, vol, D):
    s = vol * np.sqrt(T)
    d1 = np.log(F / K) / s + 0.5 * s
    return D * (F * norm.cdf(d1) - K * norm.cdf(d1 - s))


def _oracle_spots(oracle, p, n_pairs, seed, keep=None):
    keep = np.arange(p.n_obs) if keep is None else np.asarray(keep)
    col_of = np.full(p.n_obs, -1, np.int32)
    col_of[keep] = np.arange(len(keep), dtype=np.int32)
    h = paths_request(dt=p.dt, t0=p.t0, obs_step=p.obs_step, root=p.root, kind=p.kind, cvar=p.cvar, heston=p.heston,
                      same=p.same, fwd=p.fwd, n_pairs=n_pairs, seed=seed, step_row=p.step_row, lo=p.lo,
                      inv_dx=p.inv_dx, table=p.table, n_x=p.n_x, mixer=p.mixer, mix=p.mix, low_root=p.low_root,
                      col_of=col_of, n_keep=len(keep))
    oracle.paths(h)
    out = next(a for a in h.keep if isinstance(a, np.ndarray) and a.ndim == 3)
    return [out[a, : len(keep)].T for a in range(len(p.names))]


def test_simulate_local_vol_matches_the_oracle_on_the_same_plan(oracle):
    surf = workloads.lv_surface()
    model, market = M.LocalVolModel(surf), M.Market.flat(100.0, 0.02, 0.01)
    S = eng.simulate(model, market, [0.5, 1.0, 2.0], 2**13, seed=5, backend="gpu", precision="fp64")
    ref = _oracle_spots(oracle, eng.plan(model, market, [0.5, 1.0, 2.0]), 2**12, 5)[0]
    assert S.shape == ref.shape == (2**13, 3)
    assert np.abs(S / ref - 1).max() < 1e-12


def test_a_basket_with_local_correlation_and_windows_matches_the_oracle(oracle):
    names = ("A", "B", "C")
    corr = np.array([[1.0, 0.8, 0.6], [0.8, 1.0, 0.7], [0.6, 0.7, 1.0]])
    mk = M.Market.flat(100.0, 0.02, 0.0)
    b = M.Basket(names, {n: M.LocalVolModel(workloads.lv_surface()) for n in names}, {n: mk for n in names}, corr,
                 mixer=M.LocalCorrelation(sigma=0.15, down=0.3, up=0.1))
    times = np.linspace(0.1, 1.0, 10)
    p = eng.plan(b, None, times)
    spots, ext, timing = eng.run(p, 2**11, 9, keep=[4, 9], windows=[(0, 9)], precision="fp64")
    ref = _oracle_spots(oracle, p, 2**11, 9)
    assert timing["backend"] == "gpu"
    for a in range(3):
        assert np.abs(spots[a] / ref[a][:, [4, 9]] - 1).max() < 1e-12
        lo, hi = ext[a][0]
        assert np.abs(lo / ref[a].min(axis=1) - 1).max() < 1e-12 and np.abs(hi / ref[a].max(axis=1) - 1).max() < 1e-12


def test_local_vol_and_an_engine_calibrated_slv_reprice_the_surface():
    surf = workloads.lv_surface()
    market = M.Market.flat(100.0, 0.02, 0.01)
    T = 1.0
    F, D = float(market.F(T)), float(market.D(T))
    target = black(F, K, T, surf.iv(np.log(K / F), T), D)
    lv = M.LocalVolModel(surf)
    S = eng.simulate(lv, market, [T], 400_000, seed=2)[:, 0]
    p, se = calls(S, D)
    assert np.all(np.abs(p - target) < 4 * se + 0.01), (p - target, se)
    heston = M.HestonParams(0.04, 1.5, 0.04, 0.5, -0.7)
    slv = eng.calibrate_leverage(heston, surf, market, T, mix=0.5, n_particles=200_000, rng=1)
    assert isinstance(slv, M.SLVModel) and slv.leverage.values.shape[1] == 81
    S = eng.simulate(slv, market, [T], 400_000, seed=12)[:, 0]
    p, se = calls(S, D)
    assert np.all(np.abs(p - target) < 4 * se + 0.03), (p - target, se)
