"""The drop-in Engine module (optlab_b200) against the reference's own Python: the same Plan arrays from the same model
objects, the same SSVI local variance, time grid and local-correlation factors, and registration in the reference's
registry. The reference's packages are imported from the reference tree, where present."""

import os
import sys
from pathlib import Path

import numpy as np
import pytest

import optlab_b200 as eng
from optlab_b200 import models as M
from optlab_b200.surfaces import SSVI

REF = Path(os.environ.get("OPTLAB_REFERENCE", "/root/reference")) / "packages"
HAVE_REF = (REF / "core/src/optlab/core/models.py").exists()


@pytest.fixture(scope="module")
def ref():
    if not HAVE_REF:
        pytest.skip("the reference tree is not present")
    for p in ("core/src", "structured/src", "native/src", "risk/src"):
        if str(REF / p) not in sys.path:
            sys.path.insert(0, str(REF / p))
    import optlab.core.models as rm
    import optlab.core.ssvi as rs
    import optlab.native as rn
    from optlab.core.heston import HestonParams
    from optlab.core.market import Market
    from optlab.structured import localcorr as lc
    from optlab.structured import multiasset as ma

    return dict(models=rm, ssvi=rs, native=rn, Hp=HestonParams, Market=Market, lc=lc, ma=ma)


def _ssvi_args():
    T = 3.0 * np.arange(1, 41) / 40
    return (-0.6, 1.0, 0.5, T, 0.04 * T)


def test_ssvi_local_variance_matches_the_reference(ref):
    mine = SSVI.power_law(*_ssvi_args())
    theirs = ref["ssvi"].SSVI.power_law(*_ssvi_args())
    k = np.linspace(-2.5, 2.0, 301)
    for T in (0.01, 0.2, 1.0, 2.99, 3.5):
        a, b = mine.local_var(k, T), theirs.local_var(k, T)
        assert np.max(np.abs(a / b - 1)) < 1e-14
        assert np.max(np.abs(mine.w(k, T) / theirs.w(k, T) - 1)) < 1e-14


def test_time_grids_match_the_reference(ref):
    for times, dt_max, dt_min in (([0.25, 0.5, 1.0], 1 / 252, 1 / 2000), ([1, 2, 3], 1 / 252, None), ([0.1], 1 / 100, 1 / 2000)):
        assert np.array_equal(M.time_grid(times, dt_max, dt_min), ref["models"].time_grid(times, dt_max, dt_min))


def _fields(p):
    return {k: getattr(p, k) for k in ("kind", "cvar", "heston", "root", "same", "dt", "t0", "obs_step", "fwd",
                                       "step_row", "lo", "inv_dx", "table", "mixer", "mix", "low_root", "n_x")}


def _same_plan(a, b):
    fa, fb = _fields(a), _fields(b)
    for k in fa:
        x, y = fa[k], fb[k]
        if x is None or y is None:
            assert x is None and y is None, k
        elif isinstance(x, tuple):
            assert np.allclose(x, y, rtol=1e-14, atol=1e-15), k
        else:
            assert np.allclose(np.asarray(x, float), np.asarray(y, float), rtol=1e-14, atol=1e-15), k


def test_plans_match_the_references_for_every_model_kind(ref):
    rm, Hp, Market = ref["models"], ref["Hp"], ref["Market"]
    surf_r = ref["ssvi"].SSVI.power_law(*_ssvi_args())
    surf_m = SSVI.power_law(*_ssvi_args())
    mkt_r, mkt_m = Market.flat(100.0, 0.03, 0.01), M.Market.flat(100.0, 0.03, 0.01)
    hp = (0.04, 1.5, 0.04, 0.5, -0.7)
    t = np.linspace(0, 1, 11)
    lev_vals = np.array([1.0 + 0.1 * np.sin(np.linspace(0, 3, 21) + s) for s in range(11)])
    lev_x = np.tile(np.linspace(-1, 1, 21), (11, 1))
    pairs = [
        (rm.BlackScholesModel(0.2), M.BlackScholesModel(0.2)),
        (rm.HestonModel(Hp(*hp)), M.HestonModel(M.HestonParams(*hp))),
        (rm.LocalVolModel(surf_r), M.LocalVolModel(surf_m)),
        (rm.SLVModel(Hp(*hp), rm.Leverage(t, lev_x, lev_vals), 0.5),
         M.SLVModel(M.HestonParams(*hp), M.Leverage(t, lev_x, lev_vals), 0.5)),
    ]
    times = [0.25, 0.5, 1.0]
    for theirs, mine in pairs:
        _same_plan(eng.plan(mine, mkt_m, times), ref["native"].plan(theirs, mkt_r, times))
        # the reference's own objects go through this engine's plan() unchanged
        _same_plan(eng.plan(theirs, mkt_r, times), ref["native"].plan(theirs, mkt_r, times))


def test_a_basket_with_local_correlation_plans_like_the_reference(ref):
    rm, ma, lc, Market = ref["models"], ref["ma"], ref["lc"], ref["Market"]
    names = ("A", "B", "C")
    corr = np.array([[1.0, 0.8, 0.6], [0.8, 1.0, 0.7], [0.6, 0.7, 1.0]])
    mk_r, mk_m = Market.flat(100.0, 0.02, 0.0), M.Market.flat(100.0, 0.02, 0.0)
    theirs = ma.Basket(names, {n: rm.BlackScholesModel(0.2) for n in names}, {n: mk_r for n in names}, corr,
                       mixer=lc.LocalCorrelation(sigma=0.15, down=0.3, up=0.1))
    mine = M.Basket(names, {n: M.BlackScholesModel(0.2) for n in names}, {n: mk_m for n in names}, corr,
                    mixer=M.LocalCorrelation(sigma=0.15, down=0.3, up=0.1))
    _same_plan(eng.plan(mine, None, [0.5, 1.0]), ref["native"].plan(theirs, None, [0.5, 1.0]))


def test_unsupported_models_are_named_like_the_reference(ref):
    class Exotic:
        pass

    assert eng._model_unsupported(Exotic()) == "Exotic is not in the path engine"
    assert eng._model_unsupported(M.BlackScholesModel(0.2)) is None
    with pytest.raises(NotImplementedError, match="Exotic is not in the path engine"):
        eng.plan(Exotic(), None, [1.0])
    if not eng.gpu_available():
        assert eng.unsupported(M.BlackScholesModel(0.2)) == eng.NO_DEVICE


def test_the_module_registers_in_the_references_registry(ref):
    from optlab.core import engines

    saved = list(engines._compiled)
    try:
        eng.register()
        assert engines.compiled() is eng
        if not eng.gpu_available():
            with pytest.raises(engines.EngineError, match="no CUDA device"):
                engines.choose("gpu", M.BlackScholesModel(0.2))
            assert engines.choose("auto", M.BlackScholesModel(0.2)) == ("numpy", eng.NO_DEVICE)
        else:
            assert engines.choose("auto", M.BlackScholesModel(0.2)) == ("gpu", None)
    finally:
        engines._compiled[:] = saved


def test_the_cpu_backend_is_refused_there_is_no_fallback():
    p = eng.plan(M.BlackScholesModel(0.2), M.Market.flat(100.0), [1.0])
    with pytest.raises(eng.EngineError, match="GPU only"):
        eng.run(p, 8, 1, backend="cpu")


def test_the_entry_point_is_declared():
    text = (Path(__file__).resolve().parent.parent / "option-pricing-lab_b200" / "pyproject.toml").read_text()
    assert '[project.entry-points."optlab.engines"]' in text and 'native = "optlab_b200"' in text


def test_the_monotone_cubic_is_the_pchip_the_reference_fits_with():
    """MonotoneCubic against scipy's PchipInterpolator (the reference's interpolant of theta(T) and the wings):
    values and slopes on monotone, flat-stretched and sign-changing data, ends included."""
    from scipy.interpolate import PchipInterpolator

    from optlab_b200.surfaces import MonotoneCubic

    rng = np.random.default_rng(3)
    cases = [
        (np.append(0.0, np.cumsum(rng.uniform(0.1, 1.0, 12))), np.append(0.0, np.cumsum(rng.uniform(0, 1, 12)))),
        (np.arange(8.0), np.array([0.0, 1.0, 1.0, 1.0, 2.0, 5.0, 5.5, 9.0])),
        (np.cumsum(rng.uniform(0.2, 1.0, 10)), rng.normal(size=10)),
        (np.array([0.0, 1.0]), np.array([2.0, -1.0])),
        (np.array([0.0, 0.5, 2.0]), np.array([0.0, 3.0, 2.5])),
    ]
    for x, y in cases:
        ref = PchipInterpolator(x, y, extrapolate=False)
        t = np.concatenate([x, np.linspace(x[0], x[-1], 257)])
        v, s = MonotoneCubic(x, y).at(t)
        scale = np.abs(y).max() + 1.0
        assert np.max(np.abs(v - ref(t))) <= 1e-13 * scale
        assert np.max(np.abs(s - ref.derivative()(t))) <= 1e-12 * scale / np.diff(x).min()


def test_a_basket_of_several_tabled_names_plans_like_the_reference(ref):
    """Two local-vol names and an SLV name: their tables stack in the names' order, each name's step rows offset by
    the rows before it, as the reference's plan stacks them."""
    rm, ma, Hp, Market = ref["models"], ref["ma"], ref["Hp"], ref["Market"]
    T = 3.0 * np.arange(1, 41) / 40
    s1r, s2r = ref["ssvi"].SSVI.power_law(-0.6, 1.0, 0.5, T, 0.04 * T), ref["ssvi"].SSVI.power_law(-0.4, 1.0, 0.5, T, 0.05 * T)
    s1m, s2m = SSVI.power_law(-0.6, 1.0, 0.5, T, 0.04 * T), SSVI.power_law(-0.4, 1.0, 0.5, T, 0.05 * T)
    t = np.linspace(0, 1, 11)
    lev_vals = np.array([1.0 + 0.1 * np.sin(np.linspace(0, 3, 21) + s) for s in range(11)])
    lev_x = np.tile(np.linspace(-1, 1, 21), (11, 1))
    hp = (0.04, 1.5, 0.04, 0.5, -0.7)
    names = ("A", "B", "C")
    corr = np.array([[1.0, 0.5, 0.4], [0.5, 1.0, 0.3], [0.4, 0.3, 1.0]])
    mk_r, mk_m = Market.flat(100.0, 0.02, 0.01), M.Market.flat(100.0, 0.02, 0.01)
    theirs = ma.Basket(names, {"A": rm.LocalVolModel(s1r), "B": rm.SLVModel(Hp(*hp), rm.Leverage(t, lev_x, lev_vals), 0.5),
                               "C": rm.LocalVolModel(s2r)}, {n: mk_r for n in names}, corr)
    mine = M.Basket(names, {"A": M.LocalVolModel(s1m),
                            "B": M.SLVModel(M.HestonParams(*hp), M.Leverage(t, lev_x, lev_vals), 0.5),
                            "C": M.LocalVolModel(s2m)}, {n: mk_m for n in names}, corr)
    times = [0.25, 0.5, 1.0]
    _same_plan(eng.plan(mine, None, times), ref["native"].plan(theirs, None, times))
