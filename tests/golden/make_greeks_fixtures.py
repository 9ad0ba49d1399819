"""Writes tests/golden/reference_greeks.json: the reference's own bump-and-revalue Greeks of a 3-name worst-of autocall
under local vol, and samples of its tent-bumped local-variance tables.

The Greeks come from the reference's risk package as a desk would ask for them (optlab.risk.greeks.compute: deltas
central at +-h of spot, node vegas one-sided at +v on the implied-vol tents of its risk grid, risk/greeks.py:107-128,
199-244), with its structured engine's native path on the reference's compiled CPU engine (optlab::api::paths, built
from the reference's sources into oracle/_ref and reached through a ctypes stand-in for its nanobind module,
RN/src/optlab/native/_ext.pyi). The CPU engine draws the same Philox streams as this repository's kernels, so the GPU
test can run its adjoint on the very paths these Greeks were revalued on. Two bump sizes: the reference's defaults (1 %
of spot, one vol point) and small ones (1e-4 of spot, 1e-4 of vol), whose differences converge to the derivatives.

The tables: for a few nodes, the reference's TentBumpedSurface (risk/surfaces.py:95-167) bumped by +-1e-4 at that node,
tabulated per step as its engine does (local_var_rows on the base's grid), minus the base, at sampled steps and points:
what pins this repository's restatement of the tents and of their Jacobian.

Run where the reference tree and oracle/_ref are present:
    python tests/golden/make_greeks_fixtures.py [reference root; default $OPTLAB_REFERENCE, else /root/reference]
"""

from __future__ import annotations

import json
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent

NAMES = ("A", "B", "C")
C_RATE = (0.03, 0.045, 0.06)  # theta_t = c t per name
RHO = (-0.7, -0.55, -0.4)
CORR = 0.6
R, Q, S0 = 0.02, 0.01, 100.0
N_PATHS = 2**14
SEED = 20261204
NODES = [(5, 3), (2, 2), (8, 1)]  # (strike, tenor) nodes whose bumped tables are sampled


def worst_of_script(years: float = 1.0, per_year: int = 4, coupon=0.02, cb=0.7, call=1.0, ki=0.6, K=1.0) -> str:
    """The worst-of Phoenix of the adjoint's benchmark on NAMES, with its knock-in observed at maturity: quarterly,
    coupon with memory at cb, autocall at `call` (not on the last date), the worst below ki at maturity pays the put
    at K. (A daily knock-in window would read 252 daily fixings, while the reference's default grid is graded, with
    more steps than fixings in its first months; observed at the event dates only, the payoff reads grid points that
    both engines share.)"""
    n_obs = int(round(years * per_year))
    worst = f"min(min({NAMES[0]} / S0, {NAMES[1]} / S0), {NAMES[2]} / S0)"
    lines = [f"underlying {n}" for n in NAMES]
    lines += ["param S0 = 100", f"param cb = {cb!r}", f"param cpn = {coupon!r}", f"param call = {call!r}",
              f"param ki = {ki!r}", f"param K = {K!r}"]
    for j in range(1, n_obs + 1):
        t = j / per_year
        lines.append(f"event t={t!r} pay t={t!r}")
        if j == 1:
            lines.append("  missed = 0")
        lines += [f"  perf = {worst}", "  if perf >= cb then", "    pay cpn * (1 + missed) as coupon",
                  "    missed = 0", "  else", "    missed = missed + 1", "  end"]
        if j < n_obs:
            lines += ["  if perf >= call then", "    pay 1 as redemption", "    terminate", "  end"]
        else:
            lines += ["  knocked = perf < ki", "  if knocked then", "    pay 1 - max(K - perf, 0) as redemption",
                      "  else", "    pay 1 as redemption", "  end"]
        lines.append("end")
    return "\n".join(lines) + "\n"


def install_ext_stand_in():
    """`optlab.native._ext` over the reference's compiled CPU engine (oracle/_ref): the functions its Python engine
    module calls, with the nanobind module's signatures."""
    sys.path[:0] = [str(ROOT / "option-pricing-lab_b200"), str(ROOT / "oracle")]
    from oracle import Reference

    from optlab_b200.requests import paths_request

    ref = Reference()
    ext = types.ModuleType("optlab.native._ext")
    ext.gpu_count = lambda: 0
    ext.has_cuda = lambda: False
    ext.cpu_threads = lambda: os.cpu_count() or 1
    ext.gpu_name = lambda: ""
    ext.device_info = lambda device: None

    def paths(dt, t0, obs_step, root, kind, cvar, heston, same, step_row, row_lo, row_inv_dx, table, fwd, mixer, mix,
              low_root, n_x, n_pairs, first_pair, seed, col_of, n_keep, win_lo, win_hi, out, backend, n_threads=0):
        if backend != 0:
            raise RuntimeError("only the CPU backend is built here")
        held = paths_request(
            dt=dt, t0=t0, obs_step=obs_step, root=root, kind=kind, cvar=cvar, heston=heston, same=same, fwd=fwd,
            n_pairs=n_pairs, seed=seed, first_pair=first_pair, step_row=step_row if step_row.size else None,
            lo=row_lo if row_lo.size else None, inv_dx=row_inv_dx if row_inv_dx.size else None,
            table=table if table.size else None, n_x=n_x, mixer=mixer, mix=mix,
            low_root=low_root if low_root.size else None, col_of=col_of, n_keep=n_keep, win_lo=win_lo, win_hi=win_hi,
            out=out)
        ref.paths(held, n_threads)
        return 0.0, 0.0

    def unsupported(*a, **k):
        raise RuntimeError("not needed by these fixtures")

    ext.paths, ext.price, ext.leverage = paths, unsupported, unsupported
    sys.modules["optlab.native._ext"] = ext


def main(ref_root: str = os.environ.get("OPTLAB_REFERENCE", "/root/reference")) -> None:
    pk = Path(ref_root) / "packages"
    for p in ("core/src", "structured/src", "native/src", "risk/src"):
        sys.path.insert(0, str(pk / p))
    install_ext_stand_in()
    import datetime as dt

    import optlab.native as native
    from optlab.core import engines
    from optlab.core.market import Market
    from optlab.core.ssvi import SSVI
    from optlab.risk import RiskGroup, RiskSettings
    from optlab.risk import grid as rgrid
    from optlab.risk.greeks import Bumps, GreekOptions, compute
    from optlab.risk.surfaces import TentBumpedSurface
    from optlab.structured.multiasset import BasketContext
    from optlab.structured.portfolio import Book, Position

    engines._compiled[:] = [native]
    T = 3.0 * np.arange(1, 41) / 40
    surfaces = {n: SSVI.power_law(RHO[a], 1.0, 0.5, T, C_RATE[a] * T) for a, n in enumerate(NAMES)}
    corr = np.full((3, 3), CORR) + (1 - CORR) * np.eye(3)
    ctx = BasketContext(NAMES, {n: Market.flat(S0, R, Q) for n in NAMES}, surfaces, corr, dt.date(2026, 12, 4))
    script = worst_of_script()
    opts = GreekOptions(kxt="all", curves=False, sticky_strike=False, realistic=False, cross=False, theta=False)
    book = Book([Position("wo", script, 1.0)])
    sim_times = np.unique(np.concatenate([it["timeline"].sim_times for it in book._prepare(ctx)]))
    out = {"names": NAMES, "c_rate": C_RATE, "rho": RHO, "corr": CORR, "r": R, "q": Q, "spot": S0,
           "sim_times": sim_times.tolist(),
           "n_paths": N_PATHS, "seed": SEED, "key": engines.seed64(SEED), "smoothing": 0.005, "script": script,
           "strike_labels": list(rgrid.STRIKE_LABELS), "tenor_labels": list(rgrid.TENOR_LABELS), "greeks": {}}
    for label, bumps in (("default", Bumps()), ("small", Bumps(spot=1e-4, vol=1e-4))):
        rep = compute([RiskGroup("wo", book, ctx, SEED)], bumps=bumps, options=opts,
                      settings=RiskSettings(n_paths=N_PATHS, engine="cpu", smoothing=0.005))
        pos = rep.positions[0]
        g = pos["greeks"]
        entry = {"value": [pos["value"], pos["value_se"]], "spot_bump": bumps.spot, "vol_bump": bumps.vol,
                 "delta": {n: g[f"delta|{n}|"] for n in NAMES}, "vega_node": {}}
        for n in NAMES:
            entry["vega_node"][n] = [[g[f"vega_node|{n}|{k}@{t}"] for t in rgrid.TENOR_LABELS]
                                     for k in rgrid.STRIKE_LABELS]
        out["greeks"][label] = entry
        print(label, "value", entry["value"], "delta", entry["delta"])
    # the tent-bumped tables, as the reference's engine tabulates them (one step per 1/252 over the year)
    t0 = np.arange(252) / 252.0
    rng = np.random.default_rng(4)
    steps = np.sort(rng.choice(252, 12, replace=False))
    pts = np.sort(rng.choice(801, 48, replace=False))
    base = surfaces["B"]
    lo, inv, rows0 = native._local_var_rows(base, t0, 801)
    tables = {"name": "B", "steps": steps.tolist(), "points": pts.tolist(), "h": 1e-4,
              "base": rows0[np.ix_(steps, pts)].tolist(), "lo": lo[steps].tolist(), "inv_dx": inv[steps].tolist(),
              "nodes": []}
    for i, j in NODES:
        d = []
        for sgn in (1.0, -1.0):
            H = np.zeros((len(rgrid.STRIKES), len(rgrid.TENORS)))
            H[i, j] = sgn * 1e-4
            _, _, rows = TentBumpedSurface(base, nodes=H).local_var_rows(t0, 801)
            d.append(rows[np.ix_(steps, pts)])
        tables["nodes"].append({"node": [i, j], "plus": d[0].tolist(), "minus": d[1].tolist()})
    out["tables"] = tables
    # the tents themselves on a few points
    kk = np.linspace(-0.8, 0.5, 27)
    TT = np.array([0.02, 0.1, 0.3, 0.75, 1.2, 2.5, 6.0])
    Kg, Tg = np.meshgrid(kk, TT, indexing="ij")
    phi = rgrid.strike_tents(Kg, Tg)
    psi = rgrid.tenor_tents(TT, order=1)
    out["tents"] = {"k": kk.tolist(), "T": TT.tolist(), "strike": [np.asarray(p).tolist() for p in phi],
                    "tenor": [np.asarray(p).tolist() for p in psi]}
    (HERE / "reference_greeks.json").write_text(json.dumps(out))
    print("wrote", HERE / "reference_greeks.json")


if __name__ == "__main__":
    main(*sys.argv[1:])
