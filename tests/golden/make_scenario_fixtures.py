"""Writes tests/golden/reference_scenarios.json: the reference's own risk scenarios on a small book, and its moved
implied-vol surfaces' local variance at sample points.

- Moved surfaces: the reference's bumped_surface (packages/risk/src/optlab/risk/surfaces.py:204; VolMove.apply,
  risk/shocks.py:63-108) under parallel and skew moves of its implied vols, with Dupire's local variance read at
  sampled (log-moneyness, expiry) points: what pins this repository's scenario tables (optlab_b200.ivnodes).
- A book of four trades under local vol (a call-and-put ladder, a daily down-and-in put, a Phoenix autocall, a 2-name
  worst-of autocall; one year), each valued with the reference's risk engine (optlab.risk.engine.run_group, its
  structured engine's native path on its compiled CPU engine reached through a ctypes stand-in for the nanobind
  module) under spot moves of +-5 %, parallel implied-vol moves of +-2 points and skew moves of +-2 points: per
  scenario the value and, against the base on the same random numbers, the P&L and its standard error.

Run where the reference tree and oracle/_ref are present:
    python tests/golden/make_scenario_fixtures.py [reference root; default $OPTLAB_REFERENCE, else /root/reference]
"""

from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from make_greeks_fixtures import install_ext_stand_in  # noqa: E402

R, Q, S0 = 0.02, 0.01, 100.0
N_PATHS = 2**16
SURFACES = {"A": (0.04, -0.6), "B": (0.05, -0.5), "C": (0.035, -0.7)}  # theta_t = c t, rho
MOVES = {"spot+": ("spot", 0.05), "spot-": ("spot", -0.05), "vol+": ("parallel", 0.02), "vol-": ("parallel", -0.02),
         "skew+": ("skew", 0.02), "skew-": ("skew", -0.02)}


def phoenix(names, ki_window: bool, years=1.0, per_year=4, coupon=0.02, cb=0.7, call=1.0, ki=0.6, K=1.0) -> str:
    """A Phoenix autocall on the worst of `names` (quarterly, coupon with memory, autocall at `call`, knock-in put
    at maturity: on the lowest daily close of the worst with ki_window, else on the worst at maturity)."""
    n_obs = int(round(years * per_year))
    perf = f"{names[0]} / S0"
    for n in names[1:]:
        perf = f"min({perf}, {n} / S0)"
    lines = [f"underlying {n}" for n in names]
    lines += ["param S0 = 100", f"param cb = {cb!r}", f"param cpn = {coupon!r}", f"param call = {call!r}",
              f"param ki = {ki!r}", f"param K = {K!r}"]
    for j in range(1, n_obs + 1):
        t = j / per_year
        lines.append(f"event t={t!r} pay t={t!r}")
        if j == 1:
            lines.append("  missed = 0")
        lines += [f"  perf = {perf}", "  if perf >= cb then", "    pay cpn * (1 + missed) as coupon",
                  "    missed = 0", "  else", "    missed = missed + 1", "  end"]
        if j < n_obs:
            lines += ["  if perf >= call then", "    pay 1 as redemption", "    terminate", "  end"]
        else:
            if ki_window:
                low = f"lowest({names[0]}, t=0, t={t!r}, n={int(round(years * 252))})"
                lines.append(f"  knocked = {low} < ki * S0")
            else:
                lines.append("  knocked = perf < ki")
            lines += ["  if knocked then", "    pay 1 - max(K - perf, 0) as redemption", "  else",
                      "    pay 1 as redemption", "  end"]
        lines.append("end")
    return "\n".join(lines) + "\n"


TRADES = [
    {"label": "ladder-A", "names": ["A"], "seed": 101, "product": "ladder",
     "legs": [[1, 1.0, 0, 0.0], [2, 0.9, 0, 0.0]],
     "script": "underlying A\nparam S0 = 100\nevent t=1.0 pay t=1.0\n"
               "  pay max(A / S0 - 1.0, 0) + max(0.9 - A / S0, 0) as redemption\nend\n"},
    {"label": "down-in-put-B", "names": ["B"], "seed": 102, "product": "ladder",
     "legs": [[2, 1.0, 4, 0.75]],
     "script": "underlying B\nparam S0 = 100\nevent t=1.0 pay t=1.0\n"
               "  if lowest(B, t=0, t=1.0, n=252) <= 0.75 * S0 then\n"
               "    pay max(1.0 - B / S0, 0) as redemption\n  else\n    pay 0 as redemption\n  end\nend\n"},
    {"label": "phoenix-A", "names": ["A"], "seed": 103, "product": "autocall", "ki_daily": 1,
     "script": phoenix(["A"], True)},
    {"label": "worst-of-A-C", "names": ["A", "C"], "seed": 104, "product": "autocall", "ki_daily": 0, "corr": 0.5,
     "script": phoenix(["A", "C"], False)},
]


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
    from optlab.risk.engine import run_group
    from optlab.risk.shocks import Shock, VolMove
    from optlab.risk.surfaces import bumped_surface
    from optlab.structured.multiasset import BasketContext
    from optlab.structured.portfolio import Book, Position

    engines._compiled[:] = [native]
    T = 3.0 * np.arange(1, 41) / 40
    surf = {n: SSVI.power_law(rho, 1.0, 0.5, T, c * T) for n, (c, rho) in SURFACES.items()}
    out = {"r": R, "q": Q, "spot": S0, "n_paths": N_PATHS, "surfaces": SURFACES,
           "moves": {k: list(v) for k, v in MOVES.items()}, "trades": []}
    # the moved surfaces' local variance at sampled points
    rng = np.random.default_rng(9)
    k = rng.uniform(-1.2, 0.6, 200)
    Tq = rng.uniform(0.002, 3.5, 200)
    moved = {}
    for key, (kind, h) in MOVES.items():
        if kind == "spot":
            continue
        s = bumped_surface(surf["A"], parallel=h if kind == "parallel" else 0.0, skew=h if kind == "skew" else 0.0)
        moved[key] = np.asarray(s.local_var(k, Tq), dtype=float).tolist()
    out["moved_local_var"] = {"surface": "A", "k": k.tolist(), "T": Tq.tolist(), "base": surf["A"].local_var(k, Tq)
                              .tolist(), "moved": moved}
    for tr in TRADES:
        names = tuple(tr["names"])
        c = float(tr.get("corr", 0.0))
        corr = np.full((len(names), len(names)), c) + (1 - c) * np.eye(len(names))
        ctx = BasketContext(names, {n: Market.flat(S0, R, Q) for n in names}, {n: surf[n] for n in names}, corr,
                            dt.date(2026, 12, 4))
        shocks = {}
        for key, (kind, h) in MOVES.items():
            if kind == "spot":
                shocks[key] = Shock(spot={n: h for n in names})
            elif kind == "parallel":
                shocks[key] = Shock(vol={n: VolMove(parallel=h) for n in names})
            else:
                shocks[key] = Shock(vol={n: VolMove(skew=h) for n in names})
        run = run_group(RiskGroup(tr["label"], Book([Position(tr["label"], tr["script"], 1.0)]), ctx, tr["seed"]),
                        shocks, settings=RiskSettings(n_paths=N_PATHS, engine="cpu", model="lv"))
        entry = dict(tr, key=engines.seed64(tr["seed"]), base=[run.values["base"][0], run.base_se[0]],
                     method=run.method, model=run.model, values={}, pnl={})
        for key in MOVES:
            entry["values"][key] = run.values[key][0]
            entry["pnl"][key] = [run.pnl[key][0][0], run.pnl[key][1][0]]
        out["trades"].append(entry)
        print(tr["label"], run.method, run.model, entry["base"], {k: round(v[0], 5) for k, v in entry["pnl"].items()})
    (HERE / "reference_scenarios.json").write_text(json.dumps(out))
    print("wrote", HERE / "reference_scenarios.json")


if __name__ == "__main__":
    main(*sys.argv[1:])
