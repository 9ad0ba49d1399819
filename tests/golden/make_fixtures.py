"""Writes tests/golden/reference_paths.json: the reference's own golden path vectors with the inputs that produced them.

Source: the reference's tests/golden/native_cpu.json (paths of its compiled CPU engine, recorded by its golden.py
`native_cpu` group, tests/golden/golden.py:409-423) and tests/golden/calibration_simulated.json (the calibrated
Heston parameters and SVI surface of its "simulated" market, golden.py:249-326). The inputs are rebuilt here with the
reference's own Python (optlab.core from the reference tree): the Black-Scholes volatility is the surface's ATM vol at
one year (structured/context.py:154-164), the Heston model is the recorded fit, the market is Market.flat(100, 0.04,
0.012), and the time grid is models.time_grid([0.25, 0.5, 1], 1/252, 1/2000) (Black-Scholes: one step per date).

Run where the reference tree is present:  python tests/golden/make_fixtures.py [reference root; default $OPTLAB_REFERENCE, else /root/reference]
"""

from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def main(ref_root: str = os.environ.get("OPTLAB_REFERENCE", "/root/reference")) -> None:
    ref = Path(ref_root)
    sys.path[:0] = [str(ref / "packages/core/src")]
    from optlab.core.market import Market
    from optlab.core.models import time_grid
    from optlab.core.svi import SVISurface

    cal = json.loads((ref / "tests/golden/calibration_simulated.json").read_text())["values"]
    gold = json.loads((ref / "tests/golden/native_cpu.json").read_text())["values"]
    market = Market.flat(100.0, 0.04, 0.012)
    times = [0.25, 0.5, 1.0]
    surface = SVISurface.from_dict(cal["surface"])
    vol = float(surface.iv(0.0, 1.0))
    hp = cal["heston"]
    out = {
        "source": "reference tests/golden/native_cpu.json (paths) and calibration_simulated.json (inputs)",
        "seed": 7,
        "n_paths": 20000,
        "times": times,
        "fwd": [float(x) for x in market.F(np.array(times))],
        "cases": {
            "bs": {
                "kind": 0,
                "cvar": vol * vol,
                "heston": [0.0, 1.0, 1.0, 0.0, 0.0],
                "grid": [0.0, *times],
                "expected": gold["paths"]["bs"],
            },
            "heston": {
                "kind": 2,
                "cvar": 0.0,
                "heston": [hp["v0"], hp["kappa"], hp["theta"], hp["xi"], hp["rho"]],
                "grid": [float(x) for x in time_grid(np.array(times), 1 / 252, 1 / 2000)],
                "expected": gold["paths"]["heston"],
            },
        },
    }
    (HERE / "reference_paths.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", HERE / "reference_paths.json")


if __name__ == "__main__":
    main(*sys.argv[1:])
