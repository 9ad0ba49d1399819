"""optlab_b200: a B200 (sm_100a) Monte Carlo path engine behind the reference's engine-by-name interface."""

from __future__ import annotations

from ._abi import EngineError, load

__all__ = ["EngineError", "load"]
