"""Build the C ABI's request structs from NumPy arrays, keeping the arrays alive as long as the struct.

`PathsSpec` holds what a path request needs besides the pairs (the reference's `Plan`,
packages/native/src/optlab/native/__init__.py:215-240); `McSpec` adds a product for the fused kernel.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import ObMcRequest, ObPathsRequest, ptr

_I = C.c_int


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


@dataclass
class Held:
    """A request struct and the arrays its pointers point into."""

    struct: C.Structure
    keep: list = field(default_factory=list)

    def ref(self):
        return C.byref(self.struct)


def paths_request(
    *,
    dt,
    t0,
    obs_step,
    root,
    kind,
    cvar,
    heston,
    same,
    fwd,
    n_pairs,
    seed,
    first_pair=0,
    step_row=None,
    lo=None,
    inv_dx=None,
    table=None,
    n_x=0,
    mixer=0,
    mix=(0.0,) * 8,
    low_root=None,
    col_of=None,
    n_keep=None,
    win_lo=(),
    win_hi=(),
    out=None,
) -> Held:
    """An ObPathsRequest (the reference's optlab_paths_request) over arrays converted here; `out` is allocated as
    (names, n_cols, 2 n_pairs) float64 when not given."""
    a = {
        "dt": f64(dt),
        "t0": f64(t0),
        "obs_step": i32(obs_step),
        "root": f64(root),
        "kind": i32(kind),
        "cvar": f64(cvar),
        "heston": f64(heston),
        "fwd": f64(fwd),
        "step_row": i32(step_row) if step_row is not None else np.empty(0, np.int32),
        "lo": f64(lo) if lo is not None else np.empty(0),
        "inv_dx": f64(inv_dx) if inv_dx is not None else np.empty(0),
        "table": f64(table) if table is not None else np.empty(0),
        "low_root": f64(low_root) if low_root is not None else np.empty(0),
        "win_lo": i32(win_lo),
        "win_hi": i32(win_hi),
    }
    n_names, n_obs = len(a["kind"]), len(a["obs_step"])
    if col_of is None:
        col_of = np.arange(n_obs, dtype=np.int32)
    a["col_of"] = i32(col_of)
    if n_keep is None:
        n_keep = int(a["col_of"].max()) + 1 if n_obs else 0
    n_cols = n_keep + 2 * len(a["win_lo"])
    if out is None:
        out = np.empty((n_names, n_cols, 2 * n_pairs))
    a["out"] = out
    s = ObPathsRequest()
    s.n_names, s.n_steps, s.n_obs, s.n_x = n_names, len(a["dt"]), n_obs, int(n_x)
    s.n_rows = len(a["lo"])
    s.n_pairs, s.first_pair, s.seed = int(n_pairs), int(first_pair), int(seed) & (2**64 - 1)
    s.dt, s.t0, s.obs_step, s.root = ptr(a["dt"]), ptr(a["t0"]), ptr(a["obs_step"], _I), ptr(a["root"])
    s.kind, s.cvar, s.heston, s.same = ptr(a["kind"], _I), ptr(a["cvar"]), ptr(a["heston"]), int(same)
    s.step_row, s.row_lo, s.row_inv_dx = ptr(a["step_row"], _I), ptr(a["lo"]), ptr(a["inv_dx"])
    s.table, s.fwd, s.mixer = ptr(a["table"]), ptr(a["fwd"]), int(mixer)
    for k in range(8):
        s.mix[k] = float(mix[k])
    s.low_root = ptr(a["low_root"])
    s.n_cols, s.n_keep, s.col_of = n_cols, int(n_keep), ptr(a["col_of"], _I)
    s.n_windows, s.win_lo, s.win_hi = len(a["win_lo"]), ptr(a["win_lo"], _I), ptr(a["win_hi"], _I)
    s.out = ptr(out)
    return Held(s, list(a.values()))


def mc_request(
    *,
    model: int,
    dt,
    t0,
    spot,
    n_pairs,
    seed,
    first_pair=0,
    root=None,
    kind=None,
    cvar=None,
    heston=None,
    same=1,
    log_fwd=None,
    step_row=None,
    lo=None,
    inv_dx=None,
    table=None,
    n_x=0,
    r=0.0,
    q=0.0,
    product: int,
    leg_type=(),
    leg_strike=(),
    leg_barrier=(),
    leg_level=(),
    discount=1.0,
    obs_step=(),
    obs_discount=(),
    trigger=(),
    coupon_barrier=0.0,
    coupon=0.0,
    ki_barrier=0.0,
    put_strike=1.0,
    memory=0,
    ki_daily=0,
    mixer=0,
    mix=(0.0,) * 8,
    low_root=None,
) -> Held:
    """An ObMcRequest: a model (OB_MODEL_PATHS or OB_MODEL_HESTON_QE) plus a product (ladder or autocall); mixer,
    mix and low_root: a local-correlation basket (the reference plan's fields of the same names)."""
    spot = f64(np.atleast_1d(spot))
    n = len(spot)
    a = {
        "dt": f64(dt),
        "t0": f64(t0),
        "spot": spot,
        "root": f64(root if root is not None else np.eye(n)),
        "kind": i32(kind if kind is not None else np.zeros(n)),
        "cvar": f64(cvar if cvar is not None else np.zeros(n)),
        "heston": f64(heston if heston is not None else np.tile([0.0, 1.0, 1.0, 0.0, 0.0], n)),
        "log_fwd": f64(log_fwd) if log_fwd is not None else np.empty(0),
        "step_row": i32(step_row) if step_row is not None else np.empty(0, np.int32),
        "lo": f64(lo) if lo is not None else np.empty(0),
        "inv_dx": f64(inv_dx) if inv_dx is not None else np.empty(0),
        "table": f64(table) if table is not None else np.empty(0),
        "leg_type": i32(leg_type),
        "leg_strike": f64(leg_strike),
        "leg_barrier": i32(leg_barrier) if len(leg_barrier) else np.zeros(len(leg_type), np.int32),
        "leg_level": f64(leg_level) if len(leg_level) else np.zeros(len(leg_type)),
        "obs_step": i32(obs_step),
        "obs_discount": f64(obs_discount),
        "trigger": f64(trigger),
        "low_root": f64(low_root) if low_root is not None else np.empty(0),
    }
    s = ObMcRequest()
    s.model, s.n_names, s.n_steps = int(model), n, len(a["dt"])
    s.n_pairs, s.first_pair, s.seed = int(n_pairs), int(first_pair), int(seed) & (2**64 - 1)
    s.dt, s.t0, s.root, s.kind = ptr(a["dt"]), ptr(a["t0"]), ptr(a["root"]), ptr(a["kind"], _I)
    s.cvar, s.heston, s.same = ptr(a["cvar"]), ptr(a["heston"]), int(same)
    s.n_x, s.n_rows = int(n_x), len(a["lo"])
    s.step_row, s.row_lo, s.row_inv_dx, s.table = ptr(a["step_row"], _I), ptr(a["lo"]), ptr(a["inv_dx"]), ptr(a["table"])
    s.spot, s.log_fwd, s.r, s.q = ptr(a["spot"]), ptr(a["log_fwd"]), float(r), float(q)
    s.product = int(product)
    s.n_legs = len(a["leg_type"])
    s.leg_type, s.leg_strike = ptr(a["leg_type"], _I), ptr(a["leg_strike"])
    s.leg_barrier, s.leg_level, s.discount = ptr(a["leg_barrier"], _I), ptr(a["leg_level"]), float(discount)
    s.n_obs, s.obs_step = len(a["obs_step"]), ptr(a["obs_step"], _I)
    s.obs_discount, s.trigger = ptr(a["obs_discount"]), ptr(a["trigger"])
    s.coupon_barrier, s.coupon, s.ki_barrier, s.put_strike = (
        float(coupon_barrier),
        float(coupon),
        float(ki_barrier),
        float(put_strike),
    )
    s.memory, s.ki_daily = int(memory), int(ki_daily)
    s.mixer, s.low_root = int(mixer), ptr(a["low_root"])
    for k in range(8):
        s.mix[k] = float(mix[k])
    return Held(s, list(a.values()))


def result_arrays(res: _abi.ObMcResult):
    """(price, se) of a fused result as float64 arrays of n_out values."""
    n = res.n_out
    return np.array(res.price[:n]), np.array(res.se[:n])
