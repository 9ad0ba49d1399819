"""ORACLE — test infrastructure only: ctypes access to the CPU checkers.

- `Oracle`: this repository's C restatement of the reference's path algorithms (oracle/optlab_oracle.c, built into
  oracle/liboptlab_oracle.so by `make -C oracle`).
- `Reference`: the reference's own CPU engine, compiled from its sources (`make -C oracle ref`, into
  oracle/_ref/libref_optlab.so), behind the extern "C" shim oracle/ref_shim.cpp. Present only where it was built.

Only tests, the smoke check and the benchmark's CPU-baseline leg import this module; the engine never does.
"""

from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_PKG = HERE.parent / "option-pricing-lab_b200"
if str(_PKG) not in sys.path:
    sys.path.insert(0, str(_PKG))

from optlab_b200._abi import (  # noqa: E402
    ObBatchRequest,
    ObLeverageRequest,
    ObMcRequest,
    ObMcResult,
    ObPathsRequest,
    ObRequest,
    ObResult,
)

ORACLE_LIB = HERE / "liboptlab_oracle.so"
REF_LIB = HERE / "_ref" / "libref_optlab.so"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class OracleError(RuntimeError):
    pass


class Oracle:
    """The C restatement (double precision, deterministic in the thread count)."""

    def __init__(self, path: Path = ORACLE_LIB):
        if not path.exists():
            raise OracleError(f"{path} is not built: make -C oracle")
        lib = C.CDLL(str(path))
        lib.or_last_error.restype = C.c_char_p
        lib.or_paths.argtypes = [C.POINTER(ObPathsRequest), C.c_int]
        lib.or_mc_price.argtypes = [C.POINTER(ObMcRequest), C.c_int, C.POINTER(ObMcResult)]
        lib.or_price.argtypes = [C.POINTER(ObRequest), C.c_int, C.POINTER(ObResult)]
        lib.or_leverage.argtypes = [C.POINTER(ObLeverageRequest)]
        lib.or_autocall_smooth.argtypes = [C.POINTER(ObMcRequest), C.c_double, C.c_int, C.POINTER(ObMcResult)]
        lib.or_philox_normals.argtypes = [
            C.c_ulonglong,
            C.c_longlong,
            C.c_longlong,
            C.c_uint,
            C.c_ulonglong,
            C.c_int,
            C.POINTER(C.c_uint),
            _dp,
        ]
        lib.or_philox.argtypes = [C.POINTER(C.c_uint), C.c_uint, C.c_uint, C.POINTER(C.c_uint)]
        lib.or_batch_trade.argtypes = [C.POINTER(ObBatchRequest), C.c_int, C.c_int, _dp, _dp]
        self.lib = lib

    def _check(self, st: int) -> None:
        if st:
            raise OracleError(self.lib.or_last_error().decode())

    def paths(self, held, threads: int = 0) -> None:
        self._check(self.lib.or_paths(held.ref(), int(threads) or _cores()))

    def mc_price(self, held, threads: int = 0) -> ObMcResult:
        res = ObMcResult()
        self._check(self.lib.or_mc_price(held.ref(), int(threads) or _cores(), C.byref(res)))
        return res

    def autocall_smooth(self, held, eps: float, threads: int = 0):
        """(price, SE) of the smoothed autocall (the reference evaluator's ramps of relative width eps)."""
        res = ObMcResult()
        self._check(self.lib.or_autocall_smooth(held.ref(), float(eps), int(threads) or _cores(), C.byref(res)))
        return res.price[0], res.se[0]

    def batch_trade(self, book, trade: int, threads: int = 0):
        """(price, se) of one trade of a batch under each of its scenarios (base, spot, carry, vol and correlation
        moves), each scenario its own simulation on the trade's seed."""
        n = book.n_scenarios
        price, se = np.empty(n), np.empty(n)
        self._check(self.lib.or_batch_trade(C.byref(book.struct), int(trade), int(threads) or _cores(),
                                            price.ctypes.data_as(_dp), se.ctypes.data_as(_dp)))
        return price, se

    def price(self, rq: ObRequest, threads: int = 0) -> ObResult:
        res = ObResult()
        self._check(self.lib.or_price(C.byref(rq), int(threads) or _cores(), C.byref(res)))
        return res

    def leverage(self, held) -> None:
        self._check(self.lib.or_leverage(held.ref()))

    def philox_normals(self, seed, first_pair, n_pairs, tag, first_block, n_blocks):
        u = np.empty((n_pairs, n_blocks, 4), np.uint32)
        z = np.empty((n_pairs, n_blocks, 4))
        self._check(
            self.lib.or_philox_normals(
                seed,
                first_pair,
                n_pairs,
                tag,
                first_block,
                n_blocks,
                u.ctypes.data_as(C.POINTER(C.c_uint)),
                z.ctypes.data_as(_dp),
            )
        )
        return u, z

    def philox(self, counter, k0, k1):
        c = (C.c_uint * 4)(*[int(x) for x in counter])
        out = (C.c_uint * 4)()
        self.lib.or_philox(c, k0, k1, out)
        return list(out)


class Reference:
    """The reference's CPU engine (optlab::api) and the composed QE harness of oracle/ref_shim.cpp."""

    def __init__(self, path: Path = REF_LIB):
        if not path.exists():
            raise OracleError(f"{path} is not built: make -C oracle ref (needs the reference tree)")
        lib = C.CDLL(str(path))
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_paths.argtypes = [C.POINTER(ObPathsRequest), C.c_int]
        lib.ref_leverage.argtypes = [C.POINTER(ObLeverageRequest), C.c_int]
        lib.ref_price.argtypes = [C.POINTER(ObRequest), C.c_int, C.POINTER(ObResult)]
        lib.ref_philox_normals.argtypes = [
            C.c_ulonglong,
            C.c_longlong,
            C.c_longlong,
            C.c_uint,
            C.c_ulonglong,
            C.c_int,
            C.POINTER(C.c_uint),
            _dp,
        ]
        lib.ref_qe_ladder.argtypes = [
            C.c_double,
            C.c_double,
            C.c_double,
            C.c_double,
            C.c_int,
            _dp,
            C.c_longlong,
            C.c_longlong,
            C.c_ulonglong,
            C.c_int,
            _ip,
            _dp,
            _ip,
            _dp,
            C.c_int,
            _dp,
            _dp,
        ]
        self.lib = lib

    def _check(self, st: int) -> None:
        if st:
            raise OracleError(self.lib.ref_last_error().decode())

    def paths(self, held, threads: int = 0) -> None:
        self._check(self.lib.ref_paths(held.ref(), int(threads)))

    def leverage(self, held, threads: int = 1) -> None:
        self._check(self.lib.ref_leverage(held.ref(), int(threads)))

    def price(self, rq: ObRequest, threads: int = 1) -> ObResult:
        res = ObResult()
        self._check(self.lib.ref_price(C.byref(rq), int(threads), C.byref(res)))
        return res

    def philox_normals(self, seed, first_pair, n_pairs, tag, first_block, n_blocks):
        u = np.empty((n_pairs, n_blocks, 4), np.uint32)
        z = np.empty((n_pairs, n_blocks, 4))
        self._check(
            self.lib.ref_philox_normals(
                seed,
                first_pair,
                n_pairs,
                tag,
                first_block,
                n_blocks,
                u.ctypes.data_as(C.POINTER(C.c_uint)),
                z.ctypes.data_as(_dp),
            )
        )
        return u, z

    def qe_ladder(self, S0, r, q, T, n_steps, heston, n_pairs, seed, leg_type, leg_strike, leg_up_out, leg_level,
                  first_pair=0, threads=0):
        """Prices and SEs of the QE ladder (legs, then E[S_T]) on the reference's own QE step and Philox stream."""
        h = np.ascontiguousarray(heston, dtype=np.float64)
        lt = np.ascontiguousarray(leg_type, dtype=np.int32)
        ls = np.ascontiguousarray(leg_strike, dtype=np.float64)
        lu = np.ascontiguousarray(leg_up_out, dtype=np.int32)
        ll = np.ascontiguousarray(leg_level, dtype=np.float64)
        price, se = np.empty(len(lt) + 1), np.empty(len(lt) + 1)
        self._check(
            self.lib.ref_qe_ladder(
                S0, r, q, T, n_steps, h.ctypes.data_as(_dp), n_pairs, first_pair, seed, len(lt),
                lt.ctypes.data_as(_ip), ls.ctypes.data_as(_dp), lu.ctypes.data_as(_ip), ll.ctypes.data_as(_dp),
                threads, price.ctypes.data_as(_dp), se.ctypes.data_as(_dp),
            )
        )
        return price, se


def _cores() -> int:
    import os

    return os.cpu_count() or 1


def reference_available() -> bool:
    return REF_LIB.exists()
