"""ob_price_noalloc: ob_price for callers that cannot allocate device memory while they price (all of it belongs to
another allocator, or cudaMalloc and cudaFree are not allowed on their quote loop). Called through the C ABI, it must
give what ob_price gives on the same request, call after call, although its scratch is a fixed array that every
call reuses. This file is collected last so that a run stopping at its first failure has run every other test."""

import ctypes as C

import pytest

from optlab_b200 import _abi

pytestmark = pytest.mark.gpu


def _request(model, product, legs, strikes, n_paths, seed):
    rq = _abi.ObRequest()
    rq.model, rq.product = model, product
    for k in range(3):
        rq.legs[k], rq.strikes[k] = legs[k], strikes[k]
    rq.H, rq.n_steps, rq.S0, rq.r, rq.q, rq.T, rq.sigma = 80.0, 52, 100.0, 0.04, 0.01, 1.0, 0.2
    rq.v0, rq.kappa, rq.theta, rq.xi, rq.rho = 0.0228, 3.09, 0.0537, 1.31, -0.69
    rq.n_paths, rq.seed = n_paths, seed
    return rq


def test_the_allocation_free_entry_point_prices_like_ob_price_call_after_call():
    lib = _abi.load()
    requests = [
        (_request(1, 2, (1, 0, 0), (100.0, 0.0, 0.0), 2**18, 11), _abi.OB_FP64),
        (_request(0, 0, (1, 2, 3), (95.0, 105.0, 100.0), 2**16, 12), _abi.OB_FP64),
        (_request(1, 0, (1, 1, 2), (100.0, 119.0, 80.0), 2**17, 13), _abi.OB_FP32),
    ]
    for rq, prec in requests:  # consecutive calls, each on a request unlike the last
        got, want = _abi.ObResult(), _abi.ObResult()
        _abi.check(lib.ob_price_noalloc(C.byref(rq), C.byref(got), prec))
        _abi.check(lib.ob_price(C.byref(rq), C.byref(want), prec))
        assert got.n_paths == want.n_paths == rq.n_paths
        assert 0.0 < got.kernel_ms <= got.total_ms  # the kernels' event time, as ob_price reports it
        for k in range(4):
            tol = 1e-12 * abs(want.price[k]) + 1e-300
            assert abs(got.price[k] - want.price[k]) <= tol, (k, got.price[k], want.price[k])
            assert abs(got.se[k] - want.se[k]) <= 1e-10 * abs(want.se[k]) + 1e-300


def test_the_allocation_free_entry_point_refuses_a_bad_request_like_ob_price():
    lib = _abi.load()
    rq = _request(1, 2, (1, 0, 0), (100.0, 0.0, 0.0), 2**10, 1)
    rq.H = 150.0  # a down-and-out barrier above the spot
    res = _abi.ObResult()
    assert lib.ob_price_noalloc(C.byref(rq), C.byref(res), _abi.OB_FP64) == _abi.OB_EINVAL
    assert b"barrier" in lib.ob_last_error()


def _free_bytes(lib):
    dev = _abi.ObDevice()
    _abi.check(lib.ob_device_info(0, C.byref(dev)))
    return dev.free_mem


def test_the_allocation_free_entry_point_leaves_device_memory_as_it_was():
    """After one call has loaded the library's device code, further calls take no device memory: the device's free
    memory is the same before and after a series of them."""
    lib = _abi.load()
    rq = _request(1, 2, (1, 0, 0), (100.0, 0.0, 0.0), 2**17, 21)
    res = _abi.ObResult()
    for prec in (_abi.OB_FP64, _abi.OB_FP32):
        _abi.check(lib.ob_price_noalloc(C.byref(rq), C.byref(res), prec))
    before = _free_bytes(lib)
    for i in range(6):
        rq.seed = 22 + i
        _abi.check(lib.ob_price_noalloc(C.byref(rq), C.byref(res), (_abi.OB_FP64, _abi.OB_FP32)[i % 2]))
    assert _free_bytes(lib) == before
