"""The C ABI without a GPU: the library loads and exports every symbol include/optlab_b200.h declares, the request
structs have the reference's layouts, and bad requests fail with the reference's messages before any device work."""

import ctypes as C
import os
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from optlab_b200 import _abi, engine, workloads
from optlab_b200.requests import paths_request

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "optlab_b200.h"
REF_HEADER = Path(os.environ.get("OPTLAB_REFERENCE", "/root/reference")) / "packages/native/cuda/include/optlab_cuda/requests.hpp"


def declared_symbols():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(ob_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported_and_bound():
    lib = _abi.load()
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
        assert s in _abi.SIGNATURES, f"{s} has no ctypes signature"
    assert set(_abi.SIGNATURES) == set(syms)


def _c_layout(header: Path, structs: dict, extra_flags=()):
    """sizeof and offsetof of each struct field, from a C++ compile of the header."""
    lines = ['#include <cstdio>', '#include <cstddef>', f'#include "{header}"', "int main() {"]
    for st, fields in structs.items():
        lines.append(f'std::printf("{st} %zu\\n", sizeof({st}));')
        for f in fields:
            lines.append(f'std::printf("{st}.{f} %zu\\n", offsetof({st}, {f}));')
    lines.append("return 0; }")
    src = Path("/tmp/ob_layout.cpp")
    src.write_text("\n".join(lines))
    exe = Path("/tmp/ob_layout")
    subprocess.run(["g++", "-std=c++17", *extra_flags, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return dict(line.rsplit(" ", 1) for line in out.strip().splitlines())


PAIRS = {
    "ob_request": _abi.ObRequest,
    "ob_result": _abi.ObResult,
    "ob_paths_request": _abi.ObPathsRequest,
    "ob_device": _abi.ObDevice,
    "ob_leverage_request": _abi.ObLeverageRequest,
    "ob_mc_request": _abi.ObMcRequest,
    "ob_mc_result": _abi.ObMcResult,
    "ob_adjoint_request": _abi.ObAdjointRequest,
    "ob_adjoint_result": _abi.ObAdjointResult,
    "ob_batch_trade": _abi.ObBatchTrade,
    "ob_batch_request": _abi.ObBatchRequest,
    "ob_script_request": _abi.ObScriptRequest,
    "ob_script_result": _abi.ObScriptResult,
}


def test_ctypes_mirrors_match_the_header():
    layout = _c_layout(HEADER, {k: [f for f, _ in v._fields_] for k, v in PAIRS.items()})
    for name, cls in PAIRS.items():
        assert int(layout[name]) == C.sizeof(cls), name
        for f, _ in cls._fields_:
            assert int(layout[f"{name}.{f}"]) == getattr(cls, f).offset, (name, f)


@pytest.mark.skipif(not REF_HEADER.exists(), reason="the reference tree is not present")
def test_the_drop_in_structs_have_the_references_layouts():
    """ob_paths_request, ob_leverage_request, ob_request, ob_result and ob_device are byte-compatible with
    optlab_paths_request, optlab_leverage_request, optlab_request, optlab_result and optlab_device."""
    mirror = {
        "optlab_request": _abi.ObRequest,
        "optlab_result": _abi.ObResult,
        "optlab_paths_request": _abi.ObPathsRequest,
        "optlab_device": _abi.ObDevice,
        "optlab_leverage_request": _abi.ObLeverageRequest,
    }
    layout = _c_layout(REF_HEADER, {k: [f for f, _ in v._fields_] for k, v in mirror.items()})
    for name, cls in mirror.items():
        assert int(layout[name]) == C.sizeof(cls), name
        for f, _ in cls._fields_:
            assert int(layout[f"{name}.{f}"]) == getattr(cls, f).offset, (name, f)


def test_queries_answer_without_a_device():
    lib = _abi.load()
    assert lib.ob_has_cuda() == 1 and lib.ob_cpu_threads() >= 1 and lib.ob_version() >= 10000
    assert lib.ob_gpu_count() >= 0


def _base_paths(**over):
    kw = dict(
        dt=[0.1], t0=[0.0], obs_step=[1], root=[[1.0]], kind=[0], cvar=[0.04], heston=[0, 1, 1, 0, 0], same=1,
        fwd=[[100.0]], n_pairs=4, seed=1,
    )
    kw.update(over)
    return paths_request(**kw)


@pytest.mark.parametrize(
    "over,message",
    [
        (dict(kind=[7]), "kind must be 0 to 3"),
        (dict(obs_step=[2]), "obs_step must be nondecreasing in [0, n_steps]"),
        (dict(kind=[1], n_x=1), "a tabulated variance needs n_x >= 2, rows and step_row"),
        (dict(kind=[2], heston=[0.04, -1.0, 0.04, 0.5, -0.7]), "Heston parameters out of range"),
        (dict(win_lo=[0], win_hi=[3]), "bad window"),
        (dict(mixer=1), "bad local correlation"),
    ],
)
def test_bad_path_requests_fail_with_the_references_messages(over, message):
    """RC/src/requests.cpp:168-207: the same checks, an EngineError instead of std::invalid_argument."""
    h = _base_paths(**over)
    with pytest.raises(_abi.EngineError, match=re.escape(message)):
        engine.paths(h, "fp32")


def test_too_many_names_is_refused():
    kw = dict(dt=[0.1], t0=[0.0], obs_step=[1], root=np.eye(9), kind=[0] * 9, cvar=[0.04] * 9,
              heston=np.tile([0, 1, 1, 0, 0], 9), same=1, fwd=np.full((9, 1), 100.0), n_pairs=4, seed=1)
    with pytest.raises(_abi.EngineError, match="n_names must be 1 to 8"):
        engine.paths(paths_request(**kw), "fp64")


def test_bad_fused_requests_and_precisions_are_refused():
    h = workloads.lv_phoenix(n_paths=64)
    with pytest.raises(ValueError, match="precision"):
        engine.mc_price(h, "fp16")
    h.struct.obs_step[1] = h.struct.obs_step[0]
    with pytest.raises(_abi.EngineError, match="obs_step must be increasing"):
        engine.mc_price(h, "fp32")
    q = workloads.heston_qe_ladder(n_paths=64)
    q.struct.n_names = 2
    with pytest.raises(_abi.EngineError, match="the QE model has one name"):
        engine.mc_price(q, "fp64")


def test_a_missing_device_is_an_engine_error_not_a_crash():
    lib = _abi.load()
    if lib.ob_gpu_count() > 0:
        pytest.skip("a device is present")
    with pytest.raises(_abi.EngineError, match="no CUDA device"):
        engine.mc_price(workloads.lv_phoenix(n_paths=64), "fp32")


def test_an_adjoint_checkpoint_interval_other_than_0_1_or_4_is_refused():
    from optlab_b200.adjoint import AdjointPlan

    with pytest.raises(_abi.EngineError, match="checkpoint must be 0, 1 or 4"):
        AdjointPlan(workloads.worst_of(n_paths=2**10, years=1.0).held, 0.005, "fp32", checkpoint=2)
