"""The multi-rank path on CPU: two gloo ranks price disjoint pair ranges of one fused request on the oracle and pool
their sums with one all-reduce; the pooled price and SE equal one run over all pairs (draws depend only on the global
pair index, and the estimator is the same)."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from optlab_b200 import shard, workloads


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, n_pairs, weak, out):
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parent.parent
    for p in (root / "option-pricing-lab_b200", root / "oracle"):
        sys.path.insert(0, str(p))
    import datetime

    import torch.distributed as dist

    from oracle import Oracle
    from optlab_b200 import shard as sh
    from optlab_b200 import workloads as wl

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        first, count = sh.pair_range(n_pairs, rank, world, weak=weak)
        held = wl.heston_qe_ladder(n_paths=2 * n_pairs, n_steps=24)
        held.struct.first_pair, held.struct.n_pairs = first, count
        res = Oracle().mc_price(held, threads=2)
        price, se = sh.allreduce_result(res)
        out[rank] = (list(price), list(se))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_pairs", [4096, 4099])
def test_two_gloo_ranks_pool_to_the_single_run(oracle, n_pairs):
    held = workloads.heston_qe_ladder(n_paths=2 * n_pairs, n_steps=24)
    whole = oracle.mc_price(held, threads=2)
    k = whole.n_out
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, n_pairs, False, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        price, se = map(np.array, out[r])
        assert np.allclose(price, whole.price[:k], rtol=1e-12, atol=1e-14)
        assert np.allclose(se, whole.se[:k], rtol=1e-9, atol=1e-14)


def test_weak_ranges_are_disjoint_and_strong_ranges_cover_the_job():
    assert [shard.pair_range(100, r, 4, weak=True) for r in range(4)] == [(0, 100), (100, 100), (200, 100), (300, 100)]
    parts = [shard.pair_range(10, r, 3) for r in range(3)]
    assert parts == [(0, 4), (4, 3), (7, 3)]
    with pytest.raises(ValueError):
        shard.pair_range(10, 3, 3)


def test_combine_pools_the_raw_sums():
    """Shards pool the FP64 sums as accumulated: the pooled estimate equals the estimate of the summed sums exactly,
    also where price and se could not give the sums back (a large mean with a small spread)."""
    from types import SimpleNamespace

    rng = np.random.default_rng(0)
    y = 1e4 + 1e-3 * rng.normal(size=(1000, 3))

    def res(a):
        return SimpleNamespace(n_out=3, n_paths=2 * len(a), sum_y=list(a.sum(0)), sum_y2=list((a**2).sum(0)))

    parts = [res(y[:300]), res(y[300:])]
    p, s = shard.combine(parts)
    tot = np.concatenate([[1000.0], y[:300].sum(0) + y[300:].sum(0), (y[:300]**2).sum(0) + (y[300:]**2).sum(0)])
    m, se = shard.estimate(tot)
    assert np.array_equal(p, m) and np.array_equal(s, se)
    assert np.allclose(p, y.mean(0), rtol=1e-14)
