"""Sharding a fused request over ranks (one process per GPU) and combining the ranks' estimates.

The draws of a pair depend only on (seed, global pair index) (the reference's contract, packages/native/src/optlab/
native/__init__.py:317-323: batches and chunks are invisible), so rank r simulates its own range of global pairs and
the only exchange is the FP64 sums of the pair values: n, sum y and sum y^2 per output, combined once at the end.
`pair_range` splits a fixed job (strong scaling) or gives every rank the same count (weak scaling); `result_sums`
reads a rank's sums from its result (the engine returns them beside the estimate); `combine` and `allreduce_result`
pool them into the job's price and SE, with the same estimator as a single run (mean of pair values,
SE = sqrt((E[y^2] - mean^2) / (n - 1))). The sums are pooled as the kernels wrote them: rebuilding them from
(price, se) would subtract nearly equal numbers and lose the FP64 sums' digits.
"""

from __future__ import annotations

import numpy as np


def pair_range(n_pairs: int, rank: int, world: int, weak: bool = False) -> tuple[int, int]:
    """(first_pair, count) of a rank. Weak: every rank n_pairs pairs, rank r from r n_pairs. Strong: n_pairs split
    into contiguous ranges, the first n_pairs % world ranks one pair longer."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    if weak:
        return rank * n_pairs, n_pairs
    base, extra = divmod(int(n_pairs), world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def result_sums(res) -> np.ndarray:
    """[n, sum y_k..., sum y_k^2...] of an ob_mc_result over its n_paths / 2 pairs: the FP64 sums the engine (or the
    oracle) accumulated, as they are."""
    k = int(res.n_out)
    return np.concatenate([[res.n_paths / 2.0], np.asarray(res.sum_y[:k], float), np.asarray(res.sum_y2[:k], float)])


def estimate(sums: np.ndarray):
    """(price, se) per output from pooled sums [n, s1..., s2...]."""
    n = float(sums[0])
    k = (len(sums) - 1) // 2
    s1, s2 = np.asarray(sums[1:1 + k]), np.asarray(sums[1 + k:])
    mean = s1 / n
    se = np.sqrt(np.maximum(s2 / n - mean**2, 0.0) / (n - 1.0)) if n > 1 else np.zeros(k)
    return mean, se


def combine(parts) -> tuple[np.ndarray, np.ndarray]:
    """Pool the results of disjoint pair ranges (ob_mc_result each) into the job's (price, se)."""
    return estimate(sum(result_sums(r) for r in parts))


def allreduce_result(res, group=None, device=None):
    """The job's (price, se) from every rank's result (ob_mc_result), by one FP64 all-reduce of the sums (gloo on
    CPU tensors, NCCL on CUDA tensors)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor(result_sums(res), dtype=torch.float64, device=device)
    dist.all_reduce(t, group=group)
    return estimate(t.cpu().numpy())
