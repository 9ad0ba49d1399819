"""The node-vega parameterisation without a GPU: tent weights, the bump field and the contraction of table gradients
(the chain rule that turns dV/d(table) into vegas per node)."""

import numpy as np
import torch

from optlab_b200 import workloads
from optlab_b200.adjoint import VegaNodes, hats


def _nodes():
    w = workloads.worst_of(n_paths=64, years=1.0)
    return w, VegaNodes(w.row_name, w.row_T, w.row_lo, w.row_inv_dx, w.n_x, w.node_T, w.node_k, device="cpu")


def test_tent_weights_interpolate_and_sum_to_one():
    nodes = np.array([0.0, 1.0, 3.0])
    w = hats([-1.0, 0.0, 0.5, 2.0, 3.0, 9.0], nodes)
    assert np.allclose(w.sum(1), 1.0)
    assert np.allclose(w[2], [0.5, 0.5, 0.0]) and np.allclose(w[3], [0.0, 0.5, 0.5])
    assert np.allclose(w[0], [1, 0, 0]) and np.allclose(w[-1], [0, 0, 1])


def test_a_bump_of_every_node_of_a_name_is_a_parallel_shift_of_its_rows():
    w, n = _nodes()
    b = torch.zeros(n.shape, dtype=torch.float64)
    b[1] = 0.01
    field = n.bump_field(b).numpy()
    rows = w.row_name == 1
    assert np.allclose(field[rows], 0.01) and np.allclose(field[~rows], 0.0)


def test_the_contraction_is_the_chain_rule_of_the_bumped_table():
    """d/d(bump) of sum(G * table(bump)) at zero equals contract(G): autograd through table() against the closed form,
    and the batched contraction against the one-at-a-time one."""
    w, n = _nodes()
    rng = np.random.default_rng(3)
    base = torch.tensor(rng.uniform(0.01, 0.09, (len(w.row_name), w.n_x)))
    G = torch.tensor(rng.normal(size=(4, len(w.row_name), w.n_x)))
    bumps = torch.zeros(n.shape, dtype=torch.float64, requires_grad=True)
    (auto,) = torch.autograd.grad((G[0] * n.table(base, bumps)).sum(), bumps)
    assert torch.allclose(auto, n.contract(G[0], base), rtol=1e-12, atol=1e-14)
    stacked = torch.stack([n.contract(G[k], base) for k in range(4)])
    assert torch.allclose(n.contract_batches(G, base), stacked, rtol=1e-12, atol=1e-14)
