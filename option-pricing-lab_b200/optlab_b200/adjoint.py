"""Adjoint Greeks behind a torch.autograd.Function: delta per name and vega per node of the local-vol surface.

`AdjointPlan` drives the C ABI's ob_adjoint_* (csrc/adjoint.cu): one forward pass with checkpoints and one backward
pass give the price of a smoothed autocall under local vol, its deltas, and the gradient of the price with respect to
every entry of the local-variance table. `AutocallPrice` exposes that as a differentiable function of the table, so
any parameterisation of the table that torch can differentiate gets its sensitivities by the chain rule; `VegaNodes`
is the one of the benchmark: tent bumps of the local volatility on a grid of expiries x log-strikes per name,
sigma_loc(T, k) + sum_es b_es phi_e(T) psi_s(k), the table being its square. This replaces the reference's node vegas
by bump-and-revalue (packages/risk/src/optlab/risk/greeks.py:199-244, one simulation per bumped node).

Standard errors of the vegas come from batch means: the backward pass keeps one gradient per batch of pairs.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from ._abi import OB_ADJ_BATCHES, ObAdjointRequest, ObAdjointResult, check, load
from .engine import precision_code


class AdjointPlan:
    """A local-vol autocall request (OB_MODEL_PATHS, kinds 1, OB_PRODUCT_AUTOCALL) uploaded for adjoint runs.
    checkpoint: the steps between the states the forward keeps for the backward (1: every step, the backward
    recomputes nothing; 4: every fourth, a quarter of the memory; 0: every step up to 24 GiB of states)."""

    def __init__(self, held, smoothing: float = 0.005, precision="fp32", checkpoint: int = 0):
        self._held = held
        rq = ObAdjointRequest()
        rq.base = held.struct
        rq.smoothing = float(smoothing)
        rq.checkpoint = int(checkpoint)
        self._rq = rq
        self._p = C.c_void_p()
        check(load().ob_adjoint_plan_create(C.byref(rq), precision_code(precision), C.byref(self._p)))
        s = held.struct
        self.n_rows, self.n_x, self.n_names, self.n_pairs = s.n_rows, s.n_x, s.n_names, s.n_pairs
        self.gradient = None      # E[d(pair value) / d(table)], (n_rows, n_x)
        self.batch_grad = None    # per batch sums, (OB_ADJ_BATCHES, n_rows, n_x)
        self.batch_pairs = None   # pairs of each batch
        self.last = None          # the last run's ObAdjointResult

    def run(self, table: torch.Tensor | None = None, grad: bool = True, stream=None) -> ObAdjointResult:
        """One forward pass (and the backward pass with grad). table: CUDA (n_rows, n_x) local variance replacing the
        current one, or None. The result holds the price, its SE and the deltas."""
        lib = load()
        dev = torch.device("cuda", torch.cuda.current_device())
        t = None
        if table is not None:
            t = table.detach().to(dev, torch.float64).contiguous()
            if t.shape != (self.n_rows, self.n_x):
                raise ValueError(f"table must be ({self.n_rows}, {self.n_x}), not {tuple(t.shape)}")
        g = torch.empty((OB_ADJ_BATCHES, self.n_rows, self.n_x), dtype=torch.float64, device=dev) if grad else None
        st = stream or torch.cuda.current_stream()
        check(
            lib.ob_adjoint_run(
                self._p,
                C.c_void_p(t.data_ptr()) if t is not None else None,
                C.c_void_p(g.data_ptr()) if g is not None else None,
                C.c_void_p(st.cuda_stream),
            )
        )
        res = ObAdjointResult()
        bp = (C.c_longlong * OB_ADJ_BATCHES)()
        check(lib.ob_adjoint_result_get(self._p, C.byref(res), bp))
        self.last = res
        if g is not None:
            self.batch_grad = g
            self.batch_pairs = torch.tensor(list(bp), dtype=torch.float64, device=dev)
            self.gradient = g.sum(0) / self.n_pairs
        return res

    def close(self) -> None:
        if self._p:
            load().ob_adjoint_plan_destroy(self._p)
            self._p = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 (interpreter shutdown)
            pass


class AutocallPrice(torch.autograd.Function):
    """price = f(table): forward and backward passes of the engine; the gradient is dV/d(table)."""

    @staticmethod
    def forward(ctx, table: torch.Tensor, plan: AdjointPlan):
        res = plan.run(table, grad=True)
        ctx.save_for_backward(plan.gradient)
        return torch.tensor(res.price, dtype=torch.float64, device=table.device)

    @staticmethod
    def backward(ctx, g):
        (G,) = ctx.saved_tensors
        return g * G, None


def hats(points, nodes) -> np.ndarray:
    """Tent weights (len(points), len(nodes)) of piecewise-linear interpolation on `nodes`, flat beyond both ends, so
    that the weights of a point sum to one (a bump of every node is a parallel bump)."""
    points, nodes = np.asarray(points, float), np.asarray(nodes, float)
    w = np.zeros((points.size, nodes.size))
    x = np.clip(points.ravel(), nodes[0], nodes[-1])
    j = np.clip(np.searchsorted(nodes, x, side="right") - 1, 0, nodes.size - 2)
    f = (x - nodes[j]) / (nodes[j + 1] - nodes[j])
    rows = np.arange(x.size)
    w[rows, j] = 1.0 - f
    w[rows, j + 1] += f
    return w


@dataclass
class VegaNodes:
    """Tent bumps of local volatility on node_T x node_k per name, for the rows of each name in a stacked table.

    row_name[r] is the name a table row belongs to, row_T[r] its expiry, row_lo / row_inv_dx its log-strike grid.
    The weights live on `device` (default: the current CUDA device when there is one, else the CPU)."""

    row_name: np.ndarray
    row_T: np.ndarray
    row_lo: np.ndarray
    row_inv_dx: np.ndarray
    n_x: int
    node_T: np.ndarray
    node_k: np.ndarray
    device: object = None

    def __post_init__(self):
        if self.device is not None:
            dev = torch.device(self.device)
        elif torch.cuda.is_available():
            dev = torch.device("cuda", torch.cuda.current_device())
        else:
            dev = torch.device("cpu")
        k = self.row_lo[:, None] + np.arange(self.n_x)[None, :] / self.row_inv_dx[:, None]
        self.phi = torch.tensor(hats(self.row_T, self.node_T), dtype=torch.float64, device=dev)  # (rows, E)
        psi = hats(k.ravel(), self.node_k).reshape(k.shape[0], self.n_x, -1)
        self.psi = torch.tensor(psi, dtype=torch.float64, device=dev)  # (rows, n_x, K)
        self.onehot = torch.tensor(np.eye(int(self.row_name.max()) + 1)[self.row_name], dtype=torch.float64, device=dev)

    @property
    def shape(self):
        return (self.onehot.shape[1], len(self.node_T), len(self.node_k))

    def bump_field(self, bumps: torch.Tensor) -> torch.Tensor:
        """(rows, n_x) local-vol bump of node bumps (names, E, K)."""
        return torch.einsum("rn,re,rjk,nek->rj", self.onehot, self.phi, self.psi, bumps)

    def table(self, base_var: torch.Tensor, bumps: torch.Tensor) -> torch.Tensor:
        """The local-variance table (sqrt(base) + bump field)^2, differentiable in the bumps."""
        return (torch.sqrt(base_var) + self.bump_field(bumps)) ** 2

    def contract(self, table_grad: torch.Tensor, base_var: torch.Tensor) -> torch.Tensor:
        """Node vegas (names, E, K) of a table gradient at zero bumps: sum 2 sigma dV/dvar phi psi."""
        h = 2.0 * torch.sqrt(base_var) * table_grad
        return torch.einsum("rn,re,rjk,rj->nek", self.onehot, self.phi, self.psi, h)

    def contract_batches(self, table_grads: torch.Tensor, base_var: torch.Tensor) -> torch.Tensor:
        """contract of a stack of table gradients (B, rows, n_x): (B, names, E, K)."""
        h = 2.0 * torch.sqrt(base_var)[None] * table_grads
        per_row = torch.einsum("rjk,brj->brk", self.psi, h)
        return torch.einsum("rn,re,brk->bnek", self.onehot, self.phi, per_row)


def autocall_greeks(held, nodes: VegaNodes, smoothing: float = 0.005, precision="fp32", plan: AdjointPlan | None = None):
    """Price, deltas and node vegas (each with its standard error) of a local-vol autocall, by one forward and one
    backward pass; the vegas go through torch autograd (AutocallPrice of VegaNodes.table)."""
    own = plan is None
    plan = plan or AdjointPlan(held, smoothing, precision)
    try:
        s = held.struct
        dev = torch.device("cuda", torch.cuda.current_device())
        table = np.ctypeslib.as_array(s.table, shape=(s.n_rows * s.n_x,)).reshape(s.n_rows, s.n_x)
        base = torch.tensor(table, dtype=torch.float64, device=dev)
        bumps = torch.zeros(nodes.shape, dtype=torch.float64, device=dev, requires_grad=True)
        price = AutocallPrice.apply(nodes.table(base, bumps), plan)
        (vega,) = torch.autograd.grad(price, bumps)
        res = plan.last
        # batch means: each batch's vegas from its own gradient, all batches in one contraction
        pairs = plan.batch_pairs
        vb = nodes.contract_batches(plan.batch_grad / pairs.clamp(min=1.0)[:, None, None], base)
        w = pairs / pairs.sum()
        mean = (w[:, None, None, None] * vb).sum(0)
        var = (w[:, None, None, None] * (vb - mean) ** 2).sum(0) * (len(pairs) / (len(pairs) - 1)) / len(pairs)
        n = s.n_names
        return {
            "price": res.price,
            "price_se": res.price_se,
            "delta": np.array(res.delta[:n]),
            "delta_se": np.array(res.delta_se[:n]),
            "vega": vega.cpu().numpy(),
            "vega_se": torch.sqrt(var).cpu().numpy(),
            "forward_ms": res.forward_ms,
            "backward_ms": res.backward_ms,
        }
    finally:
        if own:
            plan.close()
