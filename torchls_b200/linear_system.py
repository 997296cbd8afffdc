"""Fixed sparse linear least squares and least absolute deviations on the GPU.

Interface and semantics of torchls ``linear_system.py:15-141``
(``FixedLinearSystem``, ``LinearFactor``, ``LADResult``,
``least_absolute_deviations``): a matrix with at most ``max_dense_columns``
columns is analysed once (coalesced COO, row and column lists, the pairs of
entries of each row that meet at each normal-matrix element); products, the
weighted normal matrix A^T diag(w) A + ridge I, its Cholesky factor, the
solves and the ADMM update run in this package's kernels
(``csrc/fixed_system.cu``, ``csrc/dense.cu``). Arithmetic is float64; a
float32 system returns float32 results. CUDA tensors only.
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np
import torch
from torch import Tensor

from . import _lib as L
from . import dense
from .kernels import partials, reduce


class FixedLinearSystem:
    def __init__(self, matrix: Tensor, *, max_dense_columns: int = 2048):
        if matrix.ndim != 2 or min(matrix.shape) < 1:
            raise ValueError("matrix must be a nonempty two-dimensional tensor")
        if matrix.dtype not in (torch.float32, torch.float64):
            raise ValueError("matrix must use float32 or float64")
        if max_dense_columns < 1 or matrix.shape[1] > max_dense_columns:
            raise ValueError("matrix exceeds max_dense_columns; use an iterative solver")
        L.require_cuda(matrix, "FixedLinearSystem")
        coo = matrix.detach().to_sparse_coo().coalesce()
        values = coo.values().to(torch.float64)
        if not bool(torch.isfinite(values).all()):
            raise ValueError("matrix coefficients must be finite")
        self.shape = matrix.shape
        self.dtype, self.device = matrix.dtype, matrix.device
        m, n = self.shape
        rows, cols = (t.cpu().numpy() for t in coo.indices())  # coalesced: row-major order
        nnz = len(rows)
        row_ptr = np.concatenate(([0], np.cumsum(np.bincount(rows, minlength=m))))
        col_entry = np.lexsort((rows, cols))  # per column, ascending row
        col_ptr = np.concatenate(([0], np.cumsum(np.bincount(cols, minlength=n))))
        # normal-matrix pairs: every ordered pair of entries of a row
        deg = np.diff(row_ptr)
        left, right = [], []
        for d in np.unique(deg[deg > 0]):
            starts = row_ptr[:-1][deg == d]
            ii, jj = np.meshgrid(np.arange(d), np.arange(d), indexing="ij")
            left.append((starts[:, None] + ii.reshape(1, -1)).reshape(-1))
            right.append((starts[:, None] + jj.reshape(1, -1)).reshape(-1))
        left = np.concatenate(left) if left else np.zeros(0, np.int64)
        right = np.concatenate(right) if right else np.zeros(0, np.int64)
        key = cols[left].astype(np.int64) * n + cols[right]
        order = np.lexsort((right, left, key))
        key, left, right = key[order], left[order], right[order]
        targets, first = np.unique(key, return_index=True)
        t_ptr = np.concatenate((first, [len(key)]))
        put = lambda a, dt=torch.int32: torch.from_numpy(np.ascontiguousarray(a)).to(device=self.device, dtype=dt)  # noqa: E731
        self._dev = dict(row_ptr=put(row_ptr), row=put(rows), col=put(cols), val=values.contiguous(),
                         col_ptr=put(col_ptr), col_entry=put(col_entry), target=put(targets, torch.int64),
                         target_ptr=put(t_ptr), pair_left=put(left), pair_right=put(right))
        s = L.FixedSystem()
        s.m, s.n, s.nnz, s.ntargets = m, n, nnz, len(targets)
        for name, t in self._dev.items():
            setattr(s, name, t.data_ptr())
        self._desc = s
        self.values = values

    def _input(self, value, rows):
        if value.ndim not in (1, 2) or value.shape[0] != rows:
            raise ValueError("incompatible vector or matrix shape")
        if value.device != self.device or value.dtype != self.dtype:
            raise ValueError("input and system must have matching device and dtype")
        return value[:, None] if value.ndim == 1 else value

    def _product(self, name, value, rows_in, rows_out):
        v = self._input(value, rows_in).to(torch.float64).contiguous()
        out = torch.empty((rows_out, v.shape[1]), dtype=torch.float64, device=self.device)
        L.call(name, C.byref(self._desc), v.data_ptr(), v.shape[1], out.data_ptr(), L.stream_handle(self.device))
        out = out.to(self.dtype)
        return out[:, 0] if value.ndim == 1 else out

    def matvec(self, value: Tensor) -> Tensor:
        return self._product("tls_fixed_matvec", value, self.shape[1], self.shape[0])

    def rmatvec(self, value: Tensor) -> Tensor:
        return self._product("tls_fixed_rmatvec", value, self.shape[0], self.shape[1])

    def factor(self, weights: Tensor | None = None, *, ridge: float = 0.0):
        """Cholesky factor of A^T diag(weights) A + ridge I (linear_system.py:54-73)."""
        if not math.isfinite(ridge) or ridge < 0:
            raise ValueError("ridge must be finite and nonnegative")
        w64 = None
        if weights is not None:
            if weights.ndim != 1:
                raise ValueError("weights must have one entry per matrix row")
            self._input(weights, self.shape[0])
            if not bool(torch.isfinite(weights).all() & (weights >= 0).all()):
                raise ValueError("weights must be finite and nonnegative")
            weights = weights.detach().clone()
            w64 = weights.to(torch.float64).contiguous()
        n = self.shape[1]
        normal = torch.empty((n, n), dtype=torch.float64, device=self.device)
        L.call("tls_fixed_normal", C.byref(self._desc), L.ptr(w64), float(ridge), normal.data_ptr(),
               L.stream_handle(self.device))
        return LinearFactor(self, dense.cholesky(normal), weights)


@dataclass
class LinearFactor:
    system: FixedLinearSystem
    cholesky: Tensor
    weights: Tensor | None

    def solve(self, rhs: Tensor) -> Tensor:
        """Solve the factored normal system for one or several right-hand sides."""
        value = self.system._input(rhs, self.system.shape[1])
        out = dense.cholesky_solve(value.to(torch.float64), self.cholesky).to(self.system.dtype)
        return out[:, 0] if rhs.ndim == 1 else out

    def least_squares(self, target: Tensor) -> Tensor:
        """Solve min ||sqrt(weights) (A x - target)||^2 + ridge ||x||^2."""
        self.system._input(target, self.system.shape[0])
        weighted = target
        if self.weights is not None:
            weighted = target * (self.weights if target.ndim == 1 else self.weights[:, None])
        return self.solve(self.system.rmatvec(weighted))


@dataclass
class LADResult:
    solution: Tensor
    iterations: int
    converged: bool


def least_absolute_deviations(system: FixedLinearSystem, target: Tensor, *, factor: LinearFactor | None = None,
                              max_iterations: int = 100, rho: float = 1.0, absolute_tolerance: float = 1e-4,
                              relative_tolerance: float = 1e-2) -> LADResult:
    """ADMM for entrywise ||A X - target||_1 sharing one factor across RHS
    columns (linear_system.py:103-141): per iteration a least-squares solve,
    one fused update of z, u and the stopping norms, two A^T products, and one
    host read of the norms."""
    if (max_iterations < 1 or not math.isfinite(rho) or rho <= 0
            or not all(math.isfinite(v) and v >= 0 for v in (absolute_tolerance, relative_tolerance))):
        raise ValueError("invalid ADMM iteration limit, rho or tolerance")
    system._input(target, system.shape[0])
    factor = system.factor() if factor is None else factor
    if factor.system is not system or factor.weights is not None:
        raise ValueError("ADMM requires an unweighted factor of this system")
    t64 = target.to(torch.float64).contiguous()
    z, u, zdiff, nxt = (torch.zeros_like(t64) for _ in range(4))
    nxt.copy_(t64)
    out = torch.empty(3, dtype=torch.float64, device=system.device)
    buf = partials(system.device)
    columns = 1 if target.ndim == 1 else target.shape[1]
    target_norm = float(reduce(t64, 1).sqrt())
    eps_primal = math.sqrt(target.numel()) * absolute_tolerance
    eps_dual = math.sqrt(system.shape[1] * columns) * absolute_tolerance
    stream = L.stream_handle(system.device)
    x = None
    for iteration in range(1, max_iterations + 1):
        x = factor.least_squares(nxt.to(system.dtype))
        ax = system.matvec(x).to(torch.float64).contiguous()
        L.call("tls_admm_step", t64.numel(), ax.data_ptr(), t64.data_ptr(), z.data_ptr(), u.data_ptr(),
               zdiff.data_ptr(), nxt.data_ptr(), 1.0 / rho, buf.data_ptr(), out.data_ptr(), stream)
        atu = system.rmatvec(u.to(system.dtype))
        atd = system.rmatvec(zdiff.to(system.dtype))
        pr2, ax2, z2, u2, d2 = torch.cat((out, reduce(atu, 1)[None], reduce(atd, 1)[None])).tolist()
        primal_limit = eps_primal + relative_tolerance * max(target_norm, math.sqrt(ax2), math.sqrt(z2))
        dual_limit = eps_dual + relative_tolerance * rho * math.sqrt(u2)
        dual = rho * math.sqrt(d2)
        if math.sqrt(pr2) < primal_limit and dual < dual_limit:
            return LADResult(x, iteration, True)
    return LADResult(x, max_iterations, False)
