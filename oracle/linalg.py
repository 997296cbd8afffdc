"""Block-sparse Jacobian products, block-Jacobi and PCG (numpy, float64).

Restates torchls sparse.py:25-143, preconditioning.py:12-134 and
solvers.py:167-285.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch
from scipy.linalg import solve_triangular


def add_rows(out, rows, vals):
    """out[rows[k]] += vals[k], repeated rows summed in input order (what
    np.add.at does), through torch's CPU index_add_ on views of the arrays."""
    k = int(np.prod(out.shape[1:], dtype=np.int64))
    target = torch.from_numpy(out.reshape(out.shape[0], k))  # a view: updates `out` in place
    src = torch.from_numpy(np.ascontiguousarray(vals, dtype=np.float64).reshape(-1, k))
    target.index_add_(0, torch.from_numpy(np.asarray(rows, dtype=np.int64).reshape(-1)), src)


class LinAlgError(Exception):
    """Raised when a damped block is not positive definite."""


class BlockJacobian:
    """groups: list of dict(blocks=[N,r,d] per slot, columns=[N,d], types, rows)."""

    def __init__(self, groups, layout, shape):
        self.groups, self.layout, self.shape = groups, layout, shape

    def matvec(self, v):
        """sparse.py:31-41."""
        out = []
        for g in self.groups:
            acc = sum(np.einsum("nrd,nd->nr", b, v[c]) for b, c in zip(g["blocks"], g["columns"]))
            out.append(acc.reshape(-1))
        return np.concatenate(out)

    def rmatvec(self, u):
        """sparse.py:43-55 (index_add scatter)."""
        out = np.zeros(self.shape[1])
        off = 0
        for g in self.groups:
            n, r, _ = g["blocks"][0].shape
            local = u[off : off + n * r].reshape(n, r)
            for b, c in zip(g["blocks"], g["columns"]):
                add_rows(out, c.reshape(-1), np.einsum("nrd,nr->nd", b, local).reshape(-1))
            off += n * r
        return out

    def normal_matvec(self, v, damping=0.0):
        """sparse.py:83-84."""
        return self.rmatvec(self.matvec(v)) + damping * v

    def squared_matvec_norm(self, v):
        """||J v||^2 with slots summed before squaring (sparse.py:57-81)."""
        return float(np.sum(self.matvec(v) ** 2))

    def scale_columns(self, scale):
        """sparse.py:86-102."""
        groups = []
        for g in self.groups:
            groups.append(dict(g, blocks=[b * scale[c][:, None, :] for b, c in zip(g["blocks"], g["columns"])]))
        return BlockJacobian(groups, self.layout, self.shape)

    def diagonal_blocks(self):
        """Exact per-variable J^T J blocks incl. aliased slots (sparse.py:104-121)."""
        diag = [np.zeros((e.count, e.dim, e.dim)) for e in self.layout]
        for g in self.groups:
            for s, (b, t, rows) in enumerate(zip(g["blocks"], g["types"], g["rows"])):
                gram = np.einsum("nri,nrj->nij", b, b)
                for o in range(s):
                    if g["types"][o] == t:
                        cross = np.einsum("nri,nrj->nij", b, g["blocks"][o])
                        mask = (rows == g["rows"][o])[:, None, None]
                        gram = gram + (cross + np.swapaxes(cross, -1, -2)) * mask
                add_rows(diag[t], rows, gram)
        return diag

    def to_dense(self):
        """sparse.py:123-143."""
        dense = np.zeros(self.shape)
        off = 0
        for g in self.groups:
            n, r, _ = g["blocks"][0].shape
            rid = off + np.arange(n * r).reshape(n, r)
            for b, c in zip(g["blocks"], g["columns"]):
                np.add.at(dense, (np.broadcast_to(rid[:, :, None], b.shape).reshape(-1),
                                  np.broadcast_to(c[:, None, :], b.shape).reshape(-1)), b.reshape(-1))
            off += n * r
        return dense


def cholesky(blocks):
    """Batched Cholesky; raises LinAlgError on a non-PD block (torch.linalg.cholesky)."""
    try:
        return np.linalg.cholesky(blocks)
    except np.linalg.LinAlgError as err:  # pragma: no cover - exercised in tests
        raise LinAlgError(str(err)) from err


def cholesky_apply(rhs, factor):
    """Solve L L^T x = rhs per block (preconditioning.py:12-17)."""
    out = np.empty_like(rhs)
    for i in range(len(factor)):
        y = solve_triangular(factor[i], rhs[i], lower=True)
        out[i] = solve_triangular(factor[i].T, y, lower=False)
    return out


def block_apply(factor, rhs):
    """Vectorised two-triangular-solve apply for [N,d,d] factors and [N,d] rhs."""
    n, d, _ = factor.shape
    y = np.zeros_like(rhs)
    for i in range(d):
        y[:, i] = (rhs[:, i] - np.einsum("nk,nk->n", factor[:, i, :i], y[:, :i])) / factor[:, i, i]
    x = np.zeros_like(rhs)
    for i in reversed(range(d)):
        x[:, i] = (y[:, i] - np.einsum("nk,nk->n", factor[:, i + 1 :, i], x[:, i + 1 :])) / factor[:, i, i]
    return x


def block_jacobi(layout, diagonal, damping):
    """Damped per-group block factors and their apply (solvers.py:259-285)."""
    factors = [cholesky(b + damping * np.eye(b.shape[-1])) for b in diagonal]

    def apply(v):
        parts = []
        for e, f in zip(layout, factors):
            part = v[e.offset : e.offset + e.count * e.dim].reshape(e.count, e.dim)
            parts.append(block_apply(f, part).reshape(-1))
        return np.concatenate(parts)

    return apply


class JointBlocks:
    """Joint variable-group preconditioner blocks (preconditioning.py:47-134)."""

    def __init__(self, layout, groups):
        lookup = {e.key: i for i, e in enumerate(layout)}
        grouped, chosen = [], set()
        for grp in groups:
            members = tuple(lookup[k] for k in grp)
            grouped.append(members)
            chosen.update(members)
        grouped.extend((i,) for i in range(len(layout)) if i not in chosen)
        self.layout = layout
        self.blocks, self.where = [], {}
        for bi, members in enumerate(grouped):
            off, cols = 0, []
            for i in members:
                e = layout[i]
                self.where[i] = (bi, off)
                cols.append(e.offset + np.arange(e.count)[:, None] * e.dim + np.arange(e.dim)[None, :])
                off += e.dim
            self.blocks.append((members, layout[members[0]].count, off, np.concatenate(cols, 1)))

    def normal_blocks(self, jac, diag):
        out = [np.zeros((cnt, dim, dim)) for _, cnt, dim, _ in self.blocks]
        for i, e in enumerate(self.layout):
            b, o = self.where[i]
            out[b][:, o : o + e.dim, o : o + e.dim] = diag[i]
        for g in jac.groups:
            for p, i in enumerate(g["types"]):
                bi, a = self.where[i]
                for q in range(p):
                    j = g["types"][q]
                    bj, c = self.where[j]
                    if bi == bj and i != j:
                        mask = g["rows"][p] == g["rows"][q]
                        cross = np.einsum("nri,nrj->nij", g["blocks"][p], g["blocks"][q]) * mask[:, None, None]
                        da, db = cross.shape[-2:]
                        rows = g["rows"][p]
                        np.add.at(out[bi][:, a : a + da, c : c + db], rows, cross)
                        np.add.at(out[bi][:, c : c + db, a : a + da], rows, np.swapaxes(cross, -1, -2))
        return out

    def factor(self, blocks, damping):
        factors = [cholesky(b + damping * np.eye(b.shape[-1])) for b in blocks]

        def apply(v):
            out = np.empty_like(v)
            for (_, _, dim, cols), f in zip(self.blocks, factors):
                out[cols.reshape(-1)] = block_apply(f, v[cols]).reshape(-1)
            return out

        return apply


@dataclass
class PCGResult:
    solution: np.ndarray
    iterations: int
    residual_norm: float
    converged: bool
    reason: str
    restarts: int = 0
    residual_checks: int = 0
    rhs_norm: float = 0.0


def pcg(matvec, rhs, preconditioner=None, *, rtol=1e-6, atol=1e-10, max_iterations=200,
        residual_check_interval=50, restart_strategy="adaptive", residual_drift_tolerance=0.1):
    """PCG with true-residual checks and restarts (solvers.py:167-256)."""
    M = (lambda x: x) if preconditioner is None else preconditioner
    x = np.zeros_like(rhs)
    r = rhs.copy()
    rhs_norm = float(np.linalg.norm(rhs))
    thr = max(atol, rtol * rhs_norm)
    if not math.isfinite(rhs_norm):
        return PCGResult(x, 0, rhs_norm, False, "nonfinite", rhs_norm=rhs_norm)
    if rhs_norm <= thr:
        return PCGResult(x, 0, rhs_norm, True, "residual_tolerance", rhs_norm=rhs_norm)
    z = M(r)
    rz = float(np.dot(r, z))
    p = z.copy()
    it = restarts = checks = 0
    reason = "max_iterations"
    for it in range(1, max_iterations + 1):
        ap = matvec(p)
        curv = float(np.dot(p, ap))
        if not (math.isfinite(curv) and math.isfinite(rz)):
            reason = "nonfinite"
            break
        if curv <= 0 or rz <= 0:
            reason = "nonpositive_curvature"
            break
        alpha = rz / curv
        x = x + alpha * p
        r = r - alpha * ap
        rec = float(np.linalg.norm(r))
        periodic = residual_check_interval > 0 and it % residual_check_interval == 0
        if rec <= thr or periodic:
            tr = rhs - matvec(x)
            checks += 1
            tn = float(np.linalg.norm(tr))
            if not math.isfinite(tn):
                return PCGResult(x, it, tn, False, "nonfinite", restarts, checks, rhs_norm)
            if tn <= thr:
                return PCGResult(x, it, tn, True, "residual_tolerance", restarts, checks, rhs_norm)
            drift = float(np.linalg.norm(tr - r))
            if rec <= thr or restart_strategy == "periodic" or drift > residual_drift_tolerance * max(tn, thr):
                r = tr
                z = M(r)
                rz = float(np.dot(r, z))
                p = z.copy()
                restarts += 1
                continue
        z = M(r)
        rz_new = float(np.dot(r, z))
        p = z + (rz_new / rz) * p
        rz = rz_new
    tn = float(np.linalg.norm(rhs - matvec(x)))
    checks += 1
    conv = math.isfinite(tn) and tn <= thr
    if conv:
        reason = "residual_tolerance"
    elif not math.isfinite(tn):
        reason = "nonfinite"
    return PCGResult(x, it, tn, conv, reason, restarts, checks, rhs_norm)
