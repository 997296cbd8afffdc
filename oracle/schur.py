"""Schur elimination of one independent group (numpy). Restates torchls schur.py:17-397."""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import torch

from .linalg import BlockJacobian, JointBlocks, add_rows, block_apply, cholesky


class RetainedEntry:
    def __init__(self, key, count, dim, offset):
        self.key, self.count, self.dim, self.offset = key, count, dim, offset


class SchurPlan:
    """Symbolic structure: retained layout, unique edges, W's CSR (schur.py:17-161)."""

    def __init__(self, problem, eliminate, preconditioner_groups=()):
        layout = problem.groups
        matches = [i for i, g in enumerate(layout) if g.key == eliminate]
        if len(matches) != 1:
            raise ValueError("eliminate must identify one parameter group by name or Var type")
        self.eliminated = matches[0]
        self.e = layout[self.eliminated]
        self.retained = tuple(i for i in range(len(layout)) if i != self.eliminated)
        if not self.retained:
            raise ValueError("Schur elimination needs a retained parameter group")
        self.original = layout
        self.layout, off, gidx = [], 0, []
        for i in self.retained:
            g = layout[i]
            self.layout.append(RetainedEntry(g.key, g.count, g.dim, off))
            gidx.append(np.arange(g.offset, g.offset + g.count * g.dim))
            off += g.count * g.dim
        self.dim = off
        self.global_indices = np.concatenate(gidx)
        local = {orig: k for k, orig in enumerate(self.retained)}
        records = {i: [] for i in self.retained}
        self.retained_groups, self.off_diagonal = [], []
        for gi, b in enumerate(problem.batches):
            eslots = [s for s, t in enumerate(b.groups) if t == self.eliminated]
            if eslots and any(not np.array_equal(b.rows[s], b.rows[eslots[0]]) for s in eslots[1:]):
                raise ValueError("Eliminated variables must be independent")
            rslots = [s for s, t in enumerate(b.groups) if t != self.eliminated]
            if rslots:
                cols = []
                for s in rslots:
                    ent = self.layout[local[b.groups[s]]]
                    cols.append(b.rows[s][:, None] * ent.dim + ent.offset + np.arange(ent.dim)[None, :])
                types = [local[b.groups[s]] for s in rslots]
                self.retained_groups.append((gi, rslots, cols, types, [b.rows[s] for s in rslots]))
                for p, s in enumerate(rslots):
                    for q in range(p):
                        o = rslots[q]
                        mask = (b.rows[s] != b.rows[o]) if types[p] == types[q] else np.ones(b.count, bool)
                        if mask.any():
                            self.off_diagonal.append((gi, s, o, cols[p], cols[q], mask))
            if eslots:
                for s in rslots:
                    key = b.rows[s] * self.e.count + b.rows[eslots[0]]
                    records[b.groups[s]].append((gi, s, tuple(eslots), key))
        self.edges, self.cross_records = [], []
        counts, csr_cols, orders, nnz = [], [], [], 0
        for orig, ent in zip(self.retained, self.layout):
            keys = np.concatenate([r[3] for r in records[orig]]) if records[orig] else np.zeros(0, np.int64)
            uniq, inv = np.unique(keys, return_inverse=True)
            ri, ei = uniq // self.e.count, uniq % self.e.count
            degree = np.bincount(ri, minlength=ent.count)
            starts = np.concatenate(([0], np.cumsum(degree)))
            d, e = ent.dim, self.e.dim
            local_edge = np.arange(len(uniq)) - starts[ri]
            pos = (starts[ri, None, None] * d * e + np.arange(d)[None, :, None] * degree[ri, None, None] * e
                   + local_edge[:, None, None] * e + np.arange(e)[None, None, :])
            order = np.empty(len(uniq) * d * e, np.int64)
            order[pos.reshape(-1)] = np.arange(order.size)
            colsx = np.broadcast_to((ei[:, None, None] * e + np.arange(e)[None, None, :]), (len(uniq), d, e)).reshape(-1)
            csr_cols.append(colsx[order])
            orders.append(order + nnz)
            counts.append(np.repeat(degree * e, d))
            nnz += order.size
            self.edges.append((ri, ei))
            cur, recs = 0, []
            for gi, s, es, key in records[orig]:
                recs.append((gi, s, es, inv[cur : cur + len(key)]))
                cur += len(key)
            self.cross_records.append(recs)
        cnt = np.concatenate(counts)
        self.row_ptr = np.concatenate(([0], np.cumsum(cnt))).astype(np.int64)
        self.columns = np.concatenate(csr_cols).astype(np.int64)
        self.value_order = np.concatenate(orders)
        # W^T's CSR pattern and the permutation from W's values to W^T's, built
        # once (a damped system then only permutes its values)
        ncols = self.e.count * self.e.dim
        probe = sp.csr_matrix((np.arange(len(self.columns), dtype=np.float64), self.columns, self.row_ptr),
                              shape=(self.dim, ncols)).T.tocsr()
        self.t_ptr, self.t_cols = probe.indptr.astype(np.int64), probe.indices.astype(np.int64)
        self.t_perm = probe.data.astype(np.int64)
        self.joint = JointBlocks(self.layout, preconditioner_groups) if preconditioner_groups else None
        self.pre_edges = []
        if self.joint is not None:
            for members, _, _, _ in self.joint.blocks:
                if len(members) == 1:
                    self.pre_edges.append(None)
                    continue
                keys = [self.edges[i][0] * self.e.count + self.edges[i][1] for i in members]
                uniq, inv = np.unique(np.concatenate(keys), return_inverse=True)
                maps = np.split(inv, np.cumsum([len(k) for k in keys])[:-1])
                self.pre_edges.append((uniq // self.e.count, maps))


class SchurLinearization:
    """Cross blocks and retained Jacobian (schur.py:192-257)."""

    def __init__(self, jac, diag, plan, dense=False):
        self.plan, self.diag = plan, diag
        groups = []
        for gi, slots, cols, types, rows in plan.retained_groups:
            g = jac.groups[gi]
            groups.append(dict(blocks=[g["blocks"][s] for s in slots], columns=cols, types=types, rows=rows))
        self.retained_jacobian = (
            BlockJacobian(groups, plan.layout, (sum(g["blocks"][0].shape[0] * g["blocks"][0].shape[1] for g in groups), plan.dim))
            if groups else None
        )
        self.pre_blocks = (plan.joint.normal_blocks(self.retained_jacobian, [diag[i] for i in plan.retained])
                           if plan.joint is not None else None)
        self.cross = []
        for ent, (ri, _), recs in zip(plan.layout, plan.edges, plan.cross_records):
            vals = np.zeros((len(ri), ent.dim, plan.e.dim))
            for gi, s, es, eids in recs:
                blocks = jac.groups[gi]["blocks"]
                eb = sum(blocks[k] for k in es)
                add_rows(vals, eids, np.einsum("nri,nrj->nij", blocks[s], eb))
            self.cross.append(vals)
        self.base = None
        if dense:
            self.base = np.zeros((plan.dim, plan.dim))
            for i, ent in zip(plan.retained, plan.layout):
                cols = ent.offset + np.arange(ent.count)[:, None] * ent.dim + np.arange(ent.dim)[None, :]
                self.base[cols[:, :, None], cols[:, None, :]] = diag[i]
            for gi, s, o, c1, c2, mask in plan.off_diagonal:
                b = jac.groups[gi]["blocks"]
                cross = np.einsum("nri,nrj->nij", b[s], b[o]) * mask[:, None, None]
                np.add.at(self.base, (c1[:, :, None], c2[:, None, :]), cross)
                np.add.at(self.base, (c2[:, :, None], c1[:, None, :]), np.swapaxes(cross, -1, -2))

    def damped(self, damping):
        return DampedSchurSystem(self, damping)


class _Csr:
    """CSR matrix times a numpy vector through torch's (multithreaded) CPU SpMV;
    the products are those of ``scipy.sparse`` up to summation order."""

    def __init__(self, ptr, cols, values, shape):
        self.shape = shape
        self.t = torch.sparse_csr_tensor(torch.from_numpy(ptr), torch.from_numpy(cols), torch.from_numpy(values),
                                         size=shape, check_invariants=False)
        self.ptr, self.cols, self.values = ptr, cols, values

    def __matmul__(self, v):
        return (self.t @ torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64))).numpy()

    def scipy(self):
        return sp.csr_matrix((self.values, self.cols, self.ptr), shape=self.shape)


class DampedSchurSystem:
    """schur.py:263-397."""

    def __init__(self, lin, damping):
        self.lin, self.plan, self.damping = lin, lin.plan, damping
        c = lin.diag[self.plan.eliminated]
        eye = np.eye(c.shape[-1])
        L = cholesky(c + damping * eye)
        self.inverse_l = np.linalg.inv(L)
        self.whitened = [blk @ np.swapaxes(self.inverse_l[ei], -1, -2) for blk, (_, ei) in zip(lin.cross, self.plan.edges)]
        values = np.concatenate([w.reshape(-1) for w in self.whitened])[self.plan.value_order]
        e = self.plan.e
        shape = (self.plan.dim, e.count * e.dim)
        self.w = _Csr(self.plan.row_ptr, self.plan.columns, values, shape)
        self.wt = _Csr(self.plan.t_ptr, self.plan.t_cols, values[self.plan.t_perm], shape[::-1])

    def reduced_rhs(self, rhs):
        e = self.plan.e
        b = rhs[e.offset : e.offset + e.count * e.dim].reshape(e.count, e.dim, 1)
        self.eliminated_rhs = (self.inverse_l @ b).reshape(-1)
        return rhs[self.plan.global_indices] - self.w @ self.eliminated_rhs

    def backsubstitute(self, retained):
        e = self.plan.e
        y = (self.eliminated_rhs - self.wt @ retained).reshape(e.count, e.dim, 1)
        elim = np.swapaxes(self.inverse_l, -1, -2) @ y
        total = sum(g.count * g.dim for g in self.plan.original)
        out = np.zeros(total)
        out[self.plan.global_indices] = retained
        out[e.offset : e.offset + e.count * e.dim] = elim.reshape(-1)
        return out

    def matvec(self, v):
        jac = self.lin.retained_jacobian
        if not self.plan.off_diagonal:
            parts = []
            for i, ent in zip(self.plan.retained, self.plan.layout):
                seg = v[ent.offset : ent.offset + ent.count * ent.dim].reshape(ent.count, ent.dim, 1)
                parts.append((self.lin.diag[i] @ seg).reshape(-1))
            base = np.concatenate(parts) + self.damping * v
        else:
            base = jac.normal_matvec(v, self.damping) if jac is not None else self.damping * v
        return base - self.w @ (self.wt @ v)

    def preconditioner(self):
        if self.plan.joint is not None:
            diags = []
            for (members, _, dim, _), base, ep in zip(self.plan.joint.blocks, self.lin.pre_blocks, self.plan.pre_edges):
                if ep is None:
                    i = members[0]
                    rows, _ = self.plan.edges[i]
                    wh = self.whitened[i]
                else:
                    rows, maps = ep
                    wh = np.zeros((len(rows), dim, self.plan.e.dim))
                    start = 0
                    for i, m in zip(members, maps):
                        d = self.plan.layout[i].dim
                        wh[m, start : start + d] = self.whitened[i]
                        start += d
                out = base.copy()
                add_rows(out, rows, -(wh @ np.swapaxes(wh, -1, -2)))
                diags.append(out)
            return self.plan.joint.factor(diags, self.damping)
        factors = []
        for i, ent, wh, (ri, _) in zip(self.plan.retained, self.plan.layout, self.whitened, self.plan.edges):
            d = self.lin.diag[i].copy()
            add_rows(d, ri, -(wh @ np.swapaxes(wh, -1, -2)))
            factors.append(cholesky(d + self.damping * np.eye(ent.dim)))

        def apply(v):
            return np.concatenate([
                block_apply(f, v[ent.offset : ent.offset + ent.count * ent.dim].reshape(ent.count, ent.dim)).reshape(-1)
                for ent, f in zip(self.plan.layout, factors)
            ])

        return apply

    def dense_matrix(self):
        if self.lin.base is None:
            raise ValueError("Dense Schur matrix was not requested")
        m = self.lin.base + self.damping * np.eye(self.plan.dim)
        m = m - (self.w.scipy() @ self.wt.scipy()).toarray()
        return 0.5 * (m + m.T)
