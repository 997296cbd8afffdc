"""Schur elimination for the systems the one-group path does not take.

The interface and semantics are torchls ``schur.py:17-397`` (``SchurPlan``,
``SchurLinearization``, ``DampedSchurSystem``) for any number of retained
groups, residuals that couple retained variables and joint preconditioner
groups; ``torchls_b200.schur.SchurPlan`` builds a :class:`GeneralSchurPlan`
whenever one of these is present, and the solver then uses the classes here.

Layout (device arrays, built once per problem): the reduced vector holds the
retained groups in layout order (offsets cumulative, schur.py:28-37). Each
group's edges are its unique (retained, eliminated) pairs sorted by the key
r * E + e (the reference's order, schur.py:80-93); edges are numbered group
by group, so the edges of one retained variable are contiguous. Every edge
owns a d_r x d_e block at ``edge_w`` (its cross block J_r^T J_e, summed over
the residuals that contain the pair, and its whitened W block). The kernels
(``csrc/schur_general.cu``) gather in fixed orders: deterministic results.

Retained couplings (a residual with two retained slots that name different
variables, schur.py:41-56) make the base term of the reduced operator the
normal operator of the full, column-scaled Jacobian applied to the reduced
vector padded with zeros (J x = J_r x_r when x_e = 0), instead of the
block-diagonal s U s.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .kernels import ordered_index_add_, segment_reduce
from .variables import VariableLayout


def _t(a, device, dtype=torch.int32):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dtype)


def cross_layout(problem, eliminated: int, de: int):
    """Where the linearization writes each retained slot's cross block
    J_s^T (sum of the eliminated slots): per residual batch k, ``width`` doubles
    per factor with slot s at ``slot_cross[s]``, the batch at ``base``.
    Raises when a residual connects two different eliminated variables."""
    layout = problem.layout
    info, base = [], 0
    for plan in problem.plans:
        eslots = [s for s, t in enumerate(plan.type_indices) if t == eliminated]
        rslots = [s for s, t in enumerate(plan.type_indices) if t != eliminated]
        if eslots and any(not torch.equal(plan.indices[s], plan.indices[eslots[0]]) for s in eslots[1:]):
            raise ValueError("Eliminated variables must be independent: a residual connects distinct eliminated indices")
        rec = dict(eslots=eslots, rslots=rslots, width=0, slot_cross=[-1] * L.MAX_SLOTS, base=base)
        if eslots and rslots:
            off = 0
            for s in rslots:
                rec["slot_cross"][s] = off
                off += layout[plan.type_indices[s]].dim * de
            rec["width"] = off
        info.append(rec)
        base += plan.count * rec["width"]
    return info, base


def retained_couplings(problem, eliminated: int) -> bool:
    """Whether a residual has two retained slots naming different variables
    (schur.py:41-56: then the reduced operator's base is not block-diagonal)."""
    for plan in problem.plans:
        rslots = [s for s, t in enumerate(plan.type_indices) if t != eliminated]
        for i, s in enumerate(rslots):
            for o in rslots[:i]:
                if plan.type_indices[s] != plan.type_indices[o]:
                    return True
                if bool((plan.indices[s] != plan.indices[o]).any()):
                    return True
    return False


class GeneralSchurPlan:
    """Symbolic Schur structure for the general case (schur.py:17-189)."""

    general = True

    def __init__(self, problem, eliminate, device, *, preconditioner_groups=()):
        from .solvers import normalize_groups

        layout = problem.layout
        matches = [i for i, e in enumerate(layout) if e.key == eliminate]
        if len(matches) != 1:
            raise ValueError("eliminate must identify one parameter group by name or Var type")
        self.eliminated = matches[0]
        self.e = layout[self.eliminated]
        self.retained = tuple(i for i in range(len(layout)) if i != self.eliminated)
        if not self.retained:
            raise ValueError("Schur elimination needs a retained parameter group")
        if self.e.dim > 4:
            raise ValueError("the CUDA Schur path eliminates variables of tangent dim <= 4")
        if max(layout[i].dim for i in self.retained) > 16:
            raise ValueError("the CUDA Schur path supports retained tangent dims <= 16")
        self.device = torch.device(device)
        self.original_layout = layout
        self.de = de = self.e.dim
        E = self.e.count
        self.E_count = E
        red, off = [], 0
        for i in self.retained:
            g = layout[i]
            red.append(VariableLayout(g.var_type, g.ids, off, g.name))
            off += g.size
        self.layout = tuple(red)
        self.dim = self.reduced_dim = off
        self.full_dim = sum(g.size for g in layout)
        self.global_indices = torch.cat([torch.arange(layout[i].offset, layout[i].offset + layout[i].size)
                                         for i in self.retained]).to(self.device)
        self.plan_info, self.cross_size = cross_layout(problem, self.eliminated, de)
        self.couplings = retained_couplings(problem, self.eliminated)
        # ---- edges per retained group (sorted keys r * E + e), numbered group by group
        recs = {i: [] for i in self.retained}
        for k, plan in enumerate(problem.plans):
            info = self.plan_info[k]
            if not info["width"]:
                continue
            e_idx = plan.indices[info["eslots"][0]].numpy()
            for s in info["rslots"]:
                recs[plan.type_indices[s]].append((k, s, plan.indices[s].numpy() * E + e_idx))
        var_dim, var_row, var_full, var_diag, var_ptr = [], [], [], [], [np.zeros(1, np.int64)]
        edge_var, edge_elim, edge_w, self.edges = [], [], [], []
        cross_targets = []  # (global edge id per factor, contribution offsets) per record
        eg = vbase = wbase = dbase = 0
        self.group_edges = []
        for gi, orig in enumerate(self.retained):
            g, rg = layout[orig], self.layout[gi]
            keys = np.concatenate([r[2] for r in recs[orig]]) if recs[orig] else np.zeros(0, np.int64)
            uniq, inv = np.unique(keys, return_inverse=True)
            ri, ei = uniq // E, uniq % E
            self.edges.append((torch.from_numpy(ri).to(self.device), torch.from_numpy(ei).to(self.device)))
            ne, d = len(uniq), g.dim
            var_dim.append(np.full(g.count, d, np.int32))
            var_row.append(rg.offset + np.arange(g.count, dtype=np.int64) * d)
            var_full.append(g.offset + np.arange(g.count, dtype=np.int64) * d)
            var_diag.append(dbase + np.arange(g.count, dtype=np.int64) * d * d)
            var_ptr.append(eg + np.cumsum(np.bincount(ri, minlength=g.count)))
            edge_var.append(vbase + ri)
            edge_elim.append(ei)
            edge_w.append(wbase + np.arange(ne, dtype=np.int64) * d * de)
            cur = 0
            for k, s, key in recs[orig]:
                info = self.plan_info[k]
                n = len(key)
                cross_targets.append((eg + inv[cur: cur + n],
                                      info["base"] + np.arange(n, dtype=np.int64) * info["width"]
                                      + info["slot_cross"][s], gi))
                cur += n
            self.group_edges.append((eg, ne, wbase, d))
            eg += ne
            vbase += g.count
            wbase += ne * d * de
            dbase += g.count * d * d
        self.nedges, self.nretained, self.w_size, self.diag_size = eg, vbase, wbase, dbase
        self.max_dim = max(layout[i].dim for i in self.retained)
        cat = lambda parts, dt: np.concatenate(parts).astype(dt) if parts else np.zeros(0, dt)  # noqa: E731
        edge_var_np, edge_elim_np = cat(edge_var, np.int64), cat(edge_elim, np.int64)
        order = np.lexsort((np.arange(eg), edge_elim_np))  # per eliminated variable, by edge id
        elim_ptr = np.concatenate(([0], np.cumsum(np.bincount(edge_elim_np, minlength=E))))
        dev = self.device
        self.dev = dict(
            var_dim=_t(cat(var_dim, np.int32), dev), var_row=_t(cat(var_row, np.int64), dev, torch.int64),
            var_full=_t(cat(var_full, np.int64), dev, torch.int64),
            var_diag=_t(cat(var_diag, np.int64), dev, torch.int64), var_ptr=_t(cat(var_ptr, np.int64), dev),
            edge_var=_t(edge_var_np, dev), edge_elim=_t(edge_elim_np, dev),
            edge_w=_t(cat(edge_w, np.int64), dev, torch.int64), elim_ptr=_t(elim_ptr, dev), elim_edge=_t(order, dev),
        )
        self._edge_var_np, self._edge_elim_np = edge_var_np, edge_elim_np
        self._var_dim_np = cat(var_dim, np.int32)
        self._plans_host = [(tuple(pl.type_indices), [i.numpy() for i in pl.indices], pl.count)
                            for pl in problem.plans]
        self._retained_pattern = None
        # ---- cross-block segments per retained group (fixed order: record, factor)
        self.cross_segs, self._keep = [], []
        for gi, (e0, ne, w0, d) in enumerate(self.group_edges):
            ids = [t[0] - e0 for t in cross_targets if t[2] == gi]
            offs = [t[1] for t in cross_targets if t[2] == gi]
            ids = np.concatenate(ids) if ids else np.zeros(0, np.int64)
            offs = np.concatenate(offs) if offs else np.zeros(0, np.int64)
            o = np.argsort(ids, kind="stable")
            ptr = np.concatenate(([0], np.cumsum(np.bincount(ids, minlength=ne))))
            p_t, s_t = _t(ptr, dev), _t(offs[o], dev)
            self._keep += [p_t, s_t]
            lanes = 32 if ne and len(ids) / max(ne, 1) > 8 else 1
            self.cross_segs.append(L.Segments(ne, d * de, lanes, 0, p_t.data_ptr(), s_t.data_ptr()))
        self.joint = _JointPlan(self, normalize_groups(preconditioner_groups)) if preconditioner_groups else None
        self.bad = torch.zeros(1, dtype=torch.int32, device=dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)  # no bounded waits here: stays 0
        self.wait_cycles = 0

    def retained_pattern(self) -> _RetainedPattern:
        """The block pattern of the retained normal matrix (built on first use)."""
        if self._retained_pattern is None:
            self._retained_pattern = _RetainedPattern(self)
        return self._retained_pattern

    # ---------------------------------------------------------------- linearization hooks
    def cross_buffer(self, device):
        return torch.empty(self.cross_size, dtype=torch.float64, device=device)

    def fill_cross_args(self, k, la) -> int:
        info = self.plan_info[k]
        mask = 0
        for s in info["eslots"]:
            mask |= 1 << s
        la.elim_mask = mask if info["width"] else 0
        la.elim_dim = self.de
        for s in range(L.MAX_SLOTS):
            la.slot_cross[s] = info["slot_cross"][s] if info["width"] else -1
        la.cross_width = info["width"]
        return info["base"]


class _RetainedPattern:
    """Block pattern of B = (s J_r)^T (s J_r) for ``cache_retained_matrix``
    (schur.py:171-189, 225-241): every retained variable's diagonal block and a
    block per coupled pair (a residual with two retained slots naming
    different variables), both orientations; blocks sorted by (row, column),
    values row-major back to back. Per coupling record (residual batch k,
    slots a > b) the selected factors and the value positions of their
    contributions, factor-major as the contributions are computed."""

    def __init__(self, plan: GeneralSchurPlan):
        dims = plan._var_dim_np.astype(np.int64)
        nret = plan.nretained
        base, acc = {}, 0
        for orig in plan.retained:
            base[orig] = acc
            acc += plan.original_layout[orig].count
        recs = []
        rows = [np.arange(nret, dtype=np.int64)]
        cols = [np.arange(nret, dtype=np.int64)]
        for k, (tis, idxs, count) in enumerate(plan._plans_host):
            for a in range(len(tis)):
                for b in range(a):
                    ta, tb = tis[a], tis[b]
                    if ta not in base or tb not in base:
                        continue
                    ia, ib = idxs[a].astype(np.int64), idxs[b].astype(np.int64)
                    sel = np.flatnonzero(ia != ib) if ta == tb else np.arange(count, dtype=np.int64)
                    if not len(sel):
                        continue
                    va, vb = base[ta] + ia[sel], base[tb] + ib[sel]
                    recs.append((k, a, b, sel, va, vb))
                    rows += [va, vb]
                    cols += [vb, va]
        keys = np.unique(np.concatenate(rows) * nret + np.concatenate(cols))
        brow, bcol = keys // nret, keys % nret
        size = dims[brow] * dims[bcol]
        off = np.concatenate(([0], np.cumsum(size)))
        self.nvalues = int(off[-1])
        row_ptr = np.concatenate(([0], np.cumsum(np.bincount(brow, minlength=nret))))
        dev = plan.device
        self.row_ptr, self.block_col = _t(row_ptr, dev), _t(bcol, dev)
        self.block_off = _t(off[:-1], dev, torch.int64)
        where = lambda r, c: off[np.searchsorted(keys, r * nret + c)]  # noqa: E731
        self.diag_off = where(np.arange(nret), np.arange(nret))
        self.records = []
        for k, a, b, sel, va, vb in recs:
            tis = plan._plans_host[k][0]
            da, db = plan.original_layout[tis[a]].dim, plan.original_layout[tis[b]].dim
            r_, c_ = np.arange(da), np.arange(db)
            ab = where(va, vb)[:, None, None] + r_[None, :, None] * db + c_[None, None, :]
            ba = where(vb, va)[:, None, None] + c_[None, None, :] * da + r_[None, :, None]
            self.records.append((k, a, b, _t(sel, dev, torch.int64), _t(ab.reshape(-1), dev, torch.int64),
                                 _t(ba.reshape(-1), dev, torch.int64)))
        # per retained group: its entry in the full layout, the offset of its
        # diagonal blocks in the retained diagonal buffer, their value positions
        self.groups, dbase = [], 0
        for orig in plan.retained:
            e = plan.original_layout[orig]
            v0 = base[orig]
            pos = self.diag_off[v0 : v0 + e.count][:, None] + np.arange(e.dim * e.dim)[None, :]
            self.groups.append((e, dbase, _t(pos.reshape(-1), dev, torch.int64)))
            dbase += e.count * e.dim * e.dim

    def values(self, lin, ret_diag, scale):
        """B's values for one linearization: s U s on the diagonal blocks and
        the coupled pairs' (s J_a)^T (s J_b), each block's contributions summed
        in a fixed order (``ordered_index_add_``)."""
        dev = ret_diag.device
        vals = torch.zeros(max(self.nvalues, 1), dtype=torch.float64, device=dev)
        for e, dbase, pos in self.groups:
            U = ret_diag[dbase : dbase + e.count * e.dim * e.dim].view(e.count, e.dim, e.dim)
            if scale is not None:
                sv = scale[e.offset : e.offset + e.size].view(e.count, e.dim)
                U = U * sv[:, :, None] * sv[:, None, :]
            vals[pos] = U.reshape(-1)
        jac = lin.jacobian
        st = jac.structure
        for k, a, b, sel, ab, ba in self.records:
            cross = _slot_block(jac, st, k, a, sel, scale).transpose(-1, -2) @ _slot_block(jac, st, k, b, sel, scale)
            ordered_index_add_(vals, ab, cross.reshape(-1, 1))
            ordered_index_add_(vals, ba, cross.reshape(-1, 1))
        return vals


def _slot_block(jac, st, k, s, sel, scale):
    """Slot s's Jacobian blocks [n, r, d] (float64, column-scaled) of the
    selected factors of residual batch k."""
    R, D, N = st.rdims[k], st.D[k], st.plans[k].count
    e = jac.layout[st.plans[k].type_indices[s]]
    c0 = st.slot_col[k][s]
    blk = jac.jacs[k].view(R, D, N)[:, c0 : c0 + e.dim, :][:, :, sel].permute(2, 0, 1).to(torch.float64)
    if scale is not None:
        col = (st.index[k][s].long()[sel][:, None] * e.dim + e.offset
               + torch.arange(e.dim, device=blk.device)[None, :])
        blk = blk * scale[col][:, None, :]
    return blk


class _JointPlan:
    """Joint preconditioner blocks over retained groups with identical IDs
    (preconditioning.py:47-88 on the reduced layout, schur.py:163-189): per
    block its members; per member pair, the edges the two share (the same
    retained index and eliminated variable), grouped by retained index."""

    def __init__(self, plan: GeneralSchurPlan, groups):
        from .solvers import normalize_groups

        layout = plan.layout
        lookup = {e.key: i for i, e in enumerate(layout)}
        chosen, self.blocks = set(), []
        for grp in normalize_groups(groups):
            if any(k not in lookup for k in grp):
                raise ValueError("Unknown preconditioner key (Schur groups must be retained variables)")
            members = tuple(lookup[k] for k in grp)
            first = layout[members[0]]
            if any(not torch.equal(first.ids.cpu(), layout[i].ids.cpu()) for i in members[1:]):
                raise ValueError("Joint preconditioner groups require identical IDs in identical order")
            self.blocks.append(members)
            chosen.update(members)
        self.blocks.extend((i,) for i in range(len(layout)) if i not in chosen)
        self.where = {}
        for b, members in enumerate(self.blocks):
            off = 0
            for i in members:
                self.where[i] = (b, off)
                off += layout[i].dim
        E = plan.E_count
        self.pairs, keep = [], []
        dev = plan.device
        for members in self.blocks:
            for ia, a in enumerate(members):
                for b in members[:ia]:
                    (ea0, na, _, _), (eb0, nb, _, _) = plan.group_edges[a], plan.group_edges[b]
                    ra = _local_vars(plan, a)
                    rb = _local_vars(plan, b)
                    key_a = ra * E + plan._edge_elim_np[ea0: ea0 + na]
                    key_b = rb * E + plan._edge_elim_np[eb0: eb0 + nb]
                    common, ia_, ib_ = np.intersect1d(key_a, key_b, assume_unique=True, return_indices=True)
                    rows = common // E
                    count = layout[a].count
                    ptr = np.concatenate(([0], np.cumsum(np.bincount(rows, minlength=count))))
                    t = [_t(ptr, dev), _t(ea0 + ia_, dev), _t(eb0 + ib_, dev)]
                    keep += t
                    self.pairs.append((a, b, count, t))
        self._keep = keep


def _local_vars(plan: GeneralSchurPlan, gi: int) -> np.ndarray:
    """Retained variable index within group gi of each of the group's edges."""
    e0, ne, _, _ = plan.group_edges[gi]
    first = sum(plan.layout[g].count for g in range(gi))
    return plan._edge_var_np[e0: e0 + ne] - first


class GeneralSchurLinearization:
    """Cross blocks per edge, retained and eliminated diagonal blocks and, for
    joint preconditioner groups, the member-pair couplings of the retained
    Jacobian (schur.py:192-257), for one linearization."""

    def __init__(self, plan: GeneralSchurPlan, lin, diagonal_raw, scale, *, wdtype, vec_dtype, dense=False,
                 cache_retained=False):
        self.plan = plan
        dev = plan.device
        self.cross = torch.zeros(max(plan.w_size, 1), dtype=torch.float64, device=dev)
        for seg, (e0, ne, w0, d) in zip(plan.cross_segs, plan.group_edges):
            if ne:
                segment_reduce(seg, lin.cross_contrib, self.cross[w0: w0 + ne * d * plan.de])
        self.ret_diag = torch.cat([diagonal_raw[i].reshape(-1) for i in plan.retained]).to(torch.float64)
        self.elim_diag = diagonal_raw[plan.eliminated].to(torch.float64).contiguous()
        self.scale = None if scale is None else scale.to(torch.float64).contiguous()
        self.wdtype, self.vec_dtype, self.dense = wdtype, vec_dtype, dense
        self.w = torch.empty(max(plan.w_size, 1), dtype=wdtype, device=dev)
        self.inv_l = torch.empty((plan.e.count, plan.de, plan.de), dtype=torch.float64, device=dev)
        self.tbuf = torch.empty((plan.e.count, plan.de), dtype=torch.float64, device=dev)
        self.ybuf = torch.empty((plan.e.count, plan.de), dtype=torch.float64, device=dev)
        self.jacobian = lin.jacobian if self.scale is None else lin.jacobian.scale_columns(self.scale)
        self.retained = None
        if plan.couplings:
            self.xfull = torch.empty(plan.full_dim, dtype=torch.float64, device=dev)
            self.yfull = torch.empty(plan.full_dim, dtype=torch.float64, device=dev)
            if cache_retained:  # cache_retained_matrix (schur.py:225-241): B once per linearization
                pat = plan.retained_pattern()
                self.retained_values = pat.values(lin, self.ret_diag, self.scale)
                self.retained = L.RetainedMatrix(pat.row_ptr.data_ptr(), pat.block_col.data_ptr(),
                                                 pat.block_off.data_ptr(), self.retained_values.data_ptr())
        self.joint_couplings = self._joint_couplings() if plan.joint is not None else {}

    def _joint_couplings(self):
        """Per joint member pair (a, b): sum over residuals of (s J_a)^T (s J_b)
        where both slots name the same index (preconditioning.py:89-115)."""
        plan, out = self.plan, {}
        red_of = {orig: k for k, orig in enumerate(plan.retained)}
        pair_keys = {(a, b) for a, b, _, _ in plan.joint.pairs}
        for g in self.jacobian.groups:
            for p, ti in enumerate(g.type_indices):
                for q in range(p):
                    tj = g.type_indices[q]
                    if ti == tj or ti not in red_of or tj not in red_of:
                        continue
                    a, b = red_of[ti], red_of[tj]
                    if plan.joint.where[a][0] != plan.joint.where[b][0]:
                        continue
                    mask = (g.variable_indices[p] == g.variable_indices[q]).to(torch.float64)
                    cross = (g.blocks[p].double().transpose(-1, -2) @ g.blocks[q].double()) * mask[:, None, None]
                    key = (a, b)
                    if key not in pair_keys:  # the pair's stored orientation: (b, a), transposed
                        key, cross = (b, a), cross.transpose(-1, -2)
                    if key not in out:
                        out[key] = torch.zeros((plan.layout[a].count, *cross.shape[1:]), dtype=torch.float64,
                                               device=plan.device)
                    ordered_index_add_(out[key], g.variable_indices[p], cross)
        return out

    def damped(self, damping, check: bool = True):
        return GeneralDampedSchurSystem(self, damping, check)


class GeneralDampedSchurSystem:
    """schur.py:263-397 for the general plan: eliminated factors, whitened
    blocks, reduced rhs, the reduced operator, back-substitution, the Schur
    block preconditioner (joint groups included) and the dense matrix."""

    def __init__(self, lin: GeneralSchurLinearization, damping: float, check: bool = True):
        self.linear, self.plan, self.damping = lin, lin.plan, float(damping)
        self._normal = (lin.jacobian.normal_args(torch.float64, self.damping)
                        if self.plan.couplings and lin.retained is None else None)
        self.args = self._args()
        L.call("tls_schur_general_damp", C.byref(self.args), self.stream)
        if check and int(self.plan.bad.item()) > 0:
            raise torch.linalg.LinAlgError("damped eliminated block is not positive definite")
        self._rhs_ready = False

    def _args(self) -> L.SchurGeneralArgs:
        p, lin = self.plan, self.linear
        a = L.SchurGeneralArgs()
        a.de, a.nelim, a.nretained = p.de, p.e.count, p.nretained
        a.wdtype = L.dtype_code(lin.wdtype)
        a.nedges, a.reduced_dim, a.full_dim, a.elim_offset = p.nedges, p.dim, p.full_dim, p.e.offset
        for name, t in p.dev.items():
            setattr(a, name, t.data_ptr())
        a.cross, a.elim_diag, a.ret_diag = lin.cross.data_ptr(), lin.elim_diag.data_ptr(), lin.ret_diag.data_ptr()
        a.scale = None if lin.scale is None else lin.scale.data_ptr()
        a.inv_l, a.w = lin.inv_l.data_ptr(), lin.w.data_ptr()
        a.tbuf, a.ybuf = lin.tbuf.data_ptr(), lin.ybuf.data_ptr()
        if self._normal is not None:
            a.normal = C.pointer(self._normal)
            a.xfull, a.yfull = lin.xfull.data_ptr(), lin.yfull.data_ptr()
        if lin.retained is not None:
            a.retained = C.addressof(lin.retained)
            a.yfull = lin.yfull.data_ptr()
        a.damping = self.damping
        a.bad = p.bad.data_ptr()
        a.max_dim = p.max_dim
        return a

    @property
    def stream(self):
        return L.stream_handle(self.plan.device)

    def reduced_rhs(self, rhs: torch.Tensor) -> torch.Tensor:
        """rhs_c = b_c - W (L^-1 b_e) from the full scaled rhs b (schur.py:285-290)."""
        b = rhs.to(torch.float64).contiguous()
        out = torch.empty(self.plan.dim, dtype=torch.float64, device=b.device)
        L.call("tls_schur_general_reduced_rhs", C.byref(self.args), b.data_ptr(), out.data_ptr(), self.stream)
        self._rhs_ready = True
        return out

    def backsubstitute(self, retained: torch.Tensor) -> torch.Tensor:
        """The full step: the retained part and L^-T (L^-1 b_e - W^T x_c) (schur.py:292-301)."""
        if not self._rhs_ready:
            raise ValueError("backsubstitute requires reduced_rhs first")
        x = retained.to(torch.float64).contiguous()
        out = torch.zeros(self.plan.full_dim, dtype=torch.float64, device=x.device)
        L.call("tls_schur_general_backsubstitute", C.byref(self.args), x.data_ptr(), out.data_ptr(), self.stream)
        return out

    def matvec(self, vector: torch.Tensor) -> torch.Tensor:
        """base(v) - W (W^T v) (schur.py:303-328)."""
        v = vector.to(torch.float64).contiguous()
        out = torch.empty_like(v)
        L.call("tls_schur_general_matvec", C.byref(self.args), v.data_ptr(), out.data_ptr(),
               L.stream_handle(v.device))
        return out

    def preconditioner_blocks(self):
        """Per retained group [count, d, d]: s U s - sum_e W_e W_e^T (lambda not added)."""
        p = self.plan
        flat = torch.empty(max(p.diag_size, 1), dtype=torch.float64, device=p.device)
        L.call("tls_schur_general_preconditioner_blocks", C.byref(self.args), flat.data_ptr(), self.stream)
        out, off = [], 0
        for e in p.layout:
            out.append(flat[off: off + e.count * e.dim * e.dim].view(e.count, e.dim, e.dim))
            off += e.count * e.dim * e.dim
        return out

    def preconditioner(self, *, graph_safe: bool = False, check: bool = True):
        """Block-Jacobi on the Schur blocks (schur.py:330-378), joint groups
        assembled with their member couplings minus the shared-edge W terms."""
        from .solvers import BlockJacobiPreconditioner

        p = self.plan
        diag = self.preconditioner_blocks()
        if p.joint is None:
            specs = [(d, [(e.offset, e.dim)], e.count, e.dim) for d, e in zip(diag, p.layout)]
            return BlockJacobiPreconditioner.from_blocks(specs, self.damping, None, p.dim, check=check)
        jp, specs = p.joint, []
        blocks = []
        for members in jp.blocks:
            dim = sum(p.layout[i].dim for i in members)
            blk = torch.zeros((p.layout[members[0]].count, dim, dim), dtype=torch.float64, device=p.device)
            for i in members:
                o, d = jp.where[i][1], p.layout[i].dim
                blk[:, o: o + d, o: o + d] = diag[i]
            blocks.append(blk)
        for a, b, count, (ptr, ea, eb) in jp.pairs:
            da, db = p.layout[a].dim, p.layout[b].dim
            ww = torch.empty((count, da, db), dtype=torch.float64, device=p.device)
            L.call("tls_schur_general_pair_blocks", C.byref(self.args), count, ptr.data_ptr(), ea.data_ptr(),
                   eb.data_ptr(), da, db, ww.data_ptr(), self.stream)
            cross = self.linear.joint_couplings.get((a, b))
            term = -ww if cross is None else cross - ww
            blk, oa, ob = blocks[jp.where[a][0]], jp.where[a][1], jp.where[b][1]
            blk[:, oa: oa + da, ob: ob + db] += term
            blk[:, ob: ob + db, oa: oa + da] += term.transpose(-1, -2)
        for members, blk in zip(jp.blocks, blocks):
            specs.append((blk, [(p.layout[i].offset, p.layout[i].dim) for i in members], blk.shape[0], blk.shape[1]))
        return BlockJacobiPreconditioner.from_blocks(specs, self.damping, None, p.dim, check=check)

    def dense_matrix(self) -> torch.Tensor:
        """Dense reduced matrix base + lambda I - W W^T, symmetrised (schur.py:380-397)."""
        p, lin = self.plan, self.linear
        n = p.dim
        S = torch.zeros((n, n), dtype=torch.float64, device=p.device)
        red_of = {orig: k for k, orig in enumerate(p.retained)}
        ar = lambda d: torch.arange(d, device=p.device)  # noqa: E731
        for k, e in enumerate(p.layout):  # s U s blocks
            U = lin.ret_diag[int(sum(x.count * x.dim * x.dim for x in p.layout[:k])):][: e.count * e.dim * e.dim]
            U = U.view(e.count, e.dim, e.dim)
            orig = p.original_layout[p.retained[k]]
            if lin.scale is not None:
                s = lin.scale[orig.offset: orig.offset + orig.size].view(e.count, e.dim)
                U = U * s[:, :, None] * s[:, None, :]
            idx = e.offset + ar(e.count)[:, None] * e.dim + ar(e.dim)
            S[idx[:, :, None], idx[:, None, :]] += U
        if p.couplings:  # retained couplings of the scaled Jacobian (schur.py:242-257)
            for g in lin.jacobian.groups:
                for a_, ta in enumerate(g.type_indices):
                    for b_ in range(a_):
                        tb = g.type_indices[b_]
                        if ta not in red_of or tb not in red_of:
                            continue
                        ea, eb = p.layout[red_of[ta]], p.layout[red_of[tb]]
                        mask = ((g.variable_indices[a_] != g.variable_indices[b_]) if ta == tb
                                else torch.ones_like(g.variable_indices[a_], dtype=torch.bool)).to(torch.float64)
                        cross = (g.blocks[a_].double().transpose(-1, -2) @ g.blocks[b_].double()) * mask[:, None, None]
                        ra = ea.offset + g.variable_indices[a_][:, None] * ea.dim + ar(ea.dim)
                        rb = eb.offset + g.variable_indices[b_][:, None] * eb.dim + ar(eb.dim)
                        flat = S.view(-1)
                        ordered_index_add_(flat, (ra[:, :, None] * n + rb[:, None, :]).reshape(-1),
                                           cross.reshape(-1, 1))
                        ordered_index_add_(flat, (rb[:, :, None] * n + ra[:, None, :]).reshape(-1),
                                           cross.transpose(-1, -2).reshape(-1, 1))
        S += self.damping * torch.eye(n, dtype=torch.float64, device=p.device)
        # W W^T by column chunks of a dense W (rows: reduced indices, columns: eliminated tangent)
        de, ncols = p.de, p.e.count * p.de
        step = max(de, ((1 << 27) // max(n, 1)) // de * de)
        rows0 = p.dev["var_row"][p.dev["edge_var"].long()]
        wf = lin.w.to(torch.float64)
        for c0 in range(0, ncols, step):
            c1 = min(ncols, c0 + step)
            Wd = torch.zeros((n, c1 - c0), dtype=torch.float64, device=p.device)
            for (e0, ne, w0, d) in p.group_edges:
                sel = torch.arange(e0, e0 + ne, device=p.device)
                pe = p.dev["edge_elim"][sel].long()
                keep = (pe * de >= c0) & (pe * de < c1)
                sel, pe = sel[keep], pe[keep]
                if sel.numel() == 0:
                    continue
                vals = wf[w0 + (sel - e0)[:, None, None] * d * de + ar(d)[None, :, None] * de + ar(de)[None, None, :]]
                r_idx = (rows0[sel][:, None] + ar(d)[None, :])[:, :, None].expand(-1, d, de)
                c_idx = (pe[:, None] * de + ar(de)[None, :] - c0)[:, None, :].expand(-1, d, de)
                Wd[r_idx.reshape(-1), c_idx.reshape(-1)] = vals.reshape(-1)
            S -= Wd @ Wd.T
        return 0.5 * (S + S.T)
