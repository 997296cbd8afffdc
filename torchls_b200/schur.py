"""Schur elimination of one independent variable group on the GPU.

Interface of torchls ``schur.py``: ``SchurPlan`` (symbolic, once per problem),
``SchurLinearization`` (per linearization: cross blocks), ``DampedSchurSystem``
(per trial: reduced_rhs, matvec, preconditioner, backsubstitute,
dense_matrix).

Edges are the unique (retained variable, eliminated variable) pairs sorted by
key r * E + e, exactly as torchls orders them (schur.py:83-124); ``edges``
exposes that order. The kernels store edges in a chunked order instead: a
chunk holds whole eliminated variables (so each eliminated sum stays inside
one thread block) and within a chunk edges are sorted by retained variable
(so retained sums are contiguous runs). W is stored structure-of-arrays
[dr*de][E] in that order.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .kernels import segment_reduce


# (retained dim, eliminated dim) pairs the one-group kernels are built for
FAST_DIMS = frozenset({(6, 3), (3, 3), (7, 3), (6, 1), (3, 1), (1, 1), (2, 2), (3, 2), (2, 1), (1, 3)})


def _one_group_fits(problem, eliminate, preconditioner_groups) -> bool:
    """Whether the one-group kernels take this system: one retained group of a
    built shape, no residual with two retained slots, no joint preconditioner
    groups, every eliminated variable with at most 256 retained neighbours."""
    layout = problem.layout
    matches = [i for i, e in enumerate(layout) if e.key == eliminate]
    if len(matches) != 1 or len(layout) != 2 or preconditioner_groups:
        return False
    elim = matches[0]
    ret = 1 - elim
    if (layout[ret].dim, layout[elim].dim) not in FAST_DIMS:
        return False
    deg = np.zeros(layout[elim].count, np.int64)
    for plan in problem.plans:
        rs = [s for s, t in enumerate(plan.type_indices) if t != elim]
        es = [s for s, t in enumerate(plan.type_indices) if t == elim]
        if len(rs) > 1:
            return False
        if rs and es:
            np.add.at(deg, plan.indices[es[0]].numpy(), 1)
    return int(deg.max(initial=0)) <= 256


class SchurPlan:
    """Symbolic Schur structure. Systems the one-group kernels do not take
    (several retained groups, retained couplings, joint preconditioner groups,
    other block shapes) get a ``schur_general.GeneralSchurPlan`` instead."""

    general = False

    def __new__(cls, problem, eliminate, device, *, preconditioner_groups=()):
        if cls is SchurPlan and not _one_group_fits(problem, eliminate, preconditioner_groups):
            from .schur_general import GeneralSchurPlan

            return GeneralSchurPlan(problem, eliminate, device, preconditioner_groups=preconditioner_groups)
        return super().__new__(cls)

    def __init__(self, problem, eliminate, device, *, preconditioner_groups=()):
        layout = problem.layout
        matches = [i for i, e in enumerate(layout) if e.key == eliminate]
        if len(matches) != 1:
            raise ValueError("eliminate must identify one parameter group by name or Var type")
        self.eliminated = matches[0]
        self.e = layout[self.eliminated]
        self.retained = tuple(i for i in range(len(layout)) if i != self.eliminated)
        if not self.retained:
            raise ValueError("Schur elimination needs a retained parameter group")
        self.device = torch.device(device)
        self.r = layout[self.retained[0]]
        self.dim = self.r.size
        self.original_layout = layout
        dr, de = self.r.dim, self.e.dim
        self.dr, self.de = dr, de
        E_count = self.e.count
        keys, recs = [], []
        self.plan_info = []
        for k, plan in enumerate(problem.plans):
            eslots = [s for s, t in enumerate(plan.type_indices) if t == self.eliminated]
            rslots = [s for s, t in enumerate(plan.type_indices) if t != self.eliminated]
            if eslots and any(not torch.equal(plan.indices[s], plan.indices[eslots[0]]) for s in eslots[1:]):
                raise ValueError(
                    "Eliminated variables must be independent: a residual connects distinct eliminated indices")
            info = dict(eslots=eslots, rslots=rslots, width=0, slot_cross=[-1] * L.MAX_SLOTS, base=0)
            if eslots and rslots:
                off = 0
                for s in rslots:
                    info["slot_cross"][s] = off
                    off += layout[plan.type_indices[s]].dim * de
                info["width"] = off
                for s in rslots:
                    key = plan.indices[s].numpy() * E_count + plan.indices[eslots[0]].numpy()
                    keys.append(key)
                    recs.append((k, s, plan.count))
            self.plan_info.append(info)
        base = 0
        for k, plan in enumerate(problem.plans):
            self.plan_info[k]["base"] = base
            base += plan.count * self.plan_info[k]["width"]
        self.cross_size = base
        allkeys = np.concatenate(keys) if keys else np.zeros(0, np.int64)
        uniq, inverse = np.unique(allkeys, return_inverse=True)
        ri, ei = uniq // E_count, uniq % E_count
        self.nedges = len(uniq)
        self.edges = ((torch.from_numpy(ri).to(device), torch.from_numpy(ei).to(device)),)
        self.E_count = E_count
        self._ri, self._ei = ri, ei
        self._records = recs
        self._inverse = inverse
        self.reduced_dim = self.dim
        # reduced-vector indices into the full tangent (schur.py:28-37)
        self.global_indices = torch.arange(self.r.offset, self.r.offset + self.r.size, device=device)
        self.layout = (self.r,)
        self.bad = torch.zeros(1, dtype=torch.int32, device=device)
        # device error word of the bounded waits in the Schur kernels; cleared
        # in stream order whenever a damped system is built (once per trial)
        self.err = torch.zeros(1, dtype=torch.int32, device=device)
        # limit of each bounded device wait in SM cycles (0: about a second)
        self.wait_cycles = 0
        self._layouts = {}

    def chunks_for(self, wdtype) -> ChunkLayout:
        """Slab layout for W stored as ``wdtype`` (512 edges per chunk for
        float32, 256 for float64: 36 KB of W per chunk either way)."""
        cap = 512 if wdtype == torch.float32 else 256
        if cap not in self._layouts:
            self._layouts[cap] = ChunkLayout(self, cap)
        return self._layouts[cap]

    @property
    def chunks(self) -> ChunkLayout:
        return self.chunks_for(torch.float64)

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


class ChunkLayout:
    """Chunked, slab-padded edge layout used by the kernels.

    Eliminated variables are ordered by their smallest retained neighbour (so
    a chunk's edges touch few retained variables) and packed into chunks of
    whole variables with at most ``cap`` edges. Inside a chunk edges are
    sorted by retained variable and cut into runs that never cross a window of
    32 * (cap // 256) edges (one warp's edges; each thread takes cap // 256
    consecutive edges). Each chunk owns a fixed-size, 16-byte aligned slab: W as
    [dr*de][cap] and an int32 metadata block
        [ne, np, 0, 0][edge_r: cap][meta: cap][tail run position: cap]
        [point edge ptr: cap + 4][point edge list: cap]
    so one bulk copy brings a chunk into shared memory. Edge ``slab index``
    = chunk * cap + position. Run partials are stored retained-major
    (``rrun_ptr``), so each retained variable sums a contiguous range.
    """

    THREADS = 256

    def __init__(self, plan: SchurPlan, cap: int):
        ri, ei, E, P = plan._ri, plan._ei, plan.nedges, plan.E_count
        device = plan.device
        self.cap = cap
        deg = np.bincount(ei, minlength=P)
        max_deg = int(deg.max()) if E else 0
        if max_deg > cap:
            raise ValueError(f"an eliminated variable has {max_deg} retained neighbours; the CUDA Schur path "
                             f"supports at most {cap}")
        first = np.full(P, np.iinfo(np.int64).max)
        if E:
            np.minimum.at(first, ei, ri)
        point_order = np.lexsort((np.arange(P), first))
        rank = np.empty(P, np.int64)
        rank[point_order] = np.arange(P)
        deg_o = deg[point_order]
        start = np.cumsum(deg_o) - deg_o
        chunk_of_rank = start // max(1, cap - max_deg + 1)
        ch = chunk_of_rank[rank[ei]]
        order = np.lexsort((ei, ri, ch))
        c_r, c_e, c_raw = ri[order], ei[order], ch[order]
        newchunk = np.ones(E, bool)
        newchunk[1:] = c_raw[1:] != c_raw[:-1]
        cid = np.cumsum(newchunk) - 1
        nchunks = int(cid[-1]) + 1 if E else 0
        chunk_ptr = np.concatenate((np.flatnonzero(newchunk), [E])).astype(np.int64)
        ne = np.diff(chunk_ptr)
        local = np.arange(E) - chunk_ptr[cid] if E else np.zeros(0, np.int64)
        sidx = cid * cap + local
        # runs: equal retained variable, split at warp windows
        win = 32 * max(1, cap // self.THREADS)
        self.window = win
        newrun = newchunk.copy()
        newrun[1:] |= c_r[1:] != c_r[:-1]
        newrun |= (local % win) == 0
        run_starts = np.flatnonzero(newrun)
        nruns = len(run_starts)
        run_id = np.cumsum(newrun) - 1
        run_end = np.concatenate((run_starts[1:], [E]))
        head = (local[run_starts] % win)[run_id] if E else np.zeros(0, np.int64)
        run_r = c_r[run_starts]
        cm = np.argsort(run_r, kind="stable")  # retained-major position -> run id
        run_pos = np.empty(nruns, np.int64)
        run_pos[cm] = np.arange(nruns)
        rrun_ptr = np.concatenate(([0], np.cumsum(np.bincount(run_r, minlength=plan.r.count))))
        crun_start = sidx[run_starts][cm] if E else np.zeros(0, np.int64)
        crun_len = (run_end - run_starts)[cm]
        tail = np.zeros(E, bool)
        if E:
            tail[run_end - 1] = True
        tailpos = np.where(tail, run_pos[run_id], -1) if E else np.zeros(0, np.int64)
        # chunk points and their local edge lists
        ckey = cid * P + c_e
        uniq_cp, cp_inv = np.unique(ckey, return_inverse=True)
        cpt_chunk = uniq_cp // P
        cpt_ptr = np.searchsorted(cpt_chunk, np.arange(nchunks + 1))
        npts = np.diff(cpt_ptr)
        pl = cp_inv - cpt_ptr[cid] if E else np.zeros(0, np.int64)
        # point-local CSR: edges of each chunk point in ascending local position
        po = np.lexsort((local, pl, cid))
        pcount = np.bincount(cp_inv, minlength=len(uniq_cp))
        pstart = np.cumsum(pcount) - pcount  # global start per (chunk, point)
        # a point's sum y_p is written over t of its first edge (only the
        # thread summing that point reads that entry), so the kernel reads
        # y_p at the local position of the point's first edge
        yslot = local[po[pstart]][cp_inv] if E else np.zeros(0, np.int64)
        # meta word: y_p's entry (16 bits) | run start inside the window (6 bits) | run tail flag
        meta = yslot | (head << 16) | (tail.astype(np.int64) << 22)
        # ---- metadata slab
        self.meta_ints = 5 * cap + 8
        M = np.zeros((max(nchunks, 1), self.meta_ints), np.int64)
        off_r, off_m, off_t, off_pp, off_pe = 4, 4 + cap, 4 + 2 * cap, 4 + 3 * cap, 8 + 4 * cap
        if nchunks:
            M[:nchunks, 0] = ne
            M[:nchunks, 1] = npts
            M[cid, off_r + local] = c_r
            M[cid, off_m + local] = meta
            M[cid, off_t + local] = tailpos
            local_start = pstart - pstart[cpt_ptr[cpt_chunk]]
            M[cpt_chunk, off_pp + (np.arange(len(uniq_cp)) - cpt_ptr[cpt_chunk])] = local_start
            M[np.arange(nchunks), off_pp + npts] = ne
            rank_in_chunk = np.arange(E) - chunk_ptr[cid[po]]
            M[cid[po], off_pe + rank_in_chunk] = local[po]
        self.nchunks, self.nruns, self.nedges = nchunks, nruns, E
        self._host = (c_r, c_e, sidx, plan.r.count, P)
        self._dense_pairs = None
        self.order, self.pos_of_edge = order, np.empty(E, np.int64)
        self.pos_of_edge[order] = np.arange(E)
        self.slab_of_edge = np.empty(E, np.int64)
        self.slab_of_edge[order] = sidx  # reference edge -> slab index
        nslab = max(nchunks, 1) * cap
        slab_r = np.full(nslab, -1, np.int64)
        slab_e = np.full(nslab, -1, np.int64)
        slab_r[sidx], slab_e[sidx] = c_r, c_e
        eorder = np.lexsort((sidx, c_e))
        elim_ptr = np.concatenate(([0], np.cumsum(np.bincount(c_e, minlength=P))))
        # cross-contribution segments per slab entry
        cursor, ids, offs = 0, [], []
        for k, s_, n in plan._records:
            info = plan.plan_info[k]
            ids.append(self.slab_of_edge[plan._inverse[cursor : cursor + n]])
            offs.append(info["base"] + np.arange(n, dtype=np.int64) * info["width"] + info["slot_cross"][s_])
            cursor += n
        ids = np.concatenate(ids) if ids else np.zeros(0, np.int64)
        offs = np.concatenate(offs) if offs else np.zeros(0, np.int64)
        o = np.argsort(ids, kind="stable")
        cptr = np.concatenate(([0], np.cumsum(np.bincount(ids, minlength=nslab))))
        t = lambda a, dt=torch.int32: torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dt)
        self.nslab = nslab
        self.dev = dict(
            meta=t(M.reshape(-1)), slab_r=t(slab_r), slab_e=t(slab_e), elim_ptr=t(elim_ptr),
            elim_slab=t(sidx[eorder]), rrun_ptr=t(rrun_ptr), crun_start=t(crun_start), crun_len=t(crun_len),
            cross_ptr=t(cptr), cross_src=t(offs[o]),
        )
        self.cross_seg = L.Segments(nslab, plan.dr * plan.de, 1, 0, self.dev["cross_ptr"].data_ptr(),
                                    self.dev["cross_src"].data_ptr())


def _dense_pairs(layout: ChunkLayout):
    """Per lower block (i, j), i >= j, of the reduced matrix: the pairs of slab
    entries (a, b), retained variables i and j, of each eliminated variable
    they share, in eliminated-variable order (device int32 arrays, built once)."""
    if layout._dense_pairs is None:
        c_r, c_e, sidx, nret, P = layout._host
        order = np.lexsort((c_r, c_e))  # by eliminated variable, then retained
        r_s, s_s = c_r[order], sidx[order]
        deg = np.bincount(c_e, minlength=P)
        start = np.cumsum(deg) - deg
        pa, pb = [], []
        for d in np.unique(deg[deg > 0]):
            base = start[deg == d]
            ti, tj = np.tril_indices(int(d))
            pa.append((base[:, None] + ti[None, :]).reshape(-1))
            pb.append((base[:, None] + tj[None, :]).reshape(-1))
        pa = np.concatenate(pa) if pa else np.zeros(0, np.int64)
        pb = np.concatenate(pb) if pb else np.zeros(0, np.int64)
        key = r_s[pa] * nret + r_s[pb]
        o = np.lexsort((pb, pa, key))
        key, pa, pb = key[o], pa[o], pb[o]
        uniq, first = np.unique(key, return_index=True)
        ptr = np.concatenate((first, [len(key)]))
        dev = layout.dev["meta"].device
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=torch.int32)  # noqa: E731
        layout._dense_pairs = (t(uniq // nret), t(uniq % nret), t(ptr), t(s_s[pa]), t(s_s[pb]))
    return layout._dense_pairs


class SchurLinearization:
    """Cross blocks E_e = J_r^T J_e per edge (schur.py:192-257), in chunk order, float64."""

    def __new__(cls, plan, *args, **kwargs):
        if cls is SchurLinearization and getattr(plan, "general", False):
            from .schur_general import GeneralSchurLinearization

            return GeneralSchurLinearization(plan, *args, **kwargs)
        return super().__new__(cls)

    def __init__(self, plan: SchurPlan, lin, diagonal_raw, scale, *, wdtype, vec_dtype, dense=False,
                 cache_retained=False):
        """``cache_retained`` (cache_retained_matrix) matters only with retained
        couplings, which one retained group without them never has."""
        self.plan = plan
        dev = plan.device
        self.layout = plan.chunks_for(wdtype)
        lay = self.layout
        # the whitening kernel sums each slab entry's cross contributions
        # itself; the summed blocks are formed only on request (``cross``)
        self.cross_contrib = lin.cross_contrib
        self._cross = None
        self.ret_diag = diagonal_raw[plan.retained[0]].contiguous()
        self.elim_diag = diagonal_raw[plan.eliminated].contiguous()
        self.scale = None if scale is None else scale.to(torch.float64).contiguous()
        self.wdtype, self.vec_dtype = wdtype, vec_dtype
        self.dense = dense
        self.w = torch.empty((lay.nslab * plan.dr * plan.de,), dtype=wdtype, device=dev)
        self.inv_l = torch.empty((plan.e.count, plan.de, plan.de), dtype=torch.float64, device=dev)
        self.run_partial = torch.empty((max(lay.nruns, 1), plan.dr), dtype=torch.float64, device=dev)
        self.ybuf = torch.empty((plan.e.count, plan.de), dtype=torch.float64, device=dev)

    @property
    def cross(self) -> torch.Tensor:
        """Per slab entry the unscaled cross block J_r^T J_e ([nslab, dr, de]
        float64, zero for padding): the sums the whitening kernel forms."""
        if self._cross is None:
            plan, lay = self.plan, self.layout
            self._cross = torch.zeros((lay.nslab, plan.dr, plan.de), dtype=torch.float64, device=plan.device)
            if plan.nedges:
                segment_reduce(lay.cross_seg, self.cross_contrib, self._cross)
        return self._cross

    def damped(self, damping, check: bool = True):
        return DampedSchurSystem(self, damping, check)


class DampedSchurSystem:
    """schur.py:263-397 on the GPU."""

    def __init__(self, lin: SchurLinearization, damping: float, check: bool = True):
        """``check=False`` defers the host read of the count of eliminated blocks
        that are not positive definite (``plan.bad``) to the caller."""
        self.linear, self.plan, self.damping = lin, lin.plan, float(damping)
        self.args = self._args()
        L.call("tls_schur_damp", C.byref(self.args), L.stream_handle(self.plan.device))
        if check and int(self.plan.bad.item()) > 0:
            raise torch.linalg.LinAlgError("damped eliminated block is not positive definite")
        self._rhs_ready = False

    def _args(self) -> L.SchurArgs:
        p, lin = self.plan, self.linear
        a = L.SchurArgs()
        a.nedges, a.dr, a.de = p.nedges, p.dr, p.de
        a.nretained, a.nelim = p.r.count, p.e.count
        a.wdtype, a.vec_dtype = L.dtype_code(lin.wdtype), L.dtype_code(lin.vec_dtype)
        lay = lin.layout
        a.nchunks, a.cap, a.nruns, a.meta_ints = lay.nchunks, lay.cap, lay.nruns, lay.meta_ints
        a.retained_offset, a.elim_offset = p.r.offset, p.e.offset
        d = lay.dev
        for name in ("meta", "slab_r", "slab_e", "elim_ptr", "elim_slab", "rrun_ptr", "crun_start", "crun_len"):
            setattr(a, name, d[name].data_ptr())
        a.cross_contrib = lin.cross_contrib.data_ptr()
        a.cross_ptr, a.cross_src = d["cross_ptr"].data_ptr(), d["cross_src"].data_ptr()
        a.elim_diag = lin.elim_diag.data_ptr()
        a.ret_diag = lin.ret_diag.data_ptr()
        a.scale = None if lin.scale is None else lin.scale.data_ptr()
        a.inv_l = lin.inv_l.data_ptr()
        a.w = lin.w.data_ptr()
        a.run_partial = lin.run_partial.data_ptr()
        a.ybuf = lin.ybuf.data_ptr()
        a.damping = self.damping
        a.bad = p.bad.data_ptr()
        a.err = p.err.data_ptr()
        a.wait_cycles = int(p.wait_cycles)
        return a

    @property
    def stream(self):
        return L.stream_handle(self.plan.device)

    def reduced_rhs(self, rhs: torch.Tensor) -> torch.Tensor:
        """rhs_c = b_c - W (L^-1 b_e) from the full scaled rhs b (schur.py:285-290)."""
        b = rhs.to(torch.float64).contiguous()
        out = torch.empty(self.plan.dim, dtype=self.linear.vec_dtype, device=b.device)
        L.call("tls_schur_reduced_rhs", C.byref(self.args), b.data_ptr(), out.data_ptr(), self.stream)
        self._rhs_ready = True
        return out

    def backsubstitute(self, retained: torch.Tensor) -> torch.Tensor:
        """Full float64 step: retained part plus L^-T (L^-1 b_e - W^T x_c) (schur.py:292-301)."""
        if not self._rhs_ready:
            raise ValueError("backsubstitute requires reduced_rhs first")
        x = retained.to(self.linear.vec_dtype).contiguous()
        total = sum(e.size for e in self.plan.original_layout)
        out = torch.zeros(total, dtype=torch.float64, device=x.device)
        L.call("tls_schur_backsubstitute", C.byref(self.args), x.data_ptr(), out.data_ptr(), self.stream)
        return out

    def matvec(self, vector: torch.Tensor) -> torch.Tensor:
        """(s U s + lambda I) v - W (W^T v) (schur.py:303-328)."""
        v = vector.to(self.linear.vec_dtype).contiguous()
        out = torch.empty_like(v)
        # torch's current stream (a CUDA-graph capture stream included)
        L.call("tls_schur_matvec", C.byref(self.args), v.data_ptr(), out.data_ptr(), L.stream_handle(v.device))
        return out

    def preconditioner_blocks(self) -> torch.Tensor:
        p = self.plan
        out = torch.empty((p.r.count, p.dr, p.dr), dtype=torch.float64, device=p.device)
        L.call("tls_schur_preconditioner_blocks", C.byref(self.args), out.data_ptr(), self.stream)
        return out

    def preconditioner(self, *, graph_safe: bool = False, check: bool = True):
        """Exact Schur block-diagonal preconditioner (schur.py:353-378)."""
        from .solvers import BlockJacobiPreconditioner

        p = self.plan
        blocks = self.preconditioner_blocks()
        return BlockJacobiPreconditioner.from_blocks([(blocks, [(0, p.dr)], p.r.count, p.dr)], self.damping,
                                                     None, p.dim, check=check)

    def dense_matrix(self) -> torch.Tensor:
        """Dense reduced matrix (s U s + lambda I) - W W^T (schur.py:380-397),
        assembled from the slabs by ``tls_schur_dense_matrix``: one warp per
        camera-pair block sums the products of their shared eliminated
        variables in a fixed order; the result is exactly symmetric."""
        p = self.plan
        tr, tc, ptr, pa, pb = _dense_pairs(self.linear.layout)
        S = torch.empty((p.dim, p.dim), dtype=torch.float64, device=p.device)
        L.call("tls_schur_dense_matrix", C.byref(self.args), tr.numel(), tr.data_ptr(), tc.data_ptr(), ptr.data_ptr(),
               pa.data_ptr(), pb.data_ptr(), S.data_ptr(), self.stream)
        return S
