"""Block-sparse Jacobian on the GPU (interface of torchls ``sparse.py:11-143``).

The Jacobian of each residual batch is stored once, in structure-of-arrays
order [r*D][N]; ``groups`` exposes the reference layout (per-slot blocks
[N, r, d] plus global columns) lazily for callers that want it.
``scale_columns`` records a column scale instead of rewriting J; every
product applies it on the fly (J diag(s) x = J (s * x)).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import NamedTuple

import torch
from torch import Tensor

from . import _lib as L
from .kernels import partials, segment_reduce


@dataclass(frozen=True)
class JacobianGroup:
    """Local Jacobian blocks and global tangent columns, per slot (sparse.py:11-22)."""

    blocks: tuple
    columns: tuple
    type_indices: tuple
    variable_indices: tuple

    @property
    def num_rows(self):
        return self.blocks[0].shape[0] * self.blocks[0].shape[1]


class BlockJacobian:
    def __init__(self, structure, jacs, gram_contrib, layout, shape, scale: Tensor | None = None,
                 tile_jacs: dict | None = None):
        self.structure = structure
        self.jacs = jacs
        # J of reordered factor groups in the tile plan's order, made on first
        # use and shared by column-scaled views of this Jacobian
        self._tile_jacs = {} if tile_jacs is None else tile_jacs
        self.gram_contrib = gram_contrib
        self.layout = layout
        self.shape = shape
        self.scale = scale  # float64 [n] or None
        self._scale_cast = {}
        self._contrib = {}
        self._groups = None

    @property
    def dtype(self):
        return self.jacs[0].dtype

    @property
    def device(self):
        return self.jacs[0].device

    # ------------------------------------------------------------------ descriptors
    def _scale_as(self, dtype):
        if self.scale is None:
            return None
        if dtype not in self._scale_cast:
            self._scale_cast[dtype] = self.scale.to(dtype).contiguous()
        return self._scale_cast[dtype]

    def normal_args(self, vec_dtype: torch.dtype, damping: float = 0.0, *, tiles: bool = True) -> L.NormalArgs:
        """Descriptor of the products on this Jacobian. ``tiles`` attaches the
        structure's one-pass plan for the normal operator (when it has one);
        False keeps the two-pass route (factor pass + per-variable gather)."""
        st = self.structure
        a = L.NormalArgs()
        a.nfactor_groups = len(self.jacs)
        a.nvar_groups = len(self.layout)
        a.vec_dtype = L.dtype_code(vec_dtype)
        for k, jac in enumerate(self.jacs):
            a.fg[k] = st.factor_group(k, jac)
            a.contrib_offset[k] = st.grad_base[k]
        for i in range(len(self.layout)):
            a.vg[i] = st.vgroups[i]
            a.seg[i] = st.grad_seg[i]
        s = self._scale_as(vec_dtype)
        a.scale = None if s is None else s.data_ptr()
        if vec_dtype not in self._contrib:
            self._contrib[vec_dtype] = torch.empty(st.grad_size, dtype=vec_dtype, device=self.device)
        a.contrib = self._contrib[vec_dtype].data_ptr()
        a.damping = float(damping)
        dt = st.normal_tiles() if tiles else None
        a.tiles = dt.pointer if dt is not None else None
        if dt is not None:
            for k, jac in enumerate(self.jacs):
                if dt.perm[k] is None:
                    continue
                j2 = self._tile_jacs.get(k)
                if j2 is None:
                    n = st.plans[k].count
                    j2 = torch.empty_like(jac)
                    L.call("tls_permute_columns", jac.data_ptr(), j2.data_ptr(), L.dtype_code(jac.dtype),
                           st.rdims[k] * st.D[k], n, n, dt.perm[k].data_ptr(), L.stream_handle(jac.device))
                    self._tile_jacs[k] = j2
                a.fg[k].jac = j2.data_ptr()
        return a

    # ------------------------------------------------------------------ products
    def _check_vec(self, v, n, what):
        if v.shape != (n,):
            raise ValueError(f"{what} input has incorrect shape")
        L.require_cuda(v)
        if self.dtype == torch.float64 and v.dtype == torch.float32:
            raise ValueError("float32 vectors need a float32 Jacobian")

    def matvec(self, vector: Tensor) -> Tensor:
        """J diag(s) v (sparse.py:31-41)."""
        self._check_vec(vector, self.shape[1], "matvec")
        v = vector.contiguous()
        out = torch.empty(self.shape[0], dtype=v.dtype, device=v.device)
        a = self.normal_args(v.dtype, tiles=False)
        L.call("tls_jacobian_matvec", C.byref(a), v.data_ptr(), out.data_ptr(), L.stream_handle(v.device))
        return out

    def rmatvec(self, vector: Tensor) -> Tensor:
        """diag(s) J^T u (sparse.py:43-55), deterministic."""
        self._check_vec(vector, self.shape[0], "rmatvec")
        u = vector.contiguous()
        out = torch.empty(self.shape[1], dtype=u.dtype, device=u.device)
        a = self.normal_args(u.dtype, tiles=False)
        L.call("tls_jacobian_rmatvec", C.byref(a), u.data_ptr(), out.data_ptr(), L.stream_handle(u.device))
        return out

    def normal_matvec(self, vector: Tensor, damping: float = 0.0, *, tiles: bool = True) -> Tensor:
        """diag(s) J^T J diag(s) v + damping * v (sparse.py:83-84)."""
        self._check_vec(vector, self.shape[1], "normal_matvec")
        v = vector.contiguous()
        out = torch.empty_like(v)
        a = self.normal_args(v.dtype, damping, tiles=tiles)
        L.call("tls_normal_matvec", C.byref(a), v.data_ptr(), out.data_ptr(), L.stream_handle(v.device))
        return out

    def squared_matvec_norm(self, vector: Tensor, *, batch_size: int = 262144) -> Tensor:
        """|J v|^2 in float64, slots summed before squaring (sparse.py:57-81)."""
        if vector.shape != (self.shape[1],):
            raise ValueError("matvec input has incorrect shape")
        if batch_size < 1:
            raise ValueError("batch_size must be positive")
        v = vector.to(torch.float64).contiguous()
        a = self.normal_args(torch.float64, tiles=False)
        need = max((n + 127) // 128 for n in (p.count for p in self.structure.plans))
        buf = partials(v.device, max(L.PCG_PARTIALS, need))
        out = torch.empty((), dtype=torch.float64, device=v.device)
        L.call("tls_squared_matvec_norm", C.byref(a), v.data_ptr(), buf.data_ptr(), out.data_ptr(),
               L.stream_handle(v.device))
        return out

    def scale_columns(self, scale: Tensor) -> BlockJacobian:
        """J diag(scale), sharing the stored blocks (sparse.py:86-102)."""
        if scale.shape != (self.shape[1],):
            raise ValueError("Column scale has incorrect shape")
        s = scale.to(torch.float64)
        if self.scale is not None:
            s = self.scale * s
        return BlockJacobian(self.structure, self.jacs, self.gram_contrib, self.layout, self.shape, s.contiguous(),
                             self._tile_jacs)

    def diagonal_blocks(self) -> tuple[Tensor, ...]:
        """Exact per-variable J^T J blocks incl. aliased slots (sparse.py:104-121), float64."""
        out = []
        for gi, e in enumerate(self.layout):
            blk = torch.empty((e.count, e.dim, e.dim), dtype=torch.float64, device=self.device)
            segment_reduce(self.structure.gram_seg[gi], self.gram_contrib, blk, mode=1, dim=e.dim)
            if self.scale is not None:
                s = self.scale[e.offset : e.offset + e.size].view(e.count, e.dim)
                blk = blk * s[:, :, None] * s[:, None, :]
            out.append(blk)
        return tuple(out)

    # ------------------------------------------------------------------ reference layout
    @property
    def groups(self) -> tuple[JacobianGroup, ...]:
        if self._groups is None:
            st = self.structure
            groups = []
            for k, (plan, jac) in enumerate(zip(st.plans, self.jacs)):
                R, D, N = st.rdims[k], st.D[k], plan.count
                full = jac.view(R, D, N).permute(2, 0, 1)
                blocks, cols = [], []
                for s, t in enumerate(plan.type_indices):
                    e = self.layout[t]
                    c0 = st.slot_col[k][s]
                    col = (st.index[k][s].long()[:, None] * e.dim + e.offset
                           + torch.arange(e.dim, device=self.device)[None, :])
                    b = full[:, :, c0 : c0 + e.dim]
                    if self.scale is not None:
                        b = b * self.scale[col][:, None, :].to(b.dtype)
                    blocks.append(b.contiguous())
                    cols.append(col)
                groups.append(JacobianGroup(tuple(blocks), tuple(cols), plan.type_indices,
                                            tuple(i.long() for i in st.index[k])))
            self._groups = tuple(groups)
        return self._groups

    def to_dense(self) -> Tensor:
        """Dense copy (sparse.py:123-143; the dense_qr solver's matrix). Slots
        of one factor that name the same variable add their blocks, in slot
        order per element (``ordered_index_add_``: the same sums every run)."""
        from .kernels import ordered_index_add_

        dense = torch.zeros(self.shape, dtype=torch.float64, device=self.device)
        flat = dense.view(-1)
        ncols = self.shape[1]
        offset = 0
        for g in self.groups:
            n, r, _ = g.blocks[0].shape
            rows = torch.arange(n * r, device=self.device).reshape(n, r, 1) + offset
            idx, val = [], []
            for b, col in zip(g.blocks, g.columns):
                idx.append((rows * ncols + col[:, None, :]).reshape(-1))
                val.append(b.reshape(-1).to(torch.float64))
            ordered_index_add_(flat, torch.cat(idx), torch.cat(val).reshape(-1, 1))
            offset += n * r
        return dense.to(self.dtype)


class _ForeignPlan(NamedTuple):
    """What the device structure reads of one residual batch."""

    type_indices: tuple
    indices: tuple  # CPU int64 variable index per slot
    count: int


class _ForeignProblem(NamedTuple):
    layout: tuple
    plans: tuple


def _is_own(jacobian) -> bool:
    return isinstance(jacobian, BlockJacobian)


def _signature(jacobian):
    """Incidence structure of a reference-layout Jacobian: per batch the block
    shapes, type indices and variable indices (compared by value on bind)."""
    return tuple((tuple(tuple(b.shape) for b in g.blocks), tuple(g.type_indices),
                  tuple(i for i in g.variable_indices)) for g in jacobian.groups)


class _ForeignLayout:
    """Device structure for a Jacobian in the reference's layout
    (torchls sparse.py:11-27: per batch, per slot, blocks [N, r, d], global
    columns [N, d], type indices and variable indices; a layout of
    (offset, count, dim) groups). Built once per structure; ``pack`` brings one
    linearization into this package's storage (structure-of-arrays J plus the
    per-factor Gram contributions of the diagonal blocks) with one launch of
    the packed linearization kernel per batch."""

    def __init__(self, jacobian):
        from .problem import Structure

        groups = tuple(jacobian.groups)
        if not groups:
            raise ValueError("the Jacobian has no residual batches")
        proto = groups[0].blocks[0]
        if proto.device.type != "cuda" or proto.dtype not in (torch.float32, torch.float64):
            raise ValueError("CUDA products require CUDA float32 or float64 Jacobian blocks")
        if jacobian.shape[1] > 2**31 - 1:
            raise ValueError("CUDA products require 32-bit column indices")
        self.layout = tuple(jacobian.layout)
        self.shape = tuple(jacobian.shape)
        self.dtype, self.device = proto.dtype, proto.device
        plans, rdims = [], []
        for g in groups:
            n, r = g.blocks[0].shape[:2]
            if r > 8 or sum(b.shape[2] for b in g.blocks) > 16:
                raise ValueError("CUDA products support residual dims <= 8 and slot dims summing to <= 16")
            for b, c, t, idx in zip(g.blocks, g.columns, g.type_indices, g.variable_indices):
                e = self.layout[t]
                if b.shape != (n, r, e.dim) or b.dtype != self.dtype or b.device != self.device:
                    raise ValueError("Jacobian blocks must share shape [N, r, d_slot], dtype and device")
                want = idx.to(c.device).long()[:, None] * e.dim + e.offset + torch.arange(e.dim, device=c.device)
                if c.shape != (n, e.dim) or not torch.equal(c.long(), want):
                    raise ValueError("Jacobian columns must be variable index * dim + group offset + slot column")
            plans.append(_ForeignPlan(tuple(g.type_indices), tuple(i.detach().cpu().long() for i in g.variable_indices),
                                      int(n)))
            rdims.append(int(r))
        self.signature = _signature(jacobian)
        self.structure = Structure(_ForeignProblem(self.layout, tuple(plans)), self.device, rdims)

    def check(self, jacobian, what):
        sig = _signature(jacobian)
        same = len(sig) == len(self.signature) and all(
            a[0] == b[0] and a[1] == b[1] and all(x is y or torch.equal(x, y) for x, y in zip(a[2], b[2]))
            for a, b in zip(sig, self.signature))
        if not same or tuple(jacobian.shape) != self.shape:
            raise ValueError(f"CUDA {what} plan requires unchanged incidence structure")
        proto = jacobian.groups[0].blocks[0]
        if proto.dtype != self.dtype or proto.device != self.device:
            raise ValueError(f"CUDA {what} plan requires unchanged block shapes, dtype and device")

    def pack(self, jacobian) -> BlockJacobian:
        st = self.structure
        gram = torch.empty(st.gram_size, dtype=torch.float64, device=self.device)
        jacs, keep = [], []
        stream = L.stream_handle(self.device)
        for k, g in enumerate(jacobian.groups):
            n, r = st.plans[k].count, st.rdims[k]
            jac = torch.empty(r * st.D[k] * n, dtype=self.dtype, device=self.device)
            blocks = [b.detach().to(torch.float64).contiguous() for b in g.blocks]
            zero = torch.zeros(n * r, dtype=torch.float64, device=self.device)
            keep += [blocks, zero]
            la = L.LinearizeArgs()
            la.fg = st.factor_group(k, jac, jac_stride=n)
            la.residual_kind, la.loss_kind, la.has_loss, la.want_jacobian = L.RES_PACKED, L.LOSS_NONE, 0, 1
            la.packed_residual = zero.data_ptr()
            for si, b in enumerate(blocks):
                la.packed_blocks[si] = b.data_ptr()
            la.gram_contrib = gram.data_ptr() + 8 * st.gram_base[k]
            L.call("tls_linearize", C.byref(la), stream)
            jacs.append(jac)
        return BlockJacobian(st, tuple(jacs), gram, self.layout, self.shape)


class CudaNormalPlan:
    """Fixed incidence structure for repeated normal products.

    The interface of torchls ``WarpNormalPlan(J, max_packed_bytes=...)``,
    ``.bind(J)`` and ``.normal_matvec(v, damping)`` (warp_normal.py:125-294).
    ``J`` is either this package's ``BlockJacobian`` (already stored
    structure-of-arrays: ``bind`` checks it and returns it) or any Jacobian in
    the reference's layout (``groups`` of per-slot blocks [N, r, d] with global
    columns, ``layout``, ``shape``), such as the reference's own
    ``BlockJacobian``: the plan builds the device structure (index maps, the
    one-pass tile plan) once, and each ``bind`` packs that linearization's
    blocks into structure-of-arrays storage on the device. ``max_packed_bytes``
    is validated for interface parity; the packed copy is the only storage the
    kernels read.
    """

    def __init__(self, jacobian, *, max_packed_bytes: int = 256 * 1024**2):
        if isinstance(max_packed_bytes, bool) or not isinstance(max_packed_bytes, int) or max_packed_bytes < 0:
            raise ValueError("max_packed_bytes must be a nonnegative integer")
        if _is_own(jacobian):
            if jacobian.device.type != "cuda":
                raise ValueError("CUDA normal matvec requires a CUDA BlockJacobian")
            if jacobian.shape[1] > 2**31 - 1:
                raise ValueError("CUDA normal matvec requires 32-bit column indices")
            self._foreign = None
            self.structure = jacobian.structure
            self.dtype, self.device = jacobian.dtype, jacobian.device
        else:
            self._foreign = _ForeignLayout(jacobian)
            self.structure = self._foreign.structure
            self.dtype, self.device = self._foreign.dtype, self._foreign.device
        self.size = jacobian.shape[1]

    def bind(self, jacobian) -> BlockJacobian:
        """The linearization to multiply with; raises ValueError when its
        structure, block shapes, dtype or device differ from the plan's."""
        if self._foreign is not None:
            if _is_own(jacobian):
                raise ValueError("CUDA normal plan requires unchanged incidence structure")
            self._foreign.check(jacobian, "normal")
            return self._foreign.pack(jacobian)
        if not _is_own(jacobian) or jacobian.structure is not self.structure or jacobian.shape[1] != self.size:
            raise ValueError("CUDA normal plan requires unchanged incidence structure")
        if jacobian.dtype != self.dtype or jacobian.device != self.device:
            raise ValueError("CUDA normal plan requires unchanged block shapes, dtype and device")
        return jacobian


class CudaDiagonalPlan:
    """The interface of torchls ``WarpDiagonalPlan(J).diagonal_blocks(J)``
    (warp_diagonal.py:69-179): exact per-variable J^T J blocks, aliased slots
    included, one [count, d, d] tensor per layout entry, float64, deterministic.
    Accepts this package's ``BlockJacobian`` or the reference's layout (see
    ``CudaNormalPlan``)."""

    def __init__(self, jacobian):
        if _is_own(jacobian):
            if jacobian.device.type != "cuda":
                raise ValueError("CUDA diagonal blocks require a CUDA BlockJacobian")
            self._foreign = None
            self.structure = jacobian.structure
        else:
            self._foreign = _ForeignLayout(jacobian)
            self.structure = self._foreign.structure

    def diagonal_blocks(self, jacobian):
        if self._foreign is not None:
            if _is_own(jacobian):
                raise ValueError("CUDA diagonal plan requires unchanged incidence structure, shapes and dtype")
            self._foreign.check(jacobian, "diagonal")
            return self._foreign.pack(jacobian).diagonal_blocks()
        if not _is_own(jacobian) or jacobian.structure is not self.structure:
            raise ValueError("CUDA diagonal plan requires unchanged incidence structure, shapes and dtype")
        return jacobian.diagonal_blocks()
