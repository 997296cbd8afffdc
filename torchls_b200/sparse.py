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
        """Dense copy for diagnostics (sparse.py:123-143); the solver never calls it."""
        dense = torch.zeros(self.shape, dtype=self.dtype, device=self.device)
        offset = 0
        for g in self.groups:
            n, r, _ = g.blocks[0].shape
            rows = torch.arange(n * r, device=self.device).reshape(n, r, 1) + offset
            for b, col in zip(g.blocks, g.columns):
                dense.index_put_((rows.expand_as(b).reshape(-1), col[:, None, :].expand_as(b).reshape(-1)),
                                 b.reshape(-1), accumulate=True)
            offset += n * r
        return dense


class CudaNormalPlan:
    """Fixed incidence structure for repeated normal products.

    Mirrors torchls ``WarpNormalPlan(J, max_packed_bytes=...)`` /
    ``.bind(J)`` / ``.normal_matvec(v, damping)`` (warp_normal.py:125-294).
    ``max_packed_bytes`` is accepted for interface parity; the Jacobian is
    always stored structure-of-arrays, so no extra packed copy exists.
    """

    def __init__(self, jacobian: BlockJacobian, *, max_packed_bytes: int = 256 * 1024**2):
        if not isinstance(jacobian, BlockJacobian) or jacobian.device.type != "cuda":
            raise ValueError("CUDA normal matvec requires a CUDA BlockJacobian")
        if isinstance(max_packed_bytes, bool) or not isinstance(max_packed_bytes, int) or max_packed_bytes < 0:
            raise ValueError("max_packed_bytes must be a nonnegative integer")
        if jacobian.shape[1] > 2**31 - 1:
            raise ValueError("CUDA normal matvec requires 32-bit column indices")
        self.structure = jacobian.structure
        self.size = jacobian.shape[1]
        self.dtype, self.device = jacobian.dtype, jacobian.device

    def bind(self, jacobian: BlockJacobian) -> BlockJacobian:
        if jacobian.structure is not self.structure or jacobian.shape[1] != self.size:
            raise ValueError("CUDA normal plan requires unchanged incidence structure")
        if jacobian.dtype != self.dtype or jacobian.device != self.device:
            raise ValueError("CUDA normal plan requires unchanged block shapes, dtype and device")
        return jacobian


class CudaDiagonalPlan:
    """Mirrors torchls ``WarpDiagonalPlan(J).diagonal_blocks(J)`` (warp_diagonal.py:69-179)."""

    def __init__(self, jacobian: BlockJacobian):
        if not isinstance(jacobian, BlockJacobian) or jacobian.device.type != "cuda":
            raise ValueError("CUDA diagonal blocks require a CUDA BlockJacobian")
        self.structure = jacobian.structure

    def diagonal_blocks(self, jacobian: BlockJacobian):
        if jacobian.structure is not self.structure:
            raise ValueError("CUDA diagonal plan requires unchanged incidence structure, shapes and dtype")
        return jacobian.diagonal_blocks()
