"""Problem analysis and CUDA linearization.

Interface of torchls ``problem.py``: ``LeastSquaresProblem(costs, vars).analyze()``
returns an ``AnalyzedLeastSquaresProblem`` with ``residuals``, ``cost``,
``linearize`` and ``solve`` (problem.py:242-377). Index maps follow
problem.py:66-74 (ID -> row by searchsorted) and problem.py:138-148 (global
columns idx*dim + offset + arange(dim)); residuals are ordered batch by batch,
observation-major.

Data layout in HBM (per analysed problem, built once per device):
  * int32 variable indices per factor batch and slot;
  * per batch a Jacobian in structure-of-arrays order [r*D][N] (float32 or
    float64), float64 residuals [N][r], and float64 per-factor gradient and
    Gram contributions;
  * per variable group CSR lists of contribution offsets, so every reduction
    over a variable's factors runs in a fixed order (deterministic).
"""

from __future__ import annotations

import ctypes
from collections.abc import Iterable

import numpy as np
import torch
from torch import Tensor

from . import _lib as L
from .batching import AutoBatchSize
from .cost import Cost
from .kernels import partials, reduce, segment_reduce
from .losses import HuberLoss
from .variables import NamedValues, ParameterRef, Var, VariableLayout, VarValues, as_ids


def _is_ref(arg) -> bool:
    return isinstance(arg, (Var, ParameterRef))


def _lanes(degree_mean: float) -> int:
    """Lanes per reduction target: a power of two <= 32 for cold variables, a
    whole 256-thread block per target for hot ones (mean degree > 64)."""
    if degree_mean > 64:
        return 256
    lanes = 1
    while lanes < degree_mean and lanes < 32:
        lanes *= 2
    return lanes


class CostPlan:
    """One residual batch: slots, index maps, weights and data axes (problem.py:45-155)."""

    def __init__(self, cost: Cost, layout: tuple[VariableLayout, ...]):
        self.cost = cost
        self.slots = tuple(i for i, a in enumerate(cost.args) if _is_ref(a))
        if not self.slots:
            raise ValueError("Every cost must reference at least one variable or named parameter")
        keys = {e.key: i for i, e in enumerate(layout)}
        sizes = [as_ids(cost.args[i].id).numel() for i in self.slots if as_ids(cost.args[i].id).ndim == 1]
        self.batched = bool(sizes)
        self.count = max(sizes, default=1)
        if self.count == 0 or any(s not in (1, self.count) for s in sizes):
            raise ValueError("Variable batch lengths must match (or be one)")
        types, rows = [], []
        for slot in self.slots:
            var = cost.args[slot]
            key = var.name if isinstance(var, ParameterRef) else type(var)
            if key not in keys:
                raise ValueError(f"Undeclared parameter group {key!r}")
            t = keys[key]
            known = layout[t].ids
            ids = as_ids(var.id).reshape(-1).cpu().expand(self.count).contiguous()
            pos = torch.searchsorted(known, ids)
            if bool(torch.any(pos >= len(known))) or not torch.equal(known[pos.clamp_max(len(known) - 1)], ids):
                raise ValueError(f"Cost references undeclared IDs or out-of-range indices in {key!r}")
            types.append(t)
            rows.append(pos)
        self.type_indices = tuple(types)
        self.indices = tuple(rows)
        self._read_weights()
        for i, arg in enumerate(cost.args):
            if _is_ref(arg):
                axis = 0 if as_ids(arg.id).ndim == 1 else None
                if cost.in_dims is not None and cost.in_dims[i] != axis:
                    raise ValueError("Parameter reference in_dims must match its index shape")
                continue
            tensor = torch.as_tensor(arg)
            if self.data_axis(i, tensor) == 0 and (tensor.ndim == 0 or tensor.shape[0] not in (1, self.count)):
                raise ValueError("Data batch length must match observations; use in_dims=None for shared data")
        self._linearizers = {}
        self._batch = {}
        self._device_data = {}

    def _read_weights(self):
        cost = self.cost
        self.weights = None
        if cost.weights is not None:
            w = torch.as_tensor(cost.weights)
            if w.ndim > 1 or w.numel() not in (1, self.count) or w.is_complex():
                raise ValueError("Weights must be a real scalar or one value per observation")
            w = torch.as_tensor(cost.weights, dtype=torch.float64).detach().reshape(-1)
            if not bool((torch.isfinite(w) & (w >= 0)).all()):
                raise ValueError("Weights must be finite and nonnegative")
            self.weights = w.cpu().expand(self.count).clone()

    def refresh_data(self):
        """Re-read weights and data tensors (changed in place); indices stay."""
        self._read_weights()
        self._device_data = {k: v for k, v in self._device_data.items() if k[0] == "rows"}

    def data_axis(self, i, tensor):
        if self.cost.in_dims is not None:
            return self.cost.in_dims[i]
        return 0 if self.batched and tensor.ndim > 0 else None

    # ------------------------------------------------------------------ data on device
    def data_tensor(self, i, device, dtype):
        """Argument i as a device tensor with a leading axis of 1 (shared) or N."""
        key = (i, device, dtype)
        if key not in self._device_data:
            arg = self.cost.args[i]
            t = torch.as_tensor(arg)
            if t.is_floating_point() and not isinstance(arg, Tensor):
                t = torch.as_tensor(arg, dtype=dtype)
            if self.data_axis(i, t) is None:
                t = t.unsqueeze(0)
            t = t.to(device=device, dtype=dtype if t.is_floating_point() else t.dtype)
            self._device_data[key] = t.detach()
        return self._device_data[key]

    def gather(self, values: dict, layout, device, dtype, start=0, end=None):
        """Per-observation arguments for torch.func (problem.py:201-221)."""
        end = self.count if end is None else end
        out, si = [], 0
        dev_rows = self.device_rows(device)
        for i, arg in enumerate(self.cost.args):
            if _is_ref(arg):
                key = layout[self.type_indices[si]].key
                out.append(values[key][dev_rows[si][start:end]])
                si += 1
            else:
                t = self.data_tensor(i, device, dtype)
                out.append(t.expand(self.count, *t.shape[1:])[start:end])
        return out

    def device_rows(self, device):
        key = ("rows", device)
        if key not in self._device_data:
            self._device_data[key] = tuple(r.to(device) for r in self.indices)
        return self._device_data[key]

    def batch_size(self, values, layout, device, dtype):
        policy = self.cost.batch_size
        if not isinstance(policy, AutoBatchSize):
            return policy
        key = (policy, device, dtype)
        if key not in self._batch:
            args = self.gather(values, layout, device, dtype, 0, 1)
            sample = self.cost.residual_fn(*(a[0] for a in args))
            self._batch[key] = policy.resolve(
                count=self.count,
                input_bytes=sum(a[0].numel() * a.element_size() for a in args),
                residual_dim=sample.numel(),
                tangent_dim=sum(layout[t].dim for t in self.type_indices),
                mode=self.cost.jac_mode, itemsize=sample.element_size(), device=device,
            )
        return self._batch[key]

    # ------------------------------------------------------------------ built-in residuals
    def builtin(self, layout):
        """Return (kind, arg_slot) when a fused CUDA residual applies, else None."""
        tag = getattr(self.cost.residual_fn, "cuda_residual", None)
        if tag is None or self.cost.jacobian_fn is not None or len(self.cost.args) != 3:
            return None
        slot_of = {pos: s for s, pos in enumerate(self.slots)}
        arg_slot = [slot_of.get(i, -1) for i in range(3)] + [-1]
        if arg_slot[2] != -1:
            return None
        kinds = [getattr(layout[self.type_indices[arg_slot[i]]].var_type, "cuda_kind", None)
                 if arg_slot[i] >= 0 else None for i in range(2)]
        if tag == "reprojection":
            if arg_slot[0] >= 0 and (kinds[0] != "se3" or arg_slot[0] != 0):
                return None
            if arg_slot[1] >= 0 and (kinds[1] != "euclidean" or layout[self.type_indices[arg_slot[1]]].dim != 3):
                return None
            if arg_slot[0] < 0 and arg_slot[1] >= 0 and arg_slot[1] != 0:
                return None
            return L.RES_REPROJECTION, arg_slot
        if tag == "se3_between":
            if any(arg_slot[i] >= 0 and kinds[i] != "se3" for i in range(2)):
                return None
            return L.RES_SE3_BETWEEN, arg_slot
        if tag == "sim3_between":
            if any(arg_slot[i] >= 0 and kinds[i] != "sim3" for i in range(2)):
                return None
            return L.RES_SIM3_BETWEEN, arg_slot
        return None


class Structure:
    """Device-side symbolic structure of an analysed problem (built once per device)."""

    def __init__(self, problem: AnalyzedLeastSquaresProblem, device: torch.device, rdims: list[int]):
        self.device = device
        layout = problem.layout
        self.layout = layout
        self.rdims = rdims
        self.vgroups = (L.VarGroup * L.MAX_GROUPS)()
        if len(layout) > L.MAX_GROUPS:
            raise ValueError(f"the CUDA backend supports at most {L.MAX_GROUPS} variable groups")
        if len(problem.plans) > L.MAX_FACTOR_GROUPS:
            raise ValueError(f"the CUDA backend supports at most {L.MAX_FACTOR_GROUPS} residual batches")
        for i, e in enumerate(layout):
            self.vgroups[i] = L.VarGroup(e.offset, e.count, e.dim)
        self.plans = problem.plans
        self._tiles = None
        self.D, self.W, self.slot_col, self.slot_gram, self.index = [], [], [], [], []
        self.grad_base, self.gram_base, self.res_base, self.obs_base = [], [], [], []
        g = gr = rs = ob = 0
        for plan, r in zip(problem.plans, rdims):
            dims = [layout[t].dim for t in plan.type_indices]
            if len(dims) > L.MAX_SLOTS:
                raise ValueError(f"the CUDA backend supports at most {L.MAX_SLOTS} variable arguments")
            cols = np.concatenate(([0], np.cumsum(dims)))[:-1]
            grams = np.concatenate(([0], np.cumsum([d * (d + 1) // 2 for d in dims])))[:-1]
            self.D.append(int(sum(dims)))
            self.W.append(int(sum(d * (d + 1) // 2 for d in dims)))
            self.slot_col.append([int(c) for c in cols])
            self.slot_gram.append([int(c) for c in grams])
            self.index.append(tuple(rows.to(device=device, dtype=torch.int32) for rows in plan.indices))
            self.grad_base.append(g)
            self.gram_base.append(gr)
            self.res_base.append(rs)
            self.obs_base.append(ob)
            g += plan.count * self.D[-1]
            gr += plan.count * self.W[-1]
            rs += plan.count * r
            ob += plan.count
        self.grad_size, self.gram_size, self.res_size, self.obs_size = g, gr, rs, ob
        if max(g, gr) >= 2**31:
            raise ValueError("contribution buffers exceed the 32-bit offset range")
        # CSR of contribution offsets per variable group (fixed order: batch, slot, factor)
        self.grad_seg, self.gram_seg, self._keep = [], [], []
        for gi, e in enumerate(layout):
            ids, goff, qoff = [], [], []
            for k, plan in enumerate(problem.plans):
                f = np.arange(plan.count, dtype=np.int64)
                for s, t in enumerate(plan.type_indices):
                    if t != gi:
                        continue
                    ids.append(plan.indices[s].numpy())
                    goff.append(self.grad_base[k] + f * self.D[k] + self.slot_col[k][s])
                    qoff.append(self.gram_base[k] + f * self.W[k] + self.slot_gram[k][s])
            ids = np.concatenate(ids) if ids else np.zeros(0, np.int64)
            order = np.argsort(ids, kind="stable")
            counts = np.bincount(ids, minlength=e.count)
            ptr = np.concatenate(([0], np.cumsum(counts))).astype(np.int32)
            lanes = _lanes(float(counts.mean()) if e.count else 1.0)
            for lst, offs, width in ((self.grad_seg, goff, e.dim), (self.gram_seg, qoff, e.dim * (e.dim + 1) // 2)):
                src = (np.concatenate(offs)[order] if offs else np.zeros(0, np.int64)).astype(np.int32)
                p_t = torch.from_numpy(ptr).to(device)
                s_t = torch.from_numpy(src).to(device)
                self._keep += [p_t, s_t]
                lst.append(L.Segments(e.count, width, lanes, 0, p_t.data_ptr(), s_t.data_ptr()))

    def normal_tiles(self):
        """The one-pass normal operator's tile plan on this device (built on
        first use, kept with the structure), or None when a factor shape does
        not fit it (the operator then runs in two passes)."""
        if self._tiles is None:
            self._tiles = False
            if self.device.type == "cuda":
                from .normal_tiles import FactorGroupShape, build_tile_plan

                groups = [FactorGroupShape(plan.count, [(self.layout[t].offset, self.layout[t].dim,
                                                         plan.indices[s].numpy())
                                                        for s, t in enumerate(plan.type_indices)], r)
                          for plan, r in zip(self.plans, self.rdims)]
                vg = [(e.offset, e.count, e.dim) for e in self.layout]
                sms = torch.cuda.get_device_properties(self.device).multi_processor_count
                tp = build_tile_plan(groups, vg, sms)
                if tp is not None:
                    self._tiles = _DeviceTiles(tp, self.device)
        return self._tiles or None

    def factor_group(self, k: int, jac: Tensor | None, jac_stride: int = 0, count=None, start: int = 0):
        plan = self.plans[k]
        fg = L.FactorGroup()
        fg.count = plan.count if count is None else count
        fg.rdim = self.rdims[k]
        fg.nslots = len(plan.type_indices)
        fg.total_dim = self.D[k]
        fg.jac_dtype = L.F64 if jac is None or jac.dtype == torch.float64 else L.F32
        for s, t in enumerate(plan.type_indices):
            fg.slot_group[s] = t
            fg.slot_dim[s] = self.layout[t].dim
            fg.slot_col[s] = self.slot_col[k][s]
            fg.slot_gram[s] = self.slot_gram[k][s]
            fg.index[s] = self.index[k][s].data_ptr() + 4 * start
        fg.jac = None if jac is None else jac.data_ptr() + jac.element_size() * start
        fg.jac_stride = jac_stride
        return fg


class _DeviceTiles:
    """A tile plan's arrays on the device and the ``tls_normal_tiles`` that
    points at them (kept alive together)."""

    def __init__(self, tp, device):
        self.plan = tp
        put = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
        self._keep = []
        t = L.NormalTiles()
        t.ncta, t.ntiles = tp.ncta, tp.ntiles
        t.stage_doubles, t.acc_doubles = tp.stage_doubles, tp.acc_doubles
        t.ntargets, t.gather_lanes, t.xbuf_doubles = len(tp.target_col), tp.gather_lanes, tp.xbuf_doubles
        t.nheavy = tp.nheavy
        for k in range(len(tp.tile_factors)):
            t.tile_factors[k] = tp.tile_factors[k]
            t.tile_base[k] = tp.tile_base[k]
            if tp.pos[k] is not None:
                pk = put(tp.pos[k].view(np.int32))
                self._keep.append(pk)
                t.pos[k] = pk.data_ptr()
        for k, v in enumerate(tp.cta_base):
            t.cta_base[k] = v
        for name in ("cta_tile", "tile_run", "run_col", "run_meta", "run_dest", "run_xoff", "cta_flush", "flush_col",
                     "flush_meta", "flush_dest", "target_col", "target_dim", "target_ptr", "target_src"):
            arr = getattr(tp, name)
            d = put(arr if len(arr) else np.zeros(1, np.int32))
            self._keep.append(d)
            setattr(t, name, d.data_ptr())
        # tile-position -> factor permutations (None: the caller's order)
        self.perm = [None if q is None else put(q.astype(np.int32)) for q in tp.perm]
        self.partials = torch.empty(max(tp.npartials, 1), dtype=torch.float64, device=device)
        t.partials = self.partials.data_ptr()
        self.struct = t
        self.pointer = ctypes.pointer(t)


class Linearization:
    """Residual and Jacobian of the local model plus the true objective (problem.py:20-42).

    With a loss, ``raw_residual`` holds the original errors and ``cost`` is the
    robust objective.
    """

    def __init__(self, residual, jacobian, raw_residual=None, objective=None, gradient=None):
        self.residual = residual
        self.jacobian = jacobian
        self.raw_residual = raw_residual
        self._objective = objective  # per-factor float64, or None
        self._gradient = gradient
        self._cost = None

    @property
    def objective(self):
        return None if self._objective is None else self.cost

    @property
    def cost(self) -> Tensor:
        if self._cost is None:
            if self._objective is not None:
                self._cost = 0.5 * reduce(self._objective)
            else:
                self._cost = 0.5 * reduce(self.residual, 1)
        return self._cost

    @property
    def gradient(self) -> Tensor:
        if self._gradient is None:
            self._gradient = self.jacobian.rmatvec(self.residual)
        return self._gradient


class LeastSquaresProblem:
    def __init__(self, costs: Iterable[Cost], variables: Iterable[Var]):
        self.costs = tuple(costs)
        self.variables = tuple(variables)

    def analyze(self) -> AnalyzedLeastSquaresProblem:
        """Layout by Var type, IDs sorted and unique (problem.py:247-261)."""
        if not self.costs or not self.variables:
            raise ValueError("A problem needs costs and variables")
        by_type: dict = {}
        for var in self.variables:
            by_type.setdefault(type(var), []).append(as_ids(var.id).reshape(-1).cpu())
        layout, offset = [], 0
        for key, parts in by_type.items():
            ids = torch.cat(parts).sort().values
            if len(ids) == 0 or bool(torch.any(ids[1:] == ids[:-1])):
                raise ValueError("Declared variable IDs must be nonempty and unique per type")
            layout.append(VariableLayout(key, ids, offset))
            offset += len(ids) * key.tangent_dim
        return AnalyzedLeastSquaresProblem(tuple(layout), self.costs, offset)


class AnalyzedLeastSquaresProblem:
    def __init__(self, layout, costs, tangent_dim):
        self.layout = layout
        self.tangent_dim = tangent_dim
        self.plans = tuple(CostPlan(c, layout) for c in costs)
        self._has_loss = any(p.cost.loss is not None or p.cost.weights is not None for p in self.plans)
        self._structures = {}

    def refresh_data(self):
        """Data tensors or weights of the residuals were changed in place: drop
        the cached device copies (the symbolic analysis and plans stay)."""
        for plan in self.plans:
            plan.refresh_data()

    # ------------------------------------------------------------------ values
    def _validate_values(self, vals):
        if set(vals._values) != {e.key for e in self.layout}:
            raise ValueError("Initial value types do not match the analyzed problem")
        for e in self.layout:
            if not torch.equal(vals._ids[e.key], e.ids):
                raise ValueError("Initial value IDs do not match the analyzed problem")

    def default_values(self):
        if self.layout[0].name is not None:
            return NamedValues(
                {e.key: e.var_type.default_factory().expand(e.count, *e.var_type.default_factory().shape)
                 for e in self.layout}, self.layout)
        return VarValues.make(e.var_type(e.ids) for e in self.layout)

    @staticmethod
    def _work_values(vals):
        """float64 contiguous working copies of the values, keyed like vals._values."""
        return {k: (v if v.dtype == torch.float64 else v.double()).contiguous() for k, v in vals._values.items()}

    # ------------------------------------------------------------------ structure
    def structure(self, device) -> Structure:
        device = torch.device(device)
        if device not in self._structures:
            rdims = []
            vals = {e.key: e.var_type.default_factory().to(device=device, dtype=torch.float64)
                    .expand(e.count, *e.var_type.default_factory().shape) for e in self.layout}
            for plan in self.plans:
                b = plan.builtin(self.layout)
                if b is not None:
                    rdims.append({L.RES_REPROJECTION: 2, L.RES_SE3_BETWEEN: 6, L.RES_SIM3_BETWEEN: 7}[b[0]])
                    continue
                args = plan.gather(vals, self.layout, device, torch.float64, 0, 1)
                rdims.append(int(plan.cost.residual_fn(*(a[0] for a in args)).numel()))
            self._structures[device] = Structure(self, device, rdims)
        return self._structures[device]

    # ------------------------------------------------------------------ evaluation
    def _builtin_args(self, plan, k, st, values, la, device):
        kind, arg_slot = plan.builtin(self.layout)
        la.residual_kind = kind
        for a in range(3):
            la.arg_slot[a] = arg_slot[a]
            if arg_slot[a] >= 0:
                key = self.layout[plan.type_indices[arg_slot[a]]].key
                la.arg_data[a] = values[key].data_ptr()
                la.arg_stride[a] = 0
            else:
                t = plan.data_tensor(a, device, torch.float64)
                if not t.is_contiguous():
                    t = t.contiguous()
                    plan._device_data[(a, device, torch.float64)] = t
                la.arg_data[a] = t.data_ptr()
                la.arg_stride[a] = 0 if t.shape[0] == 1 else int(np.prod(t.shape[1:]))
        la.arg_slot[3] = -1

    def _raw_plan_residuals(self, plan, k, st, values, device, out):
        """Raw residuals [N][r] (float64) of one batch into ``out``."""
        b = plan.builtin(self.layout)
        if b is not None:
            la = L.LinearizeArgs()
            la.fg = st.factor_group(k, None)
            self._builtin_args(plan, k, st, values, la, device)
            la.loss_kind = L.LOSS_NONE
            la.has_loss = 0
            la.want_jacobian = 0
            la.raw_residual = out.data_ptr()
            L.call("tls_linearize", C_byref(la), L.stream_handle(device))
            return out
        fn = torch.func.vmap(plan.cost.residual_fn)
        batch = plan.batch_size(values, self.layout, device, torch.float64) or plan.count
        view = out.view(plan.count, -1)
        for s in range(0, plan.count, batch):
            e = min(s + batch, plan.count)
            args = plan.gather(values, self.layout, device, torch.float64, s, e)
            view[s:e] = fn(*args).reshape(e - s, -1).to(torch.float64)
        return out

    def residuals(self, vals) -> Tensor:
        """Raw residuals without robust weights or loss transforms (problem.py:292-299)."""
        self._validate_values(vals)
        device = vals.device
        L.require_cuda(next(iter(vals._values.values())))
        st = self.structure(device)
        values = self._work_values(vals)
        out = torch.empty(st.res_size, dtype=torch.float64, device=device)
        for k, plan in enumerate(self.plans):
            n = plan.count * st.rdims[k]
            self._raw_plan_residuals(plan, k, st, values, device, out[st.res_base[k] : st.res_base[k] + n])
        return out.to(vals.dtype)

    def _plan_losses(self, plan, k, st, raw, device):
        """(rho, rho', rho'') of a generic loss on a batch's squared norms, float64."""
        r = raw.view(plan.count, st.rdims[k])
        s = (r * r).sum(-1)
        rho, d1, d2 = plan.cost.loss.evaluate(s)
        f = lambda t: torch.as_tensor(t, dtype=torch.float64, device=device).expand(plan.count).contiguous()
        return f(rho), f(d1), f(d2)

    def cost(self, vals) -> Tensor:
        """True objective 0.5 * sum w * rho(s) (problem.py:301-313), float64 on device."""
        raw = self.residuals(vals).double()
        if not self._has_loss:
            return 0.5 * reduce(raw, 1)
        st = self.structure(vals.device)
        total = torch.zeros((), dtype=torch.float64, device=vals.device)
        for k, plan in enumerate(self.plans):
            seg = raw[st.res_base[k] : st.res_base[k] + plan.count * st.rdims[k]].view(plan.count, -1)
            s = (seg * seg).sum(-1)
            loss = plan.cost.loss
            v = s if loss is None else loss.value(s)
            if plan.weights is not None:
                v = plan.weights.to(vals.device) * v
            total = total + reduce(v)
        return 0.5 * total

    def linearize(self, vals, *, jacobian_dtype=None, schur=None) -> Linearization:
        """Linearize at ``vals`` with fused CUDA kernels (problem.py:350-368).

        ``jacobian_dtype`` selects the stored Jacobian precision (float64 or
        float32; default the values' dtype). ``schur`` (a SchurStructure) adds
        the per-factor cross blocks used by Schur elimination.
        """
        from .sparse import BlockJacobian

        self._validate_values(vals)
        device = vals.device
        L.require_cuda(next(iter(vals._values.values())))
        st = self.structure(device)
        jdt = jacobian_dtype or vals.dtype
        values = self._work_values(vals)
        stream = L.stream_handle(device)
        residual = torch.empty(st.res_size, dtype=torch.float64, device=device)
        raw = torch.empty(st.res_size, dtype=torch.float64, device=device) if self._has_loss else None
        objective = torch.empty(st.obs_size, dtype=torch.float64, device=device) if self._has_loss else None
        grad_c = torch.empty(st.grad_size, dtype=torch.float64, device=device)
        gram_c = torch.empty(st.gram_size, dtype=torch.float64, device=device)
        cross_c = schur.cross_buffer(device) if schur is not None else None
        jacs = []
        for k, plan in enumerate(self.plans):
            R, D, N = st.rdims[k], st.D[k], plan.count
            jac = torch.empty((R * D, N), dtype=jdt, device=device)
            jacs.append(jac)
            la = L.LinearizeArgs()
            la.has_loss = int(self._has_loss)
            la.want_jacobian = 1
            loss = plan.cost.loss
            w = plan.weights.to(device) if plan.weights is not None else None
            rb, ob, gb, qb = st.res_base[k], st.obs_base[k], st.grad_base[k], st.gram_base[k]
            generic = loss is not None and not isinstance(loss, HuberLoss)
            if isinstance(loss, HuberLoss):
                la.loss_kind, la.loss_delta = L.LOSS_HUBER, float(loss.delta)
            elif generic:
                la.loss_kind = L.LOSS_GENERIC
            cross_base = schur.fill_cross_args(k, la) if schur is not None else 0
            b = plan.builtin(self.layout)
            if b is not None:
                rho = None
                if generic:
                    tmp = raw[rb : rb + N * R]
                    self._raw_plan_residuals(plan, k, st, values, device, tmp)
                    rho = self._plan_losses(plan, k, st, tmp, device)
                self._launch_linearize(st, k, la, jac, 0, N, residual, raw, objective, grad_c, gram_c, w, rho,
                                       lambda a: self._builtin_args(plan, k, st, values, a, device),
                                       stream, cross_c, cross_base)
                if generic:
                    objective[ob : ob + N] = rho[0] * (w if w is not None else 1.0)
            else:
                lin = self._user_linearizer(plan, k, st, device)
                batch = plan.batch_size(values, self.layout, device, torch.float64) or N
                for s in range(0, N, batch):
                    e = min(s + batch, N)
                    args = plan.gather(values, self.layout, device, torch.float64, s, e)
                    blocks, res = lin(args)
                    res = res.reshape(e - s, R).to(torch.float64).contiguous()
                    blocks = [bk.to(torch.float64).contiguous() for bk in blocks]
                    for bk, t in zip(blocks, plan.type_indices):
                        if tuple(bk.shape) != (e - s, R, self.layout[t].dim):
                            raise ValueError("Incorrect local Jacobian shape")
                    rho = None
                    if generic:
                        s2 = (res * res).sum(-1)
                        r0, r1, r2 = plan.cost.loss.evaluate(s2)
                        f = lambda t_: torch.as_tensor(t_, dtype=torch.float64, device=device).expand(e - s).contiguous()
                        rho = (f(r0), f(r1), f(r2))
                        ww = w[s:e] if w is not None else None
                        objective[ob + s : ob + e] = rho[0] * (ww if ww is not None else 1.0)

                    def packed(a, res=res, blocks=blocks):
                        a.residual_kind = L.RES_PACKED
                        a.packed_residual = res.data_ptr()
                        for si, bk in enumerate(blocks):
                            a.packed_blocks[si] = bk.data_ptr()

                    self._launch_linearize(st, k, la, jac, s, e - s, residual, raw, objective, grad_c, gram_c,
                                           w, rho, packed, stream, cross_c, cross_base)
                    del args, blocks, res
        gradient = torch.empty(self.tangent_dim, dtype=torch.float64, device=device)
        for gi, e in enumerate(self.layout):
            segment_reduce(st.grad_seg[gi], grad_c, gradient[e.offset : e.offset + e.size])
        jac = BlockJacobian(st, jacs, gram_c, self.layout, (st.res_size, self.tangent_dim))
        lin = Linearization(residual, jac, raw, objective, gradient)
        lin.grad_contrib = grad_c
        lin.cross_contrib = cross_c
        return lin

    def _launch_linearize(self, st, k, la, jac, start, count, residual, raw, objective, grad_c, gram_c, w, rho,
                          fill_inputs, stream, cross_c, cross_base):
        plan = self.plans[k]
        R, D, W = st.rdims[k], st.D[k], st.W[k]
        rb, ob, gb, qb = st.res_base[k], st.obs_base[k], st.grad_base[k], st.gram_base[k]
        la.fg = st.factor_group(k, jac, jac_stride=plan.count, count=count, start=start)
        fill_inputs(la)
        f8 = 8
        la.residual = residual.data_ptr() + f8 * (rb + start * R)
        la.raw_residual = None if raw is None else raw.data_ptr() + f8 * (rb + start * R)
        la.objective = None if objective is None else objective.data_ptr() + f8 * (ob + start)
        la.grad_contrib = grad_c.data_ptr() + f8 * (gb + start * D)
        la.gram_contrib = gram_c.data_ptr() + f8 * (qb + start * W)
        la.weights = None if w is None else w.data_ptr() + f8 * start
        if rho is not None:
            la.rho1 = rho[1].data_ptr() + (0 if rho[1].numel() == count else f8 * start)
            la.rho2 = rho[2].data_ptr() + (0 if rho[2].numel() == count else f8 * start)
        if cross_c is not None and la.cross_width:
            la.cross_contrib = cross_c.data_ptr() + f8 * (cross_base + start * la.cross_width)
        else:
            la.cross_contrib = None
        L.call("tls_linearize", C_byref(la), stream)

    def _user_linearizer(self, plan, k, st, device):
        """vmap(jacrev/jacfwd) of the residual at delta = 0 through the
        retraction's first-order chart (linearization.py:62-112)."""
        key = device
        if key in plan._linearizers:
            return plan._linearizers[key]
        types = tuple(self.layout[t].var_type for t in plan.type_indices)
        fn, jfn = plan.cost.residual_fn, plan.cost.jacobian_fn
        if jfn is not None:
            bj, br = torch.func.vmap(jfn), torch.func.vmap(fn)

            def run(args):
                blocks = bj(*args)
                if not isinstance(blocks, tuple) or len(blocks) != len(types):
                    raise ValueError("Custom Jacobian must return one block per Var argument")
                return blocks, br(*args).reshape(args[0].shape[0], -1)

            plan._linearizers[key] = run
            return run
        mode = plan.cost.jac_mode
        if mode == "auto":
            mode = "reverse" if st.rdims[k] <= sum(t.tangent_dim for t in types) else "forward"
        jvps = tuple(getattr(t, "retract_jvp_fn", None) for t in types)
        slots = plan.slots

        def local(deltas, *args):
            upd = list(args)
            for pos, t, jvp, d in zip(slots, types, jvps, deltas):
                upd[pos] = args[pos] + jvp(args[pos], d) if jvp is not None else t.retract_fn(args[pos], d)
            out = fn(*upd).reshape(-1)
            return out, out

        diff = torch.func.jacrev if mode == "reverse" else torch.func.jacfwd
        nargs = len(plan.cost.args)
        batched = torch.func.vmap(diff(local, argnums=0, has_aux=True), in_dims=(None, *([0] * nargs)))
        zeros = tuple(torch.zeros(t.tangent_dim, dtype=torch.float64, device=device) for t in types)

        def run(args):
            blocks, res = batched(zeros, *args)
            return tuple(blocks), res

        plan._linearizers[key] = run
        return run

    def _evaluate_trial(self, vals, lin):
        """Objective and exact reduction at a proposed point (problem.py:315-348)."""
        device = vals.device
        st = self.structure(device)
        values = self._work_values(vals)
        new = torch.empty(st.res_size, dtype=torch.float64, device=device)
        out = torch.zeros(2, dtype=torch.float64, device=device)
        buf = partials(device)
        stream = L.stream_handle(device)
        before = lin.raw_residual if self._has_loss else lin.residual
        for k, plan in enumerate(self.plans):
            R, N, rb = st.rdims[k], plan.count, st.res_base[k]
            seg_new = new[rb : rb + N * R]
            self._raw_plan_residuals(plan, k, st, values, device, seg_new)
            seg_old = before[rb : rb + N * R]
            loss = plan.cost.loss
            kind, delta, rho_old, rho_new = L.LOSS_NONE, 0.0, None, None
            if isinstance(loss, HuberLoss):
                kind, delta = L.LOSS_HUBER, float(loss.delta)
            elif loss is not None:
                kind = L.LOSS_GENERIC
                rho_old = self._plan_losses(plan, k, st, seg_old, device)[0]
                rho_new = self._plan_losses(plan, k, st, seg_new, device)[0]
            w = plan.weights.to(device) if plan.weights is not None else None
            L.call("tls_trial_terms", N, R, L.ptr(seg_old), L.ptr(seg_new), kind, delta, L.ptr(rho_old),
                   L.ptr(rho_new), L.ptr(w), int(self._has_loss), L.ptr(buf), L.ptr(out), stream)
        return out[0], out[1]

    def solve(self, initial_vals=None, **kwargs):
        from .solvers import solve

        return solve(self, self.default_values() if initial_vals is None else initial_vals, **kwargs)


def C_byref(obj):
    import ctypes

    return ctypes.byref(obj)
