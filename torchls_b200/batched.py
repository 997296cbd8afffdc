"""Many independent least-squares problems solved together on one GPU.

``solve_batched(problems)`` merges problems with the same parameter groups and
residual batches into one block-diagonal problem and runs Levenberg-Marquardt
with PER-PROBLEM damping, acceptance and convergence:

* one linearization and one Schur elimination for all problems per trial
  (every kernel launch covers every problem); then each problem's dense
  reduced matrix S_p is assembled (``tls_batched_schur_dense``) and the CG of
  EVERY problem runs in one persistent launch (``tls_batched_pcg``): CTAs pull
  tasks of 1-8 problems from a device work queue, each problem runs its own CG
  (alpha, beta, threshold, convergence) on its own warps with no grid-wide
  synchronisation, with the tiling (warps per problem) chosen per size class
  by an autotuner (:class:`BatchedSystems`);
* per-problem damping lambda_p enters as a column scale 1/sqrt(lambda_p) with
  unit damping: (s A s + I) y = s b, x = s y equals (A + lambda_p I) x = b on
  each diagonal block, so the shared kernels need no per-problem parameter;
* per-problem trial cost, exact reduction (Huber divided difference,
  ``tls_factor_terms``), predicted reduction and gain ratio are fixed-order
  segmented sums (``tls_segment_reduce``) over each problem's factors and
  tangent entries; acceptance, damping updates, step counters and the
  cost-tolerance stop run in ``tls_batched_lm_update`` (one thread per problem);
* accepted problems keep their new values and wait for the next
  linearization; rejected ones raise lambda_p and are solved again in the
  next trial (the others contribute a zero right-hand side, so their blocks
  of the PCG iterate stay zero); converged or failed problems leave the
  active mask.

Per-problem LM decisions follow torchls solvers.py:288-696 (fixed-factor
damping, step quality 1e-4, cost and gradient tolerances); the per-problem
CG stops on its recurrence residual (no true-residual restarts).
"""

from __future__ import annotations

import ctypes as C
import math
from collections.abc import Sequence
from dataclasses import dataclass, field

import numpy as np
import torch
from torch import Tensor

from . import _lib as L
from .kernels import segment_reduce
from .losses import HuberLoss
from .named import Problem
from .variables import NamedValues, ParameterRef

__all__ = ["BatchedProblem", "BatchedSummary", "merge_problems", "partition_problems", "solve_batched"]


def merge_problems(problems: Sequence[Problem]):
    """One block-diagonal ``Problem`` from problems with identical parameter
    groups (names, manifolds, trailing shapes) and residual batches (same
    function, loss and argument kinds at each position).

    Returns ``(merged, var_problem, slices)``: ``var_problem[name]`` is the
    problem id of each variable of group ``name``; ``slices[p][name]`` the
    rows of problem p in that group.
    """
    if not problems:
        raise ValueError("no problems to merge")
    first = problems[0]
    names = list(first.parameters)
    for p in problems:
        if list(p.parameters) != names or dict(p.manifolds) != dict(first.manifolds):
            raise ValueError("problems must share parameter groups and manifolds")
        if len(p._costs) != len(first._costs):
            raise ValueError("problems must share residual batches")
    counts = {n: [int(p.parameters[n].shape[0]) for p in problems] for n in names}
    offsets = {n: np.concatenate(([0], np.cumsum(counts[n]))) for n in names}
    params = {n: torch.cat([p.parameters[n] for p in problems]) for n in names}
    merged = Problem(params, manifolds=dict(first.manifolds))
    for k, c0 in enumerate(first._costs):
        cs = [p._costs[k] for p in problems]
        if any(c.residual_fn is not c0.residual_fn or type(c.loss) is not type(c0.loss) for c in cs):
            raise ValueError(f"residual batch {k} differs between problems")
        n_obs = [_count(c) for c in cs]
        args, dims = [], []
        for i, a0 in enumerate(c0.args):
            if isinstance(a0, ParameterRef):
                ids = torch.cat([torch.as_tensor(c.args[i].id).reshape(-1) + int(offsets[a0.name][j])
                                 for j, c in enumerate(cs)])
                args.append((a0.name, ids))
                dims.append(0)
            else:
                axis = c0.in_dims[i] if c0.in_dims is not None else (0 if torch.as_tensor(a0).ndim > 0 else None)
                parts = []
                for c, n in zip(cs, n_obs):
                    t = torch.as_tensor(c.args[i])
                    parts.append(t.unsqueeze(0).expand(n, *t.shape) if axis is None else t)
                args.append(torch.cat(parts))
                dims.append(0)
        weights = None
        if c0.weights is not None:
            weights = torch.cat([torch.as_tensor(c.weights, dtype=torch.float64).reshape(-1).expand(n)
                                 for c, n in zip(cs, n_obs)])
        merged.add_residual(c0.residual_fn, *args, in_dims=tuple(dims), loss=c0.loss, weights=weights,
                            jac_mode=c0.jac_mode)
    var_problem = {n: torch.repeat_interleave(torch.arange(len(problems)), torch.tensor(counts[n])) for n in names}
    slices = [{n: slice(int(offsets[n][j]), int(offsets[n][j + 1])) for n in names} for j in range(len(problems))]
    return merged, var_problem, slices


def _count(cost) -> int:
    for a in cost.args:
        if isinstance(a, ParameterRef):
            ids = torch.as_tensor(a.id)
            if ids.ndim == 1:
                return int(ids.numel())
    raise ValueError("each residual batch needs a batched parameter reference")


@dataclass
class BatchedSummary:
    problems: int
    iterations: int = 0
    linear_solves: int = 0
    linear_iterations: int = 0
    initial_cost: Tensor | None = None
    final_cost: Tensor | None = None
    accepted_steps: Tensor | None = None
    rejected_steps: Tensor | None = None
    termination: list = field(default_factory=list)


class _Segments:
    """Fixed-order per-problem sums of a float64 vector (CSR over element ids)."""

    def __init__(self, pid: Tensor, nproblems: int, device):
        pid = pid.to(torch.int64).cpu()
        order = torch.argsort(pid, stable=True)
        ptr = torch.zeros(nproblems + 1, dtype=torch.int64)
        ptr[1:] = torch.cumsum(torch.bincount(pid, minlength=nproblems), 0)
        self.ptr = ptr.to(device=device, dtype=torch.int32)
        self.src = order.to(device=device, dtype=torch.int32)
        mean = float(pid.numel()) / max(nproblems, 1)
        lanes = 256 if mean > 64 else (32 if mean > 16 else 8)
        self.seg = L.Segments(nproblems, 1, lanes, 0, self.ptr.data_ptr(), self.src.data_ptr())
        self.n = nproblems
        self.pid = pid.to(device)

    def sum(self, x: Tensor) -> Tensor:
        out = torch.empty(self.n, dtype=torch.float64, device=x.device)
        return segment_reduce(self.seg, x.to(torch.float64).contiguous(), out)


def _user_loss_terms(loss, s_old, s_new):
    """Per-factor rho(s_new) and rho(s_old) - rho(s_new) of a loss other than
    Huber (its torch ``evaluate``, user code); Huber and no loss run in
    ``tls_factor_terms``."""
    rho_new = loss.evaluate(s_new)[0]
    rho_old = loss.evaluate(s_old)[0]
    return rho_new, rho_old - rho_new


# ---------------------------------------------------------------- batched reduced systems
_SMEM_PER_CTA = 112 * 1024  # dynamic shared memory per 256-thread CTA: two CTAs per SM
_SIZE_CLASSES = (24, 48, 96, 192, 1 << 30)  # upper bounds of a problem's reduced dimension n_p
_GROUP_CHOICES = (8, 4, 2, 1)  # problems per CTA (1, 2, 4 or 8 warps per problem)


class BatchedSystems:
    """Dense per-problem reduced matrices and the one-launch batched PCG
    (``tls_batched_schur_dense`` + ``tls_batched_pcg``).

    Problems are grouped into size classes by n_p; a class runs as tasks of
    ``k`` problems per CTA, ``k`` chosen per class and storage type by
    :meth:`tune` (each candidate timed with CUDA events on the real system;
    the choice is kept in ``tiling``). Results do not depend on the tiling."""

    def __init__(self, plan, ret_problem: Tensor, nproblems: int, device):
        self.plan, self.P, self.device = plan, nproblems, torch.device(device)
        dr = self.dr = plan.dr
        ret_problem = ret_problem.to(torch.int64).cpu()
        if ret_problem.numel() and bool((ret_problem[1:] < ret_problem[:-1]).any()):
            raise ValueError("retained variables must be grouped by problem")
        counts = torch.bincount(ret_problem, minlength=nproblems)
        ret_ptr = torch.zeros(nproblems + 1, dtype=torch.int64)
        ret_ptr[1:] = torch.cumsum(counts, 0)
        n = counts * dr
        off = torch.zeros(nproblems, dtype=torch.int64)
        off[1:] = torch.cumsum(n * n, 0)[:-1]
        self.total = int((n * n).sum())
        t = lambda a, dt=torch.int32: a.to(device=self.device, dtype=dt).contiguous()  # noqa: E731
        self.ret_ptr, self.ret_problem, self.s_off = t(ret_ptr), t(ret_problem), t(off, torch.int64)
        self.diag = torch.empty((plan.r.count, dr, dr), dtype=torch.float64, device=self.device)
        self._S = {}
        # size classes: problems by descending n_p (ties by id), largest class first in the queue
        n_list = n.tolist()
        self.blocks = counts.tolist()
        order = sorted(range(nproblems), key=lambda p: (-n_list[p], p))
        self.classes, lo = [], -1
        for ub in _SIZE_CLASSES:
            members = [p for p in order if lo < n_list[p] <= ub]
            if members:
                self.classes.append((ub, members))
            lo = ub
        self.classes.sort(key=lambda c: -c[0])
        self.tiling = {}
        self._tasks = {}
        self.queue = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.x = torch.empty(plan.dim, dtype=torch.float64, device=self.device)
        self.iterations = torch.empty(nproblems, dtype=torch.int32, device=self.device)
        self.status = torch.empty(nproblems, dtype=torch.int32, device=self.device)

    def _feasible(self, members, k, sdtype) -> bool:
        need = L.lib().tls_batched_share_bytes(self.dr, int(max(self.blocks[p] for p in members)),
                                               L.dtype_code(sdtype), 0)
        return need <= (_SMEM_PER_CTA // k) & ~15

    def _task_arrays(self, groups_of_class: dict):
        key = tuple(sorted(groups_of_class.items()))
        if key not in self._tasks:
            order, first, size, groups = [], [], [], []
            for ub, members in self.classes:
                if ub not in groups_of_class:
                    continue
                k = groups_of_class[ub]
                base = len(order)
                order.extend(members)
                for s in range(0, len(members), k):
                    first.append(base + s)
                    size.append(min(k, len(members) - s))
                    groups.append(k)
            t = lambda a: torch.tensor(a, dtype=torch.int32, device=self.device)  # noqa: E731
            self._tasks[key] = (t(order), t(first), t(size), t(groups), len(first))
        return self._tasks[key]

    def _system_struct(self, sdtype) -> L.BatchedSystems:
        if sdtype not in self._S:
            self._S[sdtype] = torch.empty(max(self.total, 1), dtype=sdtype, device=self.device)
        b = L.BatchedSystems()
        b.nproblems, b.nretained, b.dr, b.sdtype = self.P, self.plan.r.count, self.dr, L.dtype_code(sdtype)
        b.ret_ptr, b.ret_problem, b.s_off = self.ret_ptr.data_ptr(), self.ret_problem.data_ptr(), self.s_off.data_ptr()
        b.S, b.diag = self._S[sdtype].data_ptr(), self.diag.data_ptr()
        return b

    def assemble(self, system, sdtype):
        """S_p of every problem from the damped one-group Schur system."""
        from .schur import _dense_pairs

        tr, tc, ptr, pa, pb = _dense_pairs(system.linear.layout)
        self._sys = self._system_struct(sdtype)
        L.call("tls_batched_schur_dense", C.byref(system.args), C.byref(self._sys), tr.numel(), tr.data_ptr(),
               tc.data_ptr(), ptr.data_ptr(), pa.data_ptr(), pb.data_ptr(), system.stream)

    def _run(self, rhs, rtol, atol, max_iterations, groups_of_class):
        order, first, size, groups, ntasks = self._task_arrays(groups_of_class)
        a = L.BatchedPcgArgs()
        a.rhs, a.x = rhs.data_ptr(), self.x.data_ptr()
        a.iterations, a.status = self.iterations.data_ptr(), self.status.data_ptr()
        a.order, a.task_first, a.task_size, a.task_groups = (order.data_ptr(), first.data_ptr(), size.data_ptr(),
                                                             groups.data_ptr())
        a.queue, a.err = self.queue.data_ptr(), self.err.data_ptr()
        a.rtol, a.atol, a.ntasks, a.max_iterations = float(rtol), float(atol), ntasks, int(max_iterations)
        a.smem_bytes = _SMEM_PER_CTA
        L.call("tls_batched_pcg", C.byref(self._sys), C.byref(a), L.stream_handle(self.device))

    def tune(self, rhs, sdtype, rtol, atol, max_iterations, reps: int = 2):
        """Choose problems per CTA for every size class by timing each feasible
        candidate on the assembled system (CUDA events, best of ``reps``)."""
        chosen, record = {}, {}
        for ub, members in self.classes:
            times = {}
            for k in _GROUP_CHOICES:
                if len(members) < k and k != 1 or not self._feasible(members, k, sdtype):
                    continue
                best = math.inf
                for _ in range(reps):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    self._run(rhs, rtol, atol, max_iterations, {ub: k})
                    e1.record()
                    e1.synchronize()
                    best = min(best, e0.elapsed_time(e1) * 1e3)
                times[k] = best
            if not times:
                raise ValueError(f"a batched problem of reduced dimension above {ub} does not fit a CTA")
            k = min(times, key=lambda c: (times[c], c))
            chosen[ub] = k
            label = f"n_p<={ub}" if ub < _SIZE_CLASSES[-1] else f"n_p>{_SIZE_CLASSES[-2]}"
            record[label] = {"problems": len(members), "problems_per_cta": k, "warps_per_problem": 8 // k,
                             "us_by_problems_per_cta": times}
        self.tiling[sdtype] = (chosen, record)

    def solve(self, system, rhs, sdtype, rtol, atol, max_iterations):
        """Assemble every S_p and run the batched PCG; returns (x, iterations,
        status) as device tensors (views of reused buffers)."""
        self.assemble(system, sdtype)
        rhs = rhs.to(torch.float64).contiguous()
        if sdtype not in self.tiling:
            self.tune(rhs, sdtype, rtol, atol, max_iterations)
        self._run(rhs, rtol, atol, max_iterations, self.tiling[sdtype][0])
        return self.x, self.iterations, self.status


class BatchedProblem:
    """Independent problems merged once (structure, segments and Schur plan
    are analysed here) and solved many times with :meth:`solve`."""

    def __init__(self, problems: Sequence[Problem], *, eliminate: str | None = "points"):
        from .schur import SchurPlan

        self.merged, self.var_problem, self.slices = merge_problems(problems)
        self.P = len(problems)
        self.eliminate = eliminate
        an, vals = self.merged._state(None)
        self.device = vals.device
        L.require_cuda(next(iter(vals._values.values())), "batched solve")
        self.initial = {k: v.clone() for k, v in self.merged.parameters.items()}
        layout = an.layout
        P, device = self.P, self.device
        # problem id per tangent entry and per factor (structure order)
        self.pid_t = torch.cat([self.var_problem[e.key].repeat_interleave(e.dim) for e in layout]).to(device)
        pid_f = []
        for plan in an.plans:
            for a in plan.cost.args:
                if isinstance(a, ParameterRef):
                    pid_f.append(self.var_problem[a.name][torch.as_tensor(a.id)])
                    break
        self.pid_f = torch.cat(pid_f).to(device)
        self.seg_t, self.seg_f = _Segments(self.pid_t, P, device), _Segments(self.pid_f, P, device)
        an.structure(device)
        self.plan = SchurPlan(an, eliminate, device) if eliminate is not None else None
        if self.plan is not None:
            if getattr(self.plan, "general", False):
                raise ValueError("batched solves eliminate one group next to one retained group")
            self.plan.chunks_for(torch.float32)
            self.plan.chunks_for(torch.float64)
            self.systems = BatchedSystems(self.plan, self.var_problem[self.plan.r.key], P, device)
        self.var_problem_dev = {k: v.to(device) for k, v in self.var_problem.items()}
        self.weights = [None if p.weights is None else p.weights.to(device=device, dtype=torch.float64).contiguous()
                        for p in an.plans]

    def reset(self):
        """Restore the initial values of every problem."""
        self.merged.parameters = {k: v.clone() for k, v in self.initial.items()}

    def solve(self, *, precision: str = "native", max_iterations: int = 20, lambda_initial: float = 1e-3,
              lambda_factor: float = 4.0, lambda_min: float = 1e-12, lambda_max: float = 1e12,
              step_quality_min: float = 1e-4, max_trials: int = 20, cost_tolerance: float = 1e-10,
              gradient_tolerance: float = 1e-8, pcg_rtol: float = 1e-6, pcg_max_iterations: int = 200):
        """LM over every problem from the current values (see the module
        docstring). Returns ``(solutions, summary)``: one dict of solved
        parameters per problem and a :class:`BatchedSummary` with per-problem
        costs, step counts and termination reasons ("gradient_tolerance",
        "cost_tolerance", "max_iterations", "trials_exhausted")."""
        from .schur import SchurLinearization
        from .solvers import BlockJacobiPreconditioner, ConjugateGradientConfig, DevicePCG

        merged, var_problem, slices, P = self.merged, self.var_problem, self.slices, self.P
        an, vals = merged._state(None)
        layout, device, n = an.layout, self.device, an.tangent_dim
        jdt = torch.float32 if precision == "mixed" else torch.float64
        pid_t, seg_t, seg_f = self.pid_t, self.seg_t, self.seg_f
        st = an.structure(device)
        plan = self.plan
        stream = L.stream_handle(device)
        cg = ConjugateGradientConfig(rtol=pcg_rtol, max_iterations=pcg_max_iterations, precision=precision)
        pcg_ws = None if plan is not None else DevicePCG(n, torch.float64, device)
        nf_total = sum(p.count for p in an.plans)
        obj_buf = torch.empty(nf_total, dtype=torch.float64, device=device)
        red_buf = torch.empty(nf_total, dtype=torch.float64, device=device)
        sq_buf = torch.empty(nf_total, dtype=torch.float64, device=device)

        def factor_sums(rows: Tensor) -> Tensor:
            """Per-factor sums of squares of factor-major rows [sum N_k r_k]."""
            rows = rows.to(torch.float64).contiguous()
            f0 = 0
            for k, p in enumerate(an.plans):
                R, N, rb = st.rdims[k], p.count, st.res_base[k]
                L.call("tls_factor_sqnorm", N, R, rows.data_ptr() + 8 * rb, sq_buf.data_ptr() + 8 * f0, stream)
                f0 += N
            return sq_buf

        def objective_terms(lin, new_raw):
            """Per-factor new objective 1/2 w rho(s_new) and exact reduction."""
            old_raw = (lin.raw_residual if an._has_loss else lin.residual).to(torch.float64).contiguous()
            new_raw = new_raw.to(torch.float64).contiguous()
            f0 = 0
            for k, p in enumerate(an.plans):
                R, N, rb = st.rdims[k], p.count, st.res_base[k]
                loss, w = p.cost.loss, self.weights[k]
                if loss is None or isinstance(loss, HuberLoss):
                    L.call("tls_factor_terms", N, R, old_raw.data_ptr() + 8 * rb, new_raw.data_ptr() + 8 * rb,
                           0 if loss is None else 1, 0.0 if loss is None else float(loss.delta), L.ptr(w),
                           obj_buf.data_ptr() + 8 * f0, red_buf.data_ptr() + 8 * f0, stream)
                else:
                    ro, rn = old_raw[rb : rb + N * R].view(N, R), new_raw[rb : rb + N * R].view(N, R)
                    obj, red = _user_loss_terms(loss, (ro * ro).sum(-1), (rn * rn).sum(-1))
                    if w is not None:
                        obj, red = w * obj, w * red
                    obj_buf[f0 : f0 + N] = 0.5 * obj
                    red_buf[f0 : f0 + N] = 0.5 * red
                f0 += N
            return obj_buf, red_buf

        def masked(values: NamedValues, proposed: NamedValues, accept: Tensor) -> NamedValues:
            out = {}
            for e in layout:
                a = accept[self.var_problem_dev[e.key]]
                a = a.view(-1, *([1] * (proposed._values[e.key].ndim - 1)))
                out[e.key] = torch.where(a, proposed._values[e.key], values._values[e.key])
            return NamedValues(out, layout)

        lam = torch.full((P,), float(lambda_initial), dtype=torch.float64, device=device)
        active = torch.ones(P, dtype=torch.bool, device=device)
        pending = torch.zeros(P, dtype=torch.bool, device=device)
        tried = torch.zeros(P, dtype=torch.bool, device=device)
        ok = torch.zeros(P, dtype=torch.bool, device=device)
        reason = torch.full((P,), L.BATCH_MAX_ITERATIONS, dtype=torch.int32, device=device)
        accepted = torch.zeros(P, dtype=torch.int64, device=device)
        rejected = torch.zeros(P, dtype=torch.int64, device=device)
        summary = BatchedSummary(problems=P)
        lm = L.BatchedLm()
        lm.nproblems = P
        lm.lambda_factor, lm.lambda_min, lm.lambda_max = float(lambda_factor), float(lambda_min), float(lambda_max)
        lm.step_quality_min, lm.cost_tolerance = float(step_quality_min), float(cost_tolerance)
        lm.lam, lm.tried, lm.ok, lm.active, lm.pending = (lam.data_ptr(), tried.data_ptr(), ok.data_ptr(),
                                                          active.data_ptr(), pending.data_ptr())
        lm.accepted, lm.rejected, lm.reason = accepted.data_ptr(), rejected.data_ptr(), reason.data_ptr()

        lin = merged.linearize(dict(vals._values), jacobian_dtype=jdt, schur=plan)
        first_obj, _ = objective_terms(lin, lin.raw_residual if an._has_loss else lin.residual)
        cost = seg_f.sum(first_obj)
        lm.cost = cost.data_ptr()
        summary.initial_cost = cost.clone()
        for it in range(max_iterations):
            g = lin.gradient
            gmax = torch.zeros(P, dtype=torch.float64, device=device).scatter_reduce(0, pid_t, g.abs(), "amax")
            done_g = active & (gmax <= gradient_tolerance)
            reason.masked_fill_(done_g, L.BATCH_GRADIENT_TOLERANCE)
            active &= ~done_g
            if not bool(active.any()):
                break
            summary.iterations += 1
            raw_diag = lin.jacobian.diagonal_blocks()
            pending.copy_(active)
            any_accept = torch.zeros((), dtype=torch.bool, device=device)
            # cross blocks once per linearization; each trial sets its column scale
            slin = (SchurLinearization(plan, lin, raw_diag, None, wdtype=jdt, vec_dtype=torch.float64)
                    if plan is not None else None)
            for _ in range(max_trials):
                if not bool(pending.any()):
                    break
                s = (1.0 / lam.sqrt())[pid_t]
                mask = pending[pid_t].to(torch.float64)
                tried.copy_(pending)
                if plan is not None:
                    slin.scale = s.contiguous()
                    system = slin.damped(1.0)
                    rhs = system.reduced_rhs(-(g * s) * mask)
                    xc, its, status = self.systems.solve(system, rhs, jdt, pcg_rtol, 1e-10, pcg_max_iterations)
                    # a preconditioner block that is not positive definite rejects its
                    # problem's trial (lambda_p grows; x_p = 0)
                    badp = (status == 1) & pending
                    lam.copy_(torch.where(badp, (lam * lambda_factor).clamp_max(lambda_max), lam))
                    rejected += badp.to(torch.int64)
                    mask = mask * (~badp)[pid_t].to(torch.float64)
                    tried &= ~badp
                    delta = s * system.backsubstitute(xc)
                    flags = torch.stack((plan.err.to(torch.int64).reshape(()), self.systems.err.to(torch.int64)
                                         .reshape(()), its.max().to(torch.int64))).tolist()
                    if flags[0] != 0:
                        raise RuntimeError("Schur matvec: a bounded device wait timed out")
                    if flags[1] != 0:
                        raise RuntimeError("batched PCG: a problem did not fit its shared-memory share")
                    n_its = int(flags[2])
                else:
                    from .solvers import _layout_specs

                    scaled = lin.jacobian.scale_columns(s)
                    pre = BlockJacobiPreconditioner.from_blocks(_layout_specs(layout, raw_diag), 1.0, s, n)
                    res = pcg_ws.run(-(g * s) * mask, cg, normal_args=scaled.normal_args(torch.float64, 1.0),
                                     preconditioner=pre)
                    delta = s * res.solution.to(torch.float64)
                    n_its = int(res.iterations)
                summary.linear_solves += 1
                summary.linear_iterations += n_its
                delta = delta * mask
                proposed = vals.retract(delta, layout)
                new_raw = an.residuals(proposed)
                obj_new, red = objective_terms(lin, new_raw)
                actual = seg_f.sum(red)
                jd = lin.jacobian.matvec(delta)
                predicted = -seg_t.sum(g * delta) - 0.5 * seg_f.sum(factor_sums(jd))
                new_cost = seg_f.sum(obj_new)
                lm.actual, lm.predicted, lm.new_cost = actual.data_ptr(), predicted.data_ptr(), new_cost.data_ptr()
                L.call("tls_batched_lm_update", C.byref(lm), stream)
                vals = masked(vals, proposed, ok)
                any_accept |= ok.any()
            reason.masked_fill_(pending, L.BATCH_TRIALS_EXHAUSTED)
            active &= ~pending
            if bool(any_accept):
                lin = merged.linearize(dict(vals._values), jacobian_dtype=jdt, schur=plan)
        summary.final_cost = cost
        summary.accepted_steps = accepted
        summary.rejected_steps = rejected
        names = {L.BATCH_MAX_ITERATIONS: "max_iterations", L.BATCH_GRADIENT_TOLERANCE: "gradient_tolerance",
                 L.BATCH_COST_TOLERANCE: "cost_tolerance", L.BATCH_TRIALS_EXHAUSTED: "trials_exhausted"}
        summary.termination = [names[c] for c in reason.tolist()]
        merged.parameters.update(dict(vals._values))
        sols = [{k: vals._values[k][sl[k]] for k in vals._values} for sl in slices]
        return sols, summary


def solve_batched(problems: Sequence[Problem], *, eliminate: str | None = "points", **options):
    """Merge ``problems`` (see :class:`BatchedProblem`) and solve them once."""
    return BatchedProblem(problems, eliminate=eliminate).solve(**options)


def partition_problems(work: Sequence[float], parts: int) -> list[list[int]]:
    """Split problems across ``parts`` GPUs by estimated work (for example
    observations x iterations): longest-processing-time first, each problem to
    the currently lightest part; ties go to the lowest part index, so every
    rank computes the same partition. Problems solve independently, so the
    only exchange is gathering the solutions at the end."""
    if parts < 1:
        raise ValueError("parts must be positive")
    order = sorted(range(len(work)), key=lambda j: (-float(work[j]), j))
    load = [0.0] * parts
    out = [[] for _ in range(parts)]
    for j in order:
        k = min(range(parts), key=lambda i: (load[i], i))
        out[k].append(j)
        load[k] += float(work[j])
    return [sorted(o) for o in out]
