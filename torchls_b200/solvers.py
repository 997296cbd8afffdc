"""Configs, PCG, block-Jacobi and the LM / GN driver on the GPU.

Interface of torchls ``solvers.py``: ``ConjugateGradientConfig``,
``TrustRegionConfig``, ``TerminationConfig``, ``PCGResult``, ``SolveSummary``,
``pcg``, ``block_jacobi`` and ``solve`` keep their fields, defaults, reason
strings and validation (solvers.py:19-164). The backend is ``"cuda"``: every
linear-algebra step runs in this package's kernels; there is no CPU path.
``precision="mixed"`` stores Jacobians and Schur W blocks in float32 (half
the bytes of every matvec) while PCG vectors, gradients, costs, dot
products, gain ratios and small-block factorizations stay float64; the outer
LM iterations refine the float32-operator inner solves.
"""

from __future__ import annotations

import ctypes as C
import itertools
import math
import time
from collections.abc import Callable
from contextlib import contextmanager
from dataclasses import dataclass, field
from functools import partial

import torch
from torch import Tensor

from . import _lib as L
from . import dense
from .bounds import BoundsPlan
from .kernels import ordered_index_add_, reduce
from .schur import DampedSchurSystem, SchurLinearization, SchurPlan
from .sparse import BlockJacobian

# Backend names a ConjugateGradientConfig accepts: this package's "cuda" and
# the reference's "torch" and "warp" (solvers.py:49-52), so that configs written
# for torchls construct unchanged. All three run this package's CUDA kernels:
# there is one implementation here, and it computes what the reference's
# backends compute (same algorithm, same stopping rules, results within the
# tolerances the parity tests state).
_BACKENDS = ("cuda", "torch", "warp")

# Keys that let one PCG solve's repeated tls_pcg_run calls launch the CUDA
# graph recorded by its first call (a new key per solve).
_GRAPH_KEYS = itertools.count(1)


def normalize_groups(groups):
    """preconditioning.py:20-36."""
    from .variables import Var

    if not isinstance(groups, (tuple, list)):
        raise ValueError("preconditioner_groups must be a sequence of groups")
    out, seen = [], set()
    for group in groups:
        if not isinstance(group, (tuple, list)) or len(group) < 2:
            raise ValueError("Each joint preconditioner group needs at least two variable keys")
        for key in group:
            if not ((isinstance(key, str) and key) or (isinstance(key, type) and issubclass(key, Var))):
                raise ValueError("Preconditioner keys must be parameter names or Var types")
            if key in seen:
                raise ValueError("A variable may occur in only one preconditioner group")
            seen.add(key)
        out.append(tuple(group))
    return tuple(out)


@dataclass(frozen=True)
class ConjugateGradientConfig:
    rtol: float = 1e-6
    atol: float = 1e-10
    max_iterations: int = 200
    preconditioner: str | None = "block_jacobi"
    preconditioner_groups: tuple[tuple, ...] = ()
    residual_check_interval: int = 50
    restart_strategy: str = "adaptive"
    residual_drift_tolerance: float = 0.1
    backend: str = "cuda"
    normal_matvec: str = "cuda"
    normal_max_packed_bytes: int = 256 * 1024**2
    # Operator applications between host status reads of the device PCG.
    graph_batch_iterations: int = 16
    cache_retained_matrix: bool = False
    # "native": Jacobian and Schur W stored in the parameter dtype;
    # "mixed": float32 Jacobian / Schur W storage, float64 vectors and reductions.
    precision: str = "native"

    def __post_init__(self):
        if (isinstance(self.normal_max_packed_bytes, bool) or not isinstance(self.normal_max_packed_bytes, int)
                or self.normal_max_packed_bytes < 0):
            raise ValueError("normal_max_packed_bytes must be a nonnegative integer")
        if (isinstance(self.graph_batch_iterations, bool) or not isinstance(self.graph_batch_iterations, int)
                or self.graph_batch_iterations < 1):
            raise ValueError("graph_batch_iterations must be a positive integer")
        if self.normal_matvec not in _BACKENDS:
            raise ValueError("normal_matvec must be cuda, torch or warp (all run the CUDA kernels)")
        if self.backend not in _BACKENDS:
            raise ValueError("CG backend must be cuda, torch or warp (all run the CUDA kernels)")
        if self.rtol < 0 or self.atol < 0 or self.max_iterations < 1:
            raise ValueError("Invalid CG tolerance or iteration limit")
        if self.preconditioner not in ("block_jacobi", None):
            raise ValueError("preconditioner must be block_jacobi or None")
        object.__setattr__(self, "preconditioner_groups", normalize_groups(self.preconditioner_groups))
        if self.preconditioner_groups and self.preconditioner is None:
            raise ValueError("Joint groups require block_jacobi preconditioning")
        if (isinstance(self.residual_check_interval, bool) or not isinstance(self.residual_check_interval, int)
                or self.residual_check_interval < 0):
            raise ValueError("residual_check_interval must be a nonnegative integer")
        if self.restart_strategy not in ("adaptive", "periodic"):
            raise ValueError("restart_strategy must be adaptive or periodic")
        if not math.isfinite(self.residual_drift_tolerance) or self.residual_drift_tolerance <= 0:
            raise ValueError("residual_drift_tolerance must be finite and positive")
        if self.precision not in ("native", "mixed"):
            raise ValueError("precision must be native or mixed")


@dataclass(frozen=True)
class TrustRegionConfig:
    lambda_initial: float = 1e-3
    lambda_min: float = 1e-12
    lambda_max: float = 1e12
    lambda_factor: float = 4.0
    step_quality_min: float = 1e-4
    max_trials: int = 20
    strategy: str = "fixed_factor"
    damping_mode: str = "identity"
    diagonal_min: float = 1e-6
    diagonal_max: float = 1e32

    def __post_init__(self):
        if not (0 < self.lambda_min <= self.lambda_initial <= self.lambda_max):
            raise ValueError("Require 0 < lambda_min <= lambda_initial <= lambda_max")
        if self.lambda_factor <= 1 or self.max_trials < 1 or not (0 <= self.step_quality_min < 1):
            raise ValueError("Invalid trust region settings")
        if self.strategy not in ("fixed_factor", "adaptive"):
            raise ValueError("Trust region strategy must be fixed_factor or adaptive")
        if self.damping_mode not in ("identity", "diagonal"):
            raise ValueError("damping_mode must be identity or diagonal")
        if not (0 < self.diagonal_min <= self.diagonal_max < math.inf):
            raise ValueError("Require finite positive diagonal damping bounds")


@dataclass(frozen=True)
class TerminationConfig:
    max_iterations: int = 50
    cost_tolerance: float = 1e-10
    gradient_tolerance: float = 1e-8
    parameter_tolerance: float = 1e-10
    target_cost: float | None = None
    max_time_seconds: float | None = None

    def __post_init__(self):
        if self.max_iterations < 1 or min(self.cost_tolerance, self.gradient_tolerance,
                                           self.parameter_tolerance) < 0:
            raise ValueError("Invalid termination settings")
        if self.target_cost is not None and (not math.isfinite(self.target_cost) or self.target_cost < 0):
            raise ValueError("target_cost must be finite and nonnegative")
        if self.max_time_seconds is not None and (
            not math.isfinite(self.max_time_seconds) or self.max_time_seconds <= 0
        ):
            raise ValueError("max_time_seconds must be finite and positive")


_DEFAULT_CG = ConjugateGradientConfig()
_DEFAULT_TRUST_REGION = TrustRegionConfig()
_DEFAULT_TERMINATION = TerminationConfig()


@dataclass(frozen=True)
class PCGResult:
    solution: Tensor
    iterations: int
    residual_norm: float
    converged: bool
    reason: str
    restarts: int = 0
    residual_checks: int = 0
    rhs_norm: float = 0.0


@dataclass
class SolveSummary:
    """Histories include the initial point and each accepted update."""

    initial_cost: float
    final_cost: float
    iterations: int = 0
    accepted_steps: int = 0
    rejected_steps: int = 0
    linear_iterations: int = 0
    termination_reason: str = "max_iterations"
    gradient_norm: float = math.inf
    cost_history: list[float] = field(default_factory=list)
    lambda_history: list[float] = field(default_factory=list)
    linear_iterations_history: list[int] = field(default_factory=list)
    linear_converged_history: list[bool] = field(default_factory=list)
    trial_history: list[dict] = field(default_factory=list)
    linear_solver: str = "conjugate_gradient"
    jacobi_scaling: bool = False
    reduced_dim: int | None = None
    linear_restarts: int = 0
    linear_residual_checks: int = 0
    linear_relative_residual_history: list[float | None] = field(default_factory=list)


# ============================================================================ block Jacobi
class BlockJacobiPreconditioner:
    """Damped block Cholesky factors and their apply, z = (L L^T)^-1 r per block
    (solvers.py:259-285, preconditioning.py:117-134). Factors are float64."""

    def __init__(self, groups, keep, n):
        self.groups = groups
        self._keep = keep
        self.n = n
        self._array = (L.BlockGroup * max(len(groups), 1))(*groups)

    @classmethod
    def from_blocks(cls, specs, damping, scale, n, check: bool = True):
        """specs: [(blocks [count,dim,dim] f64, [(offset, dim), ...] members, count, dim)].

        ``check=False`` skips the host read of the non-positive-definite count;
        the device word is kept as ``bad_word`` for the caller to read later
        (``DevicePCG.run`` reads it with the PCG control block)."""
        if len(specs) > L.MAX_GROUPS:
            raise ValueError("too many preconditioner groups")
        groups, keep = [], []
        device = specs[0][0].device
        sc = None if scale is None else scale.to(torch.float64).contiguous()
        for blocks, members, count, dim in specs:
            if dim > 16:
                raise ValueError("preconditioner blocks larger than 16 are not supported")
            blocks = blocks.to(torch.float64).contiguous()
            factor = torch.empty_like(blocks)
            g = L.BlockGroup()
            g.count, g.dim, g.nmembers = count, dim, len(members)
            for m, (off, d) in enumerate(members):
                g.member_offset[m] = off
                g.member_dim[m] = d
            g.blocks, g.factor = blocks.data_ptr(), factor.data_ptr()
            g.scale = None if sc is None else sc.data_ptr()
            groups.append(g)
            keep += [blocks, factor]
        keep.append(sc)
        pre = cls(groups, keep, n)
        bad = torch.zeros(1, dtype=torch.int32, device=device)
        L.call("tls_block_cholesky", pre._array, len(groups), float(damping), bad.data_ptr(),
               L.stream_handle(device))
        pre.bad_word = bad
        if check and int(bad.item()) > 0:
            raise torch.linalg.LinAlgError("damped block is not positive definite")
        return pre

    def __call__(self, vector: Tensor) -> Tensor:
        v = vector.contiguous()
        out = torch.empty_like(v)
        L.call("tls_block_solve", self._array, len(self.groups), v.data_ptr(), out.data_ptr(),
               L.dtype_code(v.dtype), L.stream_handle(v.device))
        return out


def _layout_specs(layout, diagonal):
    return [(d, [(e.offset, e.dim)], e.count, e.dim) for e, d in zip(layout, diagonal)]


def _joint_specs(layout, groups, jacobian: BlockJacobian, diagonal):
    """Joint blocks with cross terms between member groups (preconditioning.py:47-115)."""
    lookup = {e.key: i for i, e in enumerate(layout)}
    grouped, chosen = [], set()
    for grp in groups:
        if any(k not in lookup for k in grp):
            raise ValueError("Unknown preconditioner key (Schur groups must be retained variables)")
        members = tuple(lookup[k] for k in grp)
        first = layout[members[0]]
        if any(not torch.equal(first.ids.cpu(), layout[i].ids.cpu()) for i in members[1:]):
            raise ValueError("Joint preconditioner groups require identical IDs in identical order")
        grouped.append(members)
        chosen.update(members)
    grouped.extend((i,) for i in range(len(layout)) if i not in chosen)
    where, specs = {}, []
    for b, members in enumerate(grouped):
        off = 0
        for i in members:
            where[i] = (b, off)
            off += layout[i].dim
        count = layout[members[0]].count
        blk = torch.zeros((count, off, off), dtype=torch.float64, device=jacobian.device)
        for i in members:
            o = where[i][1]
            blk[:, o : o + layout[i].dim, o : o + layout[i].dim] = diagonal[i]
        specs.append([blk, [(layout[i].offset, layout[i].dim) for i in members], count, off])
    for g in jacobian.groups:
        for p, i in enumerate(g.type_indices):
            bi, a = where[i]
            for q in range(p):
                j = g.type_indices[q]
                bj, c = where[j]
                if bi == bj and i != j:
                    mask = (g.variable_indices[p] == g.variable_indices[q]).to(torch.float64)
                    cross = (g.blocks[p].double().transpose(-1, -2) @ g.blocks[q].double()) * mask[:, None, None]
                    da, db = cross.shape[-2:]
                    rows = g.variable_indices[p]
                    ordered_index_add_(specs[bi][0][:, a : a + da, c : c + db], rows, cross)
                    ordered_index_add_(specs[bi][0][:, c : c + db, a : a + da], rows, cross.transpose(-1, -2))
    return [tuple(s) for s in specs]


def block_jacobi(jacobian: BlockJacobian, damping: float, *, diagonal=None, groups=(), graph_safe=False):
    """Factor damped variable diagonal blocks without building J^T J (solvers.py:259-285)."""
    diagonal = jacobian.diagonal_blocks() if diagonal is None else diagonal
    specs = (_joint_specs(jacobian.layout, normalize_groups(groups), jacobian, diagonal) if groups
             else _layout_specs(jacobian.layout, diagonal))
    return BlockJacobiPreconditioner.from_blocks(specs, damping, None, jacobian.shape[1])


# ============================================================================ PCG
_REASONS = {L.PCG_CONVERGED: "residual_tolerance", L.PCG_NONFINITE: "nonfinite",
            L.PCG_NONPOSITIVE: "nonpositive_curvature", L.PCG_MAX_ITERATIONS: "max_iterations"}


class NormalOperator:
    """x -> diag(s) J^T J diag(s) x + damping x, runnable by the device PCG."""

    def __init__(self, jacobian: BlockJacobian, damping: float):
        self.jacobian, self.damping = jacobian, float(damping)

    def __call__(self, v):
        return self.jacobian.normal_matvec(v, self.damping)


class DevicePCG:
    """Workspace and driver for the device-resident PCG state machine."""

    def __init__(self, n, dtype, device):
        self.n, self.dtype, self.device = n, dtype, device
        mk = lambda: torch.empty(n, dtype=dtype, device=device)
        self.x, self.r, self.z, self.p, self.ap, self.ztrue, self.psave = (mk() for _ in range(7))
        self.partials = torch.empty(L.PCG_PARTIALS, dtype=torch.float64, device=device)
        nbytes = L.lib().tls_pcg_state_bytes()
        self.control = torch.zeros(nbytes, dtype=torch.uint8, device=device)
        self.host = torch.empty(C.sizeof(L.PcgControl), dtype=torch.uint8, pin_memory=True)
        self.words_host = torch.zeros(8, dtype=torch.int32, pin_memory=True)
        self.extra_host = torch.zeros(16, dtype=torch.float64, pin_memory=True)
        self._pending = None

    def run(self, rhs: Tensor, config: ConjugateGradientConfig, *, normal_args=None, schur_args=None,
            preconditioner: BlockJacobiPreconditioner | None = None, error_word: Tensor | None = None,
            bad_words=(), defer: bool = False) -> PCGResult | None:
        """``error_word``: the operator's device error flag (the Schur kernels'
        bounded bulk-copy and grid-barrier waits set it instead of hanging);
        ``bad_words``: device counts of blocks that were not positive definite
        when the operator or preconditioner was factored (raised as
        ``LinAlgError``). All are read with the last control-block read, so
        they cost no extra host synchronisation. ``defer=True`` returns right
        after the launch; :meth:`finish` completes the call."""
        a = L.PcgArgs()
        a.n = self.n
        a.vec_dtype = L.dtype_code(self.dtype)
        keep = []
        if normal_args is not None:
            a.op_kind = 0
            keep.append(normal_args)
            a.normal = C.pointer(normal_args)
        elif isinstance(schur_args, L.SchurGeneralArgs):
            a.op_kind = 2
            keep.append(schur_args)
            a.schur_general = C.addressof(schur_args)
        else:
            a.op_kind = 1
            keep.append(schur_args)
            a.schur = C.pointer(schur_args)
        if preconditioner is not None:
            a.pre = C.cast(preconditioner._array, C.POINTER(L.BlockGroup))
            a.npre = len(preconditioner.groups)
        rhs = rhs.to(self.dtype).contiguous()
        a.rhs = rhs.data_ptr()
        for name in ("x", "r", "z", "p", "ap", "ztrue", "psave"):
            setattr(a, name, getattr(self, name).data_ptr())
        a.partials = self.partials.data_ptr()
        a.control = self.control.data_ptr()
        a.graph_key = next(_GRAPH_KEYS)
        stream = L.stream_handle(self.device)
        L.call("tls_pcg_start", C.byref(a), float(config.rtol), float(config.atol), int(config.max_iterations),
               int(config.residual_check_interval), int(config.restart_strategy == "periodic"),
               float(config.residual_drift_tolerance), stream)
        words = ([error_word] if error_word is not None else []) + [w for w in bad_words if w is not None]
        batch = config.graph_batch_iterations
        if schur_args is not None:
            # small Schur systems run the whole loop in one persistent launch;
            # otherwise the library queues at most 16 steps per call
            batch = max(batch, 4 * int(config.max_iterations) + 16)
        # steps after termination are no-ops, so run first and read after
        L.call("tls_pcg_run", C.byref(a), batch, stream)
        self._pending = dict(a=a, keep=(keep, rhs), words=words, error_word=error_word, batch=batch, stream=stream)
        if defer:
            return None
        return self.finish()[0]

    def finish(self, extra: Tensor | None = None):
        """Wait for the PCG launched by ``run(..., defer=True)``; ``extra`` (a
        small float64 device tensor computed from the solution in stream order)
        is read in the same host synchronisation. Returns ``(PCGResult,
        extra_values)``; ``extra_values`` is None when the loop needed further
        host-driven steps (then ``extra`` was computed from an unfinished x)."""
        pend, self._pending = self._pending, None
        a, words, error_word = pend["a"], pend["words"], pend["error_word"]
        extra_vals = None
        first = True
        while True:
            ctrl, flags, ev = self._read(words, extra if first else None)
            if first:
                extra_vals = ev
            # a wait that ran out left the loop where it was: stop here, not
            # after further launches
            if error_word is not None and flags[0] != 0:
                raise RuntimeError("Schur PCG: a bounded device wait (bulk copy or grid barrier) timed out")
            if ctrl.status != L.PCG_ACTIVE:
                break
            first = False
            extra_vals = None
            L.call("tls_pcg_run", C.byref(a), pend["batch"], pend["stream"])
        if any(f > 0 for f in flags[1 if error_word is not None else 0 :]):
            raise torch.linalg.LinAlgError("damped block is not positive definite")
        res = PCGResult(self.x.clone(), int(ctrl.iterations), float(ctrl.residual_norm),
                        ctrl.status == L.PCG_CONVERGED, _REASONS[ctrl.status], int(ctrl.restarts),
                        int(ctrl.checks), float(ctrl.rhs_norm))
        return res, extra_vals

    def _read(self, words=(), extra: Tensor | None = None):
        for k, w in enumerate(words):
            self.words_host[k : k + 1].copy_(w.view(-1)[:1].to(torch.int32), non_blocking=True)
        ne = 0
        if extra is not None:
            ne = extra.numel()
            self.extra_host[:ne].copy_(extra.reshape(-1).to(torch.float64), non_blocking=True)
        self.host.copy_(self.control[: self.host.numel()], non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        flags = self.words_host[: len(words)].tolist()
        ev = self.extra_host[:ne].tolist() if extra is not None else None
        return L.PcgControl.from_buffer_copy(self.host.numpy().tobytes()), flags, ev


def _generic_pcg(matvec, rhs, preconditioner, config):
    """PCG for arbitrary torch callables, step for step as solvers.py:188-256."""
    apply = (lambda v: v) if preconditioner is None else preconditioner
    x = torch.zeros_like(rhs)
    residual = rhs.clone()
    rhs_norm = float(torch.linalg.vector_norm(rhs))
    thr = max(config.atol, config.rtol * rhs_norm)
    if not math.isfinite(rhs_norm):
        return PCGResult(x, 0, rhs_norm, False, "nonfinite", rhs_norm=rhs_norm)
    if rhs_norm <= thr:
        return PCGResult(x, 0, rhs_norm, True, "residual_tolerance", rhs_norm=rhs_norm)
    z = apply(residual)
    rz = torch.dot(residual, z)
    direction = z.clone()
    it = restarts = checks = 0
    reason = "max_iterations"
    for it in range(1, config.max_iterations + 1):
        product = matvec(direction)
        curv = torch.dot(direction, product)
        if not bool(torch.isfinite(curv) & torch.isfinite(rz)):
            reason = "nonfinite"
            break
        if float(curv) <= 0 or float(rz) <= 0:
            reason = "nonpositive_curvature"
            break
        alpha = rz / curv
        x = x + alpha * direction
        residual = residual - alpha * product
        rec = float(torch.linalg.vector_norm(residual))
        periodic = config.residual_check_interval > 0 and it % config.residual_check_interval == 0
        if rec <= thr or periodic:
            tr = rhs - matvec(x)
            checks += 1
            tn = float(torch.linalg.vector_norm(tr))
            if not math.isfinite(tn):
                return PCGResult(x, it, tn, False, "nonfinite", restarts, checks, rhs_norm)
            if tn <= thr:
                return PCGResult(x, it, tn, True, "residual_tolerance", restarts, checks, rhs_norm)
            drift = float(torch.linalg.vector_norm(tr - residual))
            if rec <= thr or config.restart_strategy == "periodic" or drift > (
                    config.residual_drift_tolerance * max(tn, thr)):
                residual = tr
                z = apply(residual)
                rz = torch.dot(residual, z)
                direction = z.clone()
                restarts += 1
                continue
        z = apply(residual)
        rz_new = torch.dot(residual, z)
        direction = z + (rz_new / rz) * direction
        rz = rz_new
    tn = float(torch.linalg.vector_norm(rhs - matvec(x)))
    checks += 1
    conv = math.isfinite(tn) and tn <= thr
    if conv:
        reason = "residual_tolerance"
    elif not math.isfinite(tn):
        reason = "nonfinite"
    return PCGResult(x, it, tn, conv, reason, restarts, checks, rhs_norm)


def pcg(matvec: Callable[[Tensor], Tensor], rhs: Tensor, *, preconditioner=None,
        config: ConjugateGradientConfig = _DEFAULT_CG) -> PCGResult:
    """Preconditioned CG with true-residual checks (solvers.py:167-256).

    When ``matvec`` is this package's normal operator (``NormalOperator``,
    ``partial(BlockJacobian.normal_matvec, damping=...)``) or a damped Schur
    system's ``matvec``, and the preconditioner is a block-Jacobi from this
    package (or None), the whole iteration runs in the device state machine.
    Other torch callables run the same algorithm step by step.
    """
    if rhs.ndim != 1 or rhs.numel() == 0:
        raise ValueError("PCG expects a nonempty vector")
    L.require_cuda(rhs, "CUDA PCG")
    if rhs.dtype not in (torch.float32, torch.float64):
        raise ValueError("CUDA PCG requires float32 or float64 tensors")
    pre_ok = preconditioner is None or isinstance(preconditioner, BlockJacobiPreconditioner)
    op = _operator_of(matvec)
    if op is not None and pre_ok:
        kind, obj, damping, tiles = op
        if kind == "normal":
            ws = DevicePCG(rhs.numel(), rhs.dtype, rhs.device)
            return ws.run(rhs, config, normal_args=obj.normal_args(rhs.dtype, damping, tiles=tiles),
                          preconditioner=preconditioner)
        if kind == "schur" and rhs.dtype == torch.float64:
            ws = DevicePCG(rhs.numel(), rhs.dtype, rhs.device)
            return ws.run(rhs, config, schur_args=obj.args, preconditioner=preconditioner, error_word=obj.plan.err)
    return _generic_pcg(matvec, rhs, preconditioner, config)


def _operator_of(matvec):
    if isinstance(matvec, NormalOperator):
        return "normal", matvec.jacobian, matvec.damping, True
    if isinstance(matvec, partial) and getattr(matvec.func, "__func__", None) is BlockJacobian.normal_matvec:
        kw = matvec.keywords
        return "normal", matvec.func.__self__, float(kw.get("damping", 0.0)), bool(kw.get("tiles", True))
    self_ = getattr(matvec, "__self__", None)
    if isinstance(self_, BlockJacobian) and getattr(matvec, "__func__", None) is BlockJacobian.normal_matvec:
        return "normal", self_, 0.0, True
    if isinstance(self_, DampedSchurSystem) and getattr(matvec, "__func__", None) is DampedSchurSystem.matvec:
        return "schur", self_, self_.damping, True
    from .schur_general import GeneralDampedSchurSystem

    if (isinstance(self_, GeneralDampedSchurSystem)
            and getattr(matvec, "__func__", None) is GeneralDampedSchurSystem.matvec):
        return "schur", self_, self_.damping, True
    return None


# ============================================================================ LM / GN
@contextmanager
def _region(name, enabled):
    if not enabled:
        yield
        return
    torch.cuda.nvtx.range_push("torchls/" + name)
    try:
        with torch.profiler.record_function("torchls/" + name):
            yield
    finally:
        torch.cuda.nvtx.range_pop()


def _finite(*tensors) -> bool:
    vals = torch.stack([reduce(t, 2) for t in tensors])
    return bool(torch.isfinite(vals).all())


@torch.no_grad()
def solve(problem, initial_vals, *, linear_solver: str = "conjugate_gradient",
          conjugate_gradient: ConjugateGradientConfig = _DEFAULT_CG,
          trust_region: TrustRegionConfig | None = _DEFAULT_TRUST_REGION,
          termination: TerminationConfig = _DEFAULT_TERMINATION, return_summary: bool = False,
          jacobi_scaling: bool = False, eliminate=None, profile: bool = False, record_trials: bool = False,
          bounds=None, normal_blocks_backend: str = "auto"):
    """Optimize with LM (or GN when trust_region=None) on the GPU (solvers.py:288-696)."""
    if linear_solver not in ("conjugate_gradient", "dense_qr", "schur_dense", "schur_cg"):
        raise ValueError("Unknown linear solver")
    if normal_blocks_backend not in ("auto", *_BACKENDS):
        raise ValueError("normal_blocks_backend must be auto, cuda, torch or warp")
    cg = conjugate_gradient
    is_schur = linear_solver.startswith("schur_")
    if eliminate is not None and not is_schur:
        raise ValueError("eliminate requires a Schur linear solver")
    if cg.preconditioner_groups and linear_solver not in ("conjugate_gradient", "schur_cg"):
        raise ValueError("Joint preconditioner groups require a CG linear solver")
    start_time = time.perf_counter()

    def timed_out():
        return termination.max_time_seconds is not None and (
            time.perf_counter() - start_time >= termination.max_time_seconds)

    vals = initial_vals.detach()
    device = vals.device
    if device.type != "cuda":
        raise ValueError("the CUDA backend requires parameters on a CUDA device")
    mixed = cg.precision == "mixed" or vals.dtype == torch.float32
    # Storage precision of J and Schur W; PCG vectors and every reduction stay
    # float64 so the inner solve converges to the same tolerance either way.
    jdt = torch.float32 if mixed else torch.float64
    vdt = torch.float64
    bplan = BoundsPlan(bounds, problem.layout, vals) if bounds is not None else None
    if bplan is not None and bplan.groups and trust_region is None:
        raise ValueError("Bounds require a trust-region LM solve")
    initial_cost = float(problem.cost(vals))
    if not math.isfinite(initial_cost):
        raise ValueError("Initial residuals are nonfinite")
    summary = SolveSummary(initial_cost, initial_cost, cost_history=[initial_cost], linear_solver=linear_solver,
                           jacobi_scaling=jacobi_scaling)
    damping = trust_region.lambda_initial if trust_region else 0.0
    rejection_factor = 2.0
    with _region("analyze_schur", profile):
        schur_plan = None
        if is_schur:
            # symbolic Schur structure is cached on the analysed problem
            cache = problem.__dict__.setdefault("_schur_plans", {})
            key = (eliminate, device, tuple(cg.preconditioner_groups))
            if key not in cache:
                cache[key] = SchurPlan(problem, eliminate, device, preconditioner_groups=cg.preconditioner_groups)
            schur_plan = cache[key]
    if linear_solver == "schur_dense" and schur_plan.dim > 8192:
        raise ValueError("Dense Schur is limited to 8192 retained dimensions; use schur_cg")
    summary.reduced_dim = schur_plan.dim if is_schur else None
    n = problem.tangent_dim
    pcg_ws = DevicePCG(schur_plan.dim if is_schur else n, vdt, device)
    column_scale = None
    layout = problem.layout
    with _region("linearize", profile):
        lin = problem.linearize(vals, jacobian_dtype=jdt, schur=schur_plan)
    cached_head = None
    for iteration in range(termination.max_iterations):
        if timed_out():
            summary.termination_reason = "time_limit"
            break
        summary.iterations = iteration + 1
        gradient = lin.gradient
        jacobian = lin.jacobian
        mask = None
        if bplan is not None:
            mask = bplan.free_mask(vals, gradient)
            gradient = gradient * mask
            jacobian = jacobian.scale_columns(mask)
        # one host read: finiteness of the linearization, |g|_inf and the cost
        # (already read together with the previous step's norms when possible)
        if cached_head is not None:
            head, cached_head = cached_head, None
        else:
            checks = [reduce(t, 2) for t in (lin.residual, *lin.jacobian.jacs)]
            head = torch.stack((torch.stack(checks).max(), reduce(gradient, 2), lin.cost)).tolist()
        if not math.isfinite(head[0]):
            summary.termination_reason = "nonfinite_linearization"
            break
        summary.gradient_norm = head[1]
        lin_cost = head[2]
        if termination.target_cost is not None and lin_cost <= termination.target_cost:
            summary.termination_reason = "target_cost"
            break
        if summary.gradient_norm <= termination.gradient_tolerance:
            summary.termination_reason = "gradient_tolerance"
            break
        original = jacobian
        with _region("prepare_linear_system", profile):
            diag_damping = trust_region is not None and trust_region.damping_mode == "diagonal"
            needs_diag = is_schur or (linear_solver == "conjugate_gradient" and cg.preconditioner is not None)
            raw_diag = lin.jacobian.diagonal_blocks() if (
                needs_diag or diag_damping or (jacobi_scaling and column_scale is None)) else None
            diag_entries = None
            if raw_diag is not None:
                diag_entries = torch.cat([torch.diagonal(b, dim1=-2, dim2=-1).reshape(-1) for b in raw_diag])
                if mask is not None:
                    diag_entries = diag_entries * mask
            if jacobi_scaling and column_scale is None:
                column_scale = 1 / (1 + diag_entries.clamp_min(0).sqrt())
            solve_scale = column_scale
            if diag_damping:
                nd = diag_entries if column_scale is None else diag_entries * column_scale.square()
                inv = nd.clamp(trust_region.diagonal_min, trust_region.diagonal_max).rsqrt()
                solve_scale = inv if column_scale is None else column_scale * inv
            combined = solve_scale if mask is None else (mask if solve_scale is None else mask * solve_scale)
            linear_gradient = gradient if solve_scale is None else gradient * solve_scale
            scaled = lin.jacobian if combined is None else lin.jacobian.scale_columns(combined)
            schur_lin = SchurLinearization(schur_plan, lin, raw_diag, combined, wdtype=jdt, vec_dtype=vdt,
                                           dense=linear_solver == "schur_dense",
                                           cache_retained=cg.cache_retained_matrix and linear_solver == "schur_cg"
                                           ) if is_schur else None
            joint_specs = None
            if linear_solver == "conjugate_gradient" and cg.preconditioner is not None:
                if cg.preconditioner_groups:
                    sdiag = scaled.diagonal_blocks()
                    joint_specs = _joint_specs(layout, cg.preconditioner_groups, scaled, sdiag)
                else:
                    joint_specs = _layout_specs(layout, raw_diag)
        old_cost = lin_cost
        accepted = False

        def trial_tensors(step):
            """Step in the problem's coordinates, proposed values and the device
            vector (trial objective, exact reduction, predicted reduction, max |step|)."""
            step = step.to(torch.float64)
            if solve_scale is not None:
                step = solve_scale * step
            if bplan is None:
                prop = vals.retract(step, layout)
            else:
                prop, step = bplan.retract(vals, step)
            with _region("trial_residual", profile):
                objective, reduction = problem._evaluate_trial(prop, lin)
            pred = -torch.dot(gradient, step) - 0.5 * original.squared_matvec_norm(step)
            return step, prop, torch.stack((objective, reduction, pred, reduce(step, 2)))

        for _ in range(trust_region.max_trials if trust_region else 1):
            if timed_out():
                summary.termination_reason = "time_limit"
                break
            summary.lambda_history.append(damping)
            trial = None
            try:
                if linear_solver == "dense_qr":
                    # the damped least-squares step [J; sqrt(lambda) I] delta = [-r; 0]
                    # (solvers.py:504-510, a QR there): the normal equations factored by the
                    # tensor-core Cholesky, then one correction whose residual goes through J
                    # itself (Bjorck's corrected semi-normal equations)
                    with _region("linear_solve", profile):
                        jd = scaled.to_dense().to(torch.float64)
                        r0 = lin.residual.to(torch.float64)
                        nrm = jd.T @ jd
                        nrm.diagonal().add_(damping)
                        fac, info = dense.cholesky_ex(nrm)
                        if int(info) > 0:
                            raise torch.linalg.LinAlgError("damped normal matrix is not positive definite")
                        delta = dense.cholesky_solve(-(jd.T @ r0), fac)
                        corr = jd.T @ (-r0 - jd @ delta) - damping * delta
                        delta = delta + dense.cholesky_solve(corr, fac)
                        usable = _finite(delta)
                elif is_schur:
                    with _region("prepare_schur", profile):
                        # schur_cg reads the non-positive-definite counts with the PCG control block
                        system = schur_lin.damped(damping, check=linear_solver == "schur_dense")
                        rhs = system.reduced_rhs(-linear_gradient)
                    with _region("linear_solve", profile):
                        if linear_solver == "schur_dense":
                            fac, info = dense.cholesky_ex(system.dense_matrix())
                            if int(info) > 0:
                                raise torch.linalg.LinAlgError("dense Schur matrix is not positive definite")
                            retained = dense.cholesky_solve(rhs.double(), fac)
                            its, conv = 1, True
                            usable = _finite(retained)
                            summary.linear_relative_residual_history.append(None)
                            delta = system.backsubstitute(retained)
                        else:
                            pre = system.preconditioner(check=False) if cg.preconditioner else None
                            pcg_ws.run(rhs, cg, schur_args=system.args, preconditioner=pre,
                                       error_word=schur_plan.err,
                                       bad_words=(schur_plan.bad, None if pre is None else pre.bad_word),
                                       defer=True)
                            # the trial is queued behind the (persistent) PCG launch and read back
                            # with its control block: one host synchronisation per trial
                            trial = trial_tensors(system.backsubstitute(pcg_ws.x))
                            res, values = pcg_ws.finish(extra=trial[2])
                            if values is None:  # the PCG needed host-driven steps: redo the trial
                                trial = trial_tensors(system.backsubstitute(res.solution))
                                values = trial[2].tolist()
                            trial = (trial[0], trial[1], values)
                            retained, its, conv = res.solution, res.iterations, res.converged
                            # finiteness of the step is read with the trial terms
                            usable = res.reason in ("residual_tolerance", "max_iterations")
                            summary.linear_restarts += res.restarts
                            summary.linear_residual_checks += res.residual_checks
                            summary.linear_relative_residual_history.append(
                                res.residual_norm / res.rhs_norm if res.rhs_norm else res.residual_norm)
                            delta = None
                    summary.linear_iterations += its
                    summary.linear_iterations_history.append(its)
                    summary.linear_converged_history.append(conv)
                else:
                    pre = None
                    if cg.preconditioner is not None:
                        scale_for_pre = None if cg.preconditioner_groups else combined
                        pre = BlockJacobiPreconditioner.from_blocks(joint_specs, damping, scale_for_pre, n)
                    with _region("linear_solve", profile):
                        res = pcg_ws.run((-linear_gradient).to(vdt), cg,
                                         normal_args=scaled.normal_args(vdt, damping), preconditioner=pre)
                    summary.linear_iterations += res.iterations
                    summary.linear_iterations_history.append(res.iterations)
                    summary.linear_converged_history.append(res.converged)
                    summary.linear_restarts += res.restarts
                    summary.linear_residual_checks += res.residual_checks
                    summary.linear_relative_residual_history.append(
                        res.residual_norm / res.rhs_norm if res.rhs_norm else res.residual_norm)
                    delta = res.solution.to(torch.float64)
                    usable = res.reason in ("residual_tolerance", "max_iterations")
            except torch.linalg.LinAlgError:
                usable = False
            if usable:
                if trial is None:
                    trial = trial_tensors(delta)
                    trial = (trial[0], trial[1], trial[2].tolist())
                delta, proposed, (proposed_cost, actual, predicted, step_max) = trial
                if not math.isfinite(step_max):  # an unusable step: rejected, not a trial
                    usable = False
            if usable:
                quality = actual / predicted if predicted > 0 else -math.inf
                accepted = math.isfinite(proposed_cost) and (
                    trust_region is None or (actual > 0 and quality >= trust_region.step_quality_min))
                if record_trials:
                    summary.trial_history.append(dict(damping=damping, predicted_reduction=predicted,
                                                      actual_reduction=actual, gain_ratio=quality,
                                                      accepted=accepted))
                if accepted:
                    vals = proposed
                    summary.accepted_steps += 1
                    summary.final_cost = proposed_cost
                    summary.cost_history.append(proposed_cost)
                    if trust_region:
                        if trust_region.strategy == "adaptive":
                            mult = max(1 / 3, 1 - (2 * min(quality, 1.0) - 1) ** 3)
                            damping = max(trust_region.lambda_min, min(trust_region.lambda_max, damping * mult))
                            rejection_factor = 2.0
                        elif quality > 0.75:
                            damping = max(trust_region.lambda_min, damping / trust_region.lambda_factor)
                    lin = jacobian = original = scaled = schur_lin = system = None
                    with _region("linearize", profile):
                        lin = problem.linearize(vals, jacobian_dtype=jdt, schur=schur_plan)
                    fg = lin.gradient
                    if bplan is not None:
                        fg = bplan.projected_gradient(vals, fg)
                    if bplan is None:
                        checks = [reduce(t, 2) for t in (lin.residual, *lin.jacobian.jacs)]
                        gnorm, step_norm, fin, cost_next = torch.stack(
                            (reduce(fg, 2), reduce(delta, 1).sqrt(), torch.stack(checks).max(), lin.cost)).tolist()
                        cached_head = [fin, gnorm, cost_next]  # the next iteration's opening read
                    else:
                        gnorm, step_norm = torch.stack((reduce(fg, 2), reduce(delta, 1).sqrt())).tolist()
                    summary.gradient_norm = gnorm
                    if termination.target_cost is not None and proposed_cost <= termination.target_cost:
                        summary.termination_reason = "target_cost"
                    elif summary.gradient_norm <= termination.gradient_tolerance:
                        summary.termination_reason = "gradient_tolerance"
                    elif abs(actual) <= termination.cost_tolerance * max(old_cost, torch.finfo(vals.dtype).tiny):
                        summary.termination_reason = "cost_tolerance"
                    elif step_norm <= termination.parameter_tolerance:
                        summary.termination_reason = "parameter_tolerance"
                    break
            summary.rejected_steps += 1
            if trust_region is None or damping >= trust_region.lambda_max:
                break
            if trust_region.strategy == "adaptive":
                damping = min(trust_region.lambda_max, damping * rejection_factor)
                rejection_factor = min(rejection_factor * 2, trust_region.lambda_max / trust_region.lambda_min)
            else:
                damping = min(trust_region.lambda_max, damping * trust_region.lambda_factor)
        if not accepted:
            if summary.termination_reason != "time_limit":
                summary.termination_reason = "no_acceptable_step"
            break
        if summary.termination_reason != "max_iterations":
            break
    return (vals, summary) if return_summary else vals
