"""Gradients through a converged LM solve by the implicit function theorem.

At the solution x* the objective F(x, theta) = 1/2 sum_f w_f rho(|r_f(x, theta)|^2)
is stationary in the tangent chart: g(x*, theta) = dF(x* (+) delta, theta)/d delta
at delta = 0 vanishes. Differentiating g(x*(theta), theta) = 0 gives
H dx*/dtheta = -dg/dtheta with H the chart Hessian of F at x*, so for a scalar
loss L(x*)

    dL/dtheta = -d(lambda . g(x*, theta))/dtheta,   H lambda = dL/d delta.

H lambda = b is solved by iterative refinement: every round evaluates the
exact residual b - H lambda with a float64 Hessian-vector product of F
(reverse over reverse autograd through the residual functions) and corrects
lambda with the Gauss-Newton matrix J^T J -- the same normal operator the LM
solve uses, built by the CUDA library. With an eliminated group the
correction is the Schur complement: reduced right-hand side, dense Cholesky
of the reduced matrix, back-substitution (all through the library's Schur
kernels); otherwise the library's PCG on the normal operator. J^T J misses
the second-order residual terms (relative size ~ the residuals), so each
round gains that many digits. dL/dtheta is then one reverse pass through
lambda . g(x*, theta).

The stationarity condition needs a well-posed problem: gauge directions
(for example the global scale of a bundle adjustment with one camera fixed)
must be removed by priors or fixed variables, otherwise H is singular.
"""

from __future__ import annotations

from collections.abc import Mapping, Sequence

import torch
from torch import Tensor

from .problem import _is_ref
from . import dense
from .variables import euclidean_type

__all__ = ["newton_polish", "objective", "solve_implicit"]


def _groups(problem):
    """(name, values, Var spec, tangent dim, count, offset) per parameter group."""
    out, off = [], 0
    for name, value in problem.parameters.items():
        spec = problem.manifolds.get(name) or euclidean_type(tuple(value.shape[1:]))
        dim = int(spec.tangent_dim)
        count = int(value.shape[0])
        out.append((name, spec, dim, count, off))
        off += dim * count
    return out, off


def objective(problem, values: Mapping[str, Tensor], delta: Tensor | None = None,
              data: Mapping[int, Tensor] | None = None) -> Tensor:
    """F(x (+) delta) = 1/2 sum_f w_f rho(|r_f|^2) in float64, differentiable.

    ``values``: parameter tensors by name; ``delta``: flat tangent vector in the
    problem's layout (None: zero); ``data``: replacement tensors keyed by
    ``id()`` of a residual data argument or weights tensor of ``problem``.
    """
    data = data or {}
    groups, _ = _groups(problem)
    current = {}
    for name, spec, dim, count, off in groups:
        v = values[name].to(torch.float64)
        if delta is not None:
            d = delta[off : off + dim * count].view(count, dim)
            v = spec.retract_fn(v, d) if not getattr(spec, "is_euclidean", False) else v + d.reshape(v.shape)
        current[name] = v
    total = torch.zeros((), dtype=torch.float64, device=next(iter(current.values())).device)
    for cost in problem._costs:
        args, dims = [], []
        for i, a in enumerate(cost.args):
            if _is_ref(a):
                idx = torch.as_tensor(a.id).to(current[a.name].device)
                args.append(current[a.name][idx])
                dims.append(0 if idx.ndim == 1 else None)
            else:
                t = data.get(id(a), a)
                t = torch.as_tensor(t)
                if t.is_floating_point():
                    t = t.to(torch.float64)
                args.append(t.to(total.device))
                dims.append(cost.in_dims[i] if cost.in_dims is not None else (0 if t.ndim > 0 else None))
        r = torch.func.vmap(cost.residual_fn, in_dims=tuple(dims))(*args)
        r = r.reshape(r.shape[0], -1).to(torch.float64)
        s = (r * r).sum(-1)
        rho = s if cost.loss is None else cost.loss.evaluate(s)[0]
        if cost.weights is not None:
            w = data.get(id(cost.weights), cost.weights)
            w = torch.as_tensor(w, dtype=torch.float64, device=total.device).reshape(-1)
            rho = w * rho
        total = total + 0.5 * rho.sum()
    return total


class _Operators:
    """Chart gradient, exact Hessian-vector products and Gauss-Newton solves at x*."""

    def __init__(self, problem, values, eliminate, data=None):
        self.problem, self.values, self.data = problem, values, data
        _, self.n = _groups(problem)
        dev = next(iter(values.values())).device
        self.zero = torch.zeros(self.n, dtype=torch.float64, device=dev)
        self._gn = None
        self.eliminate = eliminate

    def hvp(self, v: Tensor) -> Tensor:
        with torch.enable_grad():
            d = self.zero.clone().requires_grad_(True)
            f = objective(self.problem, self.values, d, self.data)
            (g,) = torch.autograd.grad(f, d, create_graph=True)
            (hv,) = torch.autograd.grad(g, d, grad_outputs=v)
        return hv.detach()

    def _gauss_newton(self):
        if self._gn is not None:
            return self._gn
        from .schur import SchurLinearization, SchurPlan

        prob = self.problem
        params = {k: v.detach().to(torch.float64) for k, v in self.values.items()}
        if self.eliminate is None:
            lin = prob.linearize(params, jacobian_dtype=torch.float64)
            self._gn = ("normal", lin, None, None)
            return self._gn
        an = prob._ensure_analyzed()
        device = self.zero.device
        cache = an.__dict__.setdefault("_schur_plans", {})  # shared with the LM solver
        key = (self.eliminate, device, ())
        if key not in cache:
            cache[key] = SchurPlan(an, self.eliminate, device)
        plan = cache[key]
        lin = prob.linearize(params, jacobian_dtype=torch.float64, schur=plan)
        raw = lin.jacobian.diagonal_blocks()
        slin = SchurLinearization(plan, lin, raw, None, wdtype=torch.float64, vec_dtype=torch.float64, dense=True)
        system = slin.damped(0.0)
        fac, info = dense.cholesky_ex(system.dense_matrix())
        if int(info) > 0:
            raise torch.linalg.LinAlgError(
                "Gauss-Newton reduced matrix is singular at the solution: fix the gauge (priors or fixed variables)")
        self._gn = ("schur", lin, system, fac)
        return self._gn

    def gn_solve(self, b: Tensor) -> Tensor:
        kind, lin, system, fac = self._gauss_newton()
        if kind == "schur":
            rc = system.reduced_rhs(b)
            xc = dense.cholesky_solve(rc.double(), fac)
            return system.backsubstitute(xc)
        from functools import partial

        from .solvers import ConjugateGradientConfig, block_jacobi, pcg

        J = lin.jacobian
        res = pcg(partial(J.normal_matvec, damping=0.0), b, preconditioner=block_jacobi(J, 0.0),
                  config=ConjugateGradientConfig(rtol=1e-13, atol=0.0, max_iterations=10 * self.n))
        return res.solution.to(torch.float64)


def _adjoint_solve(ops: _Operators, b: Tensor, tol: float, max_rounds: int):
    lam = torch.zeros_like(b)
    bn = float(torch.linalg.vector_norm(b))
    history = []
    if bn == 0.0:
        return lam, history
    res = b.clone()
    best = float("inf")
    for _ in range(max_rounds):
        lam = lam + ops.gn_solve(res)
        res = b - ops.hvp(lam)
        rel = float(torch.linalg.vector_norm(res)) / bn
        history.append(rel)
        if rel <= tol or rel > 0.5 * best:  # converged, or at the rounding floor
            break
        best = rel
    return lam, history


class _ImplicitSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, spec, *inputs):
        problem, names, solve_options = spec["problem"], spec["names"], spec["options"]
        sol = problem.solve(**solve_options)
        if isinstance(sol, tuple):
            sol = sol[0]
        spec["summary"] = problem.last_summary
        ctx.spec = spec
        ctx.inputs = inputs
        ctx.solution = {k: v.detach().clone() for k, v in sol.items()}
        return tuple(ctx.solution[k].clone() for k in names)

    @staticmethod
    def backward(ctx, *grads):
        spec = ctx.spec
        problem, names = spec["problem"], spec["names"]
        values = ctx.solution
        groups, n = _groups(problem)
        dev = next(iter(values.values())).device
        # dL/d delta: pull the ambient cotangents back through the retraction at x*
        with torch.enable_grad():
            d = torch.zeros(n, dtype=torch.float64, device=dev, requires_grad=True)
            outs, cots = [], []
            for (name, spec_, dim, count, off), g in zip(groups, grads):
                if g is None:
                    continue
                v = values[name].to(torch.float64)
                dd = d[off : off + dim * count].view(count, dim)
                x = spec_.retract_fn(v, dd) if not getattr(spec_, "is_euclidean", False) else v + dd.reshape(v.shape)
                outs.append(x)
                cots.append(g.to(torch.float64))
            b = torch.autograd.grad(outs, d, grad_outputs=cots, allow_unused=True)[0] if outs else None
        if b is None:
            return (None,) + tuple(None for _ in ctx.inputs)
        leaves = [t.detach().to(torch.float64).requires_grad_(True) for t in ctx.inputs]
        data = {id(orig): leaf for orig, leaf in zip(spec["originals"], leaves)}
        ops = _Operators(problem, values, spec["eliminate"], data=None)
        lam, history = _adjoint_solve(ops, b, spec["tol"], spec["max_rounds"])
        spec["refinement_history"] = history
        with torch.enable_grad():
            dz = torch.zeros(n, dtype=torch.float64, device=dev, requires_grad=True)
            f = objective(problem, values, dz, data)
            (g,) = torch.autograd.grad(f, dz, create_graph=True)
            phi = torch.dot(g, lam)
            gin = torch.autograd.grad(phi, leaves, allow_unused=True)
        out = []
        for orig, gi in zip(ctx.inputs, gin):
            out.append(None if gi is None else (-gi).to(orig.dtype))
        return (None,) + tuple(out)


def solve_implicit(problem, inputs: Sequence[Tensor], *, eliminate: str | None = None, tol: float = 1e-12,
                   max_rounds: int = 20, **solve_options) -> dict[str, Tensor]:
    """Solve ``problem`` on the GPU and return solution tensors that are
    differentiable with respect to ``inputs``.

    ``inputs`` are residual data arguments or weight tensors already used by
    ``problem`` (observations, per-residual weights, constants). The forward
    pass is ``problem.solve(eliminate=eliminate, **solve_options)``; the
    backward pass is the implicit-function-theorem adjoint described in the
    module docstring (tolerance ``tol`` on the adjoint residual). The solve
    should converge tightly (gradient tolerance well below the gradients
    wanted) for the adjoint to describe its result.
    """
    names = list(problem.parameters)
    opts = dict(solve_options)
    if eliminate is not None:
        opts["eliminate"] = eliminate
    spec = dict(problem=problem, names=names, options=opts, eliminate=eliminate, tol=tol, max_rounds=max_rounds,
                originals=list(inputs))
    outs = _ImplicitSolve.apply(spec, *inputs)
    result = dict(zip(names, outs))
    result_info = spec
    solve_implicit.last = result_info
    return result


def _retract_all(problem, values, step):
    groups, _ = _groups(problem)
    out = {}
    for name, spec, dim, count, off in groups:
        v = values[name]
        d = step[off : off + dim * count].view(count, dim)
        out[name] = spec.retract_fn(v, d) if not getattr(spec, "is_euclidean", False) else v + d.reshape(v.shape)
    return out


def newton_polish(problem, *, eliminate: str | None = None, steps: int = 2, tol: float = 1e-13,
                  max_rounds: int = 20) -> dict[str, Tensor]:
    """Refine ``problem.parameters`` (a converged LM solution) with Newton steps
    on the exact chart Hessian: each step solves H step = -g by the same
    Gauss-Newton-corrected refinement as the adjoint. LM stops on cost changes
    at rounding level, which leaves the parameters accurate to about the
    square root of the working precision; two Newton steps from there reach
    the stationary point to rounding level (needed, for example, by finite
    differences of the solution)."""
    dtypes = {k: v.dtype for k, v in problem.parameters.items()}
    values = {k: v.detach().to(torch.float64) for k, v in problem.parameters.items()}
    _, n = _groups(problem)
    for _ in range(steps):
        ops = _Operators(problem, values, eliminate)
        with torch.enable_grad():
            d = ops.zero.clone().requires_grad_(True)
            (g,) = torch.autograd.grad(objective(problem, values, d), d)
        step, _ = _adjoint_solve(ops, -g.detach(), tol, max_rounds)
        values = {k: v.detach() for k, v in _retract_all(problem, values, step).items()}
    problem.parameters.update({k: v.to(dtypes[k]) for k, v in values.items()})
    return dict(values)
