"""LM / GN driver (numpy). Restates torchls solvers.py:288-696 and bounds.py:10-75."""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
from scipy.linalg import cho_factor, cho_solve

from .linalg import JointBlocks, LinAlgError, block_jacobi, pcg
from .schur import SchurLinearization, SchurPlan


@dataclass
class Summary:
    initial_cost: float
    final_cost: float
    iterations: int = 0
    accepted_steps: int = 0
    rejected_steps: int = 0
    linear_iterations: int = 0
    termination_reason: str = "max_iterations"
    gradient_norm: float = math.inf
    cost_history: list = field(default_factory=list)
    lambda_history: list = field(default_factory=list)
    linear_iterations_history: list = field(default_factory=list)
    linear_converged_history: list = field(default_factory=list)
    trial_history: list = field(default_factory=list)
    linear_restarts: int = 0
    linear_residual_checks: int = 0
    linear_relative_residual_history: list = field(default_factory=list)
    reduced_dim: int | None = None


class Bounds:
    """bounds.py:10-75 for Euclidean groups given by key -> (lower, upper)."""

    def __init__(self, bounds, problem, values):
        self.groups = []
        index = {g.key: i for i, g in enumerate(problem.groups)}
        for key, (lo, hi) in bounds.items():
            gi = index[key]
            v = values[gi]
            lo = np.broadcast_to(np.asarray(-np.inf if lo is None else lo, np.float64), v.shape).copy()
            hi = np.broadcast_to(np.asarray(np.inf if hi is None else hi, np.float64), v.shape).copy()
            self.groups.append((gi, lo, hi))
        self.problem = problem

    def free_mask(self, values, gradient):
        mask = np.ones_like(gradient)
        for gi, lo, hi in self.groups:
            g = self.problem.groups[gi]
            a, b = g.offset, g.offset + g.count * g.dim
            v = values[gi]
            lg = gradient[a:b].reshape(v.shape)
            active = (lo == hi) | ((v <= lo) & (lg > 0)) | ((v >= hi) & (lg < 0))
            mask[a:b] = (~active).reshape(-1)
        return mask

    def retract(self, values, delta):
        proposed = self.problem.retract(values, delta)
        eff = delta.copy()
        for gi, lo, hi in self.groups:
            g = self.problem.groups[gi]
            v = np.clip(proposed[gi], lo, hi)
            proposed[gi] = v
            eff[g.offset : g.offset + g.count * g.dim] = (v - values[gi]).reshape(-1)
        return proposed, eff


def solve(problem, *, linear_solver="conjugate_gradient", eliminate=None, cg=None, trust_region=None,
          gauss_newton=False, termination=None, jacobi_scaling=False, bounds=None, record_trials=False,
          values=None):
    """Run LM (or GN with ``gauss_newton=True``). Option dicts use torchls field names."""
    cg = dict(dict(rtol=1e-6, atol=1e-10, max_iterations=200, preconditioner="block_jacobi",
                   preconditioner_groups=(), residual_check_interval=50, restart_strategy="adaptive",
                   residual_drift_tolerance=0.1), **(cg or {}))
    tr = None if gauss_newton else dict(dict(lambda_initial=1e-3, lambda_min=1e-12, lambda_max=1e12,
                                             lambda_factor=4.0, step_quality_min=1e-4, max_trials=20,
                                             strategy="fixed_factor", damping_mode="identity",
                                             diagonal_min=1e-6, diagonal_max=1e32), **(trust_region or {}))
    term = dict(dict(max_iterations=50, cost_tolerance=1e-10, gradient_tolerance=1e-8,
                     parameter_tolerance=1e-10, target_cost=None), **(termination or {}))
    pcg_opts = {k: cg[k] for k in ("rtol", "atol", "max_iterations", "residual_check_interval",
                                   "restart_strategy", "residual_drift_tolerance")}
    is_schur = linear_solver.startswith("schur_")
    vals = [v.copy() for v in (values if values is not None else problem.values())]
    bplan = Bounds(bounds, problem, vals) if bounds else None
    initial = problem.cost(vals)
    if not math.isfinite(initial):
        raise ValueError("Initial residuals are nonfinite")
    S = Summary(initial, initial, cost_history=[initial])
    damping = tr["lambda_initial"] if tr else 0.0
    rejection_factor = 2.0
    splan = SchurPlan(problem, eliminate, cg["preconditioner_groups"]) if is_schur else None
    joint = (JointBlocks(problem.groups, cg["preconditioner_groups"])
             if not is_schur and cg["preconditioner_groups"] else None)
    S.reduced_dim = splan.dim if is_schur else None
    column_scale = None
    lin = problem.linearize(vals)
    layout = problem.groups
    for iteration in range(term["max_iterations"]):
        S.iterations = iteration + 1
        residual, jac = lin.residual, lin.jacobian
        if not np.isfinite(residual).all() or any(not np.isfinite(b).all() for g in jac.groups for b in g["blocks"]):
            S.termination_reason = "nonfinite_linearization"
            break
        gradient = lin.gradient
        if bplan is not None:
            mask = bplan.free_mask(vals, gradient)
            gradient = gradient * mask
            jac = jac.scale_columns(mask)
        S.gradient_norm = float(np.max(np.abs(gradient)))
        if term["target_cost"] is not None and lin.cost <= term["target_cost"]:
            S.termination_reason = "target_cost"
            break
        if S.gradient_norm <= term["gradient_tolerance"]:
            S.termination_reason = "gradient_tolerance"
            break
        original = jac
        diag_damping = tr is not None and tr["damping_mode"] == "diagonal"
        needs_diag = is_schur or (linear_solver == "conjugate_gradient" and cg["preconditioner"] is not None)
        diag = None
        if needs_diag or diag_damping or (jacobi_scaling and column_scale is None):
            diag = jac.diagonal_blocks()
        if jacobi_scaling and column_scale is None:
            column_scale = np.concatenate(
                [(1 / (1 + np.sqrt(np.maximum(np.diagonal(b, axis1=-2, axis2=-1), 0)))).reshape(-1) for b in diag])
        solve_scale = column_scale
        if diag_damping:
            nd = np.concatenate([np.diagonal(b, axis1=-2, axis2=-1).reshape(-1) for b in diag])
            if column_scale is not None:
                nd = nd * column_scale**2
            inv = 1 / np.sqrt(np.clip(nd, tr["diagonal_min"], tr["diagonal_max"]))
            solve_scale = inv if column_scale is None else column_scale * inv
        if solve_scale is not None:
            jac = jac.scale_columns(solve_scale)
            lgrad = gradient * solve_scale
            if diag is not None:
                diag = [b * solve_scale[e.offset : e.offset + e.count * e.dim].reshape(e.count, e.dim, 1)
                        * solve_scale[e.offset : e.offset + e.count * e.dim].reshape(e.count, 1, e.dim)
                        for e, b in zip(layout, diag)]
        else:
            lgrad = gradient
        slin = SchurLinearization(jac, diag, splan, dense=linear_solver == "schur_dense") if is_schur else None
        jdiag = joint.normal_blocks(jac, diag) if joint else None
        old_cost = lin.cost
        accepted = False
        for _ in range(tr["max_trials"] if tr else 1):
            S.lambda_history.append(damping)
            try:
                if is_schur:
                    system = slin.damped(damping)
                    rhs = system.reduced_rhs(-lgrad)
                    if linear_solver == "schur_dense":
                        m = system.dense_matrix()
                        try:
                            fac = cho_factor(m, lower=True)
                        except np.linalg.LinAlgError as err:
                            raise LinAlgError(str(err)) from err
                        retained = cho_solve(fac, rhs)
                        its, conv = 1, True
                        usable = bool(np.isfinite(retained).all())
                        S.linear_relative_residual_history.append(None)
                    else:
                        res = pcg(system.matvec, rhs,
                                  system.preconditioner() if cg["preconditioner"] else None, **pcg_opts)
                        retained, its, conv = res.solution, res.iterations, res.converged
                        usable = res.reason in ("residual_tolerance", "max_iterations") and bool(np.isfinite(retained).all())
                        S.linear_restarts += res.restarts
                        S.linear_residual_checks += res.residual_checks
                        S.linear_relative_residual_history.append(
                            res.residual_norm / res.rhs_norm if res.rhs_norm else res.residual_norm)
                    delta = system.backsubstitute(retained)
                    S.linear_iterations += its
                    S.linear_iterations_history.append(its)
                    S.linear_converged_history.append(conv)
                else:
                    if cg["preconditioner"] is not None:
                        pre = joint.factor(jdiag, damping) if joint else block_jacobi(layout, diag, damping)
                    else:
                        pre = None
                    res = pcg(lambda v: jac.normal_matvec(v, damping), -lgrad, pre, **pcg_opts)
                    S.linear_iterations += res.iterations
                    S.linear_iterations_history.append(res.iterations)
                    S.linear_converged_history.append(res.converged)
                    S.linear_restarts += res.restarts
                    S.linear_residual_checks += res.residual_checks
                    S.linear_relative_residual_history.append(
                        res.residual_norm / res.rhs_norm if res.rhs_norm else res.residual_norm)
                    delta = res.solution
                    usable = res.reason in ("residual_tolerance", "max_iterations") and bool(np.isfinite(delta).all())
            except LinAlgError:
                usable = False
            if usable:
                if solve_scale is not None:
                    delta = solve_scale * delta
                if bplan is None:
                    proposed = problem.retract(vals, delta)
                else:
                    proposed, delta = bplan.retract(vals, delta)
                obj, red = problem.evaluate_trial(proposed, lin)
                predicted = float(-np.dot(gradient, delta) - 0.5 * original.squared_matvec_norm(delta))
                actual = float(red)
                quality = actual / predicted if predicted > 0 else -math.inf
                accepted = math.isfinite(obj) and (tr is None or (actual > 0 and quality >= tr["step_quality_min"]))
                if record_trials:
                    S.trial_history.append(dict(damping=damping, predicted_reduction=predicted,
                                                actual_reduction=actual, gain_ratio=quality, accepted=accepted))
                if accepted:
                    vals = proposed
                    S.accepted_steps += 1
                    S.final_cost = obj
                    S.cost_history.append(obj)
                    if tr:
                        if tr["strategy"] == "adaptive":
                            mult = max(1 / 3, 1 - (2 * min(quality, 1.0) - 1) ** 3)
                            damping = max(tr["lambda_min"], min(tr["lambda_max"], damping * mult))
                            rejection_factor = 2.0
                        elif quality > 0.75:
                            damping = max(tr["lambda_min"], damping / tr["lambda_factor"])
                    lin = problem.linearize(vals)
                    fg = lin.gradient
                    if bplan is not None:
                        fg = fg * bplan.free_mask(vals, fg)
                    S.gradient_norm = float(np.max(np.abs(fg)))
                    if term["target_cost"] is not None and obj <= term["target_cost"]:
                        S.termination_reason = "target_cost"
                    elif S.gradient_norm <= term["gradient_tolerance"]:
                        S.termination_reason = "gradient_tolerance"
                    elif abs(actual) <= term["cost_tolerance"] * max(old_cost, np.finfo(np.float64).tiny):
                        S.termination_reason = "cost_tolerance"
                    elif float(np.linalg.norm(delta)) <= term["parameter_tolerance"]:
                        S.termination_reason = "parameter_tolerance"
                    break
            S.rejected_steps += 1
            if tr is None or damping >= tr["lambda_max"]:
                break
            if tr["strategy"] == "adaptive":
                damping = min(tr["lambda_max"], damping * rejection_factor)
                rejection_factor = min(rejection_factor * 2, tr["lambda_max"] / tr["lambda_min"])
            else:
                damping = min(tr["lambda_max"], damping * tr["lambda_factor"])
        if not accepted:
            S.termination_reason = "no_acceptable_step"
            break
        if S.termination_reason != "max_iterations":
            break
    return vals, S
