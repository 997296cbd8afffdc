"""CUDA path vs fixtures produced by torchls itself (float64) and vs the oracle.

Tolerances: float64 CUDA results match the reference to 1e-12 relative for
per-linearization quantities and 1e-10 relative for final costs; parameters to
1e-8 (the reference's own final-iterate precision). Mixed precision (float32
Jacobian and PCG vectors, float64 reductions) must reach the float64 final
cost within 1e-8 relative.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gpu_helpers import SUMMARIES, check_summary, close, load, needs_gpu, stored_ba, to_np
from golden import problems as P

pytestmark = [pytest.mark.gpu, needs_gpu]

DEV = "cuda"


@pytest.fixture(scope="module")
def tls():
    import torchls_b200

    return torchls_b200


@pytest.fixture(scope="module")
def ba(tls):
    fx = load("ba_small")
    prob = P.ba_small(tls, device=DEV, data=stored_ba(fx))
    return fx, prob


def test_ba_linearization(tls, ba):
    fx, prob = ba
    lin = prob.linearize()
    close(lin.residual, fx["residual"], 1e-12, what="residual")
    close(lin.raw_residual, fx["raw_residual"], 1e-12, what="raw")
    close(lin.cost, fx["cost"], 1e-13, what="cost")
    close(lin.gradient, fx["gradient"], 1e-11, what="gradient")
    for i, d in enumerate(lin.jacobian.diagonal_blocks()):
        close(d, fx[f"diag{i}"], 1e-11, what=f"diag{i}")
    for gi, g in enumerate(lin.jacobian.groups):
        for si, b in enumerate(g.blocks):
            close(b, fx[f"block{gi}_{si}"], 1e-11, what=f"block{gi}_{si}")


def test_ba_products_and_determinism(tls, ba):
    fx, prob = ba
    J = prob.linearize().jacobian
    v = torch.from_numpy(fx["v"]).to(DEV)
    u = torch.from_numpy(fx["u"]).to(DEV)
    y1 = J.normal_matvec(v, 1e-3)
    close(y1, fx["normal_matvec"], 1e-12, what="normal_matvec")
    assert torch.equal(y1, J.normal_matvec(v, 1e-3)), "normal matvec is not bitwise reproducible"
    close(J.matvec(v), fx["matvec"], 1e-12, what="matvec")
    close(J.rmatvec(u), fx["rmatvec"], 1e-12, what="rmatvec")
    close(J.squared_matvec_norm(v), fx["squared_matvec_norm"], 1e-12, what="sqnorm")
    apply = tls.block_jacobi(J, 1e-3)
    close(apply(v), fx["block_jacobi_apply"], 1e-10, what="block_jacobi")


def test_ba_device_pcg(tls, ba):
    from functools import partial

    fx, prob = ba
    lin = prob.linearize()
    J = lin.jacobian
    res = tls.pcg(partial(J.normal_matvec, damping=1e-3), -lin.gradient, preconditioner=tls.block_jacobi(J, 1e-3),
                  config=tls.ConjugateGradientConfig())
    ref = SUMMARIES["ba_small_pcg"]
    assert (res.iterations, res.reason, res.restarts, res.residual_checks) == (
        ref["iterations"], ref["reason"], ref["restarts"], ref["residual_checks"])
    close(res.solution, fx["pcg_solution"], 1e-8, what="pcg solution")
    close(res.rhs_norm, ref["rhs_norm"], 1e-12, what="rhs_norm")


def test_ba_schur_system(tls, ba):
    from torchls_b200.schur import SchurLinearization, SchurPlan

    fx, prob = ba
    an = prob._ensure_analyzed()
    plan = SchurPlan(an, "points", torch.device(DEV))
    np.testing.assert_array_equal(to_np(plan.edges[0][0]), fx["schur_edges_r"])
    np.testing.assert_array_equal(to_np(plan.edges[0][1]), fx["schur_edges_e"])
    lin = prob.linearize(schur=plan)
    raw = lin.jacobian.diagonal_blocks()
    slin = SchurLinearization(plan, lin, raw, None, wdtype=torch.float64, vec_dtype=torch.float64)
    slab = torch.as_tensor(slin.layout.slab_of_edge, device=slin.cross.device)
    close(slin.cross[slab], fx["schur_cross"], 1e-12, what="cross")
    sys_ = slin.damped(1e-3)
    close(sys_.reduced_rhs(-lin.gradient), fx["schur_reduced_rhs"], 1e-11, what="reduced_rhs")
    vc = torch.from_numpy(fx["vc"]).to(DEV)
    close(sys_.matvec(vc), fx["schur_matvec"], 1e-11, what="schur matvec")
    close(sys_.preconditioner()(vc), fx["schur_preconditioner"], 1e-10, what="schur preconditioner")
    close(sys_.backsubstitute(vc), fx["schur_backsubstitute"], 1e-11, what="backsubstitute")
    close(sys_.dense_matrix(), fx["schur_dense"], 1e-11, what="dense")


@pytest.mark.parametrize("wdtype", [torch.float32, torch.float64])
def test_whitening_from_contributions_matches_summed_cross(tls, ba, wdtype):
    """tls_schur_damp whitens from the linearization's cross contributions
    (cross_contrib) by default; given the summed cross blocks (cross, with
    cross_contrib NULL) it must write bitwise the same W slabs."""
    import ctypes

    from torchls_b200 import _lib as L
    from torchls_b200.schur import SchurLinearization, SchurPlan

    fx, prob = ba
    an = prob._ensure_analyzed()
    plan = SchurPlan(an, "points", torch.device(DEV))
    lin = prob.linearize(schur=plan)
    raw = lin.jacobian.diagonal_blocks()
    slin = SchurLinearization(plan, lin, raw, None, wdtype=wdtype, vec_dtype=torch.float64)
    sys_ = slin.damped(1e-3)
    w_fused = slin.w.clone()
    a = sys_._args()
    a.cross = slin.cross.data_ptr()
    a.cross_contrib = None
    slin.w.zero_()
    L.call("tls_schur_damp", ctypes.byref(a), L.stream_handle(plan.device))
    torch.cuda.synchronize()
    assert torch.equal(slin.w, w_fused)


BA_RUNS = {
    "schur_cg": dict(linear_solver="schur_cg", eliminate="points", record_trials=True),
    "conjugate_gradient": dict(linear_solver="conjugate_gradient"),
    "schur_dense": dict(linear_solver="schur_dense", eliminate="points"),
    "scaled_adaptive": dict(linear_solver="schur_cg", eliminate="points", jacobi_scaling=True,
                            trust_region=dict(strategy="adaptive", damping_mode="diagonal")),
}


@pytest.mark.parametrize("run", list(BA_RUNS))
def test_ba_solve(tls, run):
    fx = load("ba_small")
    opts = dict(BA_RUNS[run])
    if "trust_region" in opts:
        opts["trust_region"] = tls.TrustRegionConfig(**opts["trust_region"])
    prob = P.ba_small(tls, device=DEV, data=stored_ba(fx))
    sol, s = prob.solve(return_summary=True, termination=tls.TerminationConfig(max_iterations=30), **opts)
    check_summary(s, SUMMARIES[f"ba_small_{run}"])
    close(sol["cams"], fx[f"solve_{run}_cams"], 1e-8, what="cams")
    close(sol["points"], fx[f"solve_{run}_points"], 1e-8, what="points")


def test_ba_mixed_precision_reaches_fp64_cost(tls):
    fx = load("ba_small")
    prob = P.ba_small(tls, device=DEV, data=stored_ba(fx))
    cfg = tls.ConjugateGradientConfig(precision="mixed")
    _, s = prob.solve(return_summary=True, linear_solver="schur_cg", eliminate="points", conjugate_gradient=cfg,
                      termination=tls.TerminationConfig(max_iterations=30))
    ref = SUMMARIES["ba_small_schur_cg"]["final_cost"]
    assert abs(s.final_cost - ref) <= 1e-8 * ref, (s.final_cost, ref)


OTHERS = {
    "ba_tiny": (P.ba_tiny, dict(linear_solver="schur_cg", eliminate="points")),
    "ba_tiny_gn": (P.ba_tiny, dict(linear_solver="conjugate_gradient", trust_region=None,
                                   termination=dict(max_iterations=8))),
    "pose_small": (P.pose_small, dict(linear_solver="conjugate_gradient", termination=dict(max_iterations=30))),
    "sim3_small": (P.sim3_small, dict(linear_solver="conjugate_gradient", termination=dict(max_iterations=30))),
    "se2_custom": (P.se2_custom, dict(linear_solver="conjugate_gradient")),
    "ba_two_groups": (P.ba_two_groups, dict(linear_solver="schur_cg", eliminate="points")),
    "ba_priors": (P.ba_priors, dict(linear_solver="schur_cg", eliminate="points")),
    "ba_priors_dense": (P.ba_priors, dict(linear_solver="schur_dense", eliminate="points")),
    "ba_intrinsics": (P.ba_intrinsics, dict(linear_solver="schur_cg", eliminate="points")),
    "ba_intrinsics_joint": (P.ba_intrinsics, dict(linear_solver="schur_cg", eliminate="points",
                                                  conjugate_gradient=dict(preconditioner_groups=(("cams", "focal"),)))),
    "curve_bounds": (P.curve_bounds, dict(bounds=P.CURVE_BOUNDS)),
    "rotations_small": (P.rotations_small, dict(jacobi_scaling=True, trust_region=dict(
        lambda_initial=1e-3, strategy="adaptive", damping_mode="diagonal"))),
    "rotations_small_qr": (P.rotations_small, dict(linear_solver="dense_qr", jacobi_scaling=True, trust_region=dict(
        lambda_initial=1e-3, strategy="adaptive", damping_mode="diagonal"))),
    "ba_tiny_qr": (P.ba_tiny, dict(linear_solver="dense_qr")),
    "alias_weights": (P.alias_weights, dict()),
    "alias_cauchy": (lambda api, **k: P.alias_weights(api, loss=P.cauchy_loss(api), **k), dict()),
    "alias_softsq": (lambda api, **k: P.alias_weights(api, loss=P.soft_square_loss(api), **k), dict()),
    "joint_groups": (P.joint_groups, dict(conjugate_gradient=dict(preconditioner_groups=(("off", "pts"),)))),
}


@pytest.mark.parametrize("name", list(OTHERS))
def test_other_problems(tls, name):
    builder, opts = OTHERS[name]
    opts = dict(opts)
    if "termination" in opts:
        opts["termination"] = tls.TerminationConfig(**opts["termination"])
    if isinstance(opts.get("trust_region"), dict):
        opts["trust_region"] = tls.TrustRegionConfig(**opts["trust_region"])
    if "conjugate_gradient" in opts:
        opts["conjugate_gradient"] = tls.ConjugateGradientConfig(**opts["conjugate_gradient"])
    fx = load(name)
    lin = builder(tls, device=DEV).linearize()
    close(lin.residual, fx["residual"], 1e-11, 1e-15, what="residual")
    close(lin.gradient, fx["gradient"], 1e-10, 1e-13, what="gradient")
    for i, d in enumerate(lin.jacobian.diagonal_blocks()):
        close(d, fx[f"diag{i}"], 1e-10, 1e-13, what=f"diag{i}")
    for gi, g in enumerate(lin.jacobian.groups):
        for si, (b, c) in enumerate(zip(g.blocks, g.columns)):
            close(b, fx[f"block{gi}_{si}"], 1e-10, 1e-13, what=f"block{gi}_{si}")
            np.testing.assert_array_equal(to_np(c), fx[f"columns{gi}_{si}"])
    prob = builder(tls, device=DEV)
    sol, s = prob.solve(return_summary=True, **opts)
    # pose_small runs ~180 CG iterations per step; allow +-2 per step there
    check_summary(s, SUMMARIES[name], cg_slack=2 if name == "pose_small" else 0)
    for key, val in sol.items():
        close(val, fx[f"solve_{key}"], 1e-7, 1e-12, what=key)


def test_typed_api_solve(tls):
    """Cost.factory / LeastSquaresProblem / VarValues with sparse unsorted IDs:
    linearization and the Schur-CG solve against the reference's fixture."""
    fx = load("typed_ba")
    problem, init = P.typed_ba(tls, device=DEV)
    lin = problem.linearize(init)
    close(lin.residual, fx["residual"], 1e-11, 1e-15, what="residual")
    close(lin.gradient, fx["gradient"], 1e-10, 1e-13, what="gradient")
    for gi, g in enumerate(lin.jacobian.groups):
        for si, (b, c) in enumerate(zip(g.blocks, g.columns)):
            close(b, fx[f"block{gi}_{si}"], 1e-10, 1e-13, what=f"block{gi}_{si}")
            np.testing.assert_array_equal(to_np(c), fx[f"columns{gi}_{si}"])
    sol, s = problem.solve(init, return_summary=True, linear_solver="schur_cg",
                           eliminate=problem.layout[0].var_type)
    check_summary(s, SUMMARIES["typed_ba"])
    for i, e in enumerate(problem.layout):
        close(sol._values[e.var_type], fx[f"solve{i}"], 1e-8, what=f"solve{i}")


GENERAL_SCHUR = {"intr": (P.ba_intrinsics, ()), "joint": (P.ba_intrinsics, (("cams", "focal"),)),
                 "priors": (P.ba_priors, ()), "two": (P.ba_two_groups, ())}


@pytest.mark.parametrize("precision", ["native", "mixed"])
@pytest.mark.parametrize("tag", list(GENERAL_SCHUR))
def test_general_schur_system(tls, tag, precision):
    """Several retained groups, retained couplings, joint groups (the general
    Schur kernels) against torchls's own Schur system (schur.py:17-397). Mixed
    precision stores W in float32: products within 1e-6 there."""
    from torchls_b200.schur import SchurLinearization, SchurPlan

    builder, groups = GENERAL_SCHUR[tag]
    fx = load("schur_general")
    prob = builder(tls, device=DEV)
    an = prob._ensure_analyzed()
    plan = SchurPlan(an, "points", torch.device(DEV), preconditioner_groups=groups)
    assert plan.general
    wdt = torch.float64 if precision == "native" else torch.float32
    lin = prob.linearize(jacobian_dtype=wdt, schur=plan)
    slin = SchurLinearization(plan, lin, lin.jacobian.diagonal_blocks(), None, wdtype=wdt, vec_dtype=torch.float64,
                              dense=True)
    system = slin.damped(1e-3)
    tol = 1e-11 if precision == "native" else 1e-6
    vc = torch.from_numpy(fx[f"{tag}_vc"]).to(DEV)
    close(system.reduced_rhs(-lin.gradient), fx[f"{tag}_reduced_rhs"], tol, what="reduced_rhs")
    close(system.matvec(vc), fx[f"{tag}_matvec"], tol, what="matvec")
    close(system.preconditioner()(vc), fx[f"{tag}_preconditioner"], max(tol, 1e-10), what="preconditioner")
    close(system.backsubstitute(vc), fx[f"{tag}_backsubstitute"], tol, what="backsubstitute")
    close(system.dense_matrix(), fx[f"{tag}_dense"], tol, what="dense")


@pytest.mark.parametrize("tag", ["priors", "intr", "two"])
def test_cached_retained_matrix(tls, tag):
    """cache_retained_matrix (schur.py:225-241): with retained couplings the
    base term comes from the cached block-sparse (s J_r)^T (s J_r) instead of
    the normal operator; torchls's product to 1e-11, the matrix-free operator
    to 1e-12 with a column scale, and the same solve as without the cache."""
    from torchls_b200.schur import SchurLinearization, SchurPlan

    f64 = torch.float64
    builder, _ = GENERAL_SCHUR[tag]
    fx = load("schur_general")
    prob = builder(tls, device=DEV)
    an = prob._ensure_analyzed()
    plan = SchurPlan(an, "points", torch.device(DEV))
    lin = prob.linearize(jacobian_dtype=f64, schur=plan)
    diag = lin.jacobian.diagonal_blocks()
    vc = torch.from_numpy(fx[f"{tag}_vc"]).to(DEV)

    def system(scale, cache, damping):
        return SchurLinearization(plan, lin, diag, scale, wdtype=f64, vec_dtype=f64,
                                  cache_retained=cache).damped(damping)

    cached = system(None, True, 1e-3)
    assert (cached.linear.retained is not None) == bool(plan.couplings)
    close(cached.matvec(vc), fx[f"{tag}_matvec"], 1e-11, what="matvec")
    g = torch.Generator().manual_seed(3)
    s = (torch.rand(an.tangent_dim, generator=g, dtype=f64) + 0.5).to(DEV)
    close(system(s, True, 0.1).matvec(vc), system(s, False, 0.1).matvec(vc), 1e-12, what="scaled matvec")
    opts = dict(linear_solver="schur_cg", eliminate="points", return_summary=True)
    _, s0 = builder(tls, device=DEV).solve(**opts)
    _, s1 = builder(tls, device=DEV).solve(conjugate_gradient=tls.ConjugateGradientConfig(cache_retained_matrix=True),
                                           **opts)
    assert s1.linear_iterations_history == s0.linear_iterations_history
    close(s1.final_cost, s0.final_cost, 1e-10, what="final cost")
