"""Generate the golden fixtures by running torchls itself (float64, CPU).

    python tests/golden/make_golden.py /path/to/torchls-checkout [--only name,name]

Writes ``tests/golden/*.npz`` (arrays) and ``tests/golden/summaries.json``.
The fixtures pin the numpy oracle (``tests/test_oracle.py``); the CUDA path
is then compared with the oracle and, for the stored-input bundle-adjustment
case, with these fixtures directly.
"""

from __future__ import annotations

import json
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def summary_dict(s):
    keys = ("initial_cost", "final_cost", "iterations", "accepted_steps", "rejected_steps",
            "linear_iterations", "termination_reason", "gradient_norm", "cost_history",
            "lambda_history", "linear_iterations_history", "linear_converged_history",
            "trial_history", "linear_restarts", "linear_residual_checks",
            "linear_relative_residual_history", "reduced_dim")
    return {k: getattr(s, k) for k in keys}


def arr(x):
    return x.detach().cpu().numpy() if torch.is_tensor(x) else np.asarray(x)


def linearization_record(prefix, lin, out, columns=True):
    out[prefix + "residual"] = arr(lin.residual)
    if lin.raw_residual is not None:
        out[prefix + "raw_residual"] = arr(lin.raw_residual)
    out[prefix + "cost"] = np.asarray(float(lin.cost))
    out[prefix + "gradient"] = arr(lin.gradient)
    for i, d in enumerate(lin.jacobian.diagonal_blocks()):
        out[f"{prefix}diag{i}"] = arr(d)
    for gi, g in enumerate(lin.jacobian.groups):
        for si, b in enumerate(g.blocks):
            out[f"{prefix}block{gi}_{si}"] = arr(b)
            if columns:
                out[f"{prefix}columns{gi}_{si}"] = arr(g.columns[si])


def main(reference, only=None):
    """Write every fixture, or (``only``) just the named problems of the
    second list, merging their summaries into the existing summaries.json."""
    sys.path.insert(0, reference)
    import torchls as tls
    from torchls.geometry import sim3_exp
    from torchls.schur import SchurLinearization, SchurPlan

    import problems as P
    from torchls_b200 import synthetic

    torch.set_num_threads(8)
    summaries = {}
    if only:
        with open(os.path.join(HERE, "summaries.json")) as fh:
            summaries = json.load(fh)

    # ---------------------------------------------------------------- Sim(3) retraction known answers
    if not only or "sim3_exp" in only:
        pose, delta = P.sim3_exp_cases()
        np.savez_compressed(os.path.join(HERE, "sim3_exp.npz"), pose=arr(pose), delta=arr(delta),
                            result=arr(pose @ sim3_exp(delta)))

    # ---------------------------------------------------------------- typed API (Cost.factory / VarValues)
    if not only or "typed_ba" in only:
        problem, init = P.typed_ba(tls)
        rec = {"offsets": np.array([e.offset for e in problem.layout]),
               "dims": np.array([e.dim for e in problem.layout])}
        for i, e in enumerate(problem.layout):
            rec[f"ids{i}"] = arr(e.ids)
        linearization_record("", problem.linearize(init), rec)
        sol, summ = problem.solve(init, return_summary=True, linear_solver="schur_cg",
                                  eliminate=problem.layout[0].var_type)
        for i, e in enumerate(problem.layout):
            rec[f"solve{i}"] = arr(sol._values[e.var_type])
        summaries["typed_ba"] = summary_dict(summ)
        np.savez_compressed(os.path.join(HERE, "typed_ba.npz"), **rec)
        print("typed_ba", summ.final_cost, summ.termination_reason, summ.iterations)

    # ---------------------------------------------------------------- fixed linear system / LAD
    if not only or "fixed_system" in only:
        from torchls.linear_system import FixedLinearSystem, least_absolute_deviations

        A, x, y, w, target = P.fixed_system_case()
        fs = FixedLinearSystem(A.to_sparse())
        rec = dict(A=arr(A), x=arr(x), y=arr(y), w=arr(w), target=arr(target))
        rec["matvec"] = arr(fs.matvec(x))
        rec["rmatvec"] = arr(fs.rmatvec(y))
        rec["matvec1"] = arr(fs.matvec(x[:, 0]))
        fac = fs.factor(w, ridge=0.1)
        rec["weighted_ls"] = arr(fac.least_squares(target))
        rec["cholesky"] = arr(fac.cholesky)
        rec["solve"] = arr(fs.factor().solve(x))
        lad = least_absolute_deviations(fs, target, rho=0.3, max_iterations=200)
        rec["lad_solution"] = arr(lad.solution)
        rec["lad_iterations"] = np.asarray(lad.iterations)
        rec["lad_converged"] = np.asarray(lad.converged)
        lad1 = least_absolute_deviations(fs, target[:, 0], rho=1.0, max_iterations=60)
        rec["lad1_solution"] = arr(lad1.solution)
        rec["lad1_iterations"] = np.asarray(lad1.iterations)
        np.savez_compressed(os.path.join(HERE, "fixed_system.npz"), **rec)
        print("fixed_system LAD", lad.iterations, lad.converged, lad1.iterations)

    # ---------------------------------------------------------------- general Schur system products
    if not only or "schur_general" in only:
        rec = {}
        g = torch.Generator().manual_seed(31)
        for tag, builder, groups in (("intr", P.ba_intrinsics, ()), ("joint", P.ba_intrinsics, (("cams", "focal"),)),
                                     ("priors", P.ba_priors, ()), ("two", P.ba_two_groups, ())):
            p = builder(tls)
            an = p._ensure_analyzed()
            lin = p.linearize()
            J = lin.jacobian
            plan = SchurPlan(an, "points", torch.device("cpu"), preconditioner_groups=groups)
            slin = SchurLinearization(J, J.diagonal_blocks(), plan, dense=True)
            system = slin.damped(1e-3)
            vc = torch.randn(plan.dim, generator=g, dtype=torch.float64)
            rec[f"{tag}_vc"] = arr(vc)
            rec[f"{tag}_reduced_rhs"] = arr(system.reduced_rhs(-lin.gradient))
            rec[f"{tag}_matvec"] = arr(system.matvec(vc))
            rec[f"{tag}_preconditioner"] = arr(system.preconditioner()(vc))
            rec[f"{tag}_backsubstitute"] = arr(system.backsubstitute(vc))
            rec[f"{tag}_dense"] = arr(system.dense_matrix())
        np.savez_compressed(os.path.join(HERE, "schur_general.npz"), **rec)

    # ---------------------------------------------------------------- small BA (stored inputs)
    data = synthetic.small_bundle_adjustment(0)
    if only:
        data = None
    if data is not None:
        _small_ba(tls, P, data, summaries, SchurLinearization, SchurPlan)

    # ---------------------------------------------------------------- other problems
    others = {
        "ba_tiny": (P.ba_tiny, dict(linear_solver="schur_cg", eliminate="points")),
        "ba_tiny_gn": (P.ba_tiny, dict(linear_solver="conjugate_gradient", trust_region=None,
                                       termination=tls.TerminationConfig(max_iterations=8))),
        "pose_small": (P.pose_small, dict(linear_solver="conjugate_gradient",
                                          termination=tls.TerminationConfig(max_iterations=30))),
        "sim3_small": (P.sim3_small, dict(linear_solver="conjugate_gradient",
                                          termination=tls.TerminationConfig(max_iterations=30))),
        "se2_custom": (P.se2_custom, dict(linear_solver="conjugate_gradient")),
        "ba_two_groups": (P.ba_two_groups, dict(linear_solver="schur_cg", eliminate="points")),
        "ba_priors": (P.ba_priors, dict(linear_solver="schur_cg", eliminate="points")),
        "ba_priors_dense": (P.ba_priors, dict(linear_solver="schur_dense", eliminate="points")),
        "ba_intrinsics": (P.ba_intrinsics, dict(linear_solver="schur_cg", eliminate="points")),
        "ba_intrinsics_joint": (P.ba_intrinsics, dict(linear_solver="schur_cg", eliminate="points",
                                                      conjugate_gradient=tls.ConjugateGradientConfig(
                                                          preconditioner_groups=(("cams", "focal"),)))),
        "curve_bounds": (P.curve_bounds, dict(bounds=P.CURVE_BOUNDS)),
        "rotations_small": (P.rotations_small, dict(jacobi_scaling=True, trust_region=tls.TrustRegionConfig(
            lambda_initial=1e-3, strategy="adaptive", damping_mode="diagonal"))),
        "rotations_small_qr": (P.rotations_small, dict(linear_solver="dense_qr", jacobi_scaling=True,
                                                       trust_region=tls.TrustRegionConfig(
                                                           lambda_initial=1e-3, strategy="adaptive",
                                                           damping_mode="diagonal"))),
        "ba_tiny_qr": (P.ba_tiny, dict(linear_solver="dense_qr")),
        "alias_weights": (P.alias_weights, dict()),
        "alias_cauchy": (lambda api, **k: P.alias_weights(api, loss=P.cauchy_loss(api)), dict()),
        "alias_softsq": (lambda api, **k: P.alias_weights(api, loss=P.soft_square_loss(api)), dict()),
        "joint_groups": (P.joint_groups, dict(conjugate_gradient=tls.ConjugateGradientConfig(
            preconditioner_groups=(("off", "pts"),)))),
    }
    for name, (builder, opts) in others.items():
        if only and name not in only:
            continue
        rec = {}
        p = builder(tls)
        linearization_record("", p.linearize(), rec)
        sol, summ = builder(tls).solve(return_summary=True, **opts)
        for k, val in sol.items():
            rec[f"solve_{k}"] = arr(val)
        summaries[name] = summary_dict(summ)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **rec)
        print(name, summ.final_cost, summ.termination_reason, summ.iterations)

    with open(os.path.join(HERE, "summaries.json"), "w") as fh:
        json.dump(summaries, fh, indent=1, default=float)
    if "ba_small_schur_cg" in summaries:
        print("ba_small", summaries["ba_small_schur_cg"]["final_cost"])


def _small_ba(tls, P, data, summaries, SchurLinearization, SchurPlan):
    """The small bundle adjustment with stored inputs: per-kernel products, the
    Schur system and full solves under several options."""
    out = {
        "cameras_true": arr(data.cameras_true), "points_true": arr(data.points_true),
        "cameras_init": arr(data.cameras_init), "points_init": arr(data.points_init),
        "camera_index": arr(data.camera_index), "point_index": arr(data.point_index), "uv": arr(data.uv),
    }
    prob = P.ba_small(tls, data=data)
    analyzed = prob._ensure_analyzed()
    out["layout_offsets"] = np.array([e.offset for e in analyzed.layout])
    lin = prob.linearize()
    linearization_record("", lin, out, columns=False)
    J = lin.jacobian
    n = J.shape[1]
    g = torch.Generator().manual_seed(1)
    v = torch.randn(n, generator=g, dtype=torch.float64)
    u = torch.randn(J.shape[0], generator=g, dtype=torch.float64)
    out["v"], out["u"] = arr(v), arr(u)
    out["normal_matvec"] = arr(J.normal_matvec(v, 1e-3))
    out["matvec"] = arr(J.matvec(v))
    out["rmatvec"] = arr(J.rmatvec(u))
    out["squared_matvec_norm"] = np.asarray(float(J.squared_matvec_norm(v)))
    apply = tls.block_jacobi(J, 1e-3)
    out["block_jacobi_apply"] = arr(apply(v))
    res = tls.pcg(lambda x: J.normal_matvec(x, 1e-3), -lin.gradient, preconditioner=apply,
                  config=tls.ConjugateGradientConfig())
    out["pcg_solution"] = arr(res.solution)
    summaries["ba_small_pcg"] = dict(iterations=res.iterations, residual_norm=res.residual_norm,
                                     converged=res.converged, reason=res.reason, restarts=res.restarts,
                                     residual_checks=res.residual_checks, rhs_norm=res.rhs_norm)
    plan = SchurPlan(analyzed, "points", torch.device("cpu"))
    out["schur_edges_r"] = arr(plan.edges[0][0])
    out["schur_edges_e"] = arr(plan.edges[0][1])
    out["schur_row_ptr"] = arr(plan.row_ptr)
    out["schur_columns"] = arr(plan.columns)
    out["schur_value_order"] = arr(plan.value_order)
    slin = SchurLinearization(J, J.diagonal_blocks(), plan, dense=True)
    system = slin.damped(1e-3)
    vc = torch.randn(plan.dim, generator=g, dtype=torch.float64)
    out["vc"] = arr(vc)
    out["schur_reduced_rhs"] = arr(system.reduced_rhs(-lin.gradient))
    out["schur_matvec"] = arr(system.matvec(vc))
    out["schur_preconditioner"] = arr(system.preconditioner()(vc))
    out["schur_backsubstitute"] = arr(system.backsubstitute(vc))
    out["schur_dense"] = arr(system.dense_matrix())
    out["schur_cross"] = arr(slin.cross[0])

    term30 = tls.TerminationConfig(max_iterations=30)
    runs = {
        "schur_cg": dict(linear_solver="schur_cg", eliminate="points", termination=term30, record_trials=True),
        "conjugate_gradient": dict(linear_solver="conjugate_gradient", termination=term30),
        "schur_dense": dict(linear_solver="schur_dense", eliminate="points", termination=term30),
        "scaled_adaptive": dict(
            linear_solver="schur_cg", eliminate="points", termination=term30, jacobi_scaling=True,
            trust_region=tls.TrustRegionConfig(strategy="adaptive", damping_mode="diagonal")),
        "forced": dict(
            linear_solver="schur_cg", eliminate="points", record_trials=True,
            termination=tls.TerminationConfig(max_iterations=30, cost_tolerance=0, gradient_tolerance=0,
                                              parameter_tolerance=0)),
    }
    for name, opts in runs.items():
        p = P.ba_small(tls, data=data)
        sol, summ = p.solve(return_summary=True, **opts)
        out[f"solve_{name}_cams"] = arr(sol["cams"])
        out[f"solve_{name}_points"] = arr(sol["points"])
        summaries[f"ba_small_{name}"] = summary_dict(summ)
    np.savez_compressed(os.path.join(HERE, "ba_small.npz"), **out)


if __name__ == "__main__":
    sys.path.insert(0, HERE)
    ref = sys.argv[1] if len(sys.argv) > 1 and not sys.argv[1].startswith("--") else os.environ.get(
        "TORCHLS_REFERENCE")
    if not ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path to the torchls checkout> "
                 "(or set TORCHLS_REFERENCE)")
    only = sys.argv[sys.argv.index("--only") + 1].split(",") if "--only" in sys.argv else None
    main(ref, only)
