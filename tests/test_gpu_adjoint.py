"""Implicit-function-theorem adjoint of the CUDA LM solve.

Checks: (1) gradients of the bundle-adjustment loss with respect to every
observation match torch.autograd through the reference's own unrolled
float64 Gauss-Newton steps (fixture from tests/golden/make_adjoint_golden.py)
to 1e-6 relative; (2) gradients with respect to observations and
per-observation weights match central finite differences (step 1e-6, float64
re-solves, each polished to the exact stationary point by two Newton steps)
to 1e-6 relative. Weights are detached in the reference, so their
gradients are pinned by finite differences alone.
"""

from __future__ import annotations

import pytest
import torch

from gpu_helpers import close, load, needs_gpu

pytestmark = [pytest.mark.gpu, needs_gpu]

DEV = "cuda"


def _tight(tls):
    return dict(linear_solver="schur_dense", eliminate="points",
                termination=tls.TerminationConfig(max_iterations=80, cost_tolerance=1e-15, gradient_tolerance=1e-16,
                                                  parameter_tolerance=1e-15))


def test_adjoint_matches_unrolled_reference_gradients():
    import torchls_b200 as tls
    from torchls_b200 import synthetic
    from torchls_b200.adjoint import solve_implicit

    fx = load("adjoint_small")
    data = synthetic.small_bundle_adjustment(0)
    prob, inp = synthetic.build_differentiable_bundle_adjustment(data, tls, device=DEV, loss=tls.HuberLoss(0.01))
    uv = [inp["uv_free"].requires_grad_(True), inp["uv_fixed"].requires_grad_(True)]
    opts = _tight(tls)
    elim = opts.pop("eliminate")
    sol = solve_implicit(prob, uv, eliminate=elim, **opts)
    loss = synthetic.differentiable_loss(sol, data)
    grads = torch.autograd.grad(loss, uv)
    close(sol["points"], fx["points"], 1e-8, what="points")
    close(sol["cams"], fx["cams"], 1e-8, what="cams")
    # the loss sums squares of (solved - true) point and camera differences of
    # about 1e-3: parameters pinned to 1e-8 relative move it by up to ~1e-7
    # relative (6e-13 absolute on 4.9e-5 in one run), so it is checked there
    close(loss.detach(), fx["loss"], 1e-7, what="loss")
    close(grads[0], fx["grad_uv_free"], 1e-6, what="d loss / d uv (free cameras)")
    close(grads[1], fx["grad_uv_fixed"], 1e-6, what="d loss / d uv (fixed camera)")
    assert solve_implicit.last["refinement_history"][-1] <= 1e-12


def test_adjoint_matches_central_finite_differences():
    import torchls_b200 as tls
    from torchls_b200 import synthetic
    from torchls_b200.adjoint import newton_polish, solve_implicit

    data = synthetic.make_bundle_adjustment(6, 80, 4, seed=5)
    prob, inp = synthetic.build_differentiable_bundle_adjustment(data, tls, device=DEV, loss=tls.HuberLoss(0.01))
    init = {k: v.clone() for k, v in prob.parameters.items()}
    theta = [inp["uv_free"].requires_grad_(True), inp["w_free"].requires_grad_(True)]
    opts = _tight(tls)
    elim = opts.pop("eliminate")
    sol = solve_implicit(prob, theta, eliminate=elim, **opts)
    grads = torch.autograd.grad(synthetic.differentiable_loss(sol, data), theta)

    def loss_now():
        prob.parameters = {k: v.clone() for k, v in init.items()}
        prob.refresh_data()
        prob.solve(eliminate=elim, **opts)
        # LM converges the cost, not the parameters, to rounding level: polish with Newton steps
        s = newton_polish(prob, eliminate=elim)
        return float(synthetic.differentiable_loss(s, data))

    gen = torch.Generator().manual_seed(9)
    h = 1e-6
    checked, errors = [], []
    for t, g in zip(theta, grads):
        flat, gflat = t.view(-1), g.reshape(-1)
        for k in torch.randperm(flat.numel(), generator=gen)[:6].tolist():
            with torch.no_grad():
                base = float(flat[k])
                flat[k] = base + h
                lp = loss_now()
                flat[k] = base - h
                lm = loss_now()
                flat[k] = base
            fd = (lp - lm) / (2 * h)
            checked.append(float(gflat[k]))
            errors.append(abs(fd - float(gflat[k])))
    prob.refresh_data()
    scale = max(abs(c) for c in checked)
    assert max(errors) <= 1e-6 * scale + 1e-12, (max(errors), scale, checked)
