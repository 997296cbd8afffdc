"""CPU checks of the implicit adjoint's ingredients (no GPU needed).

The objective used by the adjoint must equal the oracle's cost for the same
problem (weights, Huber loss, shared data and the scale prior included), its
tangent-space gradient must match finite differences, and the Hessian-vector
product must be symmetric and match finite differences of the gradient.
"""

from __future__ import annotations

import numpy as np
import torch

import oracle
import torchls_b200 as tls
from golden import problems as P
from torchls_b200 import synthetic
from torchls_b200.adjoint import _groups, objective
from torchls_b200.variables import ParameterRef


def _tiny():
    data = synthetic.make_bundle_adjustment(5, 40, 3, seed=11)
    prob, inputs = synthetic.build_differentiable_bundle_adjustment(data, tls, loss=tls.HuberLoss(0.01))
    return data, prob, inputs


def test_objective_matches_oracle_cost():
    data, prob, inputs = _tiny()
    inputs["w_free"].uniform_(0.5, 2.0, generator=torch.Generator().manual_seed(2))
    ref = P.OracleAPI.Problem({k: v for k, v in prob.parameters.items()}, prob.manifolds and {"cams": "se3"})
    for cost in prob._costs:
        args = [(a.name, torch.as_tensor(a.id)) if isinstance(a, ParameterRef) else a for a in cost.args]
        ref.add_residual(cost.residual_fn, *args, in_dims=cost.in_dims, loss=cost.loss and P.OracleAPI.HuberLoss(0.01),
                         weights=cost.weights)
    want = ref.inner.cost(ref.inner.values())
    got = float(objective(prob, prob.parameters))
    assert abs(got - want) <= 1e-13 * abs(want), (got, want)


def test_gradient_and_hvp_match_finite_differences():
    data, prob, inputs = _tiny()
    _, n = _groups(prob)
    vals = prob.parameters
    gen = torch.Generator().manual_seed(4)
    d0 = 1e-3 * torch.randn(n, generator=gen, dtype=torch.float64)
    v = torch.randn(n, generator=gen, dtype=torch.float64)
    w = torch.randn(n, generator=gen, dtype=torch.float64)

    def grad_at(d):
        d = d.clone().requires_grad_(True)
        f = objective(prob, vals, d)
        (g,) = torch.autograd.grad(f, d, create_graph=True)
        return d, g

    d, g = grad_at(d0)
    (hv,) = torch.autograd.grad(g, d, grad_outputs=v, retain_graph=True)
    (hw,) = torch.autograd.grad(g, d, grad_outputs=w)
    # symmetry of the chart Hessian: w.Hv == v.Hw
    assert abs(float(w @ hv - v @ hw)) <= 1e-10 * float(hv.norm() * w.norm())
    # directional derivative of F and of its gradient
    h = 1e-6
    fp = float(objective(prob, vals, d0 + h * v))
    fm = float(objective(prob, vals, d0 - h * v))
    np.testing.assert_allclose((fp - fm) / (2 * h), float(g.detach() @ v), rtol=1e-6)
    _, gp = grad_at(d0 + h * v)
    _, gm = grad_at(d0 - h * v)
    fd = (gp - gm).detach() / (2 * h)
    assert float((fd - hv).norm()) <= 1e-5 * float(hv.norm())


def test_objective_matches_oracle_on_small_ba():
    # the adjoint objective and the oracle restatement agree on the 4,000-observation problem
    data = synthetic.small_bundle_adjustment(0)
    prob = synthetic.build_bundle_adjustment(data, tls, loss=tls.HuberLoss(0.01))
    op = P.oracle_problem(P.ba_small)
    want = op.cost(op.values())
    assert isinstance(op, oracle.OracleProblem)
    assert abs(float(objective(prob, prob.parameters)) - want) <= 1e-12 * want
