"""Every device PCG path against the generic PCG (the reference's step order on
torch callables) on the same operator.

The device loop has four shapes, chosen by size: the persistent Schur-PCG
kernel with the vector CTA (small reduced systems), the persistent kernel
whose vector phase runs in the last CTA through the grid barrier (reduced
systems too large for one CTA's shared memory), the single-block step for
full systems with at most 8,192 preconditioner blocks, and the multi-kernel
update/direction loop beyond that. Each must take the same number of
iterations as the generic loop (within one, as dot products are summed in a
different order) and reach the same solution.
"""

from __future__ import annotations

from functools import partial

import pytest
import torch

from gpu_helpers import close, needs_gpu

pytestmark = [pytest.mark.gpu, needs_gpu]

DEV = "cuda"


def _compare(tls, matvec, rhs, pre, device_matvec=None):
    cfg = tls.ConjugateGradientConfig(rtol=1e-8, max_iterations=400)
    generic = tls.pcg(lambda v: matvec(v), rhs, preconditioner=(lambda v: pre(v)), config=cfg)
    device = tls.pcg(device_matvec or matvec, rhs, preconditioner=pre, config=cfg)
    assert device.reason == generic.reason, (device.reason, generic.reason)
    assert abs(device.iterations - generic.iterations) <= 1, (device.iterations, generic.iterations)
    close(device.solution, generic.solution, 1e-6, what="pcg solution")
    return device


def _schur_system(tls, cams, points, views, seed):
    from torchls_b200 import synthetic
    from torchls_b200.schur import SchurLinearization, SchurPlan

    data = synthetic.make_bundle_adjustment(cams, points, views, seed=seed)
    prob = synthetic.build_bundle_adjustment(data, tls, device=DEV, loss=tls.HuberLoss(0.01))
    an = prob._ensure_analyzed()
    plan = SchurPlan(an, "points", torch.device(DEV))
    lin = prob.linearize(jacobian_dtype=torch.float32, schur=plan)
    slin = SchurLinearization(plan, lin, lin.jacobian.diagonal_blocks(), None, wdtype=torch.float32,
                              vec_dtype=torch.float64)
    system = slin.damped(1e-3)
    rhs = system.reduced_rhs(-lin.gradient)
    return plan, system, rhs


@pytest.mark.parametrize("cams", [40, 420])  # 234 and 2,514 reduced unknowns
def test_persistent_schur_pcg_matches_generic(cams):
    import torchls_b200 as tls

    plan, system, rhs = _schur_system(tls, cams, 3000, 6, seed=21)
    pre = system.preconditioner()
    res = _compare(tls, system.matvec, rhs, pre)
    assert res.iterations > 5
    assert int(plan.err.item()) == 0


@pytest.mark.parametrize("points", [500, 9000])  # below and above 8,192 preconditioner blocks
def test_full_system_pcg_matches_generic(points):
    import torchls_b200 as tls
    from torchls_b200 import synthetic

    data = synthetic.make_bundle_adjustment(12, points, 4, seed=22)
    prob = synthetic.build_bundle_adjustment(data, tls, device=DEV, loss=tls.HuberLoss(0.01))
    lin = prob.linearize()
    J = lin.jacobian
    pre = tls.block_jacobi(J, 1e-3)
    matvec = partial(J.normal_matvec, damping=1e-3)
    res = _compare(tls, lambda v: J.normal_matvec(v, 1e-3), -lin.gradient, pre, device_matvec=matvec)
    assert res.iterations > 5
