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


def test_warp_tiles_match_cta_chunks():
    """Float32 W in 64-edge warp tiles (each warp streams and reduces its own
    tiles) against the 512-edge CTA chunks on the same system: the reduced
    rhs, the operator and the persistent PCG agree to rounding."""
    import torchls_b200 as tls
    from torchls_b200 import synthetic
    from torchls_b200.schur import SchurLinearization, SchurPlan

    data = synthetic.make_bundle_adjustment(40, 3000, 6, seed=21)
    prob = synthetic.build_bundle_adjustment(data, tls, device=DEV, loss=tls.HuberLoss(0.01))
    an = prob._ensure_analyzed()
    out = {}
    for name, max_dim in (("tiles", SchurPlan.TILE_MAX_DIM), ("chunks", 0)):
        plan = SchurPlan(an, "points", torch.device(DEV))
        plan.TILE_MAX_DIM = max_dim
        lin = prob.linearize(jacobian_dtype=torch.float32, schur=plan)
        slin = SchurLinearization(plan, lin, lin.jacobian.diagonal_blocks(), None, wdtype=torch.float32,
                                  vec_dtype=torch.float64)
        assert slin.layout.cap == (64 if name == "tiles" else 512)
        system = slin.damped(1e-3)
        rhs = system.reduced_rhs(-lin.gradient)
        v = torch.linspace(-1.0, 1.0, plan.dim, dtype=torch.float64, device=DEV)
        res = tls.pcg(system.matvec, rhs, preconditioner=system.preconditioner(),
                      config=tls.ConjugateGradientConfig(rtol=1e-8, max_iterations=400))
        out[name] = (rhs, system.matvec(v), res)
        assert int(plan.err.item()) == 0
    close(out["tiles"][0], out["chunks"][0], 1e-12, what="reduced rhs")
    close(out["tiles"][1], out["chunks"][1], 1e-12, what="matvec")
    assert abs(out["tiles"][2].iterations - out["chunks"][2].iterations) <= 1
    close(out["tiles"][2].solution, out["chunks"][2].solution, 1e-7, what="pcg solution")
