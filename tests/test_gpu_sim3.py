"""Sim(3) on the GPU: the retraction kernel against the reference's
``pose @ sim3_exp(delta)`` (torch.matrix_exp) fixtures, and the fused
``sim3_between`` linearization kernel against ``vmap(jacrev)`` of the same
torch residual (the path the reference takes for it).

The fused kernel evaluates r = log(Z^-1 S_i^-1 S_j) in closed form and the
Jacobian as J_j = J_r^-1(r), J_i = -J_r^-1(r) Ad(S_j^-1 S_i), with J_r^-1 taken
by forward-mode dual numbers through the log; torch.func differentiates the
torch formula of the same log. Both must agree to 1e-10 relative (blocks) and
1e-12 (residuals), including rotations near pi and scale changes of e^2.
"""

from __future__ import annotations

import types

import pytest
import torch

from gpu_helpers import close, load, needs_gpu
from golden import problems as P

pytestmark = [pytest.mark.gpu, needs_gpu]

DEV = "cuda"


def test_sim3_retraction_matches_reference_exp():
    import torchls_b200 as tls
    from torchls_b200.kernels import retract_group

    fx = load("sim3_exp")
    pose = torch.from_numpy(fx["pose"]).to(DEV)
    delta = torch.from_numpy(fx["delta"]).to(DEV)
    entry = types.SimpleNamespace(var_type=tls.Sim3Var, count=pose.shape[0], dim=7)
    got = retract_group(entry, pose.contiguous(), delta.reshape(-1))
    close(got, fx["result"], 1e-13, what="Sim(3) retraction")


def _problems(tls, hard):
    from torchls_b200 import residuals, synthetic

    data = synthetic.make_sim3_pose_graph(200, 600, seed=9, scale_sigma=0.05)
    if hard:  # large relative rotations and scales: near-pi rotations, e^(+-2) scale ratios
        g = torch.Generator().manual_seed(4)
        from torchls_b200.geometry import sim3_exp

        xi = torch.randn(len(data.measurements), 7, generator=g, dtype=torch.float64)
        xi[:, 3:6] *= 3.0 / xi[:, 3:6].norm(dim=-1, keepdim=True).clamp_min(1e-9) * torch.rand(
            len(xi), 1, generator=g, dtype=torch.float64)
        data.measurements = data.measurements @ sim3_exp(xi)
    fused = synthetic.build_pose_graph(data, tls, device=DEV, sim3=True)
    # the same torch residual without its fused-kernel tag: linearized by vmap(jacrev)
    plain = synthetic.build_pose_graph(data, tls, device=DEV, sim3=True,
                                       residual=lambda a, b, z: residuals.sim3_between(a, b, z))
    return fused, plain


@pytest.mark.parametrize("hard", [False, True])
def test_fused_sim3_between_matches_torch_func(hard):
    import torchls_b200 as tls

    fused, plain = _problems(tls, hard)
    a, b = fused.linearize(), plain.linearize()
    close(a.residual, b.residual, 1e-12, 1e-15, what="residual")
    close(a.gradient, b.gradient, 1e-10, 1e-13, what="gradient")
    for ga, gb in zip(a.jacobian.groups, b.jacobian.groups):
        for ba_, bb in zip(ga.blocks, gb.blocks):
            close(ba_, bb, 1e-10, 1e-13, what="Jacobian block")
    for da, db in zip(a.jacobian.diagonal_blocks(), b.jacobian.diagonal_blocks()):
        close(da, db, 1e-10, 1e-13, what="diagonal block")


def test_fused_sim3_between_is_the_kernel_path():
    """The tagged residual runs the fused kernel (no torch.func trace)."""
    import torchls_b200 as tls
    from torchls_b200 import _lib as L

    fused, _ = _problems(tls, False)
    an = fused._ensure_analyzed()
    kinds = [plan.builtin(an.layout) for plan in an.plans]
    assert all(k is not None and k[0] == L.RES_SIM3_BETWEEN for k in kinds)
    lin = fused.linearize()
    assert all(not plan._linearizers for plan in an.plans)
    assert torch.isfinite(lin.residual).all()
