"""The paired block update of the full-system PCG against the general one.

When the preconditioner is one group of one variable type whose blocks are
D contiguous columns with a D x D factor (a pose graph), and every vector and
factor is 16-byte aligned, the multi-kernel PCG reads and writes vectors and
factor rows in pairs. It computes what the general update computes (an
8-byte-offset right-hand side sends the same solve down the general path)
from a different code shape, and its results differ from the general path's
at rounding level: the two agree to rounding, each is bitwise reproducible
run to run, and both match the generic PCG like every device path.
"""

from __future__ import annotations

from functools import partial

import pytest
import torch

from gpu_helpers import close, needs_gpu

pytestmark = [pytest.mark.gpu, needs_gpu]

DEV = "cuda"


def test_paired_update_matches_the_general_update():
    import torchls_b200 as tls
    from torchls_b200 import synthetic

    data = synthetic.make_pose_graph(10_000, 30_000, seed=3)
    prob = synthetic.build_pose_graph(data, tls, device=DEV)
    lin = prob.linearize()
    J = lin.jacobian
    pre = tls.block_jacobi(J, 1e-3)
    assert len(pre.groups) == 1 and int(pre.groups[0].count) > 8192  # the multi-kernel path
    matvec = partial(J.normal_matvec, damping=1e-3)
    rhs = (-lin.gradient).contiguous()
    cfg = tls.ConjugateGradientConfig(rtol=1e-8, max_iterations=60)
    paired = tls.pcg(matvec, rhs, preconditioner=pre, config=cfg)
    again = tls.pcg(matvec, rhs, preconditioner=pre, config=cfg)
    assert torch.equal(paired.solution, again.solution), "not reproducible"
    shifted = torch.empty(rhs.numel() + 1, dtype=rhs.dtype, device=rhs.device)[1:]
    shifted.copy_(rhs)
    assert shifted.data_ptr() % 16 != 0
    general = tls.pcg(matvec, shifted, preconditioner=pre, config=cfg)
    assert abs(paired.iterations - general.iterations) <= 1 and general.iterations > 5
    assert paired.reason == general.reason
    close(paired.solution, general.solution, 1e-8, what="paired against general update")
    generic = tls.pcg(lambda v: J.normal_matvec(v, 1e-3), rhs, preconditioner=(lambda v: pre(v)), config=cfg)
    assert abs(paired.iterations - generic.iterations) <= 1
    close(paired.solution, generic.solution, 1e-6, what="pcg solution")
