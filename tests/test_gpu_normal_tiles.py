"""One-pass normal operator (tile plan) on the GPU.

The tiled operator y = diag(s) J^T J diag(s) x + lambda x must agree with
the two-pass operator (factor pass + per-variable gather) and with the
reference's fixture to 1e-12 relative, for float64 and float32 Jacobians,
with a column scale and damping, on the small bundle adjustment (two factor
groups: the fixed camera's observations form a one-slot group) and on a
pose graph (SE(3) between factors plus the edges of the fixed first pose;
its loop closures come in random order, so the plan reorders the factors
and the operator reads a tile-ordered copy of J). It must be bitwise reproducible, and a PCG driven through
it must take the reference's iteration count. ``tls_permute_columns`` (the
tile-ordered copy of J) must equal torch's column gather.
"""

from __future__ import annotations

import pytest
import torch

from gpu_helpers import SUMMARIES, close, load, needs_gpu, stored_ba
from golden import problems as P

pytestmark = [pytest.mark.gpu, needs_gpu]

DEV = "cuda"


@pytest.fixture(scope="module")
def tls():
    import torchls_b200 as tls

    return tls


def _ba_jacobian(tls, dtype=None):
    fx = load("ba_small")
    prob = P.ba_small(tls, device=DEV, data=stored_ba(fx))
    lin = prob.linearize(jacobian_dtype=dtype) if dtype is not None else prob.linearize()
    return fx, lin


def test_plan_is_used_and_matches_two_pass_and_fixture(tls):
    fx, lin = _ba_jacobian(tls)
    J = lin.jacobian
    assert J.structure.normal_tiles() is not None, "no tile plan for the small bundle adjustment"
    v = torch.from_numpy(fx["v"]).to(DEV)
    tiled = J.normal_matvec(v, 1e-3)
    two = J.normal_matvec(v, 1e-3, tiles=False)
    close(tiled, fx["normal_matvec"], 1e-12, what="tiled vs fixture")
    close(tiled, two, 1e-12, what="tiled vs two-pass")
    assert torch.equal(tiled, J.normal_matvec(v, 1e-3)), "tiled normal matvec is not bitwise reproducible"


@pytest.mark.parametrize("jdtype", [torch.float32, torch.float64])
def test_scaled_and_float32(tls, jdtype):
    fx, lin = _ba_jacobian(tls, jdtype)
    J = lin.jacobian
    gen = torch.Generator().manual_seed(11)
    s = (0.5 + torch.rand(J.shape[1], generator=gen, dtype=torch.float64)).to(DEV)
    Js = J.scale_columns(s)
    v = torch.randn(J.shape[1], generator=gen, dtype=torch.float64).to(DEV)
    close(Js.normal_matvec(v, 0.25), Js.normal_matvec(v, 0.25, tiles=False), 1e-12, what="scaled, float64 vectors")
    if jdtype == torch.float32:
        v32 = v.float()
        a, b = Js.normal_matvec(v32, 0.25), Js.normal_matvec(v32, 0.25, tiles=False)
        assert a.dtype == torch.float32
        close(a, b, 1e-6, what="float32 vectors")


def test_pose_graph(tls):
    from torchls_b200 import synthetic

    data = synthetic.make_pose_graph(400, 1200, seed=4)
    prob = synthetic.build_pose_graph(data, tls, device=DEV)
    J = prob.linearize().jacobian
    tiles = J.structure.normal_tiles()
    assert tiles is not None
    assert tiles.perm[0] is not None, "loop closures in random order should be put in tile order"
    gen = torch.Generator().manual_seed(5)
    v = torch.randn(J.shape[1], generator=gen, dtype=torch.float64).to(DEV)
    for damping in (0.0, 1e-2):
        a = J.normal_matvec(v, damping)
        close(a, J.normal_matvec(v, damping, tiles=False), 1e-12, what=f"pose graph, damping {damping}")
        assert torch.equal(a, J.normal_matvec(v, damping))
    stats = J.structure.normal_tiles().plan.stats
    assert stats["final_runs"] + stats["acc_runs"] + stats["partial_runs"] == stats["nruns"]


def test_device_pcg_through_tiles(tls):
    from functools import partial

    fx, lin = _ba_jacobian(tls)
    J = lin.jacobian
    res = tls.pcg(partial(J.normal_matvec, damping=1e-3), -lin.gradient, preconditioner=tls.block_jacobi(J, 1e-3),
                  config=tls.ConjugateGradientConfig())
    ref = SUMMARIES["ba_small_pcg"]
    assert (res.iterations, res.reason) == (ref["iterations"], ref["reason"])
    close(res.solution, fx["pcg_solution"], 1e-8, what="pcg solution")
    two = tls.pcg(partial(J.normal_matvec, damping=1e-3, tiles=False), -lin.gradient,
                  preconditioner=tls.block_jacobi(J, 1e-3), config=tls.ConjugateGradientConfig())
    assert two.iterations == res.iterations
    close(res.solution, two.solution, 1e-10, what="tiled vs two-pass PCG")


def test_permute_columns():
    from torchls_b200 import _lib as L

    gen = torch.Generator().manual_seed(2)
    for dtype in (torch.float32, torch.float64):
        src = torch.randn(7, 1001, generator=gen, dtype=dtype).to(DEV)
        perm = torch.randperm(1000, generator=gen).to(torch.int32).to(DEV)
        dst = torch.full((7, 1000), float("nan"), dtype=dtype, device=DEV)
        L.call("tls_permute_columns", src.data_ptr(), dst.data_ptr(), L.dtype_code(dtype), 7, 1000, 1001,
               perm.data_ptr(), L.stream_handle(src.device))
        assert torch.equal(dst, src[:, perm.long()])
