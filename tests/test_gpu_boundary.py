"""The reference-facing operator plans on Jacobians in the reference's layout.

``CudaNormalPlan(J).bind(J).normal_matvec(v, damping)`` and
``CudaDiagonalPlan(J).diagonal_blocks(J)`` are the calls torchls makes on its
GPU plans (warp_normal.py:125-294, warp_diagonal.py:69-179). Here ``J`` is a
plain stand-in with the reference's ``BlockJacobian`` fields (per batch and
slot: blocks [N, r, d], global columns [N, d], type indices, variable
indices; ``layout``; ``shape``) filled with the blocks torchls itself wrote to
the fixtures, so the products are compared with torchls's own results.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import pytest
import torch

from gpu_helpers import close, load, needs_gpu

pytestmark = [pytest.mark.gpu, needs_gpu]

DEV = "cuda"


@dataclass(frozen=True)
class Entry:
    offset: int
    count: int
    dim: int


@dataclass(frozen=True)
class Group:
    blocks: tuple
    columns: tuple
    type_indices: tuple
    variable_indices: tuple


@dataclass(frozen=True)
class RefJacobian:
    groups: tuple
    layout: tuple
    shape: tuple


def _dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a)).to(DEV)
    return t if dtype is None else t.to(dtype)


def _ba_small_jacobian(scale=1.0):
    fx = load("ba_small")
    off = fx["layout_offsets"]
    layout = (Entry(int(off[0]), 9, 6), Entry(int(off[1]), 500, 3))
    cam, pt = torch.from_numpy(fx["camera_index"]), torch.from_numpy(fx["point_index"])
    free = cam > 0
    slots = [((0, 1), (cam[free] - 1, pt[free])), ((1,), (pt[~free],))]
    groups, rows = [], 0
    for gi, (types, idxs) in enumerate(slots):
        blocks = tuple(_dev(fx[f"block{gi}_{si}"]) * scale for si in range(len(types)))
        cols = tuple((i.to(DEV)[:, None] * layout[t].dim + layout[t].offset
                      + torch.arange(layout[t].dim, device=DEV)) for t, i in zip(types, idxs))
        groups.append(Group(blocks, cols, types, tuple(i.to(DEV) for i in idxs)))
        rows += blocks[0].shape[0] * blocks[0].shape[1]
    return fx, RefJacobian(tuple(groups), layout, (rows, int(off[1]) + 1500))


def test_normal_plan_on_reference_layout():
    import torchls_b200 as tls

    fx, J = _ba_small_jacobian()
    plan = tls.CudaNormalPlan(J)
    v = _dev(fx["v"])
    close(plan.bind(J).normal_matvec(v, 1e-3), fx["normal_matvec"], 1e-12, what="normal_matvec")
    _, J2 = _ba_small_jacobian(scale=2.0)  # a new linearization of the same structure
    want = 4.0 * (torch.from_numpy(fx["normal_matvec"]) - 1e-3 * torch.from_numpy(fx["v"])) + 1e-3 * torch.from_numpy(
        fx["v"])
    close(plan.bind(J2).normal_matvec(v, 1e-3), want, 1e-12, what="rebound normal_matvec")
    # the products of the bound Jacobian are the reference's too
    close(plan.bind(J).matvec(v), fx["matvec"], 1e-12, what="matvec")
    close(plan.bind(J).rmatvec(_dev(fx["u"])), fx["rmatvec"], 1e-12, what="rmatvec")


def test_diagonal_plan_on_reference_layout():
    import torchls_b200 as tls

    fx, J = _ba_small_jacobian()
    blocks = tls.CudaDiagonalPlan(J).diagonal_blocks(J)
    for i, b in enumerate(blocks):
        close(b, fx[f"diag{i}"], 1e-12, what=f"diag{i}")
    # aliased slots (one residual's two slots naming the same variable)
    fa = load("alias_weights")
    layout = (Entry(0, 6, 2),)
    groups = []
    for gi, nslots in ((0, 2), (1, 1)):
        blocks = tuple(_dev(fa[f"block{gi}_{si}"]) for si in range(nslots))
        cols = tuple(_dev(fa[f"columns{gi}_{si}"]) for si in range(nslots))
        groups.append(Group(blocks, cols, (0,) * nslots, tuple(c[:, 0] // 2 for c in cols)))
    Ja = RefJacobian(tuple(groups), layout, (sum(b.blocks[0].shape[0] * b.blocks[0].shape[1] for b in groups), 12))
    close(tls.CudaDiagonalPlan(Ja).diagonal_blocks(Ja)[0], fa["diag0"], 1e-12, what="aliased diag")


def test_plans_reject_changed_structure():
    import torchls_b200 as tls

    _, J = _ba_small_jacobian()
    plan = tls.CudaNormalPlan(J)
    g0 = J.groups[0]
    moved = Group(g0.blocks, g0.columns, g0.type_indices,
                  (g0.variable_indices[0].flip(0), g0.variable_indices[1]))
    with pytest.raises(ValueError, match="unchanged"):
        plan.bind(RefJacobian((moved, J.groups[1]), J.layout, J.shape))
    bad = Group(g0.blocks, (g0.columns[0] + 1, g0.columns[1]), g0.type_indices, g0.variable_indices)
    with pytest.raises(ValueError, match="columns"):
        tls.CudaNormalPlan(RefJacobian((bad, J.groups[1]), J.layout, J.shape))
    with pytest.raises(ValueError, match="float32 or float64"):
        cpu = Group(tuple(b.cpu() for b in g0.blocks), g0.columns, g0.type_indices, g0.variable_indices)
        tls.CudaDiagonalPlan(RefJacobian((cpu, J.groups[1]), J.layout, J.shape))
