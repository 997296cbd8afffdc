"""Tile plan of the one-pass normal operator, checked on the CPU.

``build_tile_plan`` decides where each (slot, factor) contribution of
y = diag(s) J^T J diag(s) x + lambda x goes: a stage position inside its tile,
a run, and a destination (final, CTA accumulator, partial) plus the gather
lists. These tests replay a plan exactly as the CUDA kernels walk it (tiles
per CTA, runs per tile, accumulator flushes, partial gathers) with numpy and
compare the result with a dense J^T J x (1e-12 relative), on shapes that
reach every branch: a bundle adjustment with a fixed camera (two factor
groups), a graph with aliased slots, a one-slot prior group, a three-slot
group, an empty group and variables no factor touches; small stages and
accumulators force multi-tile CTAs and accumulator overflow. They also check
that no two pairs of a tile share stage space, that each pair's x-buffer
offset holds its own variable's x, and that every column of y is written
exactly once; that a graph whose edges come in random order is put in
tile order (a permutation of its factors) with far fewer partials; that the
tiles are spread evenly over the CTAs; and that malformed index arrays are
rejected.
"""

from __future__ import annotations

import numpy as np
import pytest

from torchls_b200.normal_tiles import FactorGroupShape, build_tile_plan


def _replay(plan, groups, jacs, x, scale, damping):
    n = len(x)
    sx = x * scale
    y = np.full(n, np.nan)
    writes = np.zeros(n, np.int64)
    partials = np.full(max(plan.npartials, 1), np.nan)
    pwrites = np.zeros(max(plan.npartials, 1), np.int64)

    def finish(col, vals):
        for c, v in enumerate(vals):
            y[col + c] = v * scale[col + c] + damping * x[col + c]
            writes[col + c] += 1

    def to_partial(off, vals):
        partials[off:off + len(vals)] = vals
        pwrites[off:off + len(vals)] += 1

    for k, g in enumerate(groups):
        T = plan.tile_factors[k]
        J = jacs[k]
        cols = np.concatenate(([0], np.cumsum([d for _, d, _ in g.slots])))
        for cta in range(plan.cta_base[k], plan.cta_base[k + 1]):
            acc = np.zeros(plan.acc_doubles)
            for t in range(plan.cta_tile[cta], plan.cta_tile[cta + 1]):
                f0 = (t - plan.tile_base[k]) * T
                nt = min(T, g.count - f0)
                # prologue: each target's scaled x once into the compact x buffer
                xbuf = np.full(plan.xbuf_doubles, np.nan)
                for r in range(plan.tile_run[t], plan.tile_run[t + 1]):
                    d = ((int(plan.run_meta[r]) >> 27) & 0xF) + 1
                    xo, col = int(plan.run_xoff[r]), int(plan.run_col[r])
                    assert xo + d <= plan.xbuf_doubles and np.isnan(xbuf[xo:xo + d]).all()
                    xbuf[xo:xo + d] = sx[col:col + d]
                stage = np.full(plan.stage_doubles, np.nan)
                used = np.zeros(plan.stage_doubles, bool)
                for f in range(f0, f0 + nt):
                    fac = f if plan.perm[k] is None else int(plan.perm[k][f])  # tile position -> factor
                    words = [int(plan.pos[k][s * g.count + f]) for s in range(len(g.slots))]
                    xs = np.concatenate([xbuf[(w >> 16):(w >> 16) + d] for w, (_, d, _) in zip(words, g.slots)])
                    want = np.concatenate([sx[off + int(idx[fac]) * d: off + int(idx[fac]) * d + d]
                                           for off, d, idx in g.slots])
                    assert np.array_equal(xs, want), "x buffer offset points at another variable"
                    q = J[fac] @ xs
                    for s, (_, d, _) in enumerate(g.slots):
                        p = words[s] & 0xFFFF
                        assert not used[p:p + d].any(), "two pairs share stage space"
                        used[p:p + d] = True
                        stage[p:p + d] = J[fac][:, cols[s]:cols[s] + d].T @ q
                for r in range(plan.tile_run[t], plan.tile_run[t + 1]):
                    meta = int(plan.run_meta[r])
                    start, length, d = meta & 0x3FFF, (meta >> 14) & 0x1FFF, ((meta >> 27) & 0xF) + 1
                    seg = stage[start:start + length * d]
                    assert used[start:start + length * d].all()
                    v = seg.reshape(length, d).sum(0)
                    dest, col = int(plan.run_dest[r]), int(plan.run_col[r])
                    if dest == -1:
                        finish(col, v)
                    elif dest < -1:
                        acc[-2 - dest:-2 - dest + d] += v
                    else:
                        to_partial(dest, v)
            for j in range(plan.cta_flush[cta], plan.cta_flush[cta + 1]):
                meta = int(plan.flush_meta[j])
                off, d = meta & 0xFFFF, ((meta >> 16) & 0xF) + 1
                v = acc[off:off + d]
                if plan.flush_dest[j] == -1:
                    finish(int(plan.flush_col[j]), v)
                else:
                    to_partial(int(plan.flush_dest[j]), v)
    assert (pwrites[:plan.npartials] == 1).all(), "a partial slot is not written exactly once"
    for t in range(len(plan.target_col)):
        d = int(plan.target_dim[t])
        v = np.zeros(d)
        for j in range(plan.target_ptr[t], plan.target_ptr[t + 1]):
            off = int(plan.target_src[j])
            v = v + partials[off:off + d]
        finish(int(plan.target_col[t]), v)
    assert (writes == 1).all(), "a column of y is not written exactly once"
    return y


def _dense(groups, jacs, n, x, scale, damping):
    rows = []
    for g, J in zip(groups, jacs):
        R = J.shape[1]
        for f in range(g.count):
            block = np.zeros((R, n))
            c0 = 0
            for off, d, idx in g.slots:
                block[:, off + int(idx[f]) * d: off + int(idx[f]) * d + d] += J[f][:, c0:c0 + d]
                c0 += d
            rows.append(block)
    A = np.concatenate(rows) if rows else np.zeros((0, n))
    As = A * scale[None, :]
    return As.T @ (As @ x) + damping * x


def _check(groups, var_groups, seed, **kw):
    rng = np.random.default_rng(seed)
    n = sum(c * d for _, c, d in var_groups)
    jacs = [rng.standard_normal((g.count, 1 + seed % 3 + 1, sum(d for _, d, _ in g.slots))) for g in groups]
    x = rng.standard_normal(n)
    scale = 0.5 + rng.random(n)
    plan = build_tile_plan(groups, var_groups, **kw)
    assert plan is not None
    y = _replay(plan, groups, jacs, x, scale, 0.3)
    ref = _dense(groups, jacs, n, x, scale, 0.3)
    assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()
    return plan


def _ba(cams=6, points=120, per_point=4, seed=0):
    rng = np.random.default_rng(seed)
    ci = np.concatenate([rng.choice(cams, per_point, replace=False) for _ in range(points)])
    pi = np.repeat(np.arange(points), per_point)
    free = ci > 0
    groups = [FactorGroupShape(int(free.sum()), [(0, 6, ci[free] - 1), ((cams - 1) * 6, 3, pi[free])]),
              FactorGroupShape(int((~free).sum()), [((cams - 1) * 6, 3, pi[~free])])]
    return groups, [(0, cams - 1, 6), ((cams - 1) * 6, points, 3)]


def test_bundle_adjustment_plan_reaches_every_destination():
    groups, vg = _ba()
    plan = _check(groups, vg, 0, num_sms=4, ctas_per_sm=1, stage_doubles=9 * 64, acc_doubles=24)
    st = plan.stats
    assert st["final_runs"] and st["acc_runs"] and st["partial_runs"] and st["flushes"]
    assert plan.ncta == plan.cta_base[-1] and plan.ncta >= 3


def test_bundle_adjustment_plan_default_sizes():
    groups, vg = _ba(cams=12, points=400, per_point=5, seed=1)
    _check(groups, vg, 1, num_sms=4)


def test_graph_with_aliased_slots_priors_and_untouched_variables():
    rng = np.random.default_rng(7)
    poses = 90
    i = rng.integers(0, poses - 10, 300)
    j = i + rng.integers(0, 10, 300)  # includes i == j: both slots on one variable
    loops = rng.integers(0, poses - 10, (40, 3))
    groups = [
        FactorGroupShape(300, [(0, 6, i), (0, 6, j)]),
        FactorGroupShape(25, [(0, 6, rng.integers(0, poses - 10, 25))]),   # prior on a pose
        FactorGroupShape(0, [(0, 6, np.zeros(0, np.int64))]),             # empty group
        FactorGroupShape(40, [(0, 6, loops[:, 0]), (poses * 6, 2, loops[:, 1]), (0, 6, loops[:, 2])]),
    ]
    # the last ten poses and half of the 2-dim variables are untouched
    vg = [(0, poses, 6), (poses * 6, 100, 2)]
    plan = _check(groups, vg, 2, num_sms=3, ctas_per_sm=1, stage_doubles=18 * 32, acc_doubles=60)
    assert plan.cta_base[2] == plan.cta_base[3]  # no CTAs for the empty group
    assert len(plan.target_col) > 0


def test_plan_declines_shapes_the_kernel_cannot_hold():
    g = [FactorGroupShape(10, [(0, 17, np.arange(10))])]
    assert build_tile_plan(g, [(0, 10, 17)], num_sms=1) is None
    g = [FactorGroupShape(10, [(0, 6, np.arange(10))] * 8)]
    assert build_tile_plan(g, [(0, 10, 6)], num_sms=1, stage_doubles=1000) is None


@pytest.mark.parametrize("sms", [1, 148])
def test_plan_is_deterministic(sms):
    groups, vg = _ba(cams=8, points=200, per_point=5, seed=3)
    a = build_tile_plan(groups, vg, num_sms=sms)
    b = build_tile_plan(groups, vg, num_sms=sms)
    for name in ("run_col", "run_meta", "run_dest", "flush_dest", "target_src"):
        assert np.array_equal(getattr(a, name), getattr(b, name))
    for pa, pb in zip(a.pos, b.pos):
        assert (pa is None and pb is None) or np.array_equal(pa, pb)


def test_random_order_graph_is_reordered_into_local_tiles():
    # odometry plus near-neighbour loop closures, added in random order
    rng = np.random.default_rng(11)
    poses = 400
    i = np.concatenate((np.arange(poses - 1), rng.integers(0, poses - 4, 800)))
    j = np.empty_like(i)
    j[:poses - 1] = np.arange(1, poses)
    j[poses - 1:] = i[poses - 1:] + rng.integers(2, 4, 800)
    shuffle = rng.permutation(len(i))
    g = [FactorGroupShape(len(i), [(0, 6, i[shuffle]), (0, 6, j[shuffle])], 6)]
    vg = [(0, poses, 6)]
    kw = dict(num_sms=2, stage_doubles=12 * 128)
    plan = _check(g, vg, 3, **kw)
    assert plan.perm[0] is not None and sorted(plan.perm[0].tolist()) == list(range(len(i)))
    kept = build_tile_plan(g, vg, reorder=False, **kw)
    assert kept.perm[0] is None
    assert plan.stats["partial_doubles"] * 5 < kept.stats["partial_doubles"]


@pytest.mark.parametrize("count,small", [(995_771, 4_229), (50_000, 0), (1_000, 10)])
def test_tiles_are_balanced_across_ctas(count, small):
    # every CTA of the main group carries the same number of tiles (the last
    # may carry fewer), and the groups together stay within the CTA budget
    rng = np.random.default_rng(0)
    pts = max(count // 10, 1)
    pidx = np.minimum(np.arange(count) // 10, pts - 1)
    groups = [FactorGroupShape(count, [(0, 6, rng.integers(0, 255, count)), (255 * 6, 3, pidx)], 2)]
    if small:
        groups.append(FactorGroupShape(small, [(255 * 6, 3, np.sort(rng.integers(0, pts, small)))], 2))
    plan = build_tile_plan(groups, [(0, 255, 6), (255 * 6, pts, 3)], num_sms=148)
    assert plan is not None
    assert plan.ncta <= 2 * 148
    per_cta = np.diff(plan.cta_tile[plan.cta_base[0]:plan.cta_base[1] + 1])
    assert per_cta.max() - per_cta[:-1].min() == 0
    assert per_cta[-1] <= per_cta[0]


def test_plan_rejects_index_arrays_of_the_wrong_length():
    g = [FactorGroupShape(10, [(0, 6, np.arange(9))])]
    with pytest.raises(ValueError, match="index"):
        build_tile_plan(g, [(0, 10, 6)], num_sms=1)
