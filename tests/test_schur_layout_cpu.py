"""Chunk-slab metadata of the one-group Schur kernels (CPU only).

The chunk kernel forms, per chunk, t_e for every edge, then each eliminated
variable's sum y_p over its edges in the order of the point-local edge list,
written over the t entry of the variable's first listed edge; phase 2 reads
y_p for edge e at the entry named by the low 16 bits of e's metadata word.
These tests replay that bookkeeping with numpy on the layout the host builds
and check it against direct per-variable sums.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch


@pytest.fixture(scope="module")
def plan():
    import torchls_b200 as tls
    from torchls_b200 import synthetic
    from torchls_b200.schur import SchurPlan

    data = synthetic.make_bundle_adjustment(num_cameras=24, num_points=1500, views=8, seed=5)
    problem = synthetic.build_bundle_adjustment(data, tls, device="cpu")
    return SchurPlan(problem._ensure_analyzed(), "points", torch.device("cpu"))


@pytest.mark.parametrize("wdtype", [torch.float32, torch.float64])
def test_variable_sums_follow_the_metadata(plan, wdtype):
    lay = plan.chunks_for(wdtype)
    cap = lay.cap
    M = lay.dev["meta"].numpy().reshape(-1, lay.meta_ints).astype(np.int64)
    c_r, c_e, sidx, _, _ = lay._host
    chunk_of = sidx // cap
    rng = np.random.default_rng(0)
    T = rng.standard_normal((lay.nslab, plan.de))
    for c in range(lay.nchunks):
        ne, npt = int(M[c, 0]), int(M[c, 1])
        meta = M[c, 4 + cap : 4 + 2 * cap]
        pp = M[c, 4 + 3 * cap : 4 + 3 * cap + npt + 1]
        pe = M[c, 8 + 4 * cap : 8 + 5 * cap]
        assert pp[0] == 0 and pp[-1] == ne and np.all(np.diff(pp) > 0)
        assert sorted(pe[:ne].tolist()) == list(range(ne))
        ts = T[c * cap : c * cap + cap].copy()
        # phase 1.5: sums in list order, each written over its first edge's entry
        for pl in range(npt):
            y = np.zeros(plan.de)
            for j in range(pp[pl], pp[pl + 1]):
                y = y + ts[pe[j]]
            ts[pe[pp[pl]]] = y
        # phase 2: every edge reads its variable's sum through its metadata word
        in_chunk = np.flatnonzero(chunk_of == c)
        for k in in_chunk:
            le = int(sidx[k] - c * cap)
            direct = T[sidx[in_chunk[c_e[in_chunk] == c_e[k]]]].sum(0)
            np.testing.assert_allclose(ts[int(meta[le]) & 0xFFFF], direct, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("wdtype", [torch.float32, torch.float64])
def test_run_partials_cover_each_retained_variable(plan, wdtype):
    """Phase 2 sums runs of equal retained variable inside windows of
    32 * (cap / 256) edges: a run starts at the window position in bits 16-21
    of its edges' metadata words and ends at the edge flagged in bit 22,
    whose partial goes to the retained-major position in the tail list. The
    gather sums retained variable i's positions rrun_ptr[i] .. rrun_ptr[i+1];
    crun_start / crun_len name each position's slab entries."""
    lay = plan.chunks_for(wdtype)
    cap, win = lay.cap, lay.window
    M = lay.dev["meta"].numpy().reshape(-1, lay.meta_ints).astype(np.int64)
    rrun_ptr = lay.dev["rrun_ptr"].numpy()
    crun_start = lay.dev["crun_start"].numpy()
    crun_len = lay.dev["crun_len"].numpy()
    slab_r = lay.dev["slab_r"].numpy()
    assert rrun_ptr[-1] == lay.nruns
    rng = np.random.default_rng(1)
    U = rng.standard_normal((lay.nslab, plan.dr))
    partial = np.full((lay.nruns, plan.dr), np.nan)
    for c in range(lay.nchunks):
        ne = int(M[c, 0])
        er = M[c, 4 : 4 + cap]
        meta = M[c, 4 + cap : 4 + 2 * cap]
        tpos = M[c, 4 + 2 * cap : 4 + 3 * cap]
        assert np.all(np.diff(er[:ne]) >= 0)  # sorted by retained variable
        for le in range(ne):
            head = (int(meta[le]) >> 16) & 63
            w0 = le - le % win
            assert head <= le % win and er[w0 + head] == er[le]
            if (int(meta[le]) >> 22) & 1:
                start = w0 + head
                assert np.all(er[start : le + 1] == er[le])
                assert partial[tpos[le], 0] != partial[tpos[le], 0]  # each position written once
                partial[tpos[le]] = U[c * cap + start : c * cap + le + 1].sum(0)
                assert crun_start[tpos[le]] == c * cap + start and crun_len[tpos[le]] == le + 1 - start
    assert not np.isnan(partial).any()
    for i in range(plan.r.count):
        mine = np.flatnonzero(slab_r == i)
        got = partial[rrun_ptr[i] : rrun_ptr[i + 1]].sum(0)
        np.testing.assert_allclose(got, U[mine].sum(0), rtol=1e-12, atol=1e-12)
