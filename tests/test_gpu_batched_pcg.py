"""Kernels of the batched solver: per-problem reduced matrices, the one-launch
batched PCG (work queue, tilings), the per-factor objective terms and the
per-problem LM decision.

The PCG is checked on hand-made systems against float64 torch solves (the CG
stops at rtol |b_p|, so the true residual is bounded by a small multiple of
it) and against itself across tilings (bitwise: the kernel's sums do not
depend on how many warps a problem gets); the assembled matrices are checked
against the diagonal blocks of the merged system's dense matrix
(``tls_schur_dense_matrix``), which sums the same pairs in another fixed
order: 1e-13 of the largest entry (float64), one float32 rounding (float32).
"""

from __future__ import annotations

import ctypes as C
import math

import pytest
import torch

from gpu_helpers import needs_gpu

pytestmark = [pytest.mark.gpu, needs_gpu]

DEV = "cuda"
SMEM = 112 * 1024


def _spd_problems(sizes, dr, seed, sdtype, bad=()):
    """Random SPD matrices S_p (blocks x dr square), stored back to back in
    sdtype; the float64 diagonal blocks of the stored values; problems in
    ``bad`` get a diagonal block that is not positive definite."""
    g = torch.Generator().manual_seed(seed)
    mats, offs, off = [], [], 0
    for p, nb in enumerate(sizes):
        n = nb * dr
        a = torch.randn(n, n + 3, generator=g, dtype=torch.float64)
        m = a @ a.T / n + 0.5 * torch.eye(n, dtype=torch.float64)
        if p in bad and n:
            m[:dr, :dr] = -torch.eye(dr, dtype=torch.float64)
        m = 0.5 * (m + m.T)
        mats.append(m.to(sdtype).to(torch.float64))
        offs.append(off)
        off += n * n
    S = torch.cat([m.reshape(-1) for m in mats] + [torch.zeros(1, dtype=torch.float64)]).to(sdtype)
    diag = torch.cat([torch.stack([m[i * dr:(i + 1) * dr, i * dr:(i + 1) * dr] for i in range(m.shape[0] // dr)])
                      for m in mats if m.numel()])
    return mats, torch.tensor(offs, dtype=torch.int64), S, diag


class _Batch:
    def __init__(self, sizes, dr=6, sdtype=torch.float64, seed=0, bad=()):
        from torchls_b200 import _lib as L

        self.L, self.sizes, self.dr, self.sdtype = L, list(sizes), dr, sdtype
        self.mats, offs, S, diag = _spd_problems(sizes, dr, seed, sdtype, bad)
        counts = torch.tensor(self.sizes, dtype=torch.int64)
        ptr = torch.zeros(len(sizes) + 1, dtype=torch.int64)
        ptr[1:] = torch.cumsum(counts, 0)
        self.ptr = ptr
        self.dev = dict(ret_ptr=ptr.to(DEV, torch.int32), ret_problem=torch.repeat_interleave(
            torch.arange(len(sizes)), counts).to(DEV, torch.int32), s_off=offs.to(DEV), S=S.to(DEV), diag=diag.to(DEV))
        b = L.BatchedSystems()
        b.nproblems, b.nretained, b.dr, b.sdtype = len(sizes), int(counts.sum()), dr, L.dtype_code(sdtype)
        for k in ("ret_ptr", "ret_problem", "s_off", "S", "diag"):
            setattr(b, k, self.dev[k].data_ptr())
        self.sys = b
        self.n = int(counts.sum()) * dr
        g = torch.Generator().manual_seed(seed + 1)
        self.rhs = torch.randn(self.n, generator=g, dtype=torch.float64).to(DEV)

    def run(self, groups, rtol=1e-10, atol=1e-30, max_iterations=500, order=None):
        """groups: problems per CTA for every task (one value for all)."""
        L = self.L
        P = len(self.sizes)
        order = list(range(P)) if order is None else order
        first, size, gr = [], [], []
        for s in range(0, P, groups):
            first.append(s)
            size.append(min(groups, P - s))
            gr.append(groups)
        t = lambda a: torch.tensor(a, dtype=torch.int32, device=DEV)  # noqa: E731
        arrs = [t(order), t(first), t(size), t(gr)]
        x = torch.full((max(self.n, 1),), float("nan"), dtype=torch.float64, device=DEV)
        its = torch.full((P,), -1, dtype=torch.int32, device=DEV)
        status = torch.full((P,), -1, dtype=torch.int32, device=DEV)
        queue = torch.zeros(1, dtype=torch.int32, device=DEV)
        err = torch.zeros(1, dtype=torch.int32, device=DEV)
        a = L.BatchedPcgArgs()
        a.rhs, a.x, a.iterations, a.status = self.rhs.data_ptr(), x.data_ptr(), its.data_ptr(), status.data_ptr()
        a.order, a.task_first, a.task_size, a.task_groups = (v.data_ptr() for v in arrs)
        a.queue, a.err = queue.data_ptr(), err.data_ptr()
        a.rtol, a.atol, a.ntasks, a.max_iterations, a.smem_bytes = rtol, atol, len(first), max_iterations, SMEM
        L.call("tls_batched_pcg", C.byref(self.sys), C.byref(a), L.stream_handle(torch.device(DEV)))
        torch.cuda.synchronize()
        return x[: self.n].cpu(), its.cpu(), status.cpu(), int(err.item())


@pytest.mark.parametrize("sdtype", [torch.float64, torch.float32])
def test_batched_pcg_solves_every_problem(sdtype):
    # sizes from 0 to 31 blocks (n_p up to 186): cached and uncached matrices
    sizes = [3, 1, 0, 31, 7, 12, 2, 20, 5, 31, 9, 16]
    b = _Batch(sizes, sdtype=sdtype, seed=3)
    x, its, status, err = b.run(groups=1)
    assert err == 0 and bool((status == 0).all()), status
    rhs = b.rhs.cpu()
    for p, nb in enumerate(sizes):
        lo, hi = int(b.ptr[p]) * 6, int(b.ptr[p + 1]) * 6
        if nb == 0:
            assert int(its[p]) == 0
            continue
        m = b.mats[p]
        res = (m @ x[lo:hi] - rhs[lo:hi]).norm()
        assert res <= 1e-8 * rhs[lo:hi].norm(), (p, float(res))
        assert 0 < int(its[p]) <= 500


def test_batched_pcg_tilings_agree_bitwise():
    sizes = [4, 4, 2, 9, 1, 6, 3, 8, 5, 5, 7, 2, 3, 1, 4, 6]  # n_p <= 54: every tiling fits
    b = _Batch(sizes, seed=5)
    runs = [b.run(groups=k, rtol=1e-6, atol=1e-10, max_iterations=200) for k in (1, 2, 4, 8)]
    for x, its, status, err in runs[1:]:
        assert err == 0
        assert torch.equal(x, runs[0][0])
        assert torch.equal(its, runs[0][1])
    # task order does not matter either
    order = list(range(len(sizes)))[::-1]
    x, its, _, _ = b.run(groups=2, rtol=1e-6, atol=1e-10, max_iterations=200, order=order)
    assert torch.equal(x, runs[0][0]) and torch.equal(its, runs[0][1])


def test_batched_pcg_matches_plain_cg_iterations():
    """Iteration counts and iterates of a float64 torch PCG with the same
    block-Jacobi preconditioner, the same threshold and the same stopping
    rule (rounding differs only in the order of the sums)."""
    sizes = [2, 5, 11, 3]
    b = _Batch(sizes, seed=11)
    x, its, status, _ = b.run(groups=1, rtol=1e-6, atol=1e-10, max_iterations=200)
    rhs = b.rhs.cpu()
    for p, nb in enumerate(sizes):
        lo, hi = int(b.ptr[p]) * 6, int(b.ptr[p + 1]) * 6
        m, bb = b.mats[p], rhs[lo:hi]
        Ls = [torch.linalg.cholesky(m[i * 6:(i + 1) * 6, i * 6:(i + 1) * 6]) for i in range(nb)]
        prec = lambda r: torch.cat([torch.cholesky_solve(r[i * 6:(i + 1) * 6, None], Ls[i])[:, 0]  # noqa: E731
                                    for i in range(nb)])
        xr = torch.zeros_like(bb)
        r = bb.clone()
        z = prec(r)
        pv = z.clone()
        rz = float(r @ z)
        thr = max(1e-6 * float(bb.norm()), 1e-10)
        k = 0
        for _ in range(200):
            ap = m @ pv
            pap = float(pv @ ap)
            k += 1
            alpha = rz / pap
            xr += alpha * pv
            r -= alpha * ap
            if not math.sqrt(float(r @ r)) > thr:
                break
            z = prec(r)
            rzn = float(r @ z)
            pv = z + (rzn / rz) * pv
            rz = rzn
        assert abs(int(its[p]) - k) <= 1, (p, int(its[p]), k)
        assert (x[lo:hi] - xr).norm() <= 1e-6 * xr.norm(), p


def test_batched_pcg_rejects_non_pd_blocks():
    sizes = [3, 4, 2, 5]
    b = _Batch(sizes, seed=7, bad=(1, 3))
    x, its, status, err = b.run(groups=2)
    assert err == 0
    assert status.tolist() == [0, 1, 0, 1]
    for p in (1, 3):
        lo, hi = int(b.ptr[p]) * 6, int(b.ptr[p + 1]) * 6
        assert int(its[p]) == 0 and bool((x[lo:hi] == 0).all())
    rhs = b.rhs.cpu()
    for p in (0, 2):
        lo, hi = int(b.ptr[p]) * 6, int(b.ptr[p + 1]) * 6
        assert (b.mats[p] @ x[lo:hi] - rhs[lo:hi]).norm() <= 1e-8 * rhs[lo:hi].norm()


def test_batched_pcg_reports_a_share_that_is_too_small():
    """31 blocks need ~16 KB of vectors and factors: 8 problems per CTA
    (14 KB shares) cannot hold them; the kernel flags it and skips the problem."""
    b = _Batch([31, 1], seed=2)
    _, its, status, err = b.run(groups=8)
    assert err == 1 and int(status[0]) == 2 and int(status[1]) == 0


def test_batched_dense_matches_merged_dense_matrix():
    import torchls_b200 as tls
    from torchls_b200 import synthetic
    from torchls_b200.batched import BatchedProblem
    from torchls_b200.schur import SchurLinearization

    datas = synthetic.batched_bundle_adjustment(6, first_seed=40)
    probs = [synthetic.build_bundle_adjustment(d, tls, device=DEV, loss=tls.HuberLoss(0.01)) for d in datas]
    bp = BatchedProblem(probs)
    an, vals = bp.merged._state(None)
    for wdtype in (torch.float64, torch.float32):
        lin = bp.merged.linearize(dict(vals._values), jacobian_dtype=wdtype, schur=bp.plan)
        s = torch.rand(an.tangent_dim, dtype=torch.float64, device=DEV) + 0.5
        slin = SchurLinearization(bp.plan, lin, lin.jacobian.diagonal_blocks(), s, wdtype=wdtype,
                                  vec_dtype=torch.float64)
        system = slin.damped(1.0)
        full = system.dense_matrix().cpu()
        sys_ = bp.systems
        ptr = sys_.ret_ptr.cpu().long()
        off = sys_.s_off.cpu()
        for sdtype in (torch.float64, torch.float32):
            sys_.assemble(system, sdtype)
            S = sys_._S[sdtype].cpu().double()
            for p in range(bp.P):
                lo, hi = int(ptr[p]) * 6, int(ptr[p + 1]) * 6
                n = hi - lo
                mine, ref = S[int(off[p]) : int(off[p]) + n * n].view(n, n), full[lo:hi, lo:hi]
                assert torch.equal(mine, mine.T), p  # mirrored entries are the same value
                tol = 1e-13 * float(ref.abs().max()) if sdtype == torch.float64 else 0.0
                if sdtype == torch.float32:
                    tol = float((ref.float().double() - ref).abs().max()) * 2 + 1e-13 * float(ref.abs().max())
                assert float((mine - ref).abs().max()) <= tol, (p, sdtype)
                assert not bool(full[lo:hi, :lo].any()) and not bool(full[lo:hi, hi:].any())
        diag = sys_.diag.cpu()
        for i in range(diag.shape[0]):
            ref = full[i * 6:(i + 1) * 6, i * 6:(i + 1) * 6]
            assert float((diag[i] - ref).abs().max()) <= 1e-13 * float(ref.abs().max())


def test_factor_terms_and_sqnorm():
    from torchls_b200 import _lib as L

    g = torch.Generator().manual_seed(9)
    N, R, delta = 5000, 2, 0.3
    old = (torch.randn(N, R, generator=g, dtype=torch.float64) * 0.4)
    new = old + torch.randn(N, R, generator=g, dtype=torch.float64) * 0.2
    w = torch.rand(N, generator=g, dtype=torch.float64) + 0.5
    od, nd, wd = old.to(DEV), new.to(DEV), w.to(DEV)
    so, sn = (old * old).sum(-1), (new * new).sum(-1)
    sq = ((old - new) * (old + new)).sum(-1)
    st = L.stream_handle(torch.device(DEV))
    for loss, wt in ((0, None), (1, wd), (1, None)):
        obj = torch.empty(N, dtype=torch.float64, device=DEV)
        red = torch.empty(N, dtype=torch.float64, device=DEV)
        L.call("tls_factor_terms", N, R, od.data_ptr(), nd.data_ptr(), loss, delta, L.ptr(wt), obj.data_ptr(),
               red.data_ptr(), st)
        if loss == 0:
            eo, er = sn, sq
        else:
            d2 = delta * delta
            no, nn = so.sqrt(), sn.sqrt()
            rn = torch.where(sn > d2, delta * (2 * nn - delta), sn)
            ro = torch.where(so > d2, delta * (2 * no - delta), so)
            er = torch.where((so <= d2) & (sn <= d2), sq, ro - rn)
            er = torch.where((so > d2) & (sn > d2), 2 * delta * sq / (no + nn), er)
            eo = rn
        ww = w if wt is not None else torch.ones_like(w)
        torch.testing.assert_close(obj.cpu(), 0.5 * ww * eo, rtol=1e-14, atol=1e-300)
        torch.testing.assert_close(red.cpu(), 0.5 * ww * er, rtol=1e-12, atol=1e-16)
    out = torch.empty(N, dtype=torch.float64, device=DEV)
    L.call("tls_factor_sqnorm", N, R, nd.data_ptr(), out.data_ptr(), st)
    torch.testing.assert_close(out.cpu(), sn, rtol=1e-15, atol=0)


def test_batched_lm_update_decisions():
    from torchls_b200 import _lib as L

    g = torch.Generator().manual_seed(4)
    P = 257
    actual = torch.randn(P, generator=g, dtype=torch.float64)
    predicted = torch.randn(P, generator=g, dtype=torch.float64).abs() * torch.where(
        torch.rand(P, generator=g) < 0.1, -1.0, 1.0).double()
    new_cost = torch.rand(P, generator=g, dtype=torch.float64) * 10
    new_cost[::17] = float("inf")
    actual[::13] = new_cost[::13] * 1e-12  # tiny reductions: the cost-tolerance stop
    predicted[::13] = actual[::13]
    cost = torch.rand(P, generator=g, dtype=torch.float64) * 10 + 1
    lam = torch.rand(P, generator=g, dtype=torch.float64) * 1e-3
    tried = torch.rand(P, generator=g) < 0.8
    active = torch.ones(P, dtype=torch.bool)
    pending = tried.clone()
    f, lmin, lmax, qmin, ctol = 4.0, 1e-12, 1e12, 1e-4, 1e-10
    # expected (the per-problem rule of the batched solver)
    q = torch.where(predicted > 0, actual / predicted, torch.full_like(actual, -math.inf))
    ok = tried & torch.isfinite(new_cost) & (actual > 0) & (q >= qmin)
    ecost = torch.where(ok, new_cost, cost)
    elam = torch.where(ok & (q > 0.75), (lam / f).clamp_min(lmin), lam)
    elam = torch.where(tried & ~ok, (elam * f).clamp_max(lmax), elam)
    conv = ok & (actual.abs() <= ctol * (ecost + actual).clamp_min(1e-300))
    d = {k: v.to(DEV) for k, v in dict(actual=actual, predicted=predicted, new_cost=new_cost, cost=cost, lam=lam,
                                         tried=tried, active=active, pending=pending).items()}
    d["ok"] = torch.zeros(P, dtype=torch.bool, device=DEV)
    d["accepted"] = torch.zeros(P, dtype=torch.int64, device=DEV)
    d["rejected"] = torch.zeros(P, dtype=torch.int64, device=DEV)
    d["reason"] = torch.zeros(P, dtype=torch.int32, device=DEV)
    m = L.BatchedLm()
    m.nproblems = P
    m.lambda_factor, m.lambda_min, m.lambda_max, m.step_quality_min, m.cost_tolerance = f, lmin, lmax, qmin, ctol
    for k, v in d.items():
        setattr(m, k, v.data_ptr())
    L.call("tls_batched_lm_update", C.byref(m), L.stream_handle(torch.device(DEV)))
    torch.cuda.synchronize()
    assert torch.equal(d["ok"].cpu(), ok)
    assert torch.equal(d["cost"].cpu(), ecost)
    assert torch.equal(d["lam"].cpu(), elam)
    assert torch.equal(d["accepted"].cpu(), ok.long())
    assert torch.equal(d["rejected"].cpu(), (tried & ~ok).long())
    assert torch.equal(d["active"].cpu(), ~conv)
    assert torch.equal(d["pending"].cpu(), pending & ~ok)
    assert torch.equal(d["reason"].cpu(), torch.where(conv, L.BATCH_COST_TOLERANCE, 0).int())
    assert bool(conv.any()) and bool((tried & ~ok).any()) and bool((ok & (q > 0.75)).any())


def test_batched_tiling_is_recorded():
    import torchls_b200 as tls
    from torchls_b200 import synthetic
    from torchls_b200.batched import BatchedProblem

    datas = synthetic.batched_bundle_adjustment(12, first_seed=60)
    bp = BatchedProblem([synthetic.build_bundle_adjustment(d, tls, device=DEV, loss=tls.HuberLoss(0.01))
                         for d in datas])
    bp.solve(max_iterations=2, precision="mixed")
    chosen, record = bp.systems.tiling[torch.float32]
    assert set(chosen.values()) <= {1, 2, 4, 8}
    assert sum(r["problems"] for r in record.values()) == 12
    for r in record.values():
        assert r["problems_per_cta"] in r["us_by_problems_per_cta"]
        assert r["warps_per_problem"] * r["problems_per_cta"] == 8
