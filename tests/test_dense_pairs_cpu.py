"""Host side of the dense reduced-matrix assembly: the pair lists that the
kernel sums (per lower camera-pair block, the slab entries of every shared
eliminated variable) reproduce W W^T for a random W on the small bundle
adjustment (numpy, no GPU)."""

from __future__ import annotations

import numpy as np
import torch

from golden import problems as P


def test_dense_pairs_reproduce_w_wt():
    import torchls_b200 as tls
    from torchls_b200.schur import SchurPlan, _dense_pairs

    prob = P.ba_small(tls)
    plan = SchurPlan(prob._ensure_analyzed(), "points", torch.device("cpu"))
    lay = plan.chunks_for(torch.float64)
    dr, de, cap = plan.dr, plan.de, lay.cap
    rng = np.random.default_rng(0)
    w = rng.standard_normal(lay.nslab * dr * de)
    slab = lambda s, k: w[((s // cap) * dr * de + k) * cap + (s % cap)]  # noqa: E731
    tr, tc, ptr, pa, pb = (t.numpy() for t in _dense_pairs(lay))
    n = plan.dim
    S = np.zeros((n, n))
    for t in range(len(tr)):
        for k in range(ptr[t], ptr[t + 1]):
            A = np.array([[slab(pa[k], r * de + b) for b in range(de)] for r in range(dr)])
            B = np.array([[slab(pb[k], r * de + b) for b in range(de)] for r in range(dr)])
            blk = A @ B.T
            S[tr[t] * dr:(tr[t] + 1) * dr, tc[t] * dr:(tc[t] + 1) * dr] += blk
            if tr[t] != tc[t]:
                S[tc[t] * dr:(tc[t] + 1) * dr, tr[t] * dr:(tr[t] + 1) * dr] += blk.T
    # W as a dense (reduced x eliminated) matrix from the same slabs
    slab_r, slab_e = lay.dev["slab_r"].numpy(), lay.dev["slab_e"].numpy()
    Wd = np.zeros((n, plan.E_count * de))
    for s_ in np.flatnonzero(slab_r >= 0):
        for r in range(dr):
            for b in range(de):
                Wd[slab_r[s_] * dr + r, slab_e[s_] * de + b] = slab(s_, r * de + b)
    np.testing.assert_allclose(S, Wd @ Wd.T, rtol=1e-12, atol=1e-12)
    assert np.all(tr >= tc)
