"""Dense float64 Cholesky kernels (blocked, FP64 tensor-core trailing updates)
against torch.linalg.cholesky / cholesky_solve on the same matrices: factors
and solutions within 1e-12 relative (both float64; only the summation order
differs), the first failing pivot reported like cholesky_ex's info."""

from __future__ import annotations

import pytest
import torch

from gpu_helpers import close, needs_gpu

pytestmark = [pytest.mark.gpu, needs_gpu]

DEV = "cuda"


def _spd(n, seed, cond=1e3):
    g = torch.Generator().manual_seed(seed)
    q, _ = torch.linalg.qr(torch.randn(n, n, generator=g, dtype=torch.float64))
    ev = torch.logspace(0, torch.log10(torch.tensor(cond)).item(), n, dtype=torch.float64)
    return ((q * ev) @ q.T).to(DEV)


@pytest.mark.parametrize("n", [1, 5, 63, 64, 65, 130, 200, 1530])
def test_cholesky_and_solve_match_torch(n):
    from torchls_b200 import dense

    A = _spd(n, n)
    L = dense.cholesky(A)
    want = torch.linalg.cholesky(A)
    close(L, want, 1e-12, what="factor")
    assert torch.equal(L, torch.tril(L))
    B = torch.randn(n, 3, dtype=torch.float64, device=DEV)
    close(dense.cholesky_solve(B, L), torch.cholesky_solve(B, want), 1e-10, what="solve")
    close(dense.cholesky_solve(B[:, 0], L), torch.cholesky_solve(B[:, :1], want)[:, 0], 1e-10, what="one rhs")
    L2 = dense.cholesky(A)
    assert torch.equal(L, L2), "not deterministic"


@pytest.mark.parametrize("n,bad", [(10, 0), (100, 37), (300, 250)])
def test_cholesky_reports_the_first_failing_pivot(n, bad):
    from torchls_b200 import dense

    A = _spd(n, 7)
    A[bad, bad] = -1.0  # leading minor of order bad + 1 is not positive definite
    _, info = dense.cholesky_ex(A)
    want = torch.linalg.cholesky_ex(A).info
    assert int(info) == int(want) == bad + 1
    with pytest.raises(torch.linalg.LinAlgError):
        dense.cholesky(A)
