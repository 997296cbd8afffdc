"""Dense float64 Cholesky factor and solve on the GPU (``csrc/dense.cu``).

The reference factors its dense matrices with ``torch.linalg.cholesky`` and
solves with ``torch.cholesky_solve`` (the reduced-camera matrix of
``schur_dense``, solvers.py:517-518; FixedLinearSystem's normal matrix,
linear_system.py:61-98); these are this package's kernels for both:
blocked right-looking with the trailing updates on the FP64 tensor cores,
deterministic.
"""

from __future__ import annotations

import torch

from . import _lib as L


def cholesky_ex(matrix: torch.Tensor):
    """Lower Cholesky factor of a symmetric (n x n) float64 CUDA matrix (its
    lower triangle is read) and a device int32 ``info``: 0, or the 1-based index
    of the first pivot that is not positive (the factor is then not usable),
    like ``torch.linalg.cholesky_ex``."""
    L.require_cuda(matrix, "dense Cholesky")
    if matrix.ndim != 2 or matrix.shape[0] != matrix.shape[1]:
        raise ValueError("dense Cholesky expects a square matrix")
    fac = matrix.to(torch.float64).contiguous().clone()
    info = torch.zeros((), dtype=torch.int32, device=matrix.device)
    n = fac.shape[0]
    L.call("tls_dense_cholesky", n, fac.data_ptr(), n, info.data_ptr(), L.stream_handle(matrix.device))
    return fac, info


def cholesky(matrix: torch.Tensor) -> torch.Tensor:
    """Like ``torch.linalg.cholesky``: raises ``LinAlgError`` when the matrix
    is not positive definite (one host read of ``info``)."""
    fac, info = cholesky_ex(matrix)
    if int(info) > 0:
        raise torch.linalg.LinAlgError(f"the leading minor of order {int(info)} is not positive definite")
    return fac


def cholesky_solve(rhs: torch.Tensor, factor: torch.Tensor) -> torch.Tensor:
    """(L L^T)^-1 rhs for one (n) or several (n x k) right-hand sides, float64."""
    L.require_cuda(rhs, "dense Cholesky solve")
    n = factor.shape[0]
    b = rhs.to(torch.float64)
    cols = b.reshape(n, -1).contiguous().clone()
    fac = factor.contiguous()
    L.call("tls_dense_cholesky_solve", n, fac.data_ptr(), n, cols.shape[1], cols.data_ptr(), cols.shape[1],
           L.stream_handle(rhs.device))
    return cols.reshape(rhs.shape)
