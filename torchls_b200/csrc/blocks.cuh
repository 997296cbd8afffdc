// Small dense block helpers (float64): Cholesky factor and two triangular
// solves, used by block-Jacobi (torchls solvers.py:259-285,
// preconditioning.py:12-17) and the Schur eliminated blocks (schur.py:263-269).
#pragma once
#include "common.cuh"

namespace tls {

constexpr int kMaxBlock = 16;

// Lower Cholesky of a (dim x dim) row-major block; returns false when a pivot
// is not positive or not finite (torch.linalg.cholesky raises LinAlgError).
__device__ __forceinline__ bool cholesky_block(const double* A, double* L, int dim, double damping) {
  bool ok = true;
  for (int j = 0; j < dim; ++j) {
    double s = A[j * dim + j] + damping;
    for (int k = 0; k < j; ++k) s -= L[j * dim + k] * L[j * dim + k];
    if (!(s > 0.0) || !isfinite(s)) {
      ok = false;
      s = 1.0;
    }
    const double d = sqrt(s);
    L[j * dim + j] = d;
    for (int i = j + 1; i < dim; ++i) {
      double t = A[i * dim + j];
      for (int k = 0; k < j; ++k) t -= L[i * dim + k] * L[j * dim + k];
      L[i * dim + j] = t / d;
    }
    for (int i = 0; i < j; ++i) L[i * dim + j] = 0.0;
  }
  return ok;
}

// z = (L L^T)^-1 r
__device__ __forceinline__ void cholesky_solve_block(const double* L, int dim, const double* r, double* z) {
  double y[kMaxBlock];
  for (int i = 0; i < dim; ++i) {
    double t = r[i];
    for (int k = 0; k < i; ++k) t -= L[i * dim + k] * y[k];
    y[i] = t / L[i * dim + i];
  }
  for (int i = dim - 1; i >= 0; --i) {
    double t = y[i];
    for (int k = i + 1; k < dim; ++k) t -= L[k * dim + i] * z[k];
    z[i] = t / L[i * dim + i];
  }
}

// Eliminated block of the Schur complement: L = chol(s C s + damping I) of the
// unscaled block C (row-major DE x DE) and column scales s; writes L^-1
// (forward substitution on unit vectors). False when a pivot fails.
template <int DE>
__device__ __forceinline__ bool eliminated_factor(const double* C_in, const double (&s)[DE], double damping,
                                                  double* inv_out) {
  double C[DE * DE], L[DE * DE];
#pragma unroll
  for (int i = 0; i < DE; ++i)
#pragma unroll
    for (int j = 0; j < DE; ++j) C[i * DE + j] = s[i] * C_in[i * DE + j] * s[j];
  const bool ok = cholesky_block(C, L, DE, damping);
  double Li[DE * DE];
#pragma unroll
  for (int col = 0; col < DE; ++col) {
#pragma unroll
    for (int i = 0; i < DE; ++i) {
      double t = (i == col) ? 1.0 : 0.0;
#pragma unroll
      for (int k = 0; k < DE; ++k)
        if (k < i) t -= L[i * DE + k] * Li[k * DE + col];
      Li[i * DE + col] = t / L[i * DE + i];
    }
  }
#pragma unroll
  for (int k = 0; k < DE * DE; ++k) inv_out[k] = Li[k];
  return ok;
}

// Column of element k of block i in a (possibly joint) block group.
__device__ __forceinline__ int64_t block_column(const tls_block_group& g, int64_t i, int k) {
  int start = 0;
  for (int m = 0; m < g.nmembers; ++m) {
    const int d = g.member_dim[m];
    if (k < start + d) return g.member_offset[m] + i * d + (k - start);
    start += d;
  }
  return -1;
}

}  // namespace tls
