// Dense float64 Cholesky factorisation and solves (row-major, lower).
//
// Replaces torch.linalg.cholesky / cholesky_solve at the reference's dense
// call sites: the reduced-camera matrix of schur_dense (torchls
// solvers.py:517-518, schur.py:380-397) and FixedLinearSystem's normal
// matrix (linear_system.py:61-98). Blocked right-looking factorisation with
// 64-column panels; per panel three launches:
//   diag    the 64 x 64 diagonal block, unblocked, in shared memory
//   panel   the rows below it times L_kk^-T (one thread per row)
//   update  the trailing lower triangle -= P P^T, one 64 x 64 tile per CTA on
//           the FP64 tensor cores (mma.sync m8n8k4 .f64; 4 warps, each a
//           32 x 32 quadrant of 16 accumulator tiles)
// Every sum runs in a fixed order: results are deterministic. A pivot that
// is not positive (or not finite) is reported as its 1-based index in *info
// (the first one), as LAPACK's potrf does; the factor is then not usable.
#include <stdint.h>

#include "common.cuh"

namespace tls {

constexpr int kNB = 64;  // panel width

// ---------------------------------------------------------------- diagonal block
// Unblocked right-looking Cholesky of A[k:k+nb, k:k+nb] in shared memory.
__global__ void __launch_bounds__(256) chol_diag_kernel(int64_t n, double* __restrict__ A, int64_t lda, int64_t k,
                                                        int32_t* __restrict__ info) {
  __shared__ double S[kNB][kNB + 1];
  const int nb = (int)((n - k) < kNB ? (n - k) : kNB);
  const int tid = threadIdx.x;
  for (int e = tid; e < nb * nb; e += 256) {
    const int i = e / nb, j = e % nb;
    S[i][j] = j <= i ? A[(k + i) * lda + k + j] : 0.0;
  }
  __syncthreads();
  for (int j = 0; j < nb; ++j) {
    if (tid == 0) {
      double d = S[j][j];
      if (!(d > 0.0) || !isfinite(d)) {
        atomicCAS(info, 0, (int32_t)(k + j + 1));
        d = 1.0;  // keep going on a usable value; the caller reads info
      }
      S[j][j] = sqrt(d);
    }
    __syncthreads();
    const double inv = 1.0 / S[j][j];
    for (int i = j + 1 + tid; i < nb; i += 256) S[i][j] *= inv;
    __syncthreads();
    // trailing lower triangle of the block: S[i][l] -= S[i][j] S[l][j], j < l <= i
    const int m = nb - j - 1;
    for (int e = tid; e < m * m; e += 256) {
      const int i = j + 1 + e / m, l = j + 1 + e % m;
      if (l <= i) S[i][l] -= S[i][j] * S[l][j];
    }
    __syncthreads();
  }
  for (int e = tid; e < nb * nb; e += 256) {
    const int i = e / nb, j = e % nb;
    if (j <= i) A[(k + i) * lda + k + j] = S[i][j];
  }
}

// ---------------------------------------------------------------- panel
// A[r, k:k+nb] <- A[r, k:k+nb] L_kk^-T for r >= k + nb: forward substitution
// x L_kk^T = a, one thread per row, L_kk in shared memory.
__global__ void __launch_bounds__(128) chol_panel_kernel(int64_t n, double* __restrict__ A, int64_t lda, int64_t k) {
  __shared__ double L[kNB][kNB + 1];
  const int nb = (int)((n - k) < kNB ? (n - k) : kNB);
  for (int e = threadIdx.x; e < nb * nb; e += 128) {
    const int i = e / nb, j = e % nb;
    L[i][j] = j <= i ? A[(k + i) * lda + k + j] : 0.0;
  }
  __syncthreads();
  const int64_t r = k + nb + (int64_t)blockIdx.x * 128 + threadIdx.x;
  if (r >= n) return;
  double* row = A + r * lda + k;
  double x[kNB];
#pragma unroll
  for (int j = 0; j < kNB; ++j) {
    if (j < nb) {
      double t = row[j];
#pragma unroll
      for (int l = 0; l < j; ++l) t -= x[l] * L[j][l];
      x[j] = t / L[j][j];
    } else {
      x[j] = 0.0;
    }
  }
#pragma unroll
  for (int j = 0; j < kNB; ++j)
    if (j < nb) row[j] = x[j];
}

// ---------------------------------------------------------------- trailing update
__device__ __forceinline__ void dmma_8x8x4(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// Tile (bi, bj), bi >= bj, of the trailing matrix (rows/cols from t0 = k + nb):
// C -= P_bi P_bj^T with P the panel columns k:k+nb (K = nb <= 64). The tile
// index enumerates the lower triangle of tiles row by row.
constexpr int kUpdateSmem = 2 * kNB * (kNB + 1) * (int)sizeof(double);

__global__ void __launch_bounds__(128) chol_update_kernel(int64_t n, double* __restrict__ A, int64_t lda, int64_t k) {
  extern __shared__ double upd_smem[];
  double (*Pa)[kNB + 1] = reinterpret_cast<double (*)[kNB + 1]>(upd_smem);
  double (*Pb)[kNB + 1] = Pa + kNB;
  const int nb = (int)((n - k) < kNB ? (n - k) : kNB);
  const int64_t t0 = k + nb;
  // tile (bi, bj) from the linear lower-triangle index
  const int64_t t = blockIdx.x;
  int64_t bi = (int64_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((bi + 1) * (bi + 2) / 2 <= t) ++bi;
  while (bi * (bi + 1) / 2 > t) --bi;
  const int64_t bj = t - bi * (bi + 1) / 2;
  const int64_t r0 = t0 + bi * kNB, c0 = t0 + bj * kNB;
  const int tid = threadIdx.x;
  for (int e = tid; e < kNB * kNB; e += 128) {
    const int i = e / kNB, j = e % kNB;
    const int64_t ra = r0 + i, rb = c0 + i;
    Pa[i][j] = (ra < n && j < nb) ? A[ra * lda + k + j] : 0.0;
    Pb[i][j] = (rb < n && j < nb) ? A[rb * lda + k + j] : 0.0;
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, q = lane & 3;  // fragment row group, thread in group
  const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
#pragma unroll 4
  for (int kk = 0; kk < kNB; kk += 4) {
    double fa[4], fb[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) fa[a] = Pa[wr + a * 8 + g][kk + q];  // A(row g, col q)
#pragma unroll
    for (int b = 0; b < 4; ++b) fb[b] = Pb[wc + b * 8 + g][kk + q];  // B(k = q, col g) = P_bj[col][k]
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) dmma_8x8x4(acc[a][b], fa[a], fb[b]);
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int64_t r = r0 + wr + a * 8 + g, c = c0 + wc + b * 8 + 2 * q + h;
        if (r < n && c < n && c <= r) A[r * lda + c] -= acc[a][b][h];
      }
}

__global__ void chol_zero_upper_kernel(int64_t n, double* __restrict__ A, int64_t lda) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * n) return;
  const int64_t i = e / n, j = e % n;
  if (j > i) A[i * lda + j] = 0.0;
}

// ---------------------------------------------------------------- solves
// L L^T x = b for one right-hand side column per CTA (b read from column c of
// B, row stride ldb, solved in shared memory, written back). Forward:
// per 64-row block, warp 0 solves the diagonal block (each step's x_j
// broadcast by shuffle), then every thread updates one later row with the
// block's columns in order. Backward: the same with L^T, block by block from
// the end; the update of an earlier row r sums column r of the block's rows.
__global__ void __launch_bounds__(256) chol_solve_kernel(int64_t n, const double* __restrict__ L, int64_t lda,
                                                         double* __restrict__ B, int64_t ldb) {
  extern __shared__ double y[];
  const int64_t col = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int64_t i = tid; i < n; i += 256) y[i] = B[i * ldb + col];
  __syncthreads();
  for (int64_t kb = 0; kb < n; kb += kNB) {
    const int nb = (int)((n - kb) < kNB ? (n - kb) : kNB);
    if (warp == 0) {
      double v0 = lane < nb ? y[kb + lane] : 0.0, v1 = lane + 32 < nb ? y[kb + lane + 32] : 0.0;
      for (int j = 0; j < nb; ++j) {
        const double bj = __shfl_sync(0xffffffffu, j < 32 ? v0 : v1, j & 31);
        const double xj = bj / L[(kb + j) * lda + kb + j];
        if (lane == (j & 31)) {
          if (j < 32) v0 = xj;
          else v1 = xj;
        }
        if (lane > j && lane < nb) v0 -= L[(kb + lane) * lda + kb + j] * xj;
        if (lane + 32 > j && lane + 32 < nb) v1 -= L[(kb + lane + 32) * lda + kb + j] * xj;
      }
      if (lane < nb) y[kb + lane] = v0;
      if (lane + 32 < nb) y[kb + lane + 32] = v1;
    }
    __syncthreads();
    for (int64_t r = kb + nb + tid; r < n; r += 256) {
      double t = y[r];
      const double* lr = L + r * lda + kb;
      for (int j = 0; j < nb; ++j) t -= lr[j] * y[kb + j];
      y[r] = t;
    }
    __syncthreads();
  }
  const int64_t last = ((n - 1) / kNB) * kNB;
  for (int64_t kb = last; kb >= 0; kb -= kNB) {
    const int nb = (int)((n - kb) < kNB ? (n - kb) : kNB);
    if (warp == 0) {
      double v0 = lane < nb ? y[kb + lane] : 0.0, v1 = lane + 32 < nb ? y[kb + lane + 32] : 0.0;
      for (int j = nb - 1; j >= 0; --j) {
        const double bj = __shfl_sync(0xffffffffu, j < 32 ? v0 : v1, j & 31);
        const double xj = bj / L[(kb + j) * lda + kb + j];
        if (lane == (j & 31)) {
          if (j < 32) v0 = xj;
          else v1 = xj;
        }
        if (lane < j) v0 -= L[(kb + j) * lda + kb + lane] * xj;
        if (lane + 32 < j) v1 -= L[(kb + j) * lda + kb + lane + 32] * xj;
      }
      if (lane < nb) y[kb + lane] = v0;
      if (lane + 32 < nb) y[kb + lane + 32] = v1;
    }
    __syncthreads();
    for (int64_t r = tid; r < kb; r += 256) {
      double t = y[r];
      for (int j = 0; j < nb; ++j) t -= L[(kb + j) * lda + r] * y[kb + j];
      y[r] = t;
    }
    __syncthreads();
  }
  for (int64_t i = tid; i < n; i += 256) B[i * ldb + col] = y[i];
}

// ---------------------------------------------------------------- reduced-camera matrix
// S = s U s + lambda I - W W^T from the one-group Schur system's slabs
// (schur.py:380-397). Pass 1 writes the block diagonal base (zeros
// elsewhere); pass 2 has one warp per lower block (i, j) sum W_a W_b^T over
// the pairs (a, b) of edges of a shared eliminated variable, in list order,
// and subtract it from block (i, j) and its mirror. W is read as stored.
__device__ __forceinline__ int64_t slab_w(int64_t s, int k, int cap, int kw) {
  return ((s / cap) * kw + k) * cap + (s % cap);
}

__global__ void schur_dense_base_kernel(tls_schur_args a, double* __restrict__ S) {
  const int64_t n = (int64_t)a.nretained * a.dr;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * n) return;
  const int64_t r = e / n, c = e % n;
  const int64_t i = r / a.dr, j = c / a.dr;
  double v = 0.0;
  if (i == j) {
    const int rr = (int)(r % a.dr), cc = (int)(c % a.dr);
    // scales in index order: entries (r, c) and (c, r) get the same bits
    const int64_t lo = r < c ? r : c, hi = r < c ? c : r;
    const double sl = a.scale ? a.scale[a.retained_offset + lo] : 1.0;
    const double sh = a.scale ? a.scale[a.retained_offset + hi] : 1.0;
    v = sl * a.ret_diag[i * a.dr * a.dr + rr * a.dr + cc] * sh + (rr == cc ? a.damping : 0.0);
  }
  S[e] = v;
}

template <typename TW>
__global__ void __launch_bounds__(128) schur_dense_pairs_kernel(tls_schur_args a, int64_t ntargets,
                                                                const int32_t* __restrict__ target_r,
                                                                const int32_t* __restrict__ target_c,
                                                                const int32_t* __restrict__ ptr,
                                                                const int32_t* __restrict__ pa,
                                                                const int32_t* __restrict__ pb,
                                                                double* __restrict__ S) {
  const int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= ntargets) return;
  const int dr = a.dr, de = a.de, kw = dr * de;
  const TW* w = reinterpret_cast<const TW*>(a.w);
  const int64_t n = (int64_t)a.nretained * dr;
  const int64_t i = target_r[t], j = target_c[t];
  for (int ent = lane; ent < dr * dr; ent += 32) {
    const int r = ent / dr, c = ent % dr;
    double acc = 0.0;
    for (int k = ptr[t]; k < ptr[t + 1]; ++k) {
      const int64_t sa = pa[k], sb = pb[k];
      double v = 0.0;
      for (int b = 0; b < de; ++b)
        v += to_d(w[slab_w(sa, r * de + b, a.cap, kw)]) * to_d(w[slab_w(sb, c * de + b, a.cap, kw)]);
      acc += v;
    }
    const int64_t row = i * dr + r, col = j * dr + c;
    S[row * n + col] -= acc;
    if (i != j) S[col * n + row] -= acc;
  }
}

}  // namespace tls

using namespace tls;

extern "C" int tls_schur_dense_matrix(const tls_schur_args* a, int64_t ntargets, const int32_t* target_r,
                                      const int32_t* target_c, const int32_t* ptr, const int32_t* pair_a,
                                      const int32_t* pair_b, double* S, tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (!a || !S) return tls_set_error(TLS_ERR_INVALID, "dense Schur matrix: bad arguments");
  const int64_t n = (int64_t)a->nretained * a->dr;
  if (n > 0) schur_dense_base_kernel<<<(unsigned)((n * n + 255) / 256), 256, 0, s>>>(*a, S);
  TLS_CHECK_LAUNCH();
  if (ntargets > 0) {
    const unsigned grid = (unsigned)((ntargets * 32 + 127) / 128);
    if (a->wdtype == TLS_F64)
      schur_dense_pairs_kernel<double><<<grid, 128, 0, s>>>(*a, ntargets, target_r, target_c, ptr, pair_a, pair_b, S);
    else
      schur_dense_pairs_kernel<float><<<grid, 128, 0, s>>>(*a, ntargets, target_r, target_c, ptr, pair_a, pair_b, S);
  }
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}

extern "C" int tls_dense_cholesky(int64_t n, double* A, int64_t lda, int32_t* info, tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (n < 0 || lda < n || !A || !info) return tls_set_error(TLS_ERR_INVALID, "dense Cholesky: bad arguments");
  cudaError_t e = cudaMemsetAsync(info, 0, sizeof(int32_t), s);
  if (e != cudaSuccess) return tls_set_cuda_error(e);
  static DeviceGridCache configured;  // the update kernel's shared-memory limit, once per device
  int unused = 0;
  if (int rc = configured.get(kUpdateSmem, &unused, [](int) -> int {
        return cudaFuncSetAttribute(chol_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kUpdateSmem) ==
                       cudaSuccess
                   ? 1
                   : -1;
      }))
    return rc;
  for (int64_t k = 0; k < n; k += kNB) {
    chol_diag_kernel<<<1, 256, 0, s>>>(n, A, lda, k, info);
    TLS_CHECK_LAUNCH();
    const int64_t below = n - k - kNB;
    if (below <= 0) break;
    chol_panel_kernel<<<(unsigned)((below + 127) / 128), 128, 0, s>>>(n, A, lda, k);
    TLS_CHECK_LAUNCH();
    const int64_t T = (below + kNB - 1) / kNB;
    chol_update_kernel<<<(unsigned)(T * (T + 1) / 2), 128, kUpdateSmem, s>>>(n, A, lda, k);
    TLS_CHECK_LAUNCH();
  }
  if (n > 0) chol_zero_upper_kernel<<<(unsigned)((n * n + 255) / 256), 256, 0, s>>>(n, A, lda);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}

extern "C" int tls_dense_cholesky_solve(int64_t n, const double* L, int64_t lda, int64_t nrhs, double* B, int64_t ldb,
                                        tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (n < 0 || nrhs < 0 || lda < n || ldb < nrhs || (n > 0 && (!L || !B)))
    return tls_set_error(TLS_ERR_INVALID, "dense Cholesky solve: bad arguments");
  if (n == 0 || nrhs == 0) return TLS_OK;
  const size_t smem = (size_t)n * sizeof(double);
  if (smem > 227 * 1024) return tls_set_error(TLS_ERR_UNSUPPORTED, "dense Cholesky solve: n above 29,056");
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(chol_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return tls_set_cuda_error(e);
  }
  chol_solve_kernel<<<(unsigned)nrhs, 256, smem, s>>>(n, L, lda, B, ldb);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}
