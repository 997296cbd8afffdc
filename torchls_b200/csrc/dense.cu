// Dense float64 Cholesky factorisation and solves (row-major, lower).
//
// Replaces torch.linalg.cholesky / cholesky_solve at the reference's dense
// call sites: the reduced-camera matrix of schur_dense (torchls
// solvers.py:517-518, schur.py:380-397) and FixedLinearSystem's normal
// matrix (linear_system.py:61-98). Blocked right-looking factorisation with
// 64-column panels; per panel two launches:
//   panel   every CTA factors the 64 x 64 diagonal block in shared memory (one
//           barrier per column; CTA 0 writes it back), then its 256 rows below
//           it times L_kk^-T (one thread per row)
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

// ---------------------------------------------------------------- diagonal block and panel
// Cholesky of the nb x nb diagonal block A[k:k+nb, k:k+nb] in shared memory
// (every CTA of the panel launch factors it; CTA 0 writes it back), then the
// rows below it times L_kk^-T. The 64 x 64 block (a partial last block is
// padded with the identity) is itself factored in four 16-column sub-panels:
//   1. the 16 x 16 diagonal sub-block, column by column (thread (i, l) of a
//      16 x 16 grid subtracts S[i][j] S[l][j] / S[j][j]; one barrier per
//      column), then normalised: L[j][j] = sqrt(pivot), L[i][j] /= L[j][j];
//   2. the rows below it inside the block times its L^-T (thread per row);
//   3. the trailing part of the block minus that panel times its transpose.
// The pivot tested is the Schur-complement diagonal (L[j][j]^2).
__device__ __forceinline__ void factor_diag_block(int64_t n, const double* __restrict__ A, int64_t lda, int64_t k,
                                                  int nb, double (*S)[kNB + 1], int32_t* info, bool report) {
  constexpr int kSub = 16;
  const int tid = threadIdx.x;  // blockDim.x == 256
  __shared__ int first_bad;
  for (int e = tid; e < kNB * kNB; e += blockDim.x) {
    const int i = e >> 6, j = e & (kNB - 1);
    S[i][j] = (i < nb && j <= i) ? A[(k + i) * lda + k + j] : (i == j ? 1.0 : 0.0);
  }
  if (tid == 0) first_bad = kNB;
  __syncthreads();
#pragma unroll 1
  for (int sb = 0; sb < kNB; sb += kSub) {
    const int ti = sb + (tid >> 4), tl = sb + (tid & (kSub - 1));
    for (int j = sb; j < sb + kSub; ++j) {
      double d = S[j][j];
      if (!(d > 0.0) || !isfinite(d)) d = 1.0;  // keep going on a usable value; info reports it
      if (tl > j && tl <= ti) S[ti][tl] -= S[ti][j] * S[tl][j] * (1.0 / d);
      __syncthreads();
    }
    if (tid < kSub) {
      const int j = sb + tid;
      double d = S[j][j];
      if (!(d > 0.0) || !isfinite(d)) {
        atomicMin(&first_bad, j);
        d = 1.0;
      }
      S[j][kNB] = sqrt(d);
    }
    __syncthreads();
    if (tl < ti) S[ti][tl] /= S[tl][kNB];
    __syncthreads();
    if (tid < kSub) S[sb + tid][sb + tid] = S[sb + tid][kNB];
    __syncthreads();
    const int m = kNB - sb - kSub;
    if (m > 0) {
      if (tid < m) {  // row sb + 16 + tid of the block: x L_T^T = p
        const int i = sb + kSub + tid;
        double x[kSub];
#pragma unroll
        for (int j = 0; j < kSub; ++j) x[j] = S[i][sb + j];
#pragma unroll
        for (int j = 0; j < kSub; ++j) {
          double t = x[j];
#pragma unroll
          for (int l = 0; l < j; ++l) t -= x[l] * S[sb + j][sb + l];
          x[j] = t / S[sb + j][sb + j];
        }
#pragma unroll
        for (int j = 0; j < kSub; ++j) S[i][sb + j] = x[j];
      }
      __syncthreads();
      for (int e = tid; e < kNB * kNB; e += blockDim.x) {
        const int i = e >> 6, l = e & (kNB - 1);
        if (l >= sb + kSub && l <= i) {
          double acc = 0.0;
#pragma unroll
          for (int q = 0; q < kSub; ++q) acc += S[i][sb + q] * S[l][sb + q];
          S[i][l] -= acc;
        }
      }
      __syncthreads();
    }
  }
  // the first failing pivot of the matrix: panels run in order, so an earlier
  // panel's report is already in *info
  if (report && tid == 0 && first_bad < nb) atomicCAS(info, 0, (int32_t)(k + first_bad + 1));
}

constexpr int kPanelThreads = 256;

__global__ void __launch_bounds__(kPanelThreads) chol_panel_kernel(int64_t n, double* __restrict__ A, int64_t lda,
                                                                   int64_t k, int32_t* __restrict__ info) {
  __shared__ double L[kNB][kNB + 1];
  const int nb = (int)((n - k) < kNB ? (n - k) : kNB);
  factor_diag_block(n, A, lda, k, nb, L, info, blockIdx.x == 0);
  if (blockIdx.x == 0)
    for (int e = threadIdx.x; e < nb * nb; e += kPanelThreads) {
      const int i = e / nb, j = e % nb;
      if (j <= i) A[(k + i) * lda + k + j] = L[i][j];
    }
  // rows below: x L_kk^T = a, one thread per row, in 16-column blocks (the
  // block loops are not unrolled, so the code stays small): a block of x is
  // the row's block minus the solved blocks times L's block, then a 16-step
  // forward substitution with the reciprocal diagonal (the padding column of
  // L); solved blocks go back to the row and are re-read from L1.
  for (int j = threadIdx.x; j < kNB; j += kPanelThreads) L[j][kNB] = 1.0 / L[j][j];
  __syncthreads();
  const int64_t r = k + nb + (int64_t)blockIdx.x * kPanelThreads + threadIdx.x;
  if (r >= n) return;
  double* row = A + r * lda + k;
  constexpr int kB = 16;
#pragma unroll 1
  for (int sb = 0; sb < nb; sb += kB) {
    double x[kB];
#pragma unroll
    for (int j = 0; j < kB; ++j) x[j] = sb + j < nb ? row[sb + j] : 0.0;
#pragma unroll 1
    for (int cb = 0; cb < sb; cb += kB) {
      double y[kB];
#pragma unroll
      for (int l = 0; l < kB; ++l) y[l] = row[cb + l];
#pragma unroll
      for (int j = 0; j < kB; ++j) {
        double t = x[j];
#pragma unroll
        for (int l = 0; l < kB; ++l) t -= y[l] * L[(sb + j) & (kNB - 1)][cb + l];
        x[j] = t;
      }
    }
#pragma unroll
    for (int j = 0; j < kB; ++j) {
      double t = x[j];
#pragma unroll
      for (int l = 0; l < j; ++l) t -= x[l] * L[(sb + j) & (kNB - 1)][sb + l];
      x[j] = t * L[(sb + j) & (kNB - 1)][kNB];
    }
#pragma unroll
    for (int j = 0; j < kB; ++j)
      if (sb + j < nb) row[sb + j] = x[j];
  }
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
  // 16-byte loads, all in flight before the stores (row starts are 16-byte
  // aligned when lda and k are even; otherwise 8-byte loads)
  if (((lda | k) & 1) == 0 && nb == kNB) {
    double2 va[16], vb[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int e = tid + q * 128, i = e >> 5, j2 = (e & 31) * 2;
      const int64_t ra = r0 + i, rb = c0 + i;
      va[q] = ra < n ? *reinterpret_cast<const double2*>(A + ra * lda + k + j2) : make_double2(0.0, 0.0);
      vb[q] = rb < n ? *reinterpret_cast<const double2*>(A + rb * lda + k + j2) : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int e = tid + q * 128, i = e >> 5, j2 = (e & 31) * 2;
      Pa[i][j2] = va[q].x;
      Pa[i][j2 + 1] = va[q].y;
      Pb[i][j2] = vb[q].x;
      Pb[i][j2 + 1] = vb[q].y;
    }
  } else {
    for (int e = tid; e < kNB * kNB; e += 128) {
      const int i = e >> 6, j = e & (kNB - 1);
      const int64_t ra = r0 + i, rb = c0 + i;
      Pa[i][j] = (ra < n && j < nb) ? A[ra * lda + k + j] : 0.0;
      Pb[i][j] = (rb < n && j < nb) ? A[rb * lda + k + j] : 0.0;
    }
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
// B, row stride ldb, solved in shared memory, written back), left-looking by
// 64-row blocks. Forward, block kb: the 32 warps subtract L[kb:kb+64, :kb] y
// (a warp per row, lanes over the columns, butterfly sums), then warp 0 solves
// the diagonal block (each step's x_j broadcast by shuffle; the block and its
// reciprocal diagonal staged in shared memory). Backward, block kb from the
// end: each warp sums its rows r >= kb + 64 of L[r, kb:kb+64] y_r per column
// (lanes over the columns), the 32 warp partials are added in warp order, and
// warp 0 solves with the block's transpose.
constexpr int kSolveThreads = 1024;
constexpr int kSolveWarps = kSolveThreads / 32;

__global__ void __launch_bounds__(kSolveThreads) chol_solve_kernel(int64_t n, const double* __restrict__ L,
                                                                   int64_t lda, double* __restrict__ B, int64_t ldb) {
  // dynamic shared memory: the current diagonal block (column kNB: 1 / D[j][j]),
  // the warp partials, then y
  extern __shared__ double solve_smem[];
  double (*D)[kNB + 1] = reinterpret_cast<double (*)[kNB + 1]>(solve_smem);
  double (*part)[kNB + 1] = D + kNB;
  double* y = solve_smem + (kNB + kSolveWarps) * (kNB + 1);
  const int64_t col = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int64_t i = tid; i < n; i += kSolveThreads) y[i] = B[i * ldb + col];
  auto stage = [&](int64_t kb, int nb) {
    for (int e = tid; e < nb * kNB; e += kSolveThreads) {
      const int i = e >> 6, j = e & (kNB - 1);
      if (j < nb) D[i][j] = L[(kb + i) * lda + kb + j];
    }
    __syncthreads();
    if (tid < nb) D[tid][kNB] = 1.0 / D[tid][tid];
  };
  __syncthreads();
  for (int64_t kb = 0; kb < n; kb += kNB) {
    const int nb = (int)((n - kb) < kNB ? (n - kb) : kNB);
    stage(kb, nb);
    for (int i = warp; i < nb; i += kSolveWarps) {
      const double* lr = L + (kb + i) * lda;
      double t = 0.0;
#pragma unroll 8
      for (int64_t c = lane; c < kb; c += 32) t += lr[c] * y[c];
      t = warp_sum(t);
      if (lane == 0) y[kb + i] -= t;
    }
    __syncthreads();
    if (warp == 0) {
      double v0 = lane < nb ? y[kb + lane] : 0.0, v1 = lane + 32 < nb ? y[kb + lane + 32] : 0.0;
      for (int j = 0; j < nb; ++j) {
        const double xj = __shfl_sync(0xffffffffu, j < 32 ? v0 : v1, j & 31) * D[j][kNB];
        if (lane == (j & 31)) {
          if (j < 32) v0 = xj;
          else v1 = xj;
        }
        if (lane > j && lane < nb) v0 -= D[lane][j] * xj;
        if (lane + 32 > j && lane + 32 < nb) v1 -= D[lane + 32][j] * xj;
      }
      if (lane < nb) y[kb + lane] = v0;
      if (lane + 32 < nb) y[kb + lane + 32] = v1;
    }
    __syncthreads();
  }
  const int64_t last = ((n - 1) / kNB) * kNB;
  for (int64_t kb = last; kb >= 0; kb -= kNB) {
    const int nb = (int)((n - kb) < kNB ? (n - kb) : kNB);
    stage(kb, nb);
    double a0 = 0.0, a1 = 0.0;
#pragma unroll 4
    for (int64_t r = kb + nb + warp; r < n; r += kSolveWarps) {
      const double* lr = L + r * lda + kb;
      const double yr = y[r];
      if (lane < nb) a0 += lr[lane] * yr;
      if (lane + 32 < nb) a1 += lr[lane + 32] * yr;
    }
    part[warp][lane] = a0;
    part[warp][lane + 32] = a1;
    __syncthreads();
    if (tid < nb) {
      double t = 0.0;
      for (int w = 0; w < kSolveWarps; ++w) t += part[w][tid];
      y[kb + tid] -= t;
    }
    __syncthreads();
    if (warp == 0) {
      double v0 = lane < nb ? y[kb + lane] : 0.0, v1 = lane + 32 < nb ? y[kb + lane + 32] : 0.0;
      for (int j = nb - 1; j >= 0; --j) {
        const double xj = __shfl_sync(0xffffffffu, j < 32 ? v0 : v1, j & 31) * D[j][kNB];
        if (lane == (j & 31)) {
          if (j < 32) v0 = xj;
          else v1 = xj;
        }
        if (lane < j) v0 -= D[j][lane] * xj;
        if (lane + 32 < j) v1 -= D[j][lane + 32] * xj;
      }
      if (lane < nb) y[kb + lane] = v0;
      if (lane + 32 < nb) y[kb + lane + 32] = v1;
    }
    __syncthreads();
  }
  for (int64_t i = tid; i < n; i += kSolveThreads) B[i * ldb + col] = y[i];
}

}  // namespace tls

using namespace tls;

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
    const int64_t below = n - k - kNB;
    const int64_t panel_ctas = below > 0 ? (below + kPanelThreads - 1) / kPanelThreads : 1;
    chol_panel_kernel<<<(unsigned)panel_ctas, kPanelThreads, 0, s>>>(n, A, lda, k, info);
    TLS_CHECK_LAUNCH();
    if (below <= 0) break;
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
  const size_t smem = ((size_t)n + (kNB + kSolveWarps) * (kNB + 1)) * sizeof(double);
  if (smem > 227 * 1024) return tls_set_error(TLS_ERR_UNSUPPORTED, "dense Cholesky solve: n above 22,816");
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(chol_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return tls_set_cuda_error(e);
  }
  chol_solve_kernel<<<(unsigned)nrhs, kSolveThreads, smem, s>>>(n, L, lda, B, ldb);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}
