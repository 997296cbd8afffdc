// Batched independent problems: one dense reduced-camera matrix per problem
// and one persistent preconditioned-CG launch over all of them.
//
// The batched solver (batched.py) merges thousands of small bundle
// adjustments into one block-diagonal system. Each problem's reduced matrix
// S_p = s U s + lambda I - W W^T (schur.py:380-397 restricted to the problem)
// has n_p = cameras x 6 <= a few hundred rows, so it is assembled once per LM
// trial (fixed-order sums over the shared points of each camera pair, one
// rounding to the storage type) and the CG iterations of all problems then
// run in ONE launch: a persistent grid whose CTAs pull tasks from a work
// queue (one device counter). A task is 1, 2, 4 or 8 problems of one size
// class sharing a 256-thread CTA (8, 4, 2 or 1 warps per problem: the
// tiling, chosen per size class by the host autotuner). Each problem runs
// its own CG (alpha, beta, threshold, convergence: batched.py's per-problem
// semantics) with group-local barriers only, so no problem waits for
// another. The matrix is copied once into shared memory (packed lower
// triangle) when it fits the group's share, else it is re-read from global
// memory each iteration.
//
// Determinism independent of the tiling: a matrix row is reduced by one warp
// (lanes over columns, butterfly), every dot product is computed redundantly
// by each warp of the group in the same lane-strided order, and vector
// updates are per block; no result depends on how many warps a problem has.
#include <stdint.h>

#include "common.cuh"

namespace tls {
namespace {

constexpr int kBatchThreads = 256;
constexpr int kHeader = 16;  // per-group shared flags

// s_r U_rc s_c + lambda [r == c], the scales multiplied in index order so
// that entries (r, c) and (c, r) of a symmetric U get the same bits.
__device__ __forceinline__ double base_entry(const tls_schur_args& a, int64_t i, int r, int c) {
  const int dr = a.dr, lo = r < c ? r : c, hi = r < c ? c : r;
  const double sl = a.scale ? a.scale[a.retained_offset + i * dr + lo] : 1.0;
  const double sh = a.scale ? a.scale[a.retained_offset + i * dr + hi] : 1.0;
  return sl * a.ret_diag[(i * dr + r) * dr + c] * sh + (r == c ? a.damping : 0.0);
}

__device__ __forceinline__ int64_t slab_index(int64_t s, int k, int cap, int kw) {
  return ((s / cap) * kw + k) * cap + (s % cap);
}

// The problem of retained variable i: its first variable, dimension and
// matrix offset; without problem arrays, one problem of every variable.
struct ProblemView {
  int64_t first, n, off;
};

__device__ __forceinline__ ProblemView problem_of(const tls_batched_systems& b, int64_t i, int dr) {
  if (!b.ret_problem) return {0, (int64_t)b.nretained * dr, 0};
  const int p = b.ret_problem[i];
  const int64_t first = b.ret_ptr[p];
  return {first, (int64_t)(b.ret_ptr[p + 1] - first) * dr, b.s_off[p]};
}

// ---------------------------------------------------------------- assembly
// One CTA per retained variable i: its dr rows of S_p (zeros outside the
// diagonal block) and its float64 diagonal block.
template <typename TS>
__global__ void __launch_bounds__(128) batched_dense_base_kernel(tls_schur_args a, tls_batched_systems b) {
  const int64_t i = blockIdx.x;
  const int dr = a.dr;
  const ProblemView pv = problem_of(b, i, dr);
  const int64_t n = pv.n, li = i - pv.first;
  TS* S = reinterpret_cast<TS*>(b.S) + pv.off;
  for (int64_t e = threadIdx.x; e < dr * n; e += blockDim.x) {
    const int r = (int)(e / n);
    const int64_t c = e % n;
    double v = 0.0;
    if (c / dr == li) {
      const int cc = (int)(c % dr);
      v = base_entry(a, i, r, cc);
      if (b.diag) b.diag[(i * dr + r) * dr + cc] = v;
    }
    S[((int64_t)li * dr + r) * n + c] = static_cast<TS>(v);
  }
}

// Warp per lower block (i, j) that shares eliminated variables: the sum of
// W_a W_b^T over its pairs in list order, one rounding to TS, written to the
// block and its mirror (the diagonal block adds its base and is also kept in
// float64 for the preconditioner).
template <typename TW, typename TS>
__global__ void __launch_bounds__(128) batched_dense_pairs_kernel(tls_schur_args a, tls_batched_systems b,
                                                                  int64_t ntargets,
                                                                  const int32_t* __restrict__ target_r,
                                                                  const int32_t* __restrict__ target_c,
                                                                  const int32_t* __restrict__ ptr,
                                                                  const int32_t* __restrict__ pa,
                                                                  const int32_t* __restrict__ pb) {
  const int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= ntargets) return;
  const int dr = a.dr, de = a.de, kw = dr * de;
  const TW* w = reinterpret_cast<const TW*>(a.w);
  const int64_t i = target_r[t], j = target_c[t];
  const ProblemView pv = problem_of(b, i, dr);
  const int64_t n = pv.n, li = i - pv.first, lj = j - pv.first;
  TS* S = reinterpret_cast<TS*>(b.S) + pv.off;
  for (int ent = lane; ent < dr * dr; ent += 32) {
    const int r = ent / dr, c = ent % dr;
    double acc = 0.0;
    for (int k = ptr[t]; k < ptr[t + 1]; ++k) {
      const int64_t sa = pa[k], sb = pb[k];
      double v = 0.0;
      for (int q = 0; q < de; ++q)
        v += to_d(w[slab_index(sa, r * de + q, a.cap, kw)]) * to_d(w[slab_index(sb, c * de + q, a.cap, kw)]);
      acc += v;
    }
    const double v = (i == j ? base_entry(a, i, r, c) : 0.0) - acc;
    S[(li * dr + r) * n + lj * dr + c] = static_cast<TS>(v);
    if (i != j)
      S[(lj * dr + c) * n + li * dr + r] = static_cast<TS>(v);
    else if (b.diag)
      b.diag[(i * dr + r) * dr + c] = v;
  }
}

// The same blocks with the pairs spread over the lanes: lane l takes the
// pairs l, l + 32, ... of its target (in list order), loads each W_a once and
// keeps all DR x DR partial sums in registers; the 32 lane partials of every
// entry are then added in lane order through shared memory. Fixed order:
// deterministic (the order differs from the list order of the generic kernel).
template <int DR, int DE, typename TW, typename TS, int H>
__global__ void __launch_bounds__(128, H == 2 ? 6 : 1) batched_dense_lanes_kernel(tls_schur_args a,
                                                                                  tls_batched_systems b,
                                                                  int64_t ntargets,
                                                                  const int32_t* __restrict__ target_r,
                                                                  const int32_t* __restrict__ target_c,
                                                                  const int32_t* __restrict__ ptr,
                                                                  const int32_t* __restrict__ pa,
                                                                  const int32_t* __restrict__ pb) {
  // rows in H parts (one pass over the pairs each, W re-read from L2): with
  // H = 2 half the sums live in registers at a time, so more warps fit an SM
  // (many blocks of few pairs: the batched problems); H = 1 reads W once
  // (few blocks of many pairs: one problem). Every entry's products and sums
  // run in the same order either way.
  static_assert(DR % H == 0, "rows split evenly");
  constexpr int RH = DR / H, NEH = RH * DR;
  __shared__ double red[4][32][NEH + 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t t = (int64_t)blockIdx.x * 4 + warp;
  if (t >= ntargets) return;
  const TW* w = reinterpret_cast<const TW*>(a.w);
  const int k0 = ptr[t], k1 = ptr[t + 1];
  const int64_t i = target_r[t], j = target_c[t];
  const ProblemView pv = problem_of(b, i, DR);
  const int64_t n = pv.n, li = i - pv.first, lj = j - pv.first;
  TS* S = reinterpret_cast<TS*>(b.S) + pv.off;
#pragma unroll 1
  for (int h = 0; h < H; ++h) {
    double acc[NEH];
#pragma unroll
    for (int e = 0; e < NEH; ++e) acc[e] = 0.0;
    for (int k = k0 + lane; k < k1; k += 32) {
      const int64_t sa = pa[k], sb = pb[k];
      const int64_t ba = (sa / a.cap) * DR * DE * a.cap + (sa % a.cap),
                    bb = (sb / a.cap) * DR * DE * a.cap + (sb % a.cap);
      double wa[RH * DE];
#pragma unroll
      for (int m = 0; m < RH * DE; ++m) wa[m] = to_d(w[ba + (int64_t)(h * RH * DE + m) * a.cap]);
#pragma unroll
      for (int c = 0; c < DR; ++c) {
        double wc[DE];
#pragma unroll
        for (int q = 0; q < DE; ++q) wc[q] = to_d(w[bb + (int64_t)(c * DE + q) * a.cap]);
#pragma unroll
        for (int r = 0; r < RH; ++r) {
          double v = 0.0;
#pragma unroll
          for (int q = 0; q < DE; ++q) v += wa[r * DE + q] * wc[q];
          acc[r * DR + c] += v;
        }
      }
    }
    __syncwarp();  // the previous half's sums have been read
#pragma unroll
    for (int e = 0; e < NEH; ++e) red[warp][lane][e] = acc[e];
    __syncwarp();
    for (int e = lane; e < NEH; e += 32) {
      double sum = 0.0;
      for (int l = 0; l < 32; ++l) sum += red[warp][l][e];
      const int r = h * RH + e / DR, c = e % DR;
      const double v = (i == j ? base_entry(a, i, r, c) : 0.0) - sum;
      S[(li * DR + r) * n + lj * DR + c] = static_cast<TS>(v);
      if (i != j)
        S[(lj * DR + c) * n + li * DR + r] = static_cast<TS>(v);
      else if (b.diag)
        b.diag[(i * DR + r) * DR + c] = v;
    }
  }
}

template <int DR, int DE, int H>
void launch_lanes(const tls_schur_args& a, const tls_batched_systems& b, int64_t ntargets, const int32_t* tr,
                  const int32_t* tc, const int32_t* ptr, const int32_t* pa, const int32_t* pb, cudaStream_t s) {
  const unsigned grid = (unsigned)((ntargets + 3) / 4);
  const bool w64 = a.wdtype == TLS_F64, s64 = b.sdtype == TLS_F64;
  if (w64 && s64)
    batched_dense_lanes_kernel<DR, DE, double, double, H><<<grid, 128, 0, s>>>(a, b, ntargets, tr, tc, ptr, pa, pb);
  else if (w64)
    batched_dense_lanes_kernel<DR, DE, double, float, H><<<grid, 128, 0, s>>>(a, b, ntargets, tr, tc, ptr, pa, pb);
  else if (s64)
    batched_dense_lanes_kernel<DR, DE, float, double, H><<<grid, 128, 0, s>>>(a, b, ntargets, tr, tc, ptr, pa, pb);
  else
    batched_dense_lanes_kernel<DR, DE, float, float, H><<<grid, 128, 0, s>>>(a, b, ntargets, tr, tc, ptr, pa, pb);
}

// ---------------------------------------------------------------- PCG
__device__ __forceinline__ void group_sync(int g, int warps) {
  if (warps == 1)
    __syncwarp();
  else
    asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(warps * 32) : "memory");
}

// sum_i a[i] b[i] by one warp (lane l takes l, l + 32, ...; then the
// butterfly): every lane of every warp that computes it gets the same bits.
__device__ __forceinline__ double warp_dot(const double* a, const double* b, int n, int lane) {
  double s = 0.0;
  for (int i = lane; i < n; i += 32) s += a[i] * b[i];
  return warp_sum(s);
}

template <typename TS>
__device__ __forceinline__ double row_packed(const TS* P, const double* v, int i, int n, int lane) {
  double s = 0.0;
  const int64_t ri = (int64_t)i * (i + 1) / 2;
  for (int j = lane; j < n; j += 32) {
    const TS m = j <= i ? P[ri + j] : P[(int64_t)j * (j + 1) / 2 + i];
    s += to_d(m) * v[j];
  }
  return warp_sum(s);
}

template <typename TS>
__device__ __forceinline__ double row_full(const TS* __restrict__ S, const double* v, int i, int n, int lane) {
  double s = 0.0;
  const TS* row = S + (int64_t)i * n;
  for (int j = lane; j < n; j += 32) s += to_d(row[j]) * v[j];
  return warp_sum(s);
}

// Lower Cholesky factor of one DR x DR block (row-major, zeros above);
// false when a pivot is not positive or not finite.
template <int DR>
__device__ __forceinline__ bool factor_block(const double* __restrict__ A, double* L) {
  double l[DR][DR];
#pragma unroll
  for (int i = 0; i < DR; ++i)
#pragma unroll
    for (int j = 0; j < DR; ++j) l[i][j] = A[i * DR + j];
  bool ok = true;
#pragma unroll
  for (int j = 0; j < DR; ++j) {
    double d = l[j][j];
#pragma unroll
    for (int k = 0; k < j; ++k) d -= l[j][k] * l[j][k];
    if (!(d > 0.0) || !isfinite(d)) {
      ok = false;
      d = 1.0;
    }
    d = sqrt(d);
    l[j][j] = d;
#pragma unroll
    for (int i = j + 1; i < DR; ++i) {
      double v = l[i][j];
#pragma unroll
      for (int k = 0; k < j; ++k) v -= l[i][k] * l[j][k];
      l[i][j] = v / d;
    }
  }
#pragma unroll
  for (int i = 0; i < DR; ++i)
#pragma unroll
    for (int j = 0; j < DR; ++j) L[i * DR + j] = j <= i ? l[i][j] : 0.0;
  return ok;
}

// z = (L L^T)^-1 r for one block.
template <int DR>
__device__ __forceinline__ void apply_block(const double* L, const double* r, double* z) {
  double y[DR];
#pragma unroll
  for (int i = 0; i < DR; ++i) {
    double v = r[i];
#pragma unroll
    for (int k = 0; k < i; ++k) v -= L[i * DR + k] * y[k];
    y[i] = v / L[i * DR + i];
  }
#pragma unroll
  for (int i = DR - 1; i >= 0; --i) {
    double v = y[i];
#pragma unroll
    for (int k = i + 1; k < DR; ++k) v -= L[k * DR + i] * y[k];
    y[i] = v / L[i * DR + i];
  }
#pragma unroll
  for (int i = 0; i < DR; ++i) z[i] = y[i];
}

// Bytes of a group's share that a problem of nb blocks needs without and
// with the packed matrix cache.
template <int DR>
__host__ __device__ __forceinline__ int64_t vector_bytes(int nb) {
  const int64_t n = (int64_t)nb * DR;
  return kHeader + (4 * n + (int64_t)nb * DR * DR) * (int64_t)sizeof(double);
}

// CG of problem p by group g (warps consecutive warps, share bytes of
// shared memory at `share`).
template <int DR, typename TS>
__device__ void solve_problem(const tls_batched_systems& sys, const tls_batched_pcg_args& a, int p, int g, int warps,
                              char* share, int64_t share_bytes) {
  const int lane = threadIdx.x & 31;
  const int T = warps * 32, gt = threadIdx.x - g * T, wg = gt >> 5;
  const int first = sys.ret_ptr[p], nb = sys.ret_ptr[p + 1] - first;
  const int n = nb * DR;
  const int64_t off = (int64_t)first * DR;
  const int64_t vb = vector_bytes<DR>(nb);
  if (vb > share_bytes) {  // the host sizes tasks so that this does not happen
    if (gt == 0) {
      a.iterations[p] = 0;
      a.status[p] = 2;
      atomicExch(a.err, 1);
    }
    return;
  }
  volatile int* flag = reinterpret_cast<volatile int*>(share);
  double* r = reinterpret_cast<double*>(share + kHeader);
  double* z = r + n;
  double* pv = z + n;
  double* ap = pv + n;
  double* Lf = ap + n;
  TS* cache = reinterpret_cast<TS*>(share + vb);
  const int64_t npk = (int64_t)n * (n + 1) / 2;
  const bool cached = vb + npk * (int64_t)sizeof(TS) <= share_bytes;
  const TS* __restrict__ S = reinterpret_cast<const TS*>(sys.S) + sys.s_off[p];
  double* __restrict__ x = a.x + off;
  const double* __restrict__ b = a.rhs + off;

  if (gt == 0) *flag = 0;
  group_sync(g, warps);
  for (int k = gt; k < nb; k += T)
    if (!factor_block<DR>(sys.diag + (int64_t)(first + k) * DR * DR, Lf + k * DR * DR)) *flag = 1;
  if (cached)
    for (int i = wg; i < n; i += warps) {
      const int64_t ri = (int64_t)i * (i + 1) / 2;
      for (int j = lane; j <= i; j += 32) cache[ri + j] = S[(int64_t)i * n + j];
    }
  for (int i = gt; i < n; i += T) r[i] = b[i];
  group_sync(g, warps);
  if (*flag) {  // a preconditioner block is not positive definite: the trial is rejected
    for (int i = gt; i < n; i += T) x[i] = 0.0;
    if (gt == 0) {
      a.iterations[p] = 0;
      a.status[p] = 1;
    }
    return;
  }
  for (int k = gt; k < nb; k += T) {
    apply_block<DR>(Lf + k * DR * DR, r + k * DR, z + k * DR);
#pragma unroll
    for (int q = 0; q < DR; ++q) {
      pv[k * DR + q] = z[k * DR + q];
      x[k * DR + q] = 0.0;
    }
  }
  group_sync(g, warps);
  const double bn = sqrt(warp_dot(r, r, n, lane));
  double rz = warp_dot(r, z, n, lane);
  const double thr = fmax(a.rtol * bn, a.atol);
  int its = 0;
  if (bn > thr) {
    for (int it = 0; it < a.max_iterations; ++it) {
      for (int i = wg; i < n; i += warps) {
        const double v = cached ? row_packed(cache, pv, i, n, lane) : row_full(S, pv, i, n, lane);
        if (lane == 0) ap[i] = v;
      }
      group_sync(g, warps);
      const double pap = warp_dot(pv, ap, n, lane);
      ++its;
      if (!(pap > 0.0) || !isfinite(pap)) break;  // alpha = 0: x and r stay
      const double alpha = rz / pap;
      for (int k = gt; k < nb; k += T) {
#pragma unroll
        for (int q = 0; q < DR; ++q) {
          const int i = k * DR + q;
          x[i] += alpha * pv[i];
          r[i] -= alpha * ap[i];
        }
        apply_block<DR>(Lf + k * DR * DR, r + k * DR, z + k * DR);
      }
      group_sync(g, warps);
      const double rr = warp_dot(r, r, n, lane);
      const double rzn = warp_dot(r, z, n, lane);
      if (!(sqrt(rr) > thr)) break;
      const double beta = rzn / rz;
      for (int i = gt; i < n; i += T) pv[i] = z[i] + beta * pv[i];
      rz = rzn;
      group_sync(g, warps);
    }
  }
  if (gt == 0) {
    a.iterations[p] = its;
    a.status[p] = 0;
  }
}

template <int DR, typename TS>
__global__ void __launch_bounds__(kBatchThreads, 2) batched_pcg_kernel(tls_batched_systems sys, tls_batched_pcg_args a) {
  extern __shared__ __align__(16) char smem[];
  __shared__ int task_s;
  for (;;) {
    if (threadIdx.x == 0) task_s = atomicAdd(a.queue, 1);
    __syncthreads();
    const int t = task_s;
    __syncthreads();
    if (t >= a.ntasks) return;
    const int k = a.task_groups[t];
    const int warps = 8 / k, g = (threadIdx.x >> 5) / warps;
    const int64_t share = ((int64_t)a.smem_bytes / k) & ~int64_t(15);
    if (g < a.task_size[t]) solve_problem<DR, TS>(sys, a, a.order[a.task_first[t] + g], g, warps, smem + g * share, share);
  }
}

template <int DR, typename TS>
int launch_pcg(const tls_batched_systems& sys, const tls_batched_pcg_args& a, cudaStream_t s) {
  static DeviceGridCache cache;
  int per_sm = 0;
  if (int rc = cache.get(a.smem_bytes, &per_sm, [&](int dev) -> int {
        if (cudaFuncSetAttribute(batched_pcg_kernel<DR, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 a.smem_bytes) != cudaSuccess)
          return -1;
        int occ = 0, sms = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batched_pcg_kernel<DR, TS>, kBatchThreads,
                                                          a.smem_bytes) != cudaSuccess)
          return -1;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
        return occ * sms;
      }))
    return rc;
  if (per_sm < 1) return tls_set_error(TLS_ERR_UNSUPPORTED, "batched PCG: shared-memory size leaves no resident CTA");
  const int grid = a.ntasks < per_sm ? a.ntasks : per_sm;
  cudaError_t e = cudaMemsetAsync(a.queue, 0, sizeof(int32_t), s);
  if (e != cudaSuccess) return tls_set_cuda_error(e);
  batched_pcg_kernel<DR, TS><<<grid, kBatchThreads, a.smem_bytes, s>>>(sys, a);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}

// ---------------------------------------------------------------- LM pieces
// Per factor: new objective 1/2 w rho(s_new) and exact reduction
// 1/2 w (rho(s_old) - rho(s_new)) of rows [nfactors][rdim] (batched.py's
// Huber divided difference, torchls losses.py:92-107).
__global__ void factor_terms_kernel(int64_t nf, int rdim, const double* __restrict__ old_raw,
                                    const double* __restrict__ new_raw, int loss, double delta,
                                    const double* __restrict__ w, double* __restrict__ obj, double* __restrict__ red) {
  const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  double so = 0.0, sn = 0.0, sq = 0.0;
  for (int k = 0; k < rdim; ++k) {
    const double ro = old_raw[f * rdim + k], rn = new_raw[f * rdim + k];
    so += ro * ro;
    sn += rn * rn;
    sq += (ro - rn) * (ro + rn);
  }
  double o = sn, d = sq;
  if (loss == 1) {
    const double d2 = delta * delta;
    const double no = sqrt(fmax(so, 0.0)), nn = sqrt(fmax(sn, 0.0));
    const double rho_n = sn > d2 ? delta * (2.0 * nn - delta) : sn;
    const double rho_o = so > d2 ? delta * (2.0 * no - delta) : so;
    o = rho_n;
    if (so <= d2 && sn <= d2)
      d = sq;
    else if (so > d2 && sn > d2)
      d = 2.0 * delta * sq / fmax(no + nn, 1e-300);
    else
      d = rho_o - rho_n;
  }
  const double wf = w ? w[f] : 1.0;
  obj[f] = 0.5 * (wf * o);
  red[f] = 0.5 * (wf * d);
}

__global__ void factor_sqnorm_kernel(int64_t nf, int rdim, const double* __restrict__ rows, double* __restrict__ out) {
  const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  double s = 0.0;
  for (int k = 0; k < rdim; ++k) {
    const double v = rows[f * rdim + k];
    s += v * v;
  }
  out[f] = s;
}

// Per-problem gain ratio, acceptance and damping update (torchls
// solvers.py:597-689 decisions, one problem per thread).
__global__ void batched_lm_update_kernel(tls_batched_lm m) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m.nproblems) return;
  const bool tried = m.tried[p] != 0;
  const double act = m.actual[p], pred = m.predicted[p], nc = m.new_cost[p];
  const double q = pred > 0.0 ? act / pred : -INFINITY;
  const bool ok = tried && isfinite(nc) && act > 0.0 && q >= m.step_quality_min;
  m.ok[p] = ok ? 1 : 0;
  double c = m.cost[p];
  if (ok) c = nc;
  m.cost[p] = c;
  double lam = m.lam[p];
  if (ok && q > 0.75) lam = fmax(lam / m.lambda_factor, m.lambda_min);
  if (tried && !ok) lam = fmin(lam * m.lambda_factor, m.lambda_max);
  m.lam[p] = lam;
  if (ok) m.accepted[p] += 1;
  if (tried && !ok) m.rejected[p] += 1;
  if (ok && fabs(act) <= m.cost_tolerance * fmax(c + act, 1e-300)) {
    m.reason[p] = TLS_BATCH_COST_TOLERANCE;
    m.active[p] = 0;
  }
  if (ok) m.pending[p] = 0;
}

}  // namespace
}  // namespace tls

using namespace tls;

namespace {

int assemble(const tls_schur_args* a, const tls_batched_systems* b, int64_t ntargets, const int32_t* target_r,
             const int32_t* target_c, const int32_t* ptr, const int32_t* pair_a, const int32_t* pair_b,
             cudaStream_t s) {
  if (b->nretained > 0) {
    if (b->sdtype == TLS_F64)
      batched_dense_base_kernel<double><<<b->nretained, 128, 0, s>>>(*a, *b);
    else
      batched_dense_base_kernel<float><<<b->nretained, 128, 0, s>>>(*a, *b);
  }
  TLS_CHECK_LAUNCH();
  const bool lanes = (a->dr == 6 || a->dr == 3) && a->de == 3;
  if (ntargets > 0 && lanes) {
    // batched problems (many blocks of few shared points): rows in two halves
    const bool halves = b->ret_problem != nullptr;
    if (a->dr == 6 && halves)
      launch_lanes<6, 3, 2>(*a, *b, ntargets, target_r, target_c, ptr, pair_a, pair_b, s);
    else if (a->dr == 6)
      launch_lanes<6, 3, 1>(*a, *b, ntargets, target_r, target_c, ptr, pair_a, pair_b, s);
    else
      launch_lanes<3, 3, 1>(*a, *b, ntargets, target_r, target_c, ptr, pair_a, pair_b, s);
  } else if (ntargets > 0) {
    const unsigned grid = (unsigned)((ntargets * 32 + 127) / 128);
    const bool w64 = a->wdtype == TLS_F64, s64 = b->sdtype == TLS_F64;
    if (w64 && s64)
      batched_dense_pairs_kernel<double, double><<<grid, 128, 0, s>>>(*a, *b, ntargets, target_r, target_c, ptr,
                                                                      pair_a, pair_b);
    else if (w64)
      batched_dense_pairs_kernel<double, float><<<grid, 128, 0, s>>>(*a, *b, ntargets, target_r, target_c, ptr,
                                                                     pair_a, pair_b);
    else if (s64)
      batched_dense_pairs_kernel<float, double><<<grid, 128, 0, s>>>(*a, *b, ntargets, target_r, target_c, ptr,
                                                                     pair_a, pair_b);
    else
      batched_dense_pairs_kernel<float, float><<<grid, 128, 0, s>>>(*a, *b, ntargets, target_r, target_c, ptr,
                                                                    pair_a, pair_b);
  }
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}

}  // namespace

extern "C" int tls_batched_schur_dense(const tls_schur_args* a, const tls_batched_systems* b, int64_t ntargets,
                                       const int32_t* target_r, const int32_t* target_c, const int32_t* ptr,
                                       const int32_t* pair_a, const int32_t* pair_b, tls_stream_t stream) {
  if (!a || !b || !b->S || b->nretained != a->nretained || b->dr != a->dr ||
      (b->ret_problem && (!b->ret_ptr || !b->s_off)))
    return tls_set_error(TLS_ERR_INVALID, "batched reduced matrices: bad arguments");
  return assemble(a, b, ntargets, target_r, target_c, ptr, pair_a, pair_b, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int tls_schur_dense_matrix(const tls_schur_args* a, int64_t ntargets, const int32_t* target_r,
                                      const int32_t* target_c, const int32_t* ptr, const int32_t* pair_a,
                                      const int32_t* pair_b, double* S, tls_stream_t stream) {
  if (!a || !S) return tls_set_error(TLS_ERR_INVALID, "dense Schur matrix: bad arguments");
  tls_batched_systems b{};
  b.nproblems = 1;
  b.nretained = a->nretained;
  b.dr = a->dr;
  b.sdtype = TLS_F64;
  b.S = S;
  return assemble(a, &b, ntargets, target_r, target_c, ptr, pair_a, pair_b, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int64_t tls_batched_share_bytes(int32_t dr, int32_t blocks, int32_t sdtype, int32_t with_cache) {
  const int64_t n = (int64_t)blocks * dr;
  int64_t v = kHeader + (4 * n + (int64_t)blocks * dr * dr) * (int64_t)sizeof(double);
  if (with_cache) v += n * (n + 1) / 2 * (sdtype == TLS_F64 ? 8 : 4);
  return v;
}

extern "C" int tls_batched_pcg(const tls_batched_systems* sys, const tls_batched_pcg_args* a, tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (!sys || !a || !a->queue || !a->err || a->ntasks < 0 || a->max_iterations < 0 || a->smem_bytes < 1024 ||
      a->smem_bytes > 227 * 1024)
    return tls_set_error(TLS_ERR_INVALID, "batched PCG: bad arguments");
  if (a->ntasks == 0) return TLS_OK;
  const bool s64 = sys->sdtype == TLS_F64;
  switch (sys->dr) {
    case 3:
      return s64 ? launch_pcg<3, double>(*sys, *a, s) : launch_pcg<3, float>(*sys, *a, s);
    case 6:
      return s64 ? launch_pcg<6, double>(*sys, *a, s) : launch_pcg<6, float>(*sys, *a, s);
    case 7:
      return s64 ? launch_pcg<7, double>(*sys, *a, s) : launch_pcg<7, float>(*sys, *a, s);
    default:
      return tls_set_error(TLS_ERR_UNSUPPORTED, "batched PCG: retained block dimension must be 3, 6 or 7");
  }
}

extern "C" int tls_factor_terms(int64_t nfactors, int32_t rdim, const double* old_raw, const double* new_raw,
                                int32_t loss, double delta, const double* weights, double* obj, double* red,
                                tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (nfactors < 0 || rdim < 1 || (loss != 0 && loss != 1) || (nfactors > 0 && (!old_raw || !new_raw || !obj || !red)))
    return tls_set_error(TLS_ERR_INVALID, "factor terms: bad arguments");
  if (nfactors > 0)
    factor_terms_kernel<<<(unsigned)((nfactors + 255) / 256), 256, 0, s>>>(nfactors, rdim, old_raw, new_raw, loss,
                                                                           delta, weights, obj, red);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}

extern "C" int tls_factor_sqnorm(int64_t nfactors, int32_t rdim, const double* rows, double* out, tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (nfactors < 0 || rdim < 1 || (nfactors > 0 && (!rows || !out)))
    return tls_set_error(TLS_ERR_INVALID, "factor squared norms: bad arguments");
  if (nfactors > 0)
    factor_sqnorm_kernel<<<(unsigned)((nfactors + 255) / 256), 256, 0, s>>>(nfactors, rdim, rows, out);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}

extern "C" int tls_batched_lm_update(const tls_batched_lm* m, tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (!m || m->nproblems < 0) return tls_set_error(TLS_ERR_INVALID, "batched LM update: bad arguments");
  if (m->nproblems > 0) batched_lm_update_kernel<<<(m->nproblems + 255) / 256, 256, 0, s>>>(*m);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}
