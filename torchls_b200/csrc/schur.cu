// Schur complement of one eliminated group (torchls schur.py:192-397).
//
// Edges (retained i, eliminated p) live in a chunked order: a chunk holds
// whole eliminated variables, and inside a chunk the edges are sorted by
// retained variable, so equal-retained edges form contiguous runs.
//
// Reduced matvec S x = (s U s + lambda I) x - W (W^T x), without forming S:
//   chunk kernel   t_e = W_e^T x_i          (W_e loaded once, kept in registers)
//                  y_p = sum_{e in p} t_e   (fixed order, shared memory)
//                  u_e = W_e y_p
//                  partial[run] = warp-segmented sum of u_e over the run
//   gather kernel  out_i = base_i - sum_{runs of i} partial[run]
// W is read from HBM exactly once per matvec; 8 bytes of edge metadata ride
// along. Every sum follows a fixed order: deterministic.
#include "blocks.cuh"
#include "common.cuh"
#include "pcg_state.cuh"

namespace tls {

template <typename TW>
__device__ __forceinline__ TW ldw(const void* w, int64_t idx) {
  return __ldg(reinterpret_cast<const TW*>(w) + idx);
}

constexpr int kChunkThreads = 256;

// One thread block per chunk. MODE 0: S x (y_p = sum_{e in p} W_e^T x_i);
// MODE 1: reduced rhs (y_p = L_p^-1 b_p taken from a.ybuf).
//   phase 1   (MODE 0) t_e = W_e^T x_i for each edge; W_e stays in registers
//   phase 1.5 y_p = sum of the t_e of p's edges, once per eliminated variable
//   phase 2   u_e = W_e y_p; warp-segmented inclusive scan over runs (a run
//             never crosses a 32-edge window); the run's last lane stores it.
template <int DR, int DE, int EPT, int MODE, typename TW>
__global__ void __launch_bounds__(kChunkThreads, 2)
schur_chunk_kernel(tls_schur_args a, const double* __restrict__ x) {
  constexpr int CAP = kChunkThreads * EPT;
  extern __shared__ double smem[];
  double* t_s = smem;             // [CAP][DE] per-edge W^T x
  double* y_s = smem + CAP * DE;  // [CAP][DE] per-variable sums
  const int c = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31;
  const int e0 = __ldg(a.chunk_ptr + c), ne = __ldg(a.chunk_ptr + c + 1) - e0;
  const int p0 = __ldg(a.cpt_ptr + c), np = __ldg(a.cpt_ptr + c + 1) - p0;
  const int64_t E = a.nedges;
  const TW* __restrict__ W = reinterpret_cast<const TW*>(a.w);
  TW w[EPT][DR * DE];
  uint32_t meta[EPT];
#pragma unroll
  for (int j = 0; j < EPT; ++j) {
    const int le = j * kChunkThreads + tid;
    meta[j] = 0;
    if (le < ne) {
      const int64_t e = e0 + le;
#pragma unroll
      for (int k = 0; k < DR * DE; ++k) w[j][k] = __ldg(W + k * E + e);
      meta[j] = __ldg(a.edge_meta + e);
    } else {
#pragma unroll
      for (int k = 0; k < DR * DE; ++k) w[j][k] = TW(0);
    }
  }
  if constexpr (MODE == 0) {
#pragma unroll
    for (int j = 0; j < EPT; ++j) {
      const int le = j * kChunkThreads + tid;
      if (le < ne) {
        const int64_t i = __ldg(a.edge_r + e0 + le);
        double xr[DR];
#pragma unroll
        for (int k = 0; k < DR; ++k) xr[k] = __ldg(x + i * DR + k);
#pragma unroll
        for (int b = 0; b < DE; ++b) {
          double acc = 0.0;
#pragma unroll
          for (int k = 0; k < DR; ++k) acc += static_cast<double>(w[j][k * DE + b]) * xr[k];
          t_s[le * DE + b] = acc;
        }
      }
    }
    __syncthreads();
    for (int pl = tid; pl < np; pl += kChunkThreads) {
      const int p = __ldg(a.chunk_points + p0 + pl);
      const int jb = __ldg(a.elim_ptr + p), je = __ldg(a.elim_ptr + p + 1);
      double y[DE];
#pragma unroll
      for (int b = 0; b < DE; ++b) y[b] = 0.0;
      for (int jj = jb; jj < je; ++jj) {
        const int lj = __ldg(a.elim_edges + jj) - e0;
#pragma unroll
        for (int b = 0; b < DE; ++b) y[b] += t_s[lj * DE + b];
      }
#pragma unroll
      for (int b = 0; b < DE; ++b) y_s[pl * DE + b] = y[b];
    }
  } else {
    for (int pl = tid; pl < np; pl += kChunkThreads) {
      const int64_t p = __ldg(a.chunk_points + p0 + pl);
#pragma unroll
      for (int b = 0; b < DE; ++b) y_s[pl * DE + b] = a.ybuf[p * DE + b];
    }
  }
  __syncthreads();
  const int wbase = __ldg(a.cw_ptr + c);
#pragma unroll
  for (int j = 0; j < EPT; ++j) {
    const int le = j * kChunkThreads + tid;
    if (j * kChunkThreads >= ne) break;  // uniform across the block
    const bool valid = le < ne;
    const uint32_t m = valid ? meta[j] : 0u;
    const int pl = m & 0xFFFFu;
    const int head = (m >> 16) & 31;
    const bool tail = valid && ((m >> 21) & 1u);
    double y[DE];
#pragma unroll
    for (int b = 0; b < DE; ++b) y[b] = valid ? y_s[pl * DE + b] : 0.0;
    const unsigned tails = __ballot_sync(0xffffffffu, tail);
    const int run = tail ? __ldg(a.win_run + wbase + (le >> 5)) + __popc(tails & ((1u << lane) - 1u)) : 0;
    // one output component at a time keeps few doubles live
#pragma unroll
    for (int k = 0; k < DR; ++k) {
      double u = 0.0;
#pragma unroll
      for (int b = 0; b < DE; ++b) u += static_cast<double>(w[j][k * DE + b]) * y[b];
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const double v = __shfl_up_sync(0xffffffffu, u, off);
        if (lane - off >= head) u += v;
      }
      if (tail) a.run_partial[(int64_t)run * DR + k] = u;
    }
  }
}

// One block per retained variable: sum its runs in a fixed order, then
// MODE 0: out = s U s x + lambda x - sum  (matvec, optional dot partial per block)
// MODE 1: out = b_retained - sum          (reduced rhs, b float64 full vector)
template <int DR, int MODE, typename TV>
__global__ void __launch_bounds__(256) schur_gather_kernel(tls_schur_args a, const TV* __restrict__ x,
                                                           const double* __restrict__ b, TV* __restrict__ out,
                                                           double* __restrict__ dot_partials, PcgState* pst) {
  __shared__ double sm[8][DR];
  __shared__ double smd[8];
  const int64_t i = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double acc[DR];
#pragma unroll
  for (int k = 0; k < DR; ++k) acc[k] = 0.0;
  const int rb = __ldg(a.rrun_ptr + i), re = __ldg(a.rrun_ptr + i + 1);
  for (int j = rb + tid; j < re; j += 256) {
    const int64_t run = __ldg(a.rrun_list + j);
#pragma unroll
    for (int k = 0; k < DR; ++k) acc[k] += a.run_partial[run * DR + k];
  }
#pragma unroll
  for (int k = 0; k < DR; ++k) {
    const double v = warp_sum(acc[k]);
    if (lane == 0) sm[warp][k] = v;
  }
  __syncthreads();
  if (tid == 0) {
    double tot[DR];
#pragma unroll
    for (int k = 0; k < DR; ++k) {
      double v = 0.0;
#pragma unroll
      for (int q = 0; q < 8; ++q) v += sm[q][k];
      tot[k] = v;
    }
    if constexpr (MODE == 0) {
      double xs[DR], xv[DR], s[DR];
#pragma unroll
      for (int k = 0; k < DR; ++k) {
        xv[k] = to_d(x[i * DR + k]);
        s[k] = a.scale ? a.scale[a.retained_offset + i * DR + k] : 1.0;
        xs[k] = s[k] * xv[k];
      }
      const double* U = a.ret_diag + i * DR * DR;
      double dot = 0.0;
#pragma unroll
      for (int k = 0; k < DR; ++k) {
        double v = 0.0;
#pragma unroll
        for (int l = 0; l < DR; ++l) v += U[k * DR + l] * xs[l];
        v = s[k] * v + a.damping * xv[k] - tot[k];
        const TV o = static_cast<TV>(v);
        out[i * DR + k] = o;
        dot += xv[k] * to_d(o);
      }
      if (dot_partials) dot_partials[i] = dot;
    } else {
#pragma unroll
      for (int k = 0; k < DR; ++k) out[i * DR + k] = static_cast<TV>(b[a.retained_offset + i * DR + k] - tot[k]);
    }
  }
  if (MODE == 0 && pst) pcg_operator_epilogue<256>(pst, dot_partials, gridDim.x, smd);
}

// Per eliminated variable: L = chol(s C s + lambda I), store L^-1; y = L^-1 b_e optional.
template <int DE>
__global__ void schur_factor_kernel(tls_schur_args a, const double* __restrict__ b) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.nelim) return;
  double C[DE * DE], L[DE * DE], s[DE];
#pragma unroll
  for (int k = 0; k < DE; ++k) s[k] = a.scale ? a.scale[a.elim_offset + p * DE + k] : 1.0;
#pragma unroll
  for (int i = 0; i < DE; ++i)
#pragma unroll
    for (int j = 0; j < DE; ++j) C[i * DE + j] = s[i] * a.elim_diag[p * DE * DE + i * DE + j] * s[j];
  const bool ok = cholesky_block(C, L, DE, a.damping);
  if (!ok) atomicAdd(a.bad, 1);
  // inverse of the lower-triangular L by forward substitution on unit vectors
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
  for (int k = 0; k < DE * DE; ++k) a.inv_l[p * DE * DE + k] = Li[k];
}

// W_e = diag(s_i) E_e diag(s_p) L_p^-T, stored SoA [dr*de][E]
template <int DR, int DE, typename TW>
__global__ void schur_whiten_kernel(tls_schur_args a) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.nedges) return;
  const int64_t i = a.edge_r[e], p = a.edge_e[e];
  double sr[DR], se[DE];
#pragma unroll
  for (int k = 0; k < DR; ++k) sr[k] = a.scale ? a.scale[a.retained_offset + i * DR + k] : 1.0;
#pragma unroll
  for (int k = 0; k < DE; ++k) se[k] = a.scale ? a.scale[a.elim_offset + p * DE + k] : 1.0;
  const double* Li = a.inv_l + p * DE * DE;
  const double* E = a.cross + e * DR * DE;
  TW* w = reinterpret_cast<TW*>(a.w);
#pragma unroll
  for (int r = 0; r < DR; ++r) {
#pragma unroll
    for (int c = 0; c < DE; ++c) {
      double v = 0.0;
#pragma unroll
      for (int k = 0; k < DE; ++k) v += sr[r] * E[r * DE + k] * se[k] * Li[c * DE + k];
      w[(int64_t)(r * DE + c) * a.nedges + e] = static_cast<TW>(v);
    }
  }
}

// y_p = L_p^-1 (b_e)_p, b full float64 vector (already scaled)
template <int DE>
__global__ void schur_elim_rhs_kernel(tls_schur_args a, const double* __restrict__ b) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.nelim) return;
  const double* Li = a.inv_l + p * DE * DE;
#pragma unroll
  for (int r = 0; r < DE; ++r) {
    double v = 0.0;
#pragma unroll
    for (int k = 0; k < DE; ++k) v += Li[r * DE + k] * b[a.elim_offset + p * DE + k];
    a.ybuf[p * DE + r] = v;
  }
}

// delta_p = L_p^-T (y_p - sum_{e in p} W_e^T x_i); delta_full retained part = x
template <int DR, int DE, typename TW, typename TV>
__global__ void schur_backsub_kernel(tls_schur_args a, const TV* __restrict__ xc, double* __restrict__ delta) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nret = (int64_t)a.nretained * DR;
  if (tid < nret) delta[a.retained_offset + tid] = to_d(xc[tid]);
  if (tid >= a.nelim) return;
  const int64_t p = tid;
  double t[DE];
#pragma unroll
  for (int b = 0; b < DE; ++b) t[b] = a.ybuf[p * DE + b];
  const int pb = a.elim_ptr[p], pe = a.elim_ptr[p + 1];
  for (int j = pb; j < pe; ++j) {
    const int e = a.elim_edges[j];
    const int64_t i = a.edge_r[e];
#pragma unroll
    for (int b = 0; b < DE; ++b) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < DR; ++k) acc += to_d(ldw<TW>(a.w, (int64_t)(k * DE + b) * a.nedges + e)) * to_d(xc[i * DR + k]);
      t[b] -= acc;
    }
  }
  const double* Li = a.inv_l + p * DE * DE;
#pragma unroll
  for (int r = 0; r < DE; ++r) {
    double v = 0.0;
#pragma unroll
    for (int k = 0; k < DE; ++k) v += Li[k * DE + r] * t[k];
    delta[a.elim_offset + p * DE + r] = v;
  }
}

// out_i = s U s - sum_{e in i} W_e W_e^T (lambda added by the Cholesky)
template <int DR, int DE, typename TW>
__global__ void __launch_bounds__(256) schur_precond_kernel(tls_schur_args a, double* __restrict__ out) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  double acc[DR * (DR + 1) / 2];
#pragma unroll
  for (int k = 0; k < DR * (DR + 1) / 2; ++k) acc[k] = 0.0;
  const bool live = warp < a.nretained;
  if (live) {
    const int rb = a.rrun_ptr[warp], re = a.rrun_ptr[warp + 1];
    for (int j = rb + lane; j < re; j += 32) {
      const int run = a.rrun_list[j];
      for (int e = a.run_ptr[run]; e < a.run_ptr[run + 1]; ++e) {
        double wv[DR][DE];
#pragma unroll
        for (int r = 0; r < DR; ++r)
#pragma unroll
          for (int c = 0; c < DE; ++c) wv[r][c] = to_d(ldw<TW>(a.w, (int64_t)(r * DE + c) * a.nedges + e));
        int idx = 0;
#pragma unroll
        for (int r = 0; r < DR; ++r)
#pragma unroll
          for (int q = r; q < DR; ++q) {
            double v = 0.0;
#pragma unroll
            for (int c = 0; c < DE; ++c) v += wv[r][c] * wv[q][c];
            acc[idx++] += v;
          }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < DR * (DR + 1) / 2; ++k) acc[k] = warp_sum(acc[k]);
  if (!live || lane != 0) return;
  const int64_t i = warp;
  double s[DR];
#pragma unroll
  for (int k = 0; k < DR; ++k) s[k] = a.scale ? a.scale[a.retained_offset + i * DR + k] : 1.0;
  const double* U = a.ret_diag + i * DR * DR;
  double* o = out + i * DR * DR;
  int idx = 0;
#pragma unroll
  for (int r = 0; r < DR; ++r)
#pragma unroll
    for (int q = r; q < DR; ++q) {
      const double v = s[r] * U[r * DR + q] * s[q] - acc[idx++];
      o[r * DR + q] = v;
      o[q * DR + r] = v;
    }
}

template <int DR, int DE>
struct SchurOps {
  template <int MODE, typename TW, int EPT>
  static int chunks_ept(const tls_schur_args& a, const double* x, cudaStream_t s) {
    constexpr size_t smem = 2 * sizeof(double) * kChunkThreads * EPT * DE;
    auto k = schur_chunk_kernel<DR, DE, EPT, MODE, TW>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<a.nchunks, kChunkThreads, smem, s>>>(a, x);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  }
  template <int MODE, typename TW>
  static int chunks(const tls_schur_args& a, const double* x, cudaStream_t s) {
    if (a.nchunks == 0) return TLS_OK;
    // 2 edges per thread: W stays in registers between the phases
    if constexpr (sizeof(TW) == 4) {
      if (a.ept != 2) return tls_set_error(TLS_ERR_INVALID, "Schur layouts use 2 edges per thread");
      return chunks_ept<MODE, TW, 2>(a, x, s);
    } else {
      if (a.ept != 2) return tls_set_error(TLS_ERR_INVALID, "float64 W needs a 2-edge-per-thread layout");
      return chunks_ept<MODE, TW, 2>(a, x, s);
    }
  }
  template <typename TW, typename TV, typename TA>
  static int matvec(const tls_schur_args& a, const TV* x, TV* out, double* dots, int* gblocks, PcgState* pst,
                    cudaStream_t s) {
    static_assert(sizeof(TV) == 8, "reduced vectors are float64");
    int rc = chunks<0, TW>(a, reinterpret_cast<const double*>(x), s);
    if (rc) return rc;
    if (gblocks) *gblocks = a.nretained;
    if (a.nretained > 0) schur_gather_kernel<DR, 0, TV><<<a.nretained, 256, 0, s>>>(a, x, nullptr, out, dots, pst);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  }
  template <typename TW, typename TV, typename TA>
  static int rhs(const tls_schur_args& a, const double* b, TV* out, cudaStream_t s) {
    if (a.nelim > 0) schur_elim_rhs_kernel<DE><<<(a.nelim + 127) / 128, 128, 0, s>>>(a, b);
    TLS_CHECK_LAUNCH();
    int rc = chunks<1, TW>(a, nullptr, s);
    if (rc) return rc;
    if (a.nretained > 0)
      schur_gather_kernel<DR, 1, TV><<<a.nretained, 256, 0, s>>>(a, nullptr, b, out, nullptr, nullptr);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  }
  template <typename TW>
  static int damp(const tls_schur_args& a, cudaStream_t s) {
    cudaMemsetAsync(a.bad, 0, sizeof(int32_t), s);
    if (a.nelim > 0) schur_factor_kernel<DE><<<(a.nelim + 127) / 128, 128, 0, s>>>(a, nullptr);
    TLS_CHECK_LAUNCH();
    if (a.nedges > 0) schur_whiten_kernel<DR, DE, TW><<<(a.nedges + 127) / 128, 128, 0, s>>>(a);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  }
  template <typename TW, typename TV>
  static int backsub(const tls_schur_args& a, const TV* xc, double* delta, cudaStream_t s) {
    const int64_t n = a.nelim > (int64_t)a.nretained * DR ? a.nelim : (int64_t)a.nretained * DR;
    if (n > 0) schur_backsub_kernel<DR, DE, TW, TV><<<(n + 127) / 128, 128, 0, s>>>(a, xc, delta);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  }
  template <typename TW>
  static int precond(const tls_schur_args& a, double* out, cudaStream_t s) {
    const int blocks = (a.nretained * 32 + 255) / 256;
    if (blocks > 0) schur_precond_kernel<DR, DE, TW><<<blocks, 256, 0, s>>>(a, out);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  }
};

template <typename F>
static int dispatch_dims(int dr, int de, F&& f) {
#define TLS_D(R, E) \
  if (dr == R && de == E) return f(SchurOps<R, E>{});
  TLS_D(6, 3)
  TLS_D(3, 3)
  TLS_D(7, 3)
  TLS_D(6, 1)
  TLS_D(3, 1)
  TLS_D(1, 1)
  TLS_D(2, 2)
  TLS_D(3, 2)
  TLS_D(6, 6)
  TLS_D(2, 1)
  TLS_D(1, 3)
  TLS_D(8, 3)
  TLS_D(6, 4)
  TLS_D(4, 3)
#undef TLS_D
  return tls_set_error(TLS_ERR_UNSUPPORTED, "Schur block dims not instantiated");
}

}  // namespace tls

using namespace tls;

int tls_schur_apply(const tls_schur_args* a, const void* x, void* out, double* dots, int* gblocks, void* pcg_state,
                    cudaStream_t s) {
  if (a->vec_dtype != TLS_F64) return tls_set_error(TLS_ERR_UNSUPPORTED, "reduced Schur vectors are float64");
  PcgState* pst = reinterpret_cast<PcgState*>(pcg_state);
  return dispatch_dims(a->dr, a->de, [&](auto ops) -> int {
    using O = decltype(ops);
    if (a->wdtype == TLS_F64)
      return O::template matvec<double, double, double>(*a, (const double*)x, (double*)out, dots, gblocks, pst, s);
    return O::template matvec<float, double, double>(*a, (const double*)x, (double*)out, dots, gblocks, pst, s);
  });
}

extern "C" int tls_schur_damp(const tls_schur_args* a, tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return dispatch_dims(a->dr, a->de, [&](auto ops) -> int {
    using O = decltype(ops);
    return a->wdtype == TLS_F64 ? O::template damp<double>(*a, s) : O::template damp<float>(*a, s);
  });
}

extern "C" int tls_schur_matvec(const tls_schur_args* a, const void* x, void* out, tls_stream_t stream) {
  return tls_schur_apply(a, x, out, nullptr, nullptr, nullptr, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int tls_schur_reduced_rhs(const tls_schur_args* a, const double* b, void* rhs_c, tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (a->vec_dtype != TLS_F64) return tls_set_error(TLS_ERR_UNSUPPORTED, "reduced Schur vectors are float64");
  return dispatch_dims(a->dr, a->de, [&](auto ops) -> int {
    using O = decltype(ops);
    return a->wdtype == TLS_F64 ? O::template rhs<double, double, double>(*a, b, (double*)rhs_c, s)
                                : O::template rhs<float, double, double>(*a, b, (double*)rhs_c, s);
  });
}

extern "C" int tls_schur_backsubstitute(const tls_schur_args* a, const void* x_c, double* delta_full,
                                        tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (a->vec_dtype != TLS_F64) return tls_set_error(TLS_ERR_UNSUPPORTED, "reduced Schur vectors are float64");
  return dispatch_dims(a->dr, a->de, [&](auto ops) -> int {
    using O = decltype(ops);
    return a->wdtype == TLS_F64 ? O::template backsub<double, double>(*a, (const double*)x_c, delta_full, s)
                                : O::template backsub<float, double>(*a, (const double*)x_c, delta_full, s);
  });
}

extern "C" int tls_schur_preconditioner_blocks(const tls_schur_args* a, double* out, tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return dispatch_dims(a->dr, a->de, [&](auto ops) -> int {
    using O = decltype(ops);
    return a->wdtype == TLS_F64 ? O::template precond<double>(*a, out, s) : O::template precond<float>(*a, out, s);
  });
}
