// Schur complement of one eliminated group (torchls schur.py:192-397).
//
// Edges (retained i, eliminated p) live in a chunked order: a chunk holds
// whole eliminated variables, and inside a chunk the edges are sorted by
// retained variable, so equal-retained edges form contiguous runs.
//
// Reduced matvec S x = (s U s + lambda I) x - W (W^T x), without forming S:
//   chunk kernel   t_e = W_e^T x_i          (edge-local, into shared memory)
//                  y_p = sum_{e in p} t_e   (fixed order, shared memory)
//                  u_e = W_e y_p            (edge-local)
//                  partial[run] = sum_{e in run} u_e
//   gather kernel  out_i = base_i - sum_{runs of i} partial[run]
// W is read once from HBM per matvec (the second, phase-2 read of a chunk's
// W hits L1/L2). Every sum follows a fixed order: deterministic.
#include "blocks.cuh"
#include "common.cuh"

namespace tls {

template <typename TW>
__device__ __forceinline__ TW ldw(const void* w, int64_t idx) {
  return __ldg(reinterpret_cast<const TW*>(w) + idx);
}

// MODE 0: matvec phase 1 from x; MODE 1: y_p taken from a->ybuf (reduced rhs)
template <int DR, int DE, int MODE, typename TW, typename TV, typename TA>
__global__ void __launch_bounds__(256) schur_chunk_kernel(tls_schur_args a, const TV* __restrict__ x) {
  extern __shared__ double smem[];
  const int c = blockIdx.x;
  const int e0 = a.chunk_ptr[c], e1 = a.chunk_ptr[c + 1];
  const int ne = e1 - e0;
  double* t_s = smem;                          // [ne][DE]
  double* u_s = smem + (size_t)a.max_chunk_edges * DE;  // [ne][DR]
  const int64_t E = a.nedges;
  if constexpr (MODE == 0) {
    for (int le = threadIdx.x; le < ne; le += blockDim.x) {
      const int e = e0 + le;
      const int i = __ldg(a.edge_r + e);
      TA xr[DR];
#pragma unroll
      for (int k = 0; k < DR; ++k) xr[k] = static_cast<TA>(__ldg(x + (int64_t)i * DR + k));
#pragma unroll
      for (int b = 0; b < DE; ++b) {
        TA acc = TA(0);
#pragma unroll
        for (int k = 0; k < DR; ++k) acc += static_cast<TA>(ldw<TW>(a.w, (int64_t)(k * DE + b) * E + e)) * xr[k];
        t_s[le * DE + b] = static_cast<double>(acc);
      }
    }
    __syncthreads();
  }
  for (int le = threadIdx.x; le < ne; le += blockDim.x) {
    const int e = e0 + le;
    const int p = __ldg(a.edge_e + e);
    double y[DE];
    if constexpr (MODE == 0) {
#pragma unroll
      for (int b = 0; b < DE; ++b) y[b] = 0.0;
      const int pb = __ldg(a.elim_ptr + p), pe = __ldg(a.elim_ptr + p + 1);
      for (int j = pb; j < pe; ++j) {
        const int lj = __ldg(a.elim_edges + j) - e0;
#pragma unroll
        for (int b = 0; b < DE; ++b) y[b] += t_s[lj * DE + b];
      }
    } else {
#pragma unroll
      for (int b = 0; b < DE; ++b) y[b] = a.ybuf[(int64_t)p * DE + b];
    }
    TA yv[DE];
#pragma unroll
    for (int b = 0; b < DE; ++b) yv[b] = static_cast<TA>(y[b]);
#pragma unroll
    for (int k = 0; k < DR; ++k) {
      TA acc = TA(0);
#pragma unroll
      for (int b = 0; b < DE; ++b) acc += static_cast<TA>(ldw<TW>(a.w, (int64_t)(k * DE + b) * E + e)) * yv[b];
      u_s[le * DR + k] = static_cast<double>(acc);
    }
  }
  __syncthreads();
  const int r0 = a.chunk_run_ptr[c], r1 = a.chunk_run_ptr[c + 1];
  for (int run = r0 + threadIdx.x; run < r1; run += blockDim.x) {
    const int b = a.run_ptr[run] - e0, e = a.run_ptr[run + 1] - e0;
    double acc[DR];
#pragma unroll
    for (int k = 0; k < DR; ++k) acc[k] = 0.0;
    for (int le = b; le < e; ++le)
#pragma unroll
      for (int k = 0; k < DR; ++k) acc[k] += u_s[le * DR + k];
#pragma unroll
    for (int k = 0; k < DR; ++k) a.run_partial[(int64_t)run * DR + k] = acc[k];
  }
}

// MODE 0: out = s U s x + lambda x - sum   (matvec, optional dot partials)
// MODE 1: out = b_retained - sum            (reduced rhs, b float64 full vector)
template <int DR, int MODE, typename TV>
__global__ void __launch_bounds__(256) schur_gather_kernel(tls_schur_args a, const TV* __restrict__ x,
                                                           const double* __restrict__ b, TV* __restrict__ out,
                                                           double* __restrict__ dot_partials) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  double acc[DR];
#pragma unroll
  for (int k = 0; k < DR; ++k) acc[k] = 0.0;
  const bool live = warp < a.nretained;
  if (live) {
    const int rb = a.rrun_ptr[warp], re = a.rrun_ptr[warp + 1];
    for (int j = rb + lane; j < re; j += 32) {
      const int run = a.rrun_list[j];
#pragma unroll
      for (int k = 0; k < DR; ++k) acc[k] += a.run_partial[(int64_t)run * DR + k];
    }
  }
#pragma unroll
  for (int k = 0; k < DR; ++k) acc[k] = warp_sum(acc[k]);
  double dot = 0.0;
  if (live && lane == 0) {
    const int64_t i = warp;
    if constexpr (MODE == 0) {
      double xs[DR], xv[DR];
#pragma unroll
      for (int k = 0; k < DR; ++k) {
        xv[k] = to_d(x[i * DR + k]);
        const double s = a.scale ? a.scale[a.retained_offset + i * DR + k] : 1.0;
        xs[k] = s * xv[k];
      }
      const double* U = a.ret_diag + i * DR * DR;
#pragma unroll
      for (int k = 0; k < DR; ++k) {
        double v = 0.0;
#pragma unroll
        for (int l = 0; l < DR; ++l) v += U[k * DR + l] * xs[l];
        const double s = a.scale ? a.scale[a.retained_offset + i * DR + k] : 1.0;
        v = s * v + a.damping * xv[k] - acc[k];
        const TV o = static_cast<TV>(v);
        out[i * DR + k] = o;
        dot += xv[k] * to_d(o);
      }
    } else {
#pragma unroll
      for (int k = 0; k < DR; ++k) out[i * DR + k] = static_cast<TV>(b[a.retained_offset + i * DR + k] - acc[k]);
    }
  }
  if (dot_partials) {
    __shared__ double sm[8];
    const double s = block_sum<256>(dot, sm);
    if (threadIdx.x == 0) dot_partials[blockIdx.x] = s;
  }
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
  template <typename TW, typename TV, typename TA>
  static int matvec(const tls_schur_args& a, const TV* x, TV* out, double* dots, int* gblocks, cudaStream_t s) {
    const size_t smem = (size_t)a.max_chunk_edges * (DE + DR) * sizeof(double);
    auto k = schur_chunk_kernel<DR, DE, 0, TW, TV, TA>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (a.nchunks > 0) k<<<a.nchunks, 256, smem, s>>>(a, x);
    TLS_CHECK_LAUNCH();
    const int blocks = (a.nretained * 32 + 255) / 256;
    if (gblocks) *gblocks = blocks;
    if (blocks > 0) schur_gather_kernel<DR, 0, TV><<<blocks, 256, 0, s>>>(a, x, nullptr, out, dots);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  }
  template <typename TW, typename TV, typename TA>
  static int rhs(const tls_schur_args& a, const double* b, TV* out, cudaStream_t s) {
    if (a.nelim > 0) schur_elim_rhs_kernel<DE><<<(a.nelim + 127) / 128, 128, 0, s>>>(a, b);
    TLS_CHECK_LAUNCH();
    const size_t smem = (size_t)a.max_chunk_edges * (DE + DR) * sizeof(double);
    auto k = schur_chunk_kernel<DR, DE, 1, TW, TV, TA>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (a.nchunks > 0) k<<<a.nchunks, 256, smem, s>>>(a, nullptr);
    TLS_CHECK_LAUNCH();
    const int blocks = (a.nretained * 32 + 255) / 256;
    if (blocks > 0) schur_gather_kernel<DR, 1, TV><<<blocks, 256, 0, s>>>(a, nullptr, b, out, nullptr);
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

int tls_schur_apply(const tls_schur_args* a, const void* x, void* out, double* dots, int* gblocks, cudaStream_t s) {
  return dispatch_dims(a->dr, a->de, [&](auto ops) -> int {
    using O = decltype(ops);
    if (a->vec_dtype == TLS_F64) {
      if (a->wdtype == TLS_F64)
        return O::template matvec<double, double, double>(*a, (const double*)x, (double*)out, dots, gblocks, s);
      return O::template matvec<float, double, double>(*a, (const double*)x, (double*)out, dots, gblocks, s);
    }
    if (a->wdtype != TLS_F32) return tls_set_error(TLS_ERR_UNSUPPORTED, "float64 W with float32 vectors");
    return O::template matvec<float, float, float>(*a, (const float*)x, (float*)out, dots, gblocks, s);
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
  return tls_schur_apply(a, x, out, nullptr, nullptr, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int tls_schur_reduced_rhs(const tls_schur_args* a, const double* b, void* rhs_c, tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return dispatch_dims(a->dr, a->de, [&](auto ops) -> int {
    using O = decltype(ops);
    if (a->vec_dtype == TLS_F64)
      return a->wdtype == TLS_F64 ? O::template rhs<double, double, double>(*a, b, (double*)rhs_c, s)
                                  : O::template rhs<float, double, double>(*a, b, (double*)rhs_c, s);
    return O::template rhs<float, float, float>(*a, b, (float*)rhs_c, s);
  });
}

extern "C" int tls_schur_backsubstitute(const tls_schur_args* a, const void* x_c, double* delta_full,
                                        tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return dispatch_dims(a->dr, a->de, [&](auto ops) -> int {
    using O = decltype(ops);
    if (a->vec_dtype == TLS_F64)
      return a->wdtype == TLS_F64 ? O::template backsub<double, double>(*a, (const double*)x_c, delta_full, s)
                                  : O::template backsub<float, double>(*a, (const double*)x_c, delta_full, s);
    return O::template backsub<float, float>(*a, (const float*)x_c, delta_full, s);
  });
}

extern "C" int tls_schur_preconditioner_blocks(const tls_schur_args* a, double* out, tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return dispatch_dims(a->dr, a->de, [&](auto ops) -> int {
    using O = decltype(ops);
    return a->wdtype == TLS_F64 ? O::template precond<double>(*a, out, s) : O::template precond<float>(*a, out, s);
  });
}
