// General Schur complement of one eliminated group (torchls schur.py:17-397)
// for the systems the one-group kernels (schur.cu) do not take: several
// retained groups of any dims <= 16, residuals coupling retained variables,
// joint preconditioner groups.
//
// Layout: retained variables in reduced order, each with its edges
// (retained variable, eliminated variable) contiguous in the reference's edge
// order; a dim x de block per edge at edge_w (J_r^T J_e in `cross`, the
// whitened W_e = s_r E_e s_e L_e^-T in `w`). The reduced operator
//   S x = base(x) - W (W^T x)
// runs as two gathers, both in a fixed order (no atomics on values):
//   elim kernel   t_p = sum_{e in p} W_e^T x_{r(e)}       one thread per p
//   ret kernel    out_v = base_v - sum_{e in v} W_e t_p   one warp per v
// with base(x) = s U s x + lambda x per variable, or, when residuals couple
// retained variables, diag(s) J^T J diag(s) x + lambda x through the normal
// operator of the full Jacobian applied to x padded with zeros (J e_elim = 0
// there, so J x = J_r x_r; schur.py:303-328).
#include <stdint.h>

#include <type_traits>

#include "blocks.cuh"
#include "common.cuh"
#include "pcg_state.cuh"

int tls_normal_apply(const tls_normal_args* a, const void* x, void* y, double* dot_partials, int* gather_blocks,
                     void* pcg_state, cudaStream_t st);

namespace tls {

constexpr int kSgMaxDim = 16;     // retained block dims
constexpr int kSgThreads = 256;   // 8 warps per block
constexpr int kSgMaxBlocks = 148 * 16;

__device__ __forceinline__ double sg_scale(const tls_schur_general_args& a, int64_t col) {
  return a.scale ? a.scale[col] : 1.0;
}

// W_e in float64 from its cross block, the scales and L_p^-1 (the arithmetic
// of the whitening): W[r][c] = sum_k s_r E[r][k] s_k (L_p^-1)[c][k].
template <int DE, int DM>
__device__ __forceinline__ void sg_whitened(const tls_schur_general_args& a, int v, int64_t e, int dim,
                                            double (&W)[DM][DE]) {
  const int64_t p = a.edge_elim[e];
  const double* E = a.cross + a.edge_w[e];
  const double* Li = a.inv_l + p * DE * DE;
  double se[DE];
#pragma unroll
  for (int k = 0; k < DE; ++k) se[k] = sg_scale(a, a.elim_offset + p * DE + k);
  const int64_t f0 = a.var_full[v];
#pragma unroll
  for (int r = 0; r < DM; ++r) {
    const double sr = r < dim ? sg_scale(a, f0 + r) : 0.0;
#pragma unroll
    for (int c = 0; c < DE; ++c) {
      double acc = 0.0;
      if (r < dim) {
#pragma unroll
        for (int k = 0; k < DE; ++k) acc += sr * E[r * DE + k] * se[k] * Li[c * DE + k];
      }
      W[r][c] = acc;
    }
  }
}

template <int DE>
__global__ void sg_factor_kernel(tls_schur_general_args a) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.nelim) return;
  double s[DE];
#pragma unroll
  for (int k = 0; k < DE; ++k) s[k] = sg_scale(a, a.elim_offset + p * DE + k);
  if (!eliminated_factor<DE>(a.elim_diag + p * DE * DE, s, a.damping, a.inv_l + p * DE * DE)) atomicAdd(a.bad, 1);
}

// One warp per retained variable: its edges' whitened blocks into w.
template <int DE, int DM, typename TW>
__global__ void __launch_bounds__(kSgThreads) sg_whiten_kernel(tls_schur_general_args a) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (kSgThreads / 32);
  TW* w = reinterpret_cast<TW*>(a.w);
  for (int64_t v = (int64_t)blockIdx.x * (kSgThreads / 32) + (threadIdx.x >> 5); v < a.nretained; v += nwarps) {
    const int dim = a.var_dim[v];
    for (int64_t e = a.var_ptr[v] + lane; e < a.var_ptr[v + 1]; e += 32) {
      double W[DM][DE];
      sg_whitened<DE, DM>(a, (int)v, e, dim, W);
      TW* dst = w + a.edge_w[e];
#pragma unroll
      for (int r = 0; r < DM; ++r)
#pragma unroll
        for (int c = 0; c < DE; ++c)
          if (r < dim) dst[r * DE + c] = static_cast<TW>(W[r][c]);
    }
  }
}

// MODE 0: t_p = sum_{e in p} W_e^T x_{r(e)} into tbuf.
// MODE 1: delta_p = L_p^-T (y_p - sum_{e in p} W_e^T x_{r(e)}) into the full step.
// One thread per eliminated variable, its edges in list order.
template <int DE, int MODE, typename TW>
__global__ void sg_elim_kernel(tls_schur_general_args a, const double* __restrict__ x, double* __restrict__ delta) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.nelim) return;
  const TW* w = reinterpret_cast<const TW*>(a.w);
  double t[DE];
#pragma unroll
  for (int c = 0; c < DE; ++c) t[c] = 0.0;
  for (int j = a.elim_ptr[p]; j < a.elim_ptr[p + 1]; ++j) {
    const int64_t e = a.elim_edge[j];
    const int v = a.edge_var[e];
    const int dim = a.var_dim[v];
    const TW* W = w + a.edge_w[e];
    const double* xv = x + a.var_row[v];
    for (int r = 0; r < dim; ++r) {
      const double xr = xv[r];
#pragma unroll
      for (int c = 0; c < DE; ++c) t[c] += to_d(W[r * DE + c]) * xr;
    }
  }
  if constexpr (MODE == 0) {
#pragma unroll
    for (int c = 0; c < DE; ++c) a.tbuf[p * DE + c] = t[c];
  } else {
    double y[DE];
#pragma unroll
    for (int c = 0; c < DE; ++c) y[c] = a.ybuf[p * DE + c] - t[c];
    const double* Li = a.inv_l + p * DE * DE;
#pragma unroll
    for (int r = 0; r < DE; ++r) {
      double v = 0.0;
#pragma unroll
      for (int k = 0; k < DE; ++k) v += Li[k * DE + r] * y[k];
      delta[a.elim_offset + p * DE + r] = v;
    }
  }
}

// y_p = L_p^-1 (b_e)_p (b full, scaled)
template <int DE>
__global__ void sg_elim_rhs_kernel(tls_schur_general_args a, const double* __restrict__ b) {
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

// dst (full tangent layout) at var_full <- x (reduced layout) at var_row.
// base = B x + lambda x from the cached retained normal matrix, written to the
// full-vector workspace at the variable's full offset (where the normal-operator
// path leaves its base too): one thread per (variable, component); blocks in
// row order, columns in order.
__global__ void sg_retained_kernel(tls_schur_general_args a, tls_retained_matrix m, const double* __restrict__ x) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t v = t / kSgMaxDim;
  const int r = (int)(t % kSgMaxDim);
  if (v >= a.nretained) return;
  const int dim = a.var_dim[v];
  if (r >= dim) return;
  double acc = 0.0;
  for (int k = m.row_ptr[v]; k < m.row_ptr[v + 1]; ++k) {
    const int j = m.block_col[k];
    const int dj = a.var_dim[j];
    const double* B = m.values + m.block_off[k] + (int64_t)r * dj;
    const double* xj = x + a.var_row[j];
    for (int c = 0; c < dj; ++c) acc += B[c] * xj[c];
  }
  a.yfull[a.var_full[v] + r] = acc + a.damping * x[a.var_row[v] + r];
}

__global__ void sg_scatter_kernel(tls_schur_general_args a, const double* __restrict__ x, double* __restrict__ dst) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= a.nretained) return;
  const int dim = a.var_dim[v];
  for (int k = 0; k < dim; ++k) dst[a.var_full[v] + k] = x[a.var_row[v] + k];
}

// One warp per retained variable, lanes over its edges (each lane in list
// order, then a fixed butterfly):
// MODE 0: out_v = base_v - sum_e W_e t_{p(e)}; with `dots`, each block's
//         x.out partial and the PCG operator epilogue (curvature, alpha).
// MODE 1: out_v = b_v - sum_e W_e y_{p(e)} (b full).
template <int DE, int DM, int MODE, typename TW>
__global__ void __launch_bounds__(kSgThreads) sg_ret_kernel(tls_schur_general_args a, const double* __restrict__ x,
                                                           const double* __restrict__ b, double* __restrict__ out,
                                                           double* __restrict__ dots, PcgState* pst) {
  __shared__ double sm[kSgThreads / 32];
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (kSgThreads / 32);
  const TW* w = reinterpret_cast<const TW*>(a.w);
  const double* src = MODE == 0 ? a.tbuf : a.ybuf;
  double dot = 0.0;
  for (int64_t v = (int64_t)blockIdx.x * (kSgThreads / 32) + (threadIdx.x >> 5); v < a.nretained; v += nwarps) {
    const int dim = a.var_dim[v];
    double acc[DM];
#pragma unroll
    for (int r = 0; r < DM; ++r) acc[r] = 0.0;
    for (int64_t e = a.var_ptr[v] + lane; e < a.var_ptr[v + 1]; e += 32) {
      const int64_t p = a.edge_elim[e];
      double y[DE];
#pragma unroll
      for (int c = 0; c < DE; ++c) y[c] = src[p * DE + c];
      const TW* W = w + a.edge_w[e];
#pragma unroll
      for (int r = 0; r < DM; ++r) {
        if (r < dim) {
#pragma unroll
          for (int c = 0; c < DE; ++c) acc[r] += to_d(W[r * DE + c]) * y[c];
        }
      }
    }
    double mine = 0.0;
#pragma unroll
    for (int r = 0; r < DM; ++r) {
      if (r < dim) {
        const double s = warp_sum(acc[r]);
        if (lane == r) mine = s;
      }
    }
    if (lane < dim) {
      const int64_t row = a.var_row[v] + lane, full = a.var_full[v] + lane;
      if constexpr (MODE == 0) {
        const double xr = x[row];
        double base;
        if (a.normal || a.retained) {
          base = a.yfull[full];
        } else {
          const double* U = a.ret_diag + a.var_diag[v] + (int64_t)lane * dim;
          double u = 0.0;
          for (int c = 0; c < dim; ++c) u += U[c] * (sg_scale(a, a.var_full[v] + c) * x[a.var_row[v] + c]);
          base = sg_scale(a, full) * u + a.damping * xr;
        }
        const double o = base - mine;
        out[row] = o;
        dot += xr * o;
      } else {
        out[row] = b[full] - mine;
      }
    }
  }
  if constexpr (MODE == 0) {
    if (dots) {
      const double s = block_sum<kSgThreads>(dot, sm);
      if (threadIdx.x == 0) dots[blockIdx.x] = s;
      if (pst) pcg_operator_epilogue<kSgThreads>(pst, dots, gridDim.x, sm);
    }
  }
}

// out_v = s U s - sum_e W_e W_e^T (upper triangle summed, both halves
// written), W in float64; one thread per retained variable (dims <= DM).
template <int DE, int DM>
__global__ void sg_precond_kernel(tls_schur_general_args a, double* __restrict__ out) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= a.nretained) return;
  const int dim = a.var_dim[v];
  double acc[DM][DM];
#pragma unroll
  for (int r = 0; r < DM; ++r)
#pragma unroll
    for (int q = 0; q < DM; ++q) acc[r][q] = 0.0;
  for (int64_t e = a.var_ptr[v]; e < a.var_ptr[v + 1]; ++e) {
    double W[DM][DE];
    sg_whitened<DE, DM>(a, (int)v, e, dim, W);
#pragma unroll
    for (int r = 0; r < DM; ++r)
#pragma unroll
      for (int q = r; q < DM; ++q) {
        double t = 0.0;
#pragma unroll
        for (int c = 0; c < DE; ++c) t += W[r][c] * W[q][c];
        acc[r][q] += t;
      }
  }
  const double* U = a.ret_diag + a.var_diag[v];
  double* o = out + a.var_diag[v];
  const int64_t f0 = a.var_full[v];
#pragma unroll
  for (int r = 0; r < DM; ++r)
#pragma unroll
    for (int q = r; q < DM; ++q) {
      if (q < dim) {
        const double val = sg_scale(a, f0 + r) * U[r * dim + q] * sg_scale(a, f0 + q) - acc[r][q];
        o[r * dim + q] = val;
        o[q * dim + r] = val;
      }
    }
}

// out[i] = sum_k W_{ea[k]} W_{eb[k]}^T (da x db), W in float64; one thread per i.
template <int DE, int DM>
__global__ void sg_pairs_kernel(tls_schur_general_args a, int32_t count, const int32_t* __restrict__ ptr,
                                const int32_t* __restrict__ ea, const int32_t* __restrict__ eb, int da, int db,
                                double* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  double acc[DM][DM];
#pragma unroll
  for (int r = 0; r < DM; ++r)
#pragma unroll
    for (int q = 0; q < DM; ++q) acc[r][q] = 0.0;
  for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
    double Wa[DM][DE], Wb[DM][DE];
    sg_whitened<DE, DM>(a, a.edge_var[ea[k]], ea[k], da, Wa);
    sg_whitened<DE, DM>(a, a.edge_var[eb[k]], eb[k], db, Wb);
#pragma unroll
    for (int r = 0; r < DM; ++r)
#pragma unroll
      for (int q = 0; q < DM; ++q) {
        double t = 0.0;
#pragma unroll
        for (int c = 0; c < DE; ++c) t += Wa[r][c] * Wb[q][c];
        acc[r][q] += t;
      }
  }
  double* o = out + i * da * db;
#pragma unroll
  for (int r = 0; r < DM; ++r)
#pragma unroll
    for (int q = 0; q < DM; ++q)
      if (r < da && q < db) o[r * db + q] = acc[r][q];
}

}  // namespace tls

using namespace tls;

namespace {

// Blocks of the retained-variable gather (one warp per variable, grid-stride):
// also the number of dot partials the PCG operator writes.
int sg_ret_blocks(const tls_schur_general_args* a) {
  const int64_t b = ((int64_t)a->nretained + kSgThreads / 32 - 1) / (kSgThreads / 32);
  return (int)(b < 1 ? 1 : (b > kSgMaxBlocks ? kSgMaxBlocks : b));
}

int sg_check(const tls_schur_general_args* a) {
  if (!a) return tls_set_error(TLS_ERR_INVALID, "general Schur: null arguments");
  if (a->de < 1 || a->de > 4) return tls_set_error(TLS_ERR_UNSUPPORTED, "general Schur: eliminated dim must be 1..4");
  if (a->wdtype != TLS_F32 && a->wdtype != TLS_F64) return tls_set_error(TLS_ERR_INVALID, "general Schur: W dtype");
  return TLS_OK;
}

// f(DE, DM, TW) over the instantiated shapes; DM bounds every retained dim
// (the host passes the largest retained dim).
template <typename F>
int sg_dispatch(const tls_schur_general_args* a, int maxdim, F&& f) {
  if (int rc = sg_check(a)) return rc;
  if (maxdim > kSgMaxDim) return tls_set_error(TLS_ERR_UNSUPPORTED, "general Schur: retained dims above 16");
  auto by_dm = [&](auto de) -> int {
    constexpr int DE = decltype(de)::value;
    if (maxdim <= 8) {
      return a->wdtype == TLS_F64 ? f(std::integral_constant<int, DE>{}, std::integral_constant<int, 8>{}, double{})
                                  : f(std::integral_constant<int, DE>{}, std::integral_constant<int, 8>{}, float{});
    }
    return a->wdtype == TLS_F64 ? f(std::integral_constant<int, DE>{}, std::integral_constant<int, 16>{}, double{})
                                : f(std::integral_constant<int, DE>{}, std::integral_constant<int, 16>{}, float{});
  };
  switch (a->de) {
    case 1: return by_dm(std::integral_constant<int, 1>{});
    case 2: return by_dm(std::integral_constant<int, 2>{});
    case 3: return by_dm(std::integral_constant<int, 3>{});
    default: return by_dm(std::integral_constant<int, 4>{});
  }
}

unsigned grid_of_n(int64_t n, int block) { return (unsigned)((n + block - 1) / block > 0 ? (n + block - 1) / block : 1); }

}  // namespace

// S x; with `dots` and `pcg_state`, each gather block's x.Sx partial and the
// PCG operator epilogue (the device PCG's operator for general Schur systems).
int tls_schur_general_apply(const tls_schur_general_args* a, const double* x, double* out, double* dots,
                            int* gblocks, void* pcg_state, cudaStream_t s) {
  const int maxdim = a ? a->max_dim : 0;
  PcgState* pst = reinterpret_cast<PcgState*>(pcg_state);
  if (gblocks) *gblocks = sg_ret_blocks(a);
  return sg_dispatch(a, maxdim, [&](auto de, auto dm, auto tw) -> int {
    constexpr int DE = decltype(de)::value, DM = decltype(dm)::value;
    using TW = decltype(tw);
    if (a->retained) {  // retained couplings, cached matrix: base = B x + lambda x
      if (!a->yfull) return tls_set_error(TLS_ERR_INVALID, "general Schur: the retained matrix needs yfull");
      // the struct lives in host memory (like `normal`): its device pointers go by value
      sg_retained_kernel<<<grid_of_n((int64_t)a->nretained * kSgMaxDim, 128), 128, 0, s>>>(*a, *a->retained, x);
      TLS_CHECK_LAUNCH();
    } else if (a->normal) {  // retained couplings: base = the normal operator on x padded with zeros
      cudaError_t e = cudaMemsetAsync(a->xfull, 0, a->full_dim * sizeof(double), s);
      if (e != cudaSuccess) return tls_set_cuda_error(e);
      if (a->nretained > 0) sg_scatter_kernel<<<grid_of_n(a->nretained, 128), 128, 0, s>>>(*a, x, a->xfull);
      TLS_CHECK_LAUNCH();
      int launched = 0;
      if (int rc = tls_normal_apply(a->normal, a->xfull, a->yfull, nullptr, &launched, nullptr, s)) return rc;
    }
    if (a->nelim > 0) sg_elim_kernel<DE, 0, TW><<<grid_of_n(a->nelim, 128), 128, 0, s>>>(*a, x, nullptr);
    TLS_CHECK_LAUNCH();
    sg_ret_kernel<DE, DM, 0, TW><<<sg_ret_blocks(a), kSgThreads, 0, s>>>(*a, x, nullptr, out, dots, pst);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  });
}

int tls_schur_general_ret_blocks(const tls_schur_general_args* a) { return sg_ret_blocks(a); }

static int sg_maxdim(const tls_schur_general_args* a) { return a->max_dim; }

extern "C" int tls_schur_general_damp(const tls_schur_general_args* a, tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return sg_dispatch(a, sg_maxdim(a), [&](auto de, auto dm, auto tw) -> int {
    constexpr int DE = decltype(de)::value, DM = decltype(dm)::value;
    using TW = decltype(tw);
    cudaError_t e = cudaMemsetAsync(a->bad, 0, sizeof(int32_t), s);
    if (e != cudaSuccess) return tls_set_cuda_error(e);
    if (a->nelim > 0) sg_factor_kernel<DE><<<grid_of_n(a->nelim, 128), 128, 0, s>>>(*a);
    TLS_CHECK_LAUNCH();
    if (a->nretained > 0) sg_whiten_kernel<DE, DM, TW><<<sg_ret_blocks(a), kSgThreads, 0, s>>>(*a);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  });
}

extern "C" int tls_schur_general_matvec(const tls_schur_general_args* a, const double* x, double* out,
                                        tls_stream_t stream) {
  return tls_schur_general_apply(a, x, out, nullptr, nullptr, nullptr, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int tls_schur_general_reduced_rhs(const tls_schur_general_args* a, const double* b, double* out,
                                             tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return sg_dispatch(a, sg_maxdim(a), [&](auto de, auto dm, auto tw) -> int {
    constexpr int DE = decltype(de)::value, DM = decltype(dm)::value;
    using TW = decltype(tw);
    if (a->nelim > 0) sg_elim_rhs_kernel<DE><<<grid_of_n(a->nelim, 128), 128, 0, s>>>(*a, b);
    TLS_CHECK_LAUNCH();
    sg_ret_kernel<DE, DM, 1, TW><<<sg_ret_blocks(a), kSgThreads, 0, s>>>(*a, nullptr, b, out, nullptr, nullptr);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  });
}

extern "C" int tls_schur_general_backsubstitute(const tls_schur_general_args* a, const double* x, double* delta_full,
                                                tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return sg_dispatch(a, sg_maxdim(a), [&](auto de, auto dm, auto tw) -> int {
    constexpr int DE = decltype(de)::value;
    using TW = decltype(tw);
    if (a->nretained > 0) sg_scatter_kernel<<<grid_of_n(a->nretained, 128), 128, 0, s>>>(*a, x, delta_full);
    TLS_CHECK_LAUNCH();
    if (a->nelim > 0) sg_elim_kernel<DE, 1, TW><<<grid_of_n(a->nelim, 128), 128, 0, s>>>(*a, x, delta_full);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  });
}

extern "C" int tls_schur_general_preconditioner_blocks(const tls_schur_general_args* a, double* out,
                                                       tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return sg_dispatch(a, sg_maxdim(a), [&](auto de, auto dm, auto) -> int {
    constexpr int DE = decltype(de)::value, DM = decltype(dm)::value;
    if (a->nretained > 0) sg_precond_kernel<DE, DM><<<grid_of_n(a->nretained, 64), 64, 0, s>>>(*a, out);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  });
}

extern "C" int tls_schur_general_pair_blocks(const tls_schur_general_args* a, int32_t count, const int32_t* ptr,
                                             const int32_t* edge_a, const int32_t* edge_b, int32_t da, int32_t db,
                                             double* out, tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int m = da > db ? da : db;
  if (da < 1 || db < 1) return tls_set_error(TLS_ERR_INVALID, "general Schur: pair block dims");
  return sg_dispatch(a, m, [&](auto de, auto dm, auto) -> int {
    constexpr int DE = decltype(de)::value, DM = decltype(dm)::value;
    if (count > 0)
      sg_pairs_kernel<DE, DM><<<grid_of_n(count, 64), 64, 0, s>>>(*a, count, ptr, edge_a, edge_b, da, db, out);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  });
}
