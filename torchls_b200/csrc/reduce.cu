// Deterministic reductions: segmented gather-reduce of per-factor
// contributions (replaces the index_add scatters of torchls sparse.py:43-55,
// sparse.py:104-121, schur.py:213-224 and the atomic accumulations of
// warp_diagonal.py:14-66), float64 vector sums, and trial-step terms
// (problem.py:315-348, losses.py:92-107).
#include "common.cuh"

namespace tls {

template <int WM, typename TC, typename TO>
__global__ void __launch_bounds__(256) segment_reduce_kernel(tls_segments seg, const TC* __restrict__ contrib,
                                                             int mode, int dim, TO* __restrict__ out) {
  __shared__ double red[8][WM];
  const bool block_mode = seg.lanes > 32;
  const int L = block_mode ? 256 : seg.lanes;
  int64_t t;
  int lane;
  if (block_mode) {
    t = blockIdx.x;
    lane = threadIdx.x;
  } else {
    const int64_t gt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    t = gt / L;
    lane = (int)(gt % L);
  }
  const int W = seg.width;
  double acc[WM];
#pragma unroll
  for (int k = 0; k < WM; ++k) acc[k] = 0.0;
  if (t < seg.count) {
    const int b = seg.ptr[t], e = seg.ptr[t + 1];
    for (int j = b + lane; j < e; j += L) {
      const TC* src = contrib + seg.src[j];
#pragma unroll
      for (int k = 0; k < WM; ++k)
        if (k < W) acc[k] += to_d(src[k]);
    }
  }
  bool writer;
  if (block_mode) {
    const int w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < WM; ++k) {
      const double v = warp_sum(acc[k]);
      if ((threadIdx.x & 31) == 0) red[w][k] = v;
    }
    __syncthreads();
    writer = threadIdx.x == 0;
    if (writer) {
#pragma unroll
      for (int k = 0; k < WM; ++k) {
        double v = 0.0;
#pragma unroll
        for (int q = 0; q < 8; ++q) v += red[q][k];
        acc[k] = v;
      }
    }
  } else {
#pragma unroll
    for (int k = 0; k < WM; ++k) acc[k] = group_sum(acc[k], L);
    writer = lane == 0;
  }
  if (t >= seg.count || !writer) return;
  if (mode == 0) {
#pragma unroll
    for (int k = 0; k < WM; ++k)
      if (k < W) out[t * W + k] = static_cast<TO>(acc[k]);
  } else {
    // packed upper Gram (row-major) -> symmetric dim x dim
    TO* o = out + t * dim * dim;
    int idx = 0;
    for (int a = 0; a < dim; ++a)
      for (int c = a; c < dim; ++c) {
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < WM; ++k)
          if (k == idx) v = acc[k];
        o[a * dim + c] = static_cast<TO>(v);
        o[c * dim + a] = static_cast<TO>(v);
        ++idx;
      }
  }
}

// Vector targets summed by one lane: one thread per (target, component), so
// consecutive threads read and write consecutive addresses when consecutive
// targets' contributions are contiguous (the Schur cross blocks: one
// contribution per edge). Each element sums its contributions in list order,
// exactly as the one-lane path of segment_reduce_kernel does.
template <typename TC, typename TO>
__global__ void __launch_bounds__(256) segment_reduce_elem_kernel(tls_segments seg, const TC* __restrict__ contrib,
                                                                  TO* __restrict__ out) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int W = seg.width;
  if (e >= (int64_t)seg.count * W) return;
  const int64_t t = e / W;
  const int k = (int)(e - t * W);
  double acc = 0.0;
  for (int j = seg.ptr[t]; j < seg.ptr[t + 1]; ++j) acc += to_d(contrib[seg.src[j] + k]);
  out[e] = static_cast<TO>(acc);
}

template <typename TC, typename TO>
static int launch_segments(const tls_segments* seg, const TC* c, int mode, int dim, TO* out, cudaStream_t st) {
  if (seg->count == 0) return TLS_OK;
  const int L = seg->lanes;
  if (L < 1 || (L <= 32 && (L & (L - 1))) || (L > 32 && L != 256))
    return tls_set_error(TLS_ERR_INVALID, "lanes must be a power of two <= 32, or 256 (block per target)");
  const int block = 256;
  const int64_t grid = L > 32 ? seg->count : ((int64_t)seg->count * L + block - 1) / block;
  const int W = seg->width;
  if (mode == 0 && L == 1 && W >= 4) {
    const int64_t elems = (int64_t)seg->count * W;
    segment_reduce_elem_kernel<TC, TO><<<(unsigned)((elems + block - 1) / block), block, 0, st>>>(*seg, c, out);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  }
  if (W <= 4)
    segment_reduce_kernel<4, TC, TO><<<grid, block, 0, st>>>(*seg, c, mode, dim, out);
  else if (W <= 8)
    segment_reduce_kernel<8, TC, TO><<<grid, block, 0, st>>>(*seg, c, mode, dim, out);
  else if (W <= 16)
    segment_reduce_kernel<16, TC, TO><<<grid, block, 0, st>>>(*seg, c, mode, dim, out);
  else if (W <= 36)
    segment_reduce_kernel<36, TC, TO><<<grid, block, 0, st>>>(*seg, c, mode, dim, out);
  else if (W <= 64)
    segment_reduce_kernel<64, TC, TO><<<grid, block, 0, st>>>(*seg, c, mode, dim, out);
  else
    return tls_set_error(TLS_ERR_UNSUPPORTED, "segment width > 64");
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}

// ------------------------------------------------------------------ plain sums
constexpr int kRedBlocks = 1024;
constexpr int kRedThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kRedThreads) reduce_partial_kernel(const T* __restrict__ x, int64_t n, int op,
                                                                     double* __restrict__ partials) {
  __shared__ double sm[kRedThreads / 32];
  double acc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = to_d(x[i]);
    if (op == TLS_SUM_PLAIN) acc += v;
    else if (op == TLS_SUM_SQUARES) acc += v * v;
    else {
      const double a = fabs(v);
      acc = (a > acc || isnan(a)) ? a : acc;
    }
  }
  if (op == TLS_SUM_ABSMAX) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double b = __shfl_xor_sync(0xffffffffu, acc, o);
      acc = (b > acc || isnan(b)) ? b : acc;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sm[w] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = sm[0];
      for (int k = 1; k < kRedThreads / 32; ++k) m = (sm[k] > m || isnan(sm[k])) ? sm[k] : m;
      partials[blockIdx.x] = m;
    }
    return;
  }
  const double s = block_sum<kRedThreads>(acc, sm);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kRedThreads) reduce_final_kernel(const double* __restrict__ partials, int count,
                                                                   int op, double* __restrict__ out, int accumulate,
                                                                   double factor) {
  __shared__ double sm[kRedThreads / 32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    const double v = partials[i];
    if (op == TLS_SUM_ABSMAX) acc = (v > acc || isnan(v)) ? v : acc;
    else acc += v;
  }
  if (op == TLS_SUM_ABSMAX) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double b = __shfl_xor_sync(0xffffffffu, acc, o);
      acc = (b > acc || isnan(b)) ? b : acc;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sm[w] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = sm[0];
      for (int k = 1; k < kRedThreads / 32; ++k) m = (sm[k] > m || isnan(sm[k])) ? sm[k] : m;
      out[0] = m;
    }
    return;
  }
  const double s = block_sum<kRedThreads>(acc, sm);
  if (threadIdx.x == 0) out[0] = accumulate ? out[0] + factor * s : factor * s;
}

// ------------------------------------------------------------------ trial terms
__global__ void __launch_bounds__(kRedThreads) trial_kernel(int64_t n, int R, const double* __restrict__ old_raw,
                                                            const double* __restrict__ new_raw, int loss_kind,
                                                            double delta, const double* __restrict__ rho_old,
                                                            const double* __restrict__ rho_new,
                                                            const double* __restrict__ weights, int has_loss,
                                                            double* __restrict__ partials) {
  __shared__ double sm[kRedThreads / 32];
  double val = 0.0, red = 0.0;
  const double tiny = 2.2250738585072014e-308;
  for (int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; f < n; f += (int64_t)gridDim.x * blockDim.x) {
    double so = 0.0, sn = 0.0, diff = 0.0;
    for (int i = 0; i < R; ++i) {
      const double a = old_raw[f * R + i], b = new_raw[f * R + i];
      so += a * a;
      sn += b * b;
      diff += (a - b) * (a + b);
    }
    double v = sn, r = diff;
    if (has_loss && loss_kind == TLS_LOSS_HUBER) {
      const double nn = sqrt(sn > tiny ? sn : tiny);
      v = sn > delta * delta ? delta * (2.0 * nn - delta) : sn;
      // divided difference of rho (losses.py:92-107)
      const double a = sqrt(so), b = sqrt(sn);
      const double lo = a < b ? a : b, hi = a < b ? b : a;
      double sh = delta - lo;
      sh = sh > 0.0 ? sh : 0.0;
      const double gap = hi - lo;
      const double apb = a + b;
      const double crossing = (2.0 * delta - sh * (sh / (gap > tiny ? gap : tiny))) / (apb > tiny ? apb : tiny);
      const double coef = hi <= delta ? 1.0 : (lo >= delta ? 2.0 * delta / (apb > tiny ? apb : tiny) : crossing);
      r = diff * coef;
    } else if (has_loss && loss_kind == TLS_LOSS_GENERIC) {
      v = rho_new[f];
      r = rho_old[f] - rho_new[f];
    }
    if (has_loss && weights) {
      v *= weights[f];
      r *= weights[f];
    }
    val += v;
    red += r;
  }
  const double sv = block_sum<kRedThreads>(val, sm);
  const double sr = block_sum<kRedThreads>(red, sm);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = sv;
    partials[kRedBlocks + blockIdx.x] = sr;
  }
}

static int red_grid(int64_t n) {
  int64_t g = (n + kRedThreads - 1) / kRedThreads;
  if (g > kRedBlocks) g = kRedBlocks;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace tls

using namespace tls;

extern "C" int tls_segment_reduce(const tls_segments* seg, const void* contrib, int32_t contrib_dtype, int32_t mode,
                                  int32_t dim, void* out, int32_t out_dtype, tls_stream_t stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (mode == 1 && out_dtype != TLS_F64) return tls_set_error(TLS_ERR_INVALID, "Gram output must be float64");
  if (contrib_dtype == TLS_F64) {
    if (out_dtype == TLS_F64)
      return launch_segments(seg, (const double*)contrib, mode, dim, (double*)out, st);
    return launch_segments(seg, (const double*)contrib, mode, dim, (float*)out, st);
  }
  if (out_dtype == TLS_F64) return launch_segments(seg, (const float*)contrib, mode, dim, (double*)out, st);
  return launch_segments(seg, (const float*)contrib, mode, dim, (float*)out, st);
}

extern "C" int tls_reduce(const void* x, int32_t dtype, int64_t n, int32_t op, double* partials, double* out,
                          tls_stream_t stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int g = red_grid(n);
  if (dtype == TLS_F64)
    reduce_partial_kernel<double><<<g, kRedThreads, 0, st>>>((const double*)x, n, op, partials);
  else
    reduce_partial_kernel<float><<<g, kRedThreads, 0, st>>>((const float*)x, n, op, partials);
  TLS_CHECK_LAUNCH();
  reduce_final_kernel<<<1, kRedThreads, 0, st>>>(partials, g, op, out, 0, 1.0);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}

extern "C" int tls_trial_terms(int64_t count, int32_t rdim, const double* old_raw, const double* new_raw,
                               int32_t loss_kind, double delta, const double* rho_old, const double* rho_new,
                               const double* weights, int32_t has_loss, double* partials, double* out,
                               tls_stream_t stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (count == 0) return TLS_OK;
  const int g = red_grid(count);
  trial_kernel<<<g, kRedThreads, 0, st>>>(count, rdim, old_raw, new_raw, loss_kind, delta, rho_old, rho_new,
                                          weights, has_loss, partials);
  TLS_CHECK_LAUNCH();
  reduce_final_kernel<<<1, kRedThreads, 0, st>>>(partials, g, TLS_SUM_PLAIN, out, 1, 0.5);
  TLS_CHECK_LAUNCH();
  reduce_final_kernel<<<1, kRedThreads, 0, st>>>(partials + kRedBlocks, g, TLS_SUM_PLAIN, out + 1, 1, 0.5);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}
