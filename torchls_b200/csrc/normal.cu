// Block-sparse Jacobian products on the SoA layout.
//
// normal_matvec: y = diag(s) J^T J diag(s) x + lambda x (torchls sparse.py:83-84,
// warp_normal.py:26-122). One factor-major pass computes q_f = J_f (s.x)
// and each slot's J_s^T q_f into a contribution buffer (coalesced SoA loads of
// J, coalesced contribution stores); a second pass sums each variable's
// contributions in a fixed list order. No atomics: results are bitwise
// reproducible run to run.
#include <mutex>

#include "common.cuh"
#include "pcg_state.cuh"

namespace tls {

struct FactorPass {
  int64_t n;
  int32_t R, D;
  int8_t col_slot[32];
  int32_t slot_col[TLS_MAX_SLOTS];
  int32_t slot_dim[TLS_MAX_SLOTS];
  int64_t slot_off[TLS_MAX_SLOTS];
  const int32_t* index[TLS_MAX_SLOTS];
  const void* jac;
  int64_t ld;
};

__host__ FactorPass make_pass(const tls_factor_group& fg, const tls_var_group* vg) {
  FactorPass p{};
  p.n = fg.count;
  p.R = fg.rdim;
  p.D = fg.total_dim;
  for (int c = 0; c < 32; ++c) p.col_slot[c] = -1;
  for (int s = 0; s < fg.nslots; ++s) {
    p.slot_col[s] = fg.slot_col[s];
    p.slot_dim[s] = fg.slot_dim[s];
    p.slot_off[s] = vg[fg.slot_group[s]].offset;
    p.index[s] = fg.index[s];
    for (int j = 0; j < fg.slot_dim[s]; ++j) p.col_slot[fg.slot_col[s] + j] = (int8_t)s;
  }
  p.jac = fg.jac;
  p.ld = fg.jac_stride ? fg.jac_stride : fg.count;
  return p;
}

// MODE 0: contributions J^T J x (per factor)   MODE 1: rows J x   MODE 2: |J x|^2 partial
// MODE 3: contributions J^T u for factor rows u (x holds u, [N][R])
template <int RM, int DM, int MODE, typename TJ, typename TV, typename TA>
__global__ void __launch_bounds__(128) factor_pass_kernel(FactorPass p, const TV* __restrict__ x,
                                                          const TV* __restrict__ scale, TV* __restrict__ out,
                                                          double* __restrict__ partials) {
  const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  TA q[RM];
#pragma unroll
  for (int i = 0; i < RM; ++i) q[i] = TA(0);
  TA xv[DM];
  const TJ* __restrict__ jac = reinterpret_cast<const TJ*>(p.jac);
  const bool live = f < p.n;
  // factor-major outputs ([N][D] or [N][R]) go through a per-warp shared stage
  // so the warp stores its contiguous range with coalesced stores
  constexpr int kStage = (MODE == 1) ? RM : DM;
  __shared__ TV stage[128 / 32][32 * kStage];
  const int lane = threadIdx.x & 31;
  TV* row_stage = stage[threadIdx.x >> 5];
  const int64_t f0 = f - lane;
  const int width = (MODE == 1) ? p.R : p.D;
  if (live) {
#pragma unroll
    for (int c = 0; c < DM; ++c) {
      const int s = p.col_slot[c];
      xv[c] = TA(0);
      if (MODE != 3 && s >= 0) {
        const int64_t col = p.slot_off[s] + (int64_t)__ldg(p.index[s] + f) * p.slot_dim[s] + (c - p.slot_col[s]);
        TA v = static_cast<TA>(__ldg(x + col));
        if (scale) v *= static_cast<TA>(__ldg(scale + col));
        xv[c] = v;
      }
    }
    // Large blocks are not held in registers (occupancy): J is streamed row by
    // row for q = J x and read again (L1/L2 hits) for J^T q. Same arithmetic order.
    constexpr bool kHold = RM * DM <= 36;
    auto jget = [&](int i, int c) -> TJ {
      return (i < p.R && c < p.D) ? __ldg(jac + (int64_t)(i * p.D + c) * p.ld + f) : TJ(0);
    };
    TJ J[kHold ? RM : 1][kHold ? DM : 1];
    if constexpr (kHold) {
#pragma unroll
      for (int i = 0; i < RM; ++i)
#pragma unroll
        for (int c = 0; c < DM; ++c) J[i][c] = jget(i, c);
    }
    if constexpr (MODE == 3) {
#pragma unroll
      for (int i = 0; i < RM; ++i)
        if (i < p.R) q[i] = static_cast<TA>(x[f * p.R + i]);
    } else {
#pragma unroll
      for (int i = 0; i < RM; ++i)
#pragma unroll
        for (int c = 0; c < DM; ++c) {
          if constexpr (kHold) q[i] += static_cast<TA>(J[i][c]) * xv[c];
          else q[i] += static_cast<TA>(jget(i, c)) * xv[c];
        }
    }
    if constexpr (MODE == 0 || MODE == 3) {
#pragma unroll
      for (int c = 0; c < DM; ++c) {
        TA y = TA(0);
#pragma unroll
        for (int i = 0; i < RM; ++i) {
          if constexpr (kHold) y += static_cast<TA>(J[i][c]) * q[i];
          else y += static_cast<TA>(jget(i, c)) * q[i];
        }
        if (c < p.D) row_stage[lane * width + c] = static_cast<TV>(y);
      }
    } else if constexpr (MODE == 1) {
#pragma unroll
      for (int i = 0; i < RM; ++i)
        if (i < p.R) row_stage[lane * width + i] = static_cast<TV>(q[i]);
    }
  }
  if constexpr (MODE != 2) {
    __syncwarp();
    if (f0 < p.n) {
      const int nvalid = (p.n - f0) < 32 ? (int)(p.n - f0) : 32;
      TV* dst = out + f0 * width;
      for (int k = lane; k < nvalid * width; k += 32) dst[k] = row_stage[k];
    }
  }
  if constexpr (MODE == 2) {
    __shared__ double sm[4];
    double acc = 0.0;
    if (live) {
#pragma unroll
      for (int i = 0; i < RM; ++i) acc += to_d(q[i]) * to_d(q[i]);
    }
    const double s = block_sum<128>(acc, sm);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
  }
}

template <int MODE, typename TJ, typename TV, typename TA>
static int launch_factor_pass(const FactorPass& p, const TV* x, const TV* scale, TV* out, double* partials,
                              cudaStream_t st) {
  if (p.n == 0) return TLS_OK;
  const int block = 128;
  const int64_t grid = (p.n + block - 1) / block;
#define TLS_FP(RM, DM)                                                                                    \
  if (p.R <= RM && p.D <= DM) {                                                                          \
    factor_pass_kernel<RM, DM, MODE, TJ, TV, TA><<<grid, block, 0, st>>>(p, x, scale, out, partials); \
    TLS_CHECK_LAUNCH();                                                                                   \
    return TLS_OK;                                                                                        \
  }
  TLS_FP(1, 4)
  TLS_FP(2, 4)
  TLS_FP(3, 4)
  TLS_FP(2, 9)
  TLS_FP(3, 6)
  TLS_FP(3, 9)
  TLS_FP(4, 8)
  TLS_FP(6, 12)
  TLS_FP(7, 14)
  TLS_FP(8, 16)
#undef TLS_FP
  return tls_set_error(TLS_ERR_UNSUPPORTED, "factor shape beyond r <= 8, D <= 16");
}

// Gather: y[col] = s[col] * sum(contrib) + lambda * x[col], deterministic order.
struct GatherGroups {
  int32_t ngroups;
  int32_t block_begin[TLS_MAX_GROUPS + 1];
  int64_t offset[TLS_MAX_GROUPS];
  int32_t dim[TLS_MAX_GROUPS];
  tls_segments seg[TLS_MAX_GROUPS];
};

// Lanes per target: 1..32 (aligned lane groups inside a warp) or, for hot
// variables, a whole 256-thread block per target ("block mode", lanes > 32).
__host__ __device__ __forceinline__ int gather_blocks_for(const tls_segments& seg) {
  if (seg.lanes > 32) return seg.count;
  const int64_t threads = (int64_t)seg.count * seg.lanes;
  return (int)((threads + 255) / 256);
}

template <int WM, typename TV>
__global__ void __launch_bounds__(256) normal_gather_kernel(GatherGroups g, const TV* __restrict__ contrib,
                                                            const TV* __restrict__ x, const TV* __restrict__ scale,
                                                            double damping, TV* __restrict__ y,
                                                            double* __restrict__ dot_partials, PcgState* pst) {
  __shared__ double red[8][WM];
  __shared__ double sm[8];
  int gi = 0;
#pragma unroll 1
  while (gi + 1 < g.ngroups && (int)blockIdx.x >= g.block_begin[gi + 1]) ++gi;
  const tls_segments& seg = g.seg[gi];
  const int d = g.dim[gi];
  const bool block_mode = seg.lanes > 32;
  const int L = block_mode ? 256 : seg.lanes;
  int64_t t;
  int lane;
  if (block_mode) {
    t = blockIdx.x - g.block_begin[gi];
    lane = threadIdx.x;
  } else {
    const int64_t local = (int64_t)(blockIdx.x - g.block_begin[gi]) * blockDim.x + threadIdx.x;
    t = local / L;
    lane = (int)(local % L);
  }
  double acc[WM];
#pragma unroll
  for (int k = 0; k < WM; ++k) acc[k] = 0.0;
  if (t < seg.count) {
    const int b = seg.ptr[t], e = seg.ptr[t + 1];
    // two entries per lane in flight per round; accumulated in list order
    for (int j0 = b + lane; j0 < e; j0 += 2 * L) {
      TV v[2][WM];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int j = j0 + u * L;
        const TV* src = j < e ? contrib + seg.src[j] : nullptr;
#pragma unroll
        for (int k = 0; k < WM; ++k) v[u][k] = (src && k < d) ? src[k] : TV(0);
      }
#pragma unroll
      for (int u = 0; u < 2; ++u)
        if (j0 + u * L < e) {
#pragma unroll
          for (int k = 0; k < WM; ++k)
            if (k < d) acc[k] += to_d(v[u][k]);
        }
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
  double dot = 0.0;
  if (t < seg.count && writer) {
    const int64_t base = g.offset[gi] + t * d;
#pragma unroll
    for (int k = 0; k < WM; ++k) {
      if (k < d) {
        const int64_t col = base + k;
        double v = acc[k];
        if (scale) v *= to_d(scale[col]);
        const double xv = x ? to_d(x[col]) : 0.0;
        v += damping * xv;
        const TV out = static_cast<TV>(v);
        y[col] = out;
        dot += xv * to_d(out);
      }
    }
  }
  if (dot_partials) {
    const double s = block_sum<256>(dot, sm);
    if (threadIdx.x == 0) dot_partials[blockIdx.x] = s;
    if (pst) pcg_operator_epilogue<256>(pst, dot_partials, gridDim.x, sm);
  }
}

}  // namespace tls

using namespace tls;

int tls_normal_gather(const tls_normal_args* a, const void* x, void* y, double* dot_partials, int* gather_blocks,
                      void* pcg_state, cudaStream_t st);

int tls_normal_tiles_apply(const tls_normal_args* a, const void* x, void* y, double* dot_partials, int* nblocks,
                           void* pcg_state, cudaStream_t st);
int tls_normal_tiles_blocks(const tls_normal_args* a);

// Number of dot partials the normal operator writes: one per gather block, or
// with a tile plan one per tile CTA plus one per gather block.
int tls_normal_gather_blocks(const tls_normal_args* a) {
  if (a->tiles) return tls_normal_tiles_blocks(a);
  int blocks = 0;
  for (int i = 0; i < a->nvar_groups; ++i) blocks += gather_blocks_for(a->seg[i]);
  return blocks;
}

// Shared by tls_normal_matvec and the PCG driver. Returns the number of dot
// partials written through *gather_blocks.
int tls_normal_apply(const tls_normal_args* a, const void* x, void* y, double* dot_partials, int* gather_blocks,
                     void* pcg_state, cudaStream_t st) {
  if (a->nfactor_groups > TLS_MAX_FACTOR_GROUPS || a->nvar_groups > TLS_MAX_GROUPS)
    return tls_set_error(TLS_ERR_INVALID, "too many groups");
  if (a->tiles) return tls_normal_tiles_apply(a, x, y, dot_partials, gather_blocks, pcg_state, st);
  for (int k = 0; k < a->nfactor_groups; ++k) {
    const tls_factor_group& fg = a->fg[k];
    FactorPass p = make_pass(fg, a->vg);
    int rc;
    if (a->vec_dtype == TLS_F64) {
      double* out = (double*)a->contrib + a->contrib_offset[k];
      if (fg.jac_dtype == TLS_F64)
        rc = launch_factor_pass<0, double, double, double>(p, (const double*)x, (const double*)a->scale, out, nullptr, st);
      else
        rc = launch_factor_pass<0, float, double, double>(p, (const double*)x, (const double*)a->scale, out, nullptr, st);
    } else {
      float* out = (float*)a->contrib + a->contrib_offset[k];
      if (fg.jac_dtype == TLS_F32)
        rc = launch_factor_pass<0, float, float, float>(p, (const float*)x, (const float*)a->scale, out, nullptr, st);
      else
        return tls_set_error(TLS_ERR_UNSUPPORTED, "float64 Jacobian with float32 vectors");
    }
    if (rc) return rc;
  }
  return tls_normal_gather(a, x, y, dot_partials, gather_blocks, pcg_state, st);
}

int tls_normal_gather(const tls_normal_args* a, const void* x, void* y, double* dot_partials, int* gather_blocks,
                      void* pcg_state, cudaStream_t st) {
  PcgState* pst = reinterpret_cast<PcgState*>(pcg_state);
  GatherGroups g{};
  g.ngroups = a->nvar_groups;
  int blocks = 0, wmax = 1;
  for (int i = 0; i < a->nvar_groups; ++i) {
    g.block_begin[i] = blocks;
    g.offset[i] = a->vg[i].offset;
    g.dim[i] = a->vg[i].dim;
    g.seg[i] = a->seg[i];
    blocks += gather_blocks_for(a->seg[i]);
    if (a->vg[i].dim > wmax) wmax = a->vg[i].dim;
  }
  g.block_begin[a->nvar_groups] = blocks;
  if (gather_blocks) *gather_blocks = blocks;
  if (blocks == 0) return TLS_OK;
#define TLS_G(WM)                                                                                        \
  if (wmax <= WM) {                                                                                      \
    if (a->vec_dtype == TLS_F64)                                                                         \
      normal_gather_kernel<WM, double><<<blocks, 256, 0, st>>>(g, (const double*)a->contrib, (const double*)x, \
                                                               (const double*)a->scale, a->damping,     \
                                                               (double*)y, dot_partials, pst);           \
    else                                                                                                 \
      normal_gather_kernel<WM, float><<<blocks, 256, 0, st>>>(g, (const float*)a->contrib, (const float*)x,   \
                                                              (const float*)a->scale, a->damping,       \
                                                              (float*)y, dot_partials, pst);             \
    TLS_CHECK_LAUNCH();                                                                                  \
    return TLS_OK;                                                                                       \
  }
  TLS_G(3)
  TLS_G(6)
  TLS_G(8)
  TLS_G(16)
#undef TLS_G
  return tls_set_error(TLS_ERR_UNSUPPORTED, "variable dim > 16");
}

extern "C" int tls_normal_matvec(const tls_normal_args* a, const void* x, void* y, tls_stream_t stream) {
  return tls_normal_apply(a, x, y, nullptr, nullptr, nullptr, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int tls_jacobian_matvec(const tls_normal_args* a, const void* x, void* out_rows, tls_stream_t stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  int64_t row = 0;
  for (int k = 0; k < a->nfactor_groups; ++k) {
    const tls_factor_group& fg = a->fg[k];
    FactorPass p = make_pass(fg, a->vg);
    int rc;
    if (a->vec_dtype == TLS_F64) {
      double* out = (double*)out_rows + row;
      rc = fg.jac_dtype == TLS_F64
               ? launch_factor_pass<1, double, double, double>(p, (const double*)x, (const double*)a->scale, out, nullptr, st)
               : launch_factor_pass<1, float, double, double>(p, (const double*)x, (const double*)a->scale, out, nullptr, st);
    } else {
      float* out = (float*)out_rows + row;
      if (fg.jac_dtype != TLS_F32) return tls_set_error(TLS_ERR_UNSUPPORTED, "float64 Jacobian with float32 vectors");
      rc = launch_factor_pass<1, float, float, float>(p, (const float*)x, (const float*)a->scale, out, nullptr, st);
    }
    if (rc) return rc;
    row += fg.count * fg.rdim;
  }
  return TLS_OK;
}

__global__ void sum_partials_kernel(const double* partials, int count, double* out, int accumulate) {
  __shared__ double sm[8];
  double acc = 0.0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) acc += partials[i];
  const double s = block_sum<256>(acc, sm);
  if (threadIdx.x == 0) out[0] = accumulate ? out[0] + s : s;
}

// Arguments of both |J x|^2 entry points: x and the column scale are read as
// float64, so a scale of another dtype would be misread.
static int check_sqnorm_args(const tls_normal_args* a, const double* x, const double* out) {
  if (!a || !x || !out) return tls_set_error(TLS_ERR_INVALID, "squared_matvec_norm: null args, x or out");
  if (a->scale && a->vec_dtype != TLS_F64)
    return tls_set_error(TLS_ERR_INVALID, "squared_matvec_norm: the column scale must be float64 (vec_dtype)");
  if (a->nfactor_groups < 0 || a->nfactor_groups > TLS_MAX_FACTOR_GROUPS)
    return tls_set_error(TLS_ERR_INVALID, "squared_matvec_norm: factor group count out of range");
  return TLS_OK;
}

extern "C" int tls_squared_matvec_norm(const tls_normal_args* a, const double* x, double* partials, double* out,
                                       tls_stream_t stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (int rc = check_sqnorm_args(a, x, out)) return rc;
  if (!partials) return tls_set_error(TLS_ERR_INVALID, "squared_matvec_norm: null partials buffer");
  // One launch per factor group; each writes its block partials, then one
  // fixed-order sum accumulates into *out.
  bool first = true;
  for (int k = 0; k < a->nfactor_groups; ++k) {
    const tls_factor_group& fg = a->fg[k];
    if (fg.count == 0) continue;
    FactorPass p = make_pass(fg, a->vg);
    const int blocks = (int)((fg.count + 127) / 128);
    if (blocks > (1 << 20)) return tls_set_error(TLS_ERR_UNSUPPORTED, "too many factors for one pass");
    int rc = fg.jac_dtype == TLS_F64
                 ? launch_factor_pass<2, double, double, double>(p, x, (const double*)a->scale, nullptr, partials, st)
                 : launch_factor_pass<2, float, double, double>(p, x, (const double*)a->scale, nullptr, partials, st);
    if (rc) return rc;
    sum_partials_kernel<<<1, 256, 0, st>>>(partials, blocks, out, first ? 0 : 1);
    TLS_CHECK_LAUNCH();
    first = false;
  }
  if (first) cudaMemsetAsync(out, 0, sizeof(double), st);
  return TLS_OK;
}

extern "C" int tls_jacobian_rmatvec(const tls_normal_args* a, const void* rows, void* out, tls_stream_t stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  int64_t row = 0;
  for (int k = 0; k < a->nfactor_groups; ++k) {
    const tls_factor_group& fg = a->fg[k];
    FactorPass p = make_pass(fg, a->vg);
    int rc;
    if (a->vec_dtype == TLS_F64) {
      double* c = (double*)a->contrib + a->contrib_offset[k];
      const double* u = (const double*)rows + row;
      rc = fg.jac_dtype == TLS_F64 ? launch_factor_pass<3, double, double, double>(p, u, nullptr, c, nullptr, st)
                                   : launch_factor_pass<3, float, double, double>(p, u, nullptr, c, nullptr, st);
    } else {
      if (fg.jac_dtype != TLS_F32) return tls_set_error(TLS_ERR_UNSUPPORTED, "float64 Jacobian with float32 vectors");
      rc = launch_factor_pass<3, float, float, float>(p, (const float*)rows + row, nullptr,
                                                      (float*)a->contrib + a->contrib_offset[k], nullptr, st);
    }
    if (rc) return rc;
    row += fg.count * fg.rdim;
  }
  tls_normal_args b = *a;
  b.damping = 0.0;
  return tls_normal_gather(&b, nullptr, out, nullptr, nullptr, nullptr, st);
}

// ---------------------------------------------------------------- |J x|^2 without caller scratch
// Some callers cannot allocate device memory at the point where they need
// this norm: code running inside another framework's allocator or memory
// pool, a host language binding with no device allocator of its own, or a
// real-time loop where an allocation may block. For them the block partials
// live in one file-scope array instead of a caller-supplied buffer. Every GPU
// that loads this library holds the array (512 KB) until the process exits.
// Each call rewrites exactly the partials it then sums, so nothing has to be
// cleared between calls; but every call on a device shares the one array, so
// calls whose kernels overlap on the GPU (different streams without ordering)
// race and may return wrong sums.
constexpr int kStaticSqnormPartials = 65536;  // one double per 128-factor block
static __device__ __align__(256) double g_sqnorm_scratch[kStaticSqnormPartials];

namespace {
constexpr int kMaxScratchDevices = 64;
std::mutex g_scratch_mu;
double* g_scratch_addr[kMaxScratchDevices] = {};

// Device address of g_sqnorm_scratch on the current device. The symbol name
// in host code is only a host-side stand-in; kernels must get this address.
int static_scratch(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return tls_set_error(TLS_ERR_CUDA, "cudaGetDevice failed");
  if (dev < 0 || dev >= kMaxScratchDevices) return tls_set_error(TLS_ERR_UNSUPPORTED, "device index beyond 63");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sqnorm_scratch);
    if (e != cudaSuccess || !p) return tls_set_error(TLS_ERR_CUDA, cudaGetErrorString(e));
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[dev];
  return TLS_OK;
}
}  // namespace

extern "C" int tls_squared_matvec_norm_static(const tls_normal_args* a, const double* x, double* out,
                                              tls_stream_t stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (int rc = check_sqnorm_args(a, x, out)) return rc;
  for (int k = 0; k < a->nfactor_groups; ++k) {
    if ((a->fg[k].count + 127) / 128 > kStaticSqnormPartials)
      return tls_set_error(TLS_ERR_INVALID,
                           "tls_squared_matvec_norm_static: a factor group has more than 8,388,608 factors "
                           "(65,536 blocks of 128); use tls_squared_matvec_norm with a caller buffer");
  }
  double* partials = nullptr;
  int rc = static_scratch(&partials);
  if (rc) return rc;
  bool first = true;
  for (int k = 0; k < a->nfactor_groups; ++k) {
    const tls_factor_group& fg = a->fg[k];
    if (fg.count == 0) continue;
    FactorPass p = make_pass(fg, a->vg);
    const int blocks = (int)((fg.count + 127) / 128);
    rc = fg.jac_dtype == TLS_F64
             ? launch_factor_pass<2, double, double, double>(p, x, (const double*)a->scale, nullptr, partials, st)
             : launch_factor_pass<2, float, double, double>(p, x, (const double*)a->scale, nullptr, partials, st);
    if (rc) return rc;
    sum_partials_kernel<<<1, 256, 0, st>>>(partials, blocks, out, first ? 0 : 1);
    TLS_CHECK_LAUNCH();
    first = false;
  }
  if (first) cudaMemsetAsync(out, 0, sizeof(double), st);
  return TLS_OK;
}
