// One-pass normal operator over a tile plan (tls_normal_tiles).
//
// y = diag(s) J^T J diag(s) x + lambda x (torchls sparse.py:83-84,
// warp_normal.py:26-122) reading J once. Per tile of consecutive factors
// each thread takes factors i, i + 256, ...: J_f from the SoA rows (coalesced
// across the warp), x gathered per slot, q = J_f (s.x) and every slot's
// J_s^T q in float64, stored to a shared-memory stage at the position the plan
// gives that (slot, factor) pair. The stage is ordered by target variable, so
// each target's contributions form one contiguous run; one thread sums a run
// in order and either finishes the target (all its contributions were in the
// run), adds it to the CTA's shared accumulator (targets that recur across the
// CTA's tiles, such as the cameras of a bundle adjustment), or stores it as a
// partial. The CTA then flushes its accumulator, and a last kernel sums each
// remaining target's partials in list order. Every order is fixed by the
// plan: bitwise reproducible, no atomics on values.
#include <atomic>

#include "common.cuh"
#include "pcg_state.cuh"

namespace tls {

constexpr int kTileThreads = 512;
// shared memory a tile CTA may use (stage + accumulator), below the 227 KB limit
constexpr int kTileSmemLimit = 200 * 1024;

struct TileLaunch {
  int64_t n;
  int32_t R, D, T, S;
  int64_t ncols;  // length of x, y and the column scale
  int8_t col_slot[32];
  int32_t slot_col[TLS_MAX_SLOTS];
  int32_t slot_dim[TLS_MAX_SLOTS];
  int64_t slot_off[TLS_MAX_SLOTS];
  const int32_t* index[TLS_MAX_SLOTS];
  const void* jac;
  int64_t ld;
  const uint32_t* pos;
  int32_t tile_base, cta_base, stage_doubles, acc_doubles, xbuf_doubles, pad2_;
  const int32_t* cta_tile;
  const int32_t* tile_run;
  const int32_t* run_col;
  const int32_t* run_meta;
  const int32_t* run_dest;
  const int32_t* run_xoff;
  const int32_t* cta_flush;
  const int32_t* flush_col;
  const int32_t* flush_meta;
  const int32_t* flush_dest;
  double* partials;
};

// Hint: bring [p, p + bytes) into L2 (bulk prefetch; only the 16-byte-aligned
// interior is requested, so nothing outside the range is touched).
__device__ __forceinline__ void prefetch_l2(const void* p, int64_t bytes) {
  uint64_t a = reinterpret_cast<uint64_t>(p), b = a + (uint64_t)(bytes > 0 ? bytes : 0);
  a = (a + 15) & ~uint64_t(15);
  b &= ~uint64_t(15);
  while (b > a) {
    const uint32_t n = (b - a) > (1u << 16) ? (1u << 16) : (uint32_t)(b - a);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(n) : "memory");
    a += n;
  }
}

// The next tile's J rows, stage-position rows and run lists go to L2 while
// this tile computes; one thread per range.
template <typename TJ>
__device__ __forceinline__ void prefetch_tile(const TileLaunch& p, int t) {
  const int64_t f0 = (int64_t)(t - p.tile_base) * p.T;
  const int64_t nt = (p.n - f0) < p.T ? (p.n - f0) : p.T;
  const int rows = p.R * p.D;
  const int k = threadIdx.x;
  const TJ* jac = reinterpret_cast<const TJ*>(p.jac);
  if (k < rows) {
    prefetch_l2(jac + (int64_t)k * p.ld + f0, nt * (int64_t)sizeof(TJ));
  } else if (k < rows + p.S) {
    prefetch_l2(p.pos + (int64_t)(k - rows) * p.n + f0, nt * 4);
  } else if (k < rows + p.S + 4) {
    const int r0 = p.tile_run[t], r1 = p.tile_run[t + 1];
    const int j = k - rows - p.S;
    const int32_t* arr = j == 0 ? p.run_meta : (j == 1 ? p.run_dest : (j == 2 ? p.run_col : p.run_xoff));
    prefetch_l2(arr + r0, (int64_t)(r1 - r0) * 4);
  }
}

template <typename TV>
__device__ __forceinline__ void finish_col(int64_t col, double sum, const TV* __restrict__ x,
                                           const TV* __restrict__ scale, double damping, TV* __restrict__ y,
                                           double& dot) {
  double v = sum;
  if (scale) v *= to_d(scale[col]);
  const double xv = to_d(x[col]);
  v += damping * xv;
  const TV out = static_cast<TV>(v);
  y[col] = out;
  dot += xv * to_d(out);
}

// Select arr[s] for a runtime slot s without dynamic register indexing.
template <int SMX>
__device__ __forceinline__ int pick(const int (&arr)[SMX], int s) {
  int v = arr[0];
#pragma unroll
  for (int k = 1; k < SMX; ++k)
    if (s == k) v = arr[k];
  return v;
}

// U factors per thread in flight, up to SMX slots per factor; J held in
// registers when RM*DM <= 54, else re-read (L1 hits) for J^T q. Every
// independent load (indices, stage positions, J) is issued before the first
// dependent one, so a thread waits about one DRAM and one L2 latency per
// round instead of one per slot.
template <int RM, int DM, int U, int SMX, typename TJ, typename TV>
__global__ void __launch_bounds__(kTileThreads, (RM * DM <= 18) ? 2 : 1)
    normal_tile_kernel(TileLaunch p, const TV* __restrict__ x, const TV* __restrict__ scale, double damping,
                       TV* __restrict__ y, double* __restrict__ dot_partials) {
  extern __shared__ __align__(16) double tile_smem[];
  __shared__ double red[kTileThreads / 32];
  asm volatile("griddepcontrol.launch_dependents;");
  double* stage = tile_smem;
  double* acc = tile_smem + p.stage_doubles;
  double* xbuf = acc + p.acc_doubles;
  const int cta = p.cta_base + blockIdx.x;
  for (int i = threadIdx.x; i < p.acc_doubles; i += kTileThreads) acc[i] = 0.0;
  const TJ* __restrict__ jac = reinterpret_cast<const TJ*>(p.jac);
  constexpr bool kHold = RM * DM <= 54;
  const int t0 = p.cta_tile[cta], t1 = p.cta_tile[cta + 1];
  double dot = 0.0;
  {
    // this CTA's share of x (and the column scale) to L2: every CTA gathers from all of it
    const int64_t share = ((p.ncols + gridDim.x - 1) / gridDim.x + 15) & ~int64_t(15);
    const int64_t c0 = (int64_t)blockIdx.x * share;
    const int64_t cnt = c0 < p.ncols ? ((p.ncols - c0) < share ? (p.ncols - c0) : share) : 0;
    if (threadIdx.x == kTileThreads - 1) prefetch_l2(x + c0, cnt * (int64_t)sizeof(TV));
    if (threadIdx.x == kTileThreads - 2 && scale) prefetch_l2(scale + c0, cnt * (int64_t)sizeof(TV));
  }
#pragma unroll 1
  for (int t = t0; t < t1; ++t) {
    const int64_t f0 = (int64_t)(t - p.tile_base) * p.T;
    const int nt = (int)((p.n - f0) < p.T ? (p.n - f0) : p.T);
    if (t + 1 < t1) prefetch_tile<TJ>(p, t + 1);
    const int r0 = p.tile_run[t], r1 = p.tile_run[t + 1];
    // ---- prologue: each target's x (times its column scale) once into the x buffer
#pragma unroll 1
    for (int r = r0 + threadIdx.x; r < r1; r += kTileThreads) {
      const int d = ((__ldg(p.run_meta + r) >> 27) & 0xf) + 1;
      const int64_t col = __ldg(p.run_col + r);
      const int xo = __ldg(p.run_xoff + r);
      double v[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) v[c] = c < d ? to_d(x[col + c]) : 0.0;
      if (scale) {
#pragma unroll
        for (int c = 0; c < 16; ++c)
          if (c < d) v[c] *= to_d(scale[col + c]);
      }
#pragma unroll
      for (int c = 0; c < 16; ++c)
        if (c < d) xbuf[xo + c] = v[c];
    }
    __syncthreads();
    // ---- phase A: contributions of this thread's factors into the stage
#pragma unroll 1
    for (int i0 = threadIdx.x; i0 < nt; i0 += kTileThreads * U) {
      int pv[U][SMX];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int i = i0 + u * kTileThreads;
        const bool live = i < nt;
        const int64_t f = f0 + i;
#pragma unroll
        for (int s = 0; s < SMX; ++s) pv[u][s] = (live && s < p.S) ? (int)__ldg(p.pos + (int64_t)s * p.n + f) : 0;
      }
      TJ J[U][kHold ? RM : 1][kHold ? DM : 1];
      if constexpr (kHold) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int i = i0 + u * kTileThreads;
          const bool live = i < nt;
          const int64_t f = f0 + i;
#pragma unroll
          for (int r = 0; r < RM; ++r)
#pragma unroll
            for (int c = 0; c < DM; ++c)
              J[u][r][c] = (live && r < p.R && c < p.D) ? __ldg(jac + (int64_t)(r * p.D + c) * p.ld + f) : TJ(0);
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int i = i0 + u * kTileThreads;
        if (i >= nt) continue;
        const int64_t f = f0 + i;
        auto jget = [&](int r, int c) -> double {
          if constexpr (kHold) return to_d(J[u][r][c]);
          else return (r < p.R && c < p.D) ? to_d(__ldg(jac + (int64_t)(r * p.D + c) * p.ld + f)) : 0.0;
        };
        double xv[DM];
#pragma unroll
        for (int c = 0; c < DM; ++c) {
          const int s = c < p.D ? p.col_slot[c] : -1;
          xv[c] = s >= 0 ? xbuf[(pick<SMX>(pv[u], s) >> 16) + c - p.slot_col[s]] : 0.0;
        }
        double q[RM];
#pragma unroll
        for (int r = 0; r < RM; ++r) {
          double a = 0.0;
#pragma unroll
          for (int c = 0; c < DM; ++c) a += jget(r, c) * xv[c];
          q[r] = a;
        }
#pragma unroll
        for (int c = 0; c < DM; ++c) {
          const int s = c < p.D ? p.col_slot[c] : -1;
          if (s < 0) continue;
          double v = 0.0;
#pragma unroll
          for (int r = 0; r < RM; ++r) v += jget(r, c) * q[r];
          stage[(pick<SMX>(pv[u], s) & 0xffff) + c - p.slot_col[s]] = v;
        }
      }
    }
    __syncthreads();
    // ---- phase B: one thread per run, summed in stage order
#pragma unroll 1
    for (int r = r0 + threadIdx.x; r < r1; r += kTileThreads) {
      const int meta = __ldg(p.run_meta + r);
      const int start = meta & 0x3fff, len = (meta >> 14) & 0x1fff, d = ((meta >> 27) & 0xf) + 1;
      const int dest = __ldg(p.run_dest + r);
      const int64_t col = __ldg(p.run_col + r);
      const int xo = dest == -1 ? __ldg(p.run_xoff + r) : 0;
      // components in chunks of four; a final run's x is in the x buffer
      // (without a column scale) or loaded with its scale before the sums
#pragma unroll 1
      for (int c0 = 0; c0 < d; c0 += 4) {
        double xs[4], sc[4], v[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          xs[c] = 0.0;
          sc[c] = 1.0;
          v[c] = 0.0;
          if (dest == -1 && c0 + c < d) {
            if (scale) {
              xs[c] = to_d(x[col + c0 + c]);
              sc[c] = to_d(scale[col + c0 + c]);
            } else {
              xs[c] = xbuf[xo + c0 + c];
            }
          }
        }
        const double* src = stage + start + c0;
#pragma unroll 1
        for (int e = 0; e < len; ++e, src += d) {
#pragma unroll
          for (int c = 0; c < 4; ++c)
            if (c0 + c < d) v[c] += src[c];
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (c0 + c >= d) continue;
          if (dest == -1) {
            const TV out = static_cast<TV>(v[c] * sc[c] + damping * xs[c]);
            y[col + c0 + c] = out;
            dot += xs[c] * to_d(out);
          } else if (dest < -1) {
            acc[-2 - dest + c0 + c] += v[c];
          } else {
            p.partials[dest + c0 + c] = v[c];
          }
        }
      }
    }
    __syncthreads();
  }
  __syncthreads();
  // ---- flush the accumulator
  const int j0 = p.cta_flush[cta], j1 = p.cta_flush[cta + 1];
#pragma unroll 1
  for (int j = j0 + threadIdx.x; j < j1; j += kTileThreads) {
    const int meta = __ldg(p.flush_meta + j);
    const int off = meta & 0xffff, d = ((meta >> 16) & 0xf) + 1;
    const int dest = __ldg(p.flush_dest + j);
    const int64_t col = __ldg(p.flush_col + j);
    for (int c = 0; c < d; ++c) {
      if (dest == -1) finish_col(col + c, acc[off + c], x, scale, damping, y, dot);
      else p.partials[dest + c] = acc[off + c];
    }
  }
  if (dot_partials) {
    const double s = block_sum<kTileThreads>(dot, red);
    if (threadIdx.x == 0) dot_partials[cta] = s;
  }
}

// ---------------------------------------------------------------------------
// Specialised kernel for the common factor shapes: one or two slots with
// compile-time residual and slot dimensions (reprojection r = 2 over a camera
// and a point, SE(3)/Sim(3) between factors, their one-slot forms). Same plan,
// same phases and the same summation orders as the generic kernel; the
// compile-time shape removes the per-column slot lookups and lets every loop
// unroll, which is what bounds the generic kernel (instruction issue).

// x (times its column scale) of one run's target into the x buffer.
template <int DD, typename TV>
__device__ __forceinline__ void load_run_x(int64_t col, int xo, const TV* __restrict__ x,
                                           const TV* __restrict__ scale, double* xbuf) {
  double v[DD];
#pragma unroll
  for (int c = 0; c < DD; ++c) v[c] = to_d(x[col + c]);
  if (scale) {
#pragma unroll
    for (int c = 0; c < DD; ++c) v[c] *= to_d(scale[col + c]);
  }
#pragma unroll
  for (int c = 0; c < DD; ++c) xbuf[xo + c] = v[c];
}

// Sum one run (len contributions of DD values, stage order) and deliver it.
template <int DD, typename TV>
__device__ __forceinline__ void deliver_run(const double* src, int len, int dest, int64_t col, int xo,
                                            const double* xbuf, double* acc, double* partials,
                                            const TV* __restrict__ x, const TV* __restrict__ scale, double damping,
                                            TV* __restrict__ y, double& dot) {
  double v[DD];
#pragma unroll
  for (int c = 0; c < DD; ++c) v[c] = 0.0;
#pragma unroll 2
  for (int e = 0; e < len; ++e, src += DD) {
#pragma unroll
    for (int c = 0; c < DD; ++c) v[c] += src[c];
  }
  if (dest == -1) {
#pragma unroll
    for (int c = 0; c < DD; ++c) {
      double xs, sc = 1.0;
      if (scale) {
        xs = to_d(x[col + c]);
        sc = to_d(scale[col + c]);
      } else {
        xs = xbuf[xo + c];
      }
      const TV out = static_cast<TV>(v[c] * sc + damping * xs);
      y[col + c] = out;
      dot += xs * to_d(out);
    }
  } else if (dest < -1) {
#pragma unroll
    for (int c = 0; c < DD; ++c) acc[-2 - dest + c] += v[c];
  } else {
#pragma unroll
    for (int c = 0; c < DD; ++c) partials[dest + c] = v[c];
  }
}

// Any dimension up to 16 (runs of a variable group of another dimension).
template <typename TV>
__device__ __forceinline__ void deliver_run_any(const double* stage, int start, int len, int d, int dest,
                                                int64_t col, int xo, const double* xbuf, double* acc,
                                                double* partials, const TV* __restrict__ x,
                                                const TV* __restrict__ scale, double damping, TV* __restrict__ y,
                                                double& dot) {
#pragma unroll 1
  for (int c0 = 0; c0 < d; c0 += 4) {
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    const double* src = stage + start + c0;
#pragma unroll 1
    for (int e = 0; e < len; ++e, src += d) {
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (c0 + c < d) v[c] += src[c];
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (c0 + c >= d) continue;
      if (dest == -1) {
        double xs, sc = 1.0;
        if (scale) {
          xs = to_d(x[col + c0 + c]);
          sc = to_d(scale[col + c0 + c]);
        } else {
          xs = xbuf[xo + c0 + c];
        }
        const TV out = static_cast<TV>(v[c] * sc + damping * xs);
        y[col + c0 + c] = out;
        dot += xs * to_d(out);
      } else if (dest < -1) {
        acc[-2 - dest + c0 + c] += v[c];
      } else {
        partials[dest + c0 + c] = v[c];
      }
    }
  }
}

// One CTA's tiles (local CTA `local` of `count` in this factor group's launch).
template <int R, int DA, int DB, typename TJ, typename TV>
__device__ __forceinline__ double tile_cta(const TileLaunch& p, int local, int count, double* tile_smem,
                                           const TV* __restrict__ x, const TV* __restrict__ scale, double damping,
                                           TV* __restrict__ y) {
  constexpr int D = DA + DB;
  constexpr bool kHold = R * D <= 54;  // larger blocks: J read twice (the second time from L1/L2)
  double* stage = tile_smem;
  double* acc = tile_smem + p.stage_doubles;
  double* xbuf = acc + p.acc_doubles;
  const int cta = p.cta_base + local;
  for (int i = threadIdx.x; i < p.acc_doubles; i += kTileThreads) acc[i] = 0.0;
  const TJ* __restrict__ jac = reinterpret_cast<const TJ*>(p.jac);
  const int t0 = p.cta_tile[cta], t1 = p.cta_tile[cta + 1];
  double dot = 0.0;
  {
    const int64_t share = ((p.ncols + count - 1) / count + 15) & ~int64_t(15);
    const int64_t c0 = (int64_t)local * share;
    const int64_t cnt = c0 < p.ncols ? ((p.ncols - c0) < share ? (p.ncols - c0) : share) : 0;
    if (threadIdx.x == kTileThreads - 1) prefetch_l2(x + c0, cnt * (int64_t)sizeof(TV));
    if (threadIdx.x == kTileThreads - 2 && scale) prefetch_l2(scale + c0, cnt * (int64_t)sizeof(TV));
  }
#pragma unroll 1
  for (int t = t0; t < t1; ++t) {
    const int64_t f0 = (int64_t)(t - p.tile_base) * p.T;
    const int nt = (int)((p.n - f0) < p.T ? (p.n - f0) : p.T);
    if (t + 1 < t1) prefetch_tile<TJ>(p, t + 1);
    const int r0 = p.tile_run[t], r1 = p.tile_run[t + 1];
    // ---- prologue: each target's x once into the x buffer
#pragma unroll 1
    for (int r = r0 + threadIdx.x; r < r1; r += kTileThreads) {
      const int d = ((__ldg(p.run_meta + r) >> 27) & 0xf) + 1;
      const int64_t col = __ldg(p.run_col + r);
      const int xo = __ldg(p.run_xoff + r);
      if (d == DA) {
        load_run_x<DA>(col, xo, x, scale, xbuf);
      } else if (DB > 0 && d == DB) {
        load_run_x<(DB > 0 ? DB : 1)>(col, xo, x, scale, xbuf);
      } else {
        for (int c = 0; c < d; ++c) {
          double v = to_d(x[col + c]);
          if (scale) v *= to_d(scale[col + c]);
          xbuf[xo + c] = v;
        }
      }
    }
    __syncthreads();
    // ---- phase A
#pragma unroll 1
    for (int i = threadIdx.x; i < nt; i += kTileThreads) {
      const int64_t f = f0 + i;
      const uint32_t wa = __ldg(p.pos + f);
      const uint32_t wb = DB > 0 ? __ldg(p.pos + p.n + f) : 0u;
      const TJ* __restrict__ jf = jac + f;
      TJ J[kHold ? R * D : 1];
      if constexpr (kHold) {
#pragma unroll
        for (int k = 0; k < R * D; ++k) J[k] = __ldg(jf + (int64_t)k * p.ld);
      }
      auto jget = [&](int r, int c) -> double {
        if constexpr (kHold) return to_d(J[r * D + c]);
        else return to_d(__ldg(jf + (int64_t)(r * D + c) * p.ld));
      };
      double xv[D];
      const double* xa = xbuf + (wa >> 16);
#pragma unroll
      for (int c = 0; c < DA; ++c) xv[c] = xa[c];
      if constexpr (DB > 0) {
        const double* xb = xbuf + (wb >> 16);
#pragma unroll
        for (int c = 0; c < DB; ++c) xv[DA + c] = xb[c];
      }
      double q[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        double a = 0.0;
#pragma unroll
        for (int c = 0; c < D; ++c) a += jget(r, c) * xv[c];
        q[r] = a;
      }
      double* sa = stage + (wa & 0xffffu);
#pragma unroll
      for (int c = 0; c < DA; ++c) {
        double v = 0.0;
#pragma unroll
        for (int r = 0; r < R; ++r) v += jget(r, c) * q[r];
        sa[c] = v;
      }
      if constexpr (DB > 0) {
        double* sb = stage + (wb & 0xffffu);
#pragma unroll
        for (int c = 0; c < DB; ++c) {
          double v = 0.0;
#pragma unroll
          for (int r = 0; r < R; ++r) v += jget(r, DA + c) * q[r];
          sb[c] = v;
        }
      }
    }
    __syncthreads();
    // ---- phase B
#pragma unroll 1
    for (int r = r0 + threadIdx.x; r < r1; r += kTileThreads) {
      const int meta = __ldg(p.run_meta + r);
      const int start = meta & 0x3fff, len = (meta >> 14) & 0x1fff, d = ((meta >> 27) & 0xf) + 1;
      const int dest = __ldg(p.run_dest + r);
      const int64_t col = __ldg(p.run_col + r);
      const int xo = dest == -1 ? __ldg(p.run_xoff + r) : 0;
      if (d == DA)
        deliver_run<DA>(stage + start, len, dest, col, xo, xbuf, acc, p.partials, x, scale, damping, y, dot);
      else if (DB > 0 && d == DB)
        deliver_run<(DB > 0 ? DB : 1)>(stage + start, len, dest, col, xo, xbuf, acc, p.partials, x, scale,
                                       damping, y, dot);
      else
        deliver_run_any(stage, start, len, d, dest, col, xo, xbuf, acc, p.partials, x, scale, damping, y, dot);
    }
    __syncthreads();
  }
  __syncthreads();
  const int j0 = p.cta_flush[cta], j1 = p.cta_flush[cta + 1];
#pragma unroll 1
  for (int j = j0 + threadIdx.x; j < j1; j += kTileThreads) {
    const int meta = __ldg(p.flush_meta + j);
    const int off = meta & 0xffff, d = ((meta >> 16) & 0xf) + 1;
    const int dest = __ldg(p.flush_dest + j);
    const int64_t col = __ldg(p.flush_col + j);
    for (int c = 0; c < d; ++c) {
      if (dest == -1) finish_col(col + c, acc[off + c], x, scale, damping, y, dot);
      else p.partials[dest + c] = acc[off + c];
    }
  }
  return dot;
}

template <int R, int DA, int DB, typename TJ, typename TV>
__global__ void __launch_bounds__(kTileThreads, (R * (DA + DB) <= 18) ? 2 : 1)
    normal_tile2_kernel(TileLaunch p, const TV* __restrict__ x, const TV* __restrict__ scale, double damping,
                        TV* __restrict__ y, double* __restrict__ dot_partials) {
  extern __shared__ __align__(16) double tile_smem[];
  __shared__ double red[kTileThreads / 32];
  asm volatile("griddepcontrol.launch_dependents;");
  const double dot = tile_cta<R, DA, DB, TJ, TV>(p, blockIdx.x, gridDim.x, tile_smem, x, scale, damping, y);
  if (dot_partials) {
    const double v = block_sum<kTileThreads>(dot, red);
    if (threadIdx.x == 0) dot_partials[p.cta_base + blockIdx.x] = v;
  }
}

// Two factor groups in one launch (a bundle adjustment's free-camera and
// fixed-camera observations; a pose graph's edges and the first pose's
// edges): CTAs [0, g1) run group p1, the rest group p2.
template <int R1, int DA1, int DB1, int R2, int DA2, int DB2, typename TJ, typename TV>
__global__ void __launch_bounds__(kTileThreads, (R1 * (DA1 + DB1) <= 18 && R2 * (DA2 + DB2) <= 18) ? 2 : 1)
    normal_tile_pair_kernel(TileLaunch p1, TileLaunch p2, int g1, const TV* __restrict__ x,
                            const TV* __restrict__ scale, double damping, TV* __restrict__ y,
                            double* __restrict__ dot_partials) {
  extern __shared__ __align__(16) double tile_smem[];
  __shared__ double red[kTileThreads / 32];
  asm volatile("griddepcontrol.launch_dependents;");
  double dot;
  if ((int)blockIdx.x < g1)
    dot = tile_cta<R1, DA1, DB1, TJ, TV>(p1, blockIdx.x, g1, tile_smem, x, scale, damping, y);
  else
    dot = tile_cta<R2, DA2, DB2, TJ, TV>(p2, blockIdx.x - g1, gridDim.x - g1, tile_smem, x, scale, damping, y);
  if (dot_partials) {
    const double v = block_sum<kTileThreads>(dot, red);
    if (threadIdx.x == 0) dot_partials[blockIdx.x] = v;
  }
}

struct TileGather {
  int32_t ntargets, lanes, nheavy, pad_;
  const int32_t* col;
  const int32_t* dim;
  const int32_t* ptr;
  const int32_t* src;
  const double* partials;
};

// One aligned lane group per target; lanes stride the target's partials and
// a fixed butterfly combines them.
template <int WM, typename TV>
__global__ void __launch_bounds__(256, 2)
    tile_gather_kernel(TileGather g, const TV* __restrict__ x, const TV* __restrict__ scale, double damping,
                       TV* __restrict__ y, double* __restrict__ dot_partials, int dot_base, PcgState* pst) {
  __shared__ double sm[8];
  constexpr int B = 4;  // partials per lane in flight
  // blocks [0, nheavy): a whole block per heavy target; then `lanes` per target
  __shared__ double hred[256 / 32][WM];
  const bool heavy = (int)blockIdx.x < g.nheavy;
  const int L = heavy ? 256 : g.lanes;
  const int64_t gt = heavy ? (int64_t)threadIdx.x
                           : (int64_t)(blockIdx.x - g.nheavy) * blockDim.x + threadIdx.x;
  const int64_t t = heavy ? (int64_t)blockIdx.x : g.nheavy + gt / L;
  const int lane = (int)(gt % L);
  const bool live = t < g.ntargets;
  // plan data and x are ready before the tile kernel ends: load them, then
  // wait for the tile kernel's partials (programmatic dependent launch)
  int d = 0, b = 0, e = 0;
  int64_t col = 0;
  if (live) {
    d = g.dim[t];
    b = g.ptr[t];
    e = g.ptr[t + 1];
    col = g.col[t];
  }
  double xs[WM], sc[WM];
#pragma unroll
  for (int c = 0; c < WM; ++c) {
    xs[c] = 0.0;
    sc[c] = 1.0;
    if (live && lane == 0 && c < d) {
      xs[c] = to_d(x[col + c]);
      if (scale) sc[c] = to_d(scale[col + c]);
    }
  }
  int off[B];
#pragma unroll
  for (int q = 0; q < B; ++q) off[q] = b + lane + q * L < e ? __ldg(g.src + b + lane + q * L) : -1;
  asm volatile("griddepcontrol.wait;" ::: "memory");
  double s[WM];
#pragma unroll
  for (int c = 0; c < WM; ++c) s[c] = 0.0;
  // B partials per lane in flight, added in list order
  for (int j = b + lane; j < e; j += B * L) {
    if (j != b + lane) {
#pragma unroll
      for (int q = 0; q < B; ++q) off[q] = j + q * L < e ? __ldg(g.src + j + q * L) : -1;
    }
    double w[B][WM];
#pragma unroll
    for (int q = 0; q < B; ++q)
#pragma unroll
      for (int c = 0; c < WM; ++c) w[q][c] = (off[q] >= 0 && c < d) ? g.partials[off[q] + c] : 0.0;
#pragma unroll
    for (int q = 0; q < B; ++q)
      if (off[q] >= 0) {
#pragma unroll
        for (int c = 0; c < WM; ++c)
          if (c < d) s[c] += w[q][c];
      }
  }
  if (heavy) {
    // fixed tree: butterfly within each warp, then the eight warp sums in order
#pragma unroll
    for (int c = 0; c < WM; ++c) s[c] = warp_sum(s[c]);
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
      for (int c = 0; c < WM; ++c) hred[threadIdx.x >> 5][c] = s[c];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
      for (int c = 0; c < WM; ++c) {
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < 256 / 32; ++w) v += hred[w][c];
        s[c] = v;
      }
    }
  } else {
#pragma unroll
    for (int c = 0; c < WM; ++c) s[c] = group_sum(s[c], L);
  }
  double dot = 0.0;
  if (live && lane == 0) {
#pragma unroll
    for (int c = 0; c < WM; ++c)
      if (c < d) {
        const TV out = static_cast<TV>(s[c] * sc[c] + damping * xs[c]);
        y[col + c] = out;
        dot += xs[c] * to_d(out);
      }
  }
  if (dot_partials) {
    const double v = block_sum<256>(dot, sm);
    if (threadIdx.x == 0) dot_partials[dot_base + blockIdx.x] = v;
    if (pst) pcg_operator_epilogue<256>(pst, dot_partials, gridDim.x, sm, dot_base + (int)gridDim.x);
  }
}

static int tile_heavy_blocks(const tls_normal_tiles* T) { return T->nheavy; }

static int tile_gather_blocks(const tls_normal_tiles* T) {
  const int64_t threads = (int64_t)(T->ntargets - T->nheavy) * T->gather_lanes;
  const int64_t b = tile_heavy_blocks(T) + (threads + 255) / 256;
  return b < 1 ? 1 : (int)b;
}

template <int RM, int DM, int U, int SMX, typename TJ, typename TV>
static int launch_tile(const TileLaunch& p, int grid, const TV* x, const TV* scale, double damping, TV* y,
                       double* dot_partials, cudaStream_t st) {
  const int smem = (p.stage_doubles + p.acc_doubles + p.xbuf_doubles) * (int)sizeof(double);
  // the dynamic shared-memory limit is a per-device function attribute: set
  // once per device and instantiation
  static std::atomic<uint64_t> configured{0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return tls_set_error(TLS_ERR_CUDA, "no current CUDA device (or index beyond 63)");
  if (!(configured.load() & (1ull << dev))) {
    cudaError_t e = cudaFuncSetAttribute(normal_tile_kernel<RM, DM, U, SMX, TJ, TV>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmemLimit);
    if (e != cudaSuccess) return tls_set_cuda_error(e);
    configured.fetch_or(1ull << dev);
  }
  normal_tile_kernel<RM, DM, U, SMX, TJ, TV><<<grid, kTileThreads, smem, st>>>(p, x, scale, damping, y, dot_partials);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}

template <int R, int DA, int DB, typename TJ, typename TV>
static int launch_tile2(const TileLaunch& p, int grid, const TV* x, const TV* scale, double damping, TV* y,
                        double* dot_partials, cudaStream_t st) {
  const int smem = (p.stage_doubles + p.acc_doubles + p.xbuf_doubles) * (int)sizeof(double);
  static std::atomic<uint64_t> configured{0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return tls_set_error(TLS_ERR_CUDA, "no current CUDA device (or index beyond 63)");
  if (!(configured.load() & (1ull << dev))) {
    cudaError_t e = cudaFuncSetAttribute(normal_tile2_kernel<R, DA, DB, TJ, TV>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmemLimit);
    if (e != cudaSuccess) return tls_set_cuda_error(e);
    configured.fetch_or(1ull << dev);
  }
  normal_tile2_kernel<R, DA, DB, TJ, TV><<<grid, kTileThreads, smem, st>>>(p, x, scale, damping, y, dot_partials);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}

template <int R1, int DA1, int DB1, int R2, int DA2, int DB2, typename TJ, typename TV>
static int launch_tile_pair(const TileLaunch& p1, const TileLaunch& p2, int g1, int g2, const TV* x, const TV* scale,
                            double damping, TV* y, double* dot_partials, cudaStream_t st) {
  const int smem = (p1.stage_doubles + p1.acc_doubles + p1.xbuf_doubles) * (int)sizeof(double);
  static std::atomic<uint64_t> configured{0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return tls_set_error(TLS_ERR_CUDA, "no current CUDA device (or index beyond 63)");
  if (!(configured.load() & (1ull << dev))) {
    cudaError_t e = cudaFuncSetAttribute(normal_tile_pair_kernel<R1, DA1, DB1, R2, DA2, DB2, TJ, TV>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmemLimit);
    if (e != cudaSuccess) return tls_set_cuda_error(e);
    configured.fetch_or(1ull << dev);
  }
  normal_tile_pair_kernel<R1, DA1, DB1, R2, DA2, DB2, TJ, TV>
      <<<g1 + g2, kTileThreads, smem, st>>>(p1, p2, g1, x, scale, damping, y, dot_partials);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}

// Two factor groups of known shapes in one launch; returns -1 when the pair
// has no combined kernel.
template <typename TJ, typename TV>
static int dispatch_tile_pair(const TileLaunch& p1, const TileLaunch& p2, int g1, int g2, const TV* x,
                              const TV* scale, double damping, TV* y, double* dot_partials, cudaStream_t st) {
  auto is = [](const TileLaunch& p, int r, int da, int db) {
    return p.R == r && p.S == (db > 0 ? 2 : 1) && p.slot_dim[0] == da && (db == 0 || p.slot_dim[1] == db);
  };
#define TLS_PAIR(R1, A1, B1, R2, A2, B2)                                                                    \
  if (is(p1, R1, A1, B1) && is(p2, R2, A2, B2))                                                             \
    return launch_tile_pair<R1, A1, B1, R2, A2, B2, TJ, TV>(p1, p2, g1, g2, x, scale, damping, y, dot_partials, st);
  TLS_PAIR(2, 6, 3, 2, 3, 0)
  TLS_PAIR(6, 6, 6, 6, 6, 0)
  TLS_PAIR(7, 7, 7, 7, 7, 0)
#undef TLS_PAIR
  return -1;
}

template <typename TJ, typename TV>
static int dispatch_tile(const TileLaunch& p, int grid, const TV* x, const TV* scale, double damping, TV* y,
                         double* dot_partials, cudaStream_t st) {
  // shapes with a specialised kernel (slot dims from the first two slots)
  const int da = p.S >= 1 ? p.slot_dim[0] : 0, db = p.S >= 2 ? p.slot_dim[1] : 0;
#define TLS_TILE2(R_, DA_, DB_)                                                                     \
  if (p.R == R_ && p.S == (DB_ > 0 ? 2 : 1) && da == DA_ && db == DB_)                              \
    return launch_tile2<R_, DA_, DB_, TJ, TV>(p, grid, x, scale, damping, y, dot_partials, st);
  TLS_TILE2(2, 6, 3)
  TLS_TILE2(2, 3, 0)
  TLS_TILE2(2, 6, 0)
  TLS_TILE2(6, 6, 6)
  TLS_TILE2(6, 6, 0)
  TLS_TILE2(7, 7, 7)
  TLS_TILE2(7, 7, 0)
#undef TLS_TILE2
#define TLS_TILE(RM, DM, U)                                                                            \
  if (p.R <= RM && p.D <= DM)                                                                          \
    return p.S <= 2 ? launch_tile<RM, DM, U, 2, TJ, TV>(p, grid, x, scale, damping, y, dot_partials, st) \
                    : launch_tile<RM, DM, U, TLS_MAX_SLOTS, TJ, TV>(p, grid, x, scale, damping, y, dot_partials, st);
  TLS_TILE(1, 4, 1)
  TLS_TILE(2, 4, 1)
  TLS_TILE(3, 4, 1)
  TLS_TILE(2, 9, 1)
  TLS_TILE(3, 6, 1)
  TLS_TILE(3, 9, 1)
  TLS_TILE(4, 8, 1)
  TLS_TILE(6, 12, 1)
  TLS_TILE(7, 14, 1)
  TLS_TILE(8, 16, 1)
#undef TLS_TILE
  return tls_set_error(TLS_ERR_UNSUPPORTED, "factor shape beyond r <= 8, D <= 16");
}

static int check_tiles(const tls_normal_args* a) {
  const tls_normal_tiles* T = a->tiles;
  if (T->ncta < 0 || T->ntiles < 0 || T->ntargets < 0 || T->stage_doubles < 0 || T->acc_doubles < 0 ||
      T->stage_doubles > 16384 || T->acc_doubles > 65536)
    return tls_set_error(TLS_ERR_INVALID, "tile plan: bad sizes");
  if (T->xbuf_doubles < 0 || T->xbuf_doubles > 16384 ||
      (int64_t)(T->stage_doubles + T->acc_doubles + T->xbuf_doubles) * 8 > kTileSmemLimit)
    return tls_set_error(TLS_ERR_INVALID, "tile plan: stage, accumulator and x buffer exceed 200 KB of shared memory");
  if (T->gather_lanes < 1 || T->gather_lanes > 32 || (T->gather_lanes & (T->gather_lanes - 1)))
    return tls_set_error(TLS_ERR_INVALID, "tile plan: gather lanes must be a power of two <= 32");
  if (T->nheavy < 0 || T->nheavy > T->ntargets)
    return tls_set_error(TLS_ERR_INVALID, "tile plan: heavy targets beyond the target count");
  if (T->cta_base[0] != 0 || T->cta_base[a->nfactor_groups] != T->ncta)
    return tls_set_error(TLS_ERR_INVALID, "tile plan: CTA ranges do not cover the factor groups");
  for (int k = 0; k < a->nfactor_groups; ++k) {
    const int ncta = T->cta_base[k + 1] - T->cta_base[k];
    if (ncta < 0 || (a->fg[k].count > 0 && (ncta == 0 || T->tile_factors[k] < 1 || !T->pos[k])))
      return tls_set_error(TLS_ERR_INVALID, "tile plan does not match the factor groups");
  }
  int wmax = 1;
  for (int i = 0; i < a->nvar_groups; ++i) wmax = a->vg[i].dim > wmax ? a->vg[i].dim : wmax;
  if (wmax > 16) return tls_set_error(TLS_ERR_UNSUPPORTED, "variable dim > 16");
  return TLS_OK;
}

template <typename TV>
static int launch_tile_gather(const tls_normal_args* a, const TV* x, const TV* scale, TV* y, double* dot_partials,
                              PcgState* pst, cudaStream_t st) {
  const tls_normal_tiles* T = a->tiles;
  TileGather g{T->ntargets, T->gather_lanes, T->nheavy, 0, T->target_col, T->target_dim,
               T->target_ptr, T->target_src, T->partials};
  const int blocks = tile_gather_blocks(T);
  int wmax = 1;
  for (int i = 0; i < a->nvar_groups; ++i) wmax = a->vg[i].dim > wmax ? a->vg[i].dim : wmax;
  // programmatic dependent launch: the gather's blocks start (and load their
  // plan data) as the tile kernel's CTAs retire; griddepcontrol.wait orders
  // their reads of the partials after the whole tile kernel
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const int nbase = T->ncta;
  const double damping = a->damping;
#define TLS_TG(WM)                                                                                        \
  if (wmax <= WM) {                                                                                       \
    cudaError_t err = cudaLaunchKernelEx(&cfg, tile_gather_kernel<WM, TV>, g, x, scale, damping, y,      \
                                         dot_partials, nbase, pst);                                       \
    if (err != cudaSuccess) return tls_set_cuda_error(err);                                             \
    TLS_CHECK_LAUNCH();                                                                                   \
    return TLS_OK;                                                                                        \
  }
  TLS_TG(3)
  TLS_TG(6)
  TLS_TG(8)
  TLS_TG(16)
#undef TLS_TG
  return tls_set_error(TLS_ERR_UNSUPPORTED, "variable dim > 16");
}

}  // namespace tls

using namespace tls;

int tls_normal_tiles_blocks(const tls_normal_args* a) { return a->tiles->ncta + tile_gather_blocks(a->tiles); }

// y = diag(s) J^T J diag(s) x + damping x through the tile plan. Dot partials
// (when given): [0, ncta) from the tile CTAs, then one per gather block; the
// gather kernel's last block finishes the PCG curvature when pcg_state is set.
int tls_normal_tiles_apply(const tls_normal_args* a, const void* x, void* y, double* dot_partials,
                           int* nblocks, void* pcg_state, cudaStream_t st) {
  int rc = check_tiles(a);
  if (rc) return rc;
  const tls_normal_tiles* T = a->tiles;
  int64_t ncols = 0;
  for (int i = 0; i < a->nvar_groups; ++i) {
    const int64_t e = a->vg[i].offset + (int64_t)a->vg[i].count * a->vg[i].dim;
    ncols = e > ncols ? e : ncols;
  }
  TileLaunch L[TLS_MAX_FACTOR_GROUPS];
  for (int k = 0; k < a->nfactor_groups; ++k) {
    const tls_factor_group& fg = a->fg[k];
    if (fg.jac_dtype != TLS_F32 && a->vec_dtype != TLS_F64)
      return tls_set_error(TLS_ERR_UNSUPPORTED, "float64 Jacobian with float32 vectors");
    if (k > 0 && fg.jac_dtype != a->fg[0].jac_dtype)
      return tls_set_error(TLS_ERR_UNSUPPORTED, "factor groups with different Jacobian dtypes");
    TileLaunch& p = L[k];
    p = TileLaunch{};
    p.n = fg.count;
    p.R = fg.rdim;
    p.D = fg.total_dim;
    p.T = T->tile_factors[k];
    p.S = fg.nslots;
    p.ncols = ncols;
    for (int c = 0; c < 32; ++c) p.col_slot[c] = -1;
    for (int s = 0; s < fg.nslots; ++s) {
      p.slot_col[s] = fg.slot_col[s];
      p.slot_dim[s] = fg.slot_dim[s];
      p.slot_off[s] = a->vg[fg.slot_group[s]].offset;
      p.index[s] = fg.index[s];
      for (int j = 0; j < fg.slot_dim[s]; ++j) p.col_slot[fg.slot_col[s] + j] = (int8_t)s;
    }
    p.jac = fg.jac;
    p.ld = fg.jac_stride ? fg.jac_stride : fg.count;
    p.pos = T->pos[k];
    p.tile_base = T->tile_base[k];
    p.cta_base = T->cta_base[k];
    p.stage_doubles = T->stage_doubles;
    p.acc_doubles = T->acc_doubles;
    p.xbuf_doubles = T->xbuf_doubles;
    p.cta_tile = T->cta_tile;
    p.tile_run = T->tile_run;
    p.run_col = T->run_col;
    p.run_meta = T->run_meta;
    p.run_dest = T->run_dest;
    p.run_xoff = T->run_xoff;
    p.cta_flush = T->cta_flush;
    p.flush_col = T->flush_col;
    p.flush_meta = T->flush_meta;
    p.flush_dest = T->flush_dest;
    p.partials = T->partials;
  }
  const bool f64 = a->vec_dtype == TLS_F64, j64 = a->nfactor_groups > 0 && a->fg[0].jac_dtype == TLS_F64;
  int k = 0;
  if (a->nfactor_groups == 2) {
    // both groups in one launch when a combined kernel exists
    const int g1 = T->cta_base[1] - T->cta_base[0], g2 = T->cta_base[2] - T->cta_base[1];
    if (g1 > 0 && g2 > 0) {
      if (f64)
        rc = j64 ? dispatch_tile_pair<double, double>(L[0], L[1], g1, g2, (const double*)x, (const double*)a->scale,
                                                      a->damping, (double*)y, dot_partials, st)
                 : dispatch_tile_pair<float, double>(L[0], L[1], g1, g2, (const double*)x, (const double*)a->scale,
                                                     a->damping, (double*)y, dot_partials, st);
      else
        rc = dispatch_tile_pair<float, float>(L[0], L[1], g1, g2, (const float*)x, (const float*)a->scale,
                                              a->damping, (float*)y, dot_partials, st);
      if (rc > 0) return rc;
      if (rc == 0) k = 2;
    }
  }
  for (; k < a->nfactor_groups; ++k) {
    const int grid = T->cta_base[k + 1] - T->cta_base[k];
    if (grid == 0) continue;
    if (f64)
      rc = j64 ? dispatch_tile<double, double>(L[k], grid, (const double*)x, (const double*)a->scale, a->damping,
                                               (double*)y, dot_partials, st)
               : dispatch_tile<float, double>(L[k], grid, (const double*)x, (const double*)a->scale, a->damping,
                                              (double*)y, dot_partials, st);
    else
      rc = dispatch_tile<float, float>(L[k], grid, (const float*)x, (const float*)a->scale, a->damping, (float*)y,
                                       dot_partials, st);
    if (rc) return rc;
  }
  PcgState* pst = reinterpret_cast<PcgState*>(pcg_state);
  rc = a->vec_dtype == TLS_F64
           ? launch_tile_gather<double>(a, (const double*)x, (const double*)a->scale, (double*)y, dot_partials, pst, st)
           : launch_tile_gather<float>(a, (const float*)x, (const float*)a->scale, (float*)y, dot_partials, pst, st);
  if (rc) return rc;
  if (nblocks) *nblocks = tls_normal_tiles_blocks(a);
  return TLS_OK;
}

// ---------------------------------------------------------------- tile-order copy of J
namespace tls {
template <typename T>
__global__ void __launch_bounds__(256) permute_columns_kernel(const T* __restrict__ src, T* __restrict__ dst,
                                                              int64_t ncols, int64_t ld, const int32_t* __restrict__ perm) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= ncols) return;
  const int64_t r = blockIdx.y;
  dst[r * ncols + p] = src[r * ld + __ldg(perm + p)];
}
}  // namespace tls

// dst[r][p] = src[r][perm[p]] for r < rows, p < ncols: the columns of an SoA
// Jacobian [rows][ld] in a tile plan's factor order (coalesced stores).
extern "C" int tls_permute_columns(const void* src, void* dst, int32_t dtype, int64_t rows, int64_t ncols,
                                   int64_t ld_src, const int32_t* perm, tls_stream_t stream) {
  if (rows < 0 || ncols < 0 || ld_src < ncols || rows > 65535 || (dtype != TLS_F32 && dtype != TLS_F64))
    return tls_set_error(TLS_ERR_INVALID, "tls_permute_columns: bad shape or dtype");
  if (rows == 0 || ncols == 0) return TLS_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const dim3 grid((unsigned)((ncols + 255) / 256), (unsigned)rows);
  if (dtype == TLS_F32)
    permute_columns_kernel<float><<<grid, 256, 0, st>>>((const float*)src, (float*)dst, ncols, ld_src, perm);
  else
    permute_columns_kernel<double><<<grid, 256, 0, st>>>((const double*)src, (double*)dst, ncols, ld_src, perm);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}

