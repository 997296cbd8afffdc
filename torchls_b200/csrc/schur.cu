// Schur complement of one eliminated group (torchls schur.py:192-397).
//
// Edges (retained i, eliminated p) live in chunks of whole eliminated
// variables. Each chunk owns a fixed-size, 16-byte aligned slab: W as
// [dr*de][cap] plus an int32 metadata block. The reduced matvec
// S x = (s U s + lambda I) x - W (W^T x) never forms S:
//
//   chunk kernel (persistent grid, 2 CTAs/SM). Thread 0 streams chunk slabs
//   into shared memory with 1-D bulk copies (cp.async.bulk, TMA) completing
//   on an mbarrier; two stages, so chunk c+grid loads while chunk c computes.
//     phase 1   t_e = W_e^T x_i                 (per edge, into shared memory;
//               each thread keeps its edges' W in registers for phase 2)
//     phase 1.5 y_p = sum_{e in p} t_e          (per eliminated variable, fixed order,
//               written over t of the variable's first listed edge)
//     phase 2   u_e = W_e y_p; each thread takes cap/256 consecutive edges,
//               sums runs of equal retained variable sequentially, then a
//               warp-segmented inclusive scan joins runs across lanes (runs
//               never cross one warp's window); the run's tail stores the
//               run partial, retained-major.
//   Products and sums are float64 (W stored as float32 or float64). x is
//   staged in shared memory when it fits next to the two slab stages.
//   gather kernel (one block per retained variable) sums its contiguous run
//   partials in a fixed order and adds the diagonal term; its last block
//   finalises the PCG curvature.
//
// W is read from HBM exactly once per matvec. Every sum follows a fixed order:
// results are bitwise reproducible. Every mbarrier wait is bounded: on
// timeout the kernel raises a.err and keeps going (it never hangs).
#include <stdint.h>

#include "blocks.cuh"
#include "common.cuh"
#include "pcg_device.cuh"
#include "pcg_state.cuh"

namespace tls {

constexpr int kChunkThreads = 256;
// Largest dynamic shared memory of the vector-CTA kernel: two CTAs (with
// their static shared memory and the per-CTA reservation) still fit an SM.
constexpr int64_t kVectorSmemMax = 110 * 1024;
constexpr int kMetaHead = 4;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// 1-D bulk copy global -> this CTA's shared memory, completing on `bar`.
// Both addresses are 16-byte aligned and `bytes` is a multiple of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Default limit of every bounded wait: 2^31 SM cycles, about one second.
constexpr long long kWaitCycles = 1LL << 31;

// The wait limit of one launch: a->wait_cycles when positive, else the default.
__host__ __device__ __forceinline__ long long wait_limit(const tls_schur_args& a) {
  return a.wait_cycles > 0 ? a.wait_cycles : kWaitCycles;
}

// Bounded wait on a bulk-copy barrier: gives up after `limit` SM cycles, flags
// the error and returns false instead of hanging. A caller that sees false
// must not read the stage (its copy may not have landed).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int32_t* err,
                                                  long long limit = kWaitCycles) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit) {
      if (err) atomicExch(err, 1);
      return false;
    }
  }
  return true;
}

// Wait (with the default limit, whatever the launch's limit) for the bulk
// copies of consumptions [from, to) that are still in flight into this CTA's
// shared memory, so that none lands after the CTA has left.
__device__ __forceinline__ void mbar_drain(uint64_t* bar, int from, int to, int32_t* err) {
  for (int k = from; k < to; ++k) mbar_wait_bounded(&bar[k & 1], (k >> 1) & 1, err);
}

template <int DR, int DE, int CAP, typename TW, typename TA>
struct SlabShape {
  static constexpr int kWBytes = DR * DE * CAP * (int)sizeof(TW);
  static constexpr int kMetaInts = 5 * CAP + 8;
  static constexpr int kMetaBytes = kMetaInts * 4;
  static constexpr int kStageBytes = kWBytes + kMetaBytes;
  static constexpr int kTBytes = CAP * 4 * (int)sizeof(TA);  // [CAP][4] per-edge / per-variable 3-vectors
  static constexpr int kBaseSmem = 2 * kStageBytes + kTBytes;
  static constexpr int kEpt = CAP / kChunkThreads;  // consecutive edges per thread
  static_assert(kWBytes % 16 == 0 && kMetaBytes % 16 == 0, "slabs must be 16-byte multiples");
  static_assert(kEpt == 1 || kEpt == 2 || kEpt == 4, "edges per thread");
  static_assert(DE <= 4, "eliminated blocks up to 4 wide");
};

// EPT consecutive shared-memory values starting at p (p aligned to EPT values).
template <int EPT, typename T>
__device__ __forceinline__ void lds_vec(const T* p, T (&v)[EPT]) {
  if constexpr (EPT == 1) {
    v[0] = p[0];
  } else if constexpr (EPT == 2 && sizeof(T) == 4) {
    const float2 q = *reinterpret_cast<const float2*>(p);
    v[0] = q.x, v[1] = q.y;
  } else if constexpr (EPT == 2 && sizeof(T) == 8) {
    const double2 q = *reinterpret_cast<const double2*>(p);
    v[0] = q.x, v[1] = q.y;
  } else if constexpr (EPT == 4 && sizeof(T) == 4) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
  } else {
#pragma unroll
    for (int j = 0; j < EPT; ++j) v[j] = p[j];
  }
}

template <typename TA>
__device__ __forceinline__ void lds4(const TA* p, TA (&v)[4]) {
  if constexpr (sizeof(TA) == 4) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
  } else {
    const double2 q0 = reinterpret_cast<const double2*>(p)[0], q1 = reinterpret_cast<const double2*>(p)[1];
    v[0] = q0.x, v[1] = q0.y, v[2] = q1.x, v[3] = q1.y;
  }
}

template <typename TA>
__device__ __forceinline__ void sts4(TA* p, const TA (&v)[4]) {
  if constexpr (sizeof(TA) == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
    reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
  }
}

// The first N (the eliminated block width) of four values held at p; the
// rest of v is zero. float64 rows of four start on 32-byte boundaries.
template <int N, typename TA>
__device__ __forceinline__ void ldsn(const TA* p, TA (&v)[4]) {
  if constexpr (sizeof(TA) == 8 && N >= 2) {
    const double2 q0 = reinterpret_cast<const double2*>(p)[0];
    v[0] = q0.x, v[1] = q0.y;
    if constexpr (N == 4) {
      const double2 q1 = reinterpret_cast<const double2*>(p)[1];
      v[2] = q1.x, v[3] = q1.y;
    } else if constexpr (N == 3) {
      v[2] = p[2], v[3] = TA(0);
    } else {
      v[2] = v[3] = TA(0);
    }
  } else if constexpr (N == 1) {
    v[0] = p[0], v[1] = v[2] = v[3] = TA(0);
  } else {
    lds4(p, v);
  }
}

template <int N, typename TA>
__device__ __forceinline__ void stsn(TA* p, const TA (&v)[4]) {
  if constexpr (sizeof(TA) == 8 && N >= 2) {
    reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
    if constexpr (N == 4) reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
    else if constexpr (N == 3) p[2] = v[2];
  } else if constexpr (N == 1) {
    p[0] = v[0];
  } else {
    sts4(p, v);
  }
}

// Compute one chunk held in shared memory (W slab `Ws`, metadata `Ms`):
// MODE 0: S x partials (phase 1 from x); MODE 1: reduced rhs (y_p = a.ybuf[p]).
// TA: arithmetic type of the per-edge products and of the run sums (float64:
// S = U - W W^T cancels heavily, and float32 products stalled CG); W is
// stored as TW. Per-variable sums y_p and every sum across runs are float64.
// XS: x was staged in shared memory (as TA). COH: x is rewritten by this
// kernel between matvecs (persistent loop): plain coherent loads after the
// grid barrier instead of the read-only (.nc) path.
template <int DR, int DE, int CAP, int MODE, typename TW, typename TA, bool XS, bool COH>
__device__ __forceinline__ void chunk_compute(const tls_schur_args& a, const double* __restrict__ x, const TA* x_s,
                                              TA* t_s, const TW* Ws, const int32_t* Ms, int c) {
  constexpr int EPT = CAP / kChunkThreads;
  const int tid = threadIdx.x, lane = tid & 31;
  const int ne = Ms[0], np = Ms[1];
  const int32_t* er = Ms + kMetaHead;
  const uint32_t* meta = reinterpret_cast<const uint32_t*>(Ms + kMetaHead + CAP);
  const int32_t* tpos = Ms + kMetaHead + 2 * CAP;
  const int32_t* pp = Ms + kMetaHead + 3 * CAP;
  const int32_t* pe = Ms + 2 * kMetaHead + 4 * CAP;
  const int le0 = tid * EPT;  // this thread's first edge
  // This thread's W entries: read from the stage once and kept in registers
  // for phases 1 and 2 (MODE 1 reads them in phase 2). Entries past ne are
  // the slab's padding and are never used.
  TW w[DR * DE][EPT];
  if constexpr (MODE == 0) {
#pragma unroll
    for (int kb = 0; kb < DR * DE; ++kb) lds_vec<EPT>(Ws + kb * CAP + le0, w[kb]);
  }
  // ---- phase 1: t_e = W_e^T x_i
  if constexpr (MODE == 0) {
    if (le0 < ne) {
#pragma unroll
      for (int j = 0; j < EPT; ++j) {
        if (le0 + j < ne) {
          const int i = er[le0 + j];
          TA xr[DR];
          if (!XS && DR % 2 == 0 && (reinterpret_cast<uintptr_t>(x) & 15) == 0) {
            // x rows of even width start on 16-byte boundaries when x does:
            // pairs per load (COH: plain loads, x is rewritten by this kernel;
            // see gather_one)
            const double2* xp = reinterpret_cast<const double2*>(x + (int64_t)i * DR);
#pragma unroll
            for (int k = 0; k < DR; k += 2) {
              const double2 v2 = COH ? xp[k / 2] : __ldg(xp + k / 2);
              xr[k] = static_cast<TA>(v2.x), xr[k + 1] = static_cast<TA>(v2.y);
            }
          } else {
#pragma unroll
            for (int k = 0; k < DR; ++k) {
              if constexpr (XS) xr[k] = x_s[i * DR + k];
              else if constexpr (COH) xr[k] = static_cast<TA>(x[(int64_t)i * DR + k]);
              else xr[k] = static_cast<TA>(__ldg(x + (int64_t)i * DR + k));
            }
          }
          TA t[4] = {TA(0), TA(0), TA(0), TA(0)};
#pragma unroll
          for (int b = 0; b < DE; ++b) {
#pragma unroll
            for (int k = 0; k < DR; ++k) t[b] = fma(static_cast<TA>(w[k * DE + b][j]), xr[k], t[b]);
          }
          stsn<DE>(t_s + (le0 + j) * 4, t);
        }
      }
    }
    __syncthreads();
  }
  // ---- phase 1.5: y_p per eliminated variable (float64 sum over its edges),
  // written over t of the variable's first edge: only this thread reads the
  // t entries of its variable's edges, so no barrier separates the sum from
  // the store (the metadata word of every edge points phase 2 at that entry)
  constexpr int PPT = CAP / kChunkThreads;
#pragma unroll
  for (int q = 0; q < PPT; ++q) {
    const int pl = tid + q * kChunkThreads;
    double yreg[DE];
#pragma unroll
    for (int b = 0; b < DE; ++b) yreg[b] = 0.0;
    if (pl < np) {
      const int slot = pe[pp[pl]];
      if constexpr (MODE == 0) {
        // four edges per round: independent shared-memory loads, fixed-order sums
        const int jb = pp[pl], je = pp[pl + 1];
        for (int j = jb; j < je; j += 4) {
          TA t[4][4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (j + u < je) ldsn<DE>(t_s + pe[j + u] * 4, t[u]);
            else t[u][0] = t[u][1] = t[u][2] = t[u][3] = TA(0);
          }
#pragma unroll
          for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int b = 0; b < DE; ++b)
              if (j + u < je) yreg[b] += static_cast<double>(t[u][b]);
        }
      } else {
        const int64_t p = __ldg(a.slab_e + (int64_t)c * CAP + slot);
#pragma unroll
        for (int b = 0; b < DE; ++b) yreg[b] = a.ybuf[p * DE + b];
      }
      TA y[4] = {TA(0), TA(0), TA(0), TA(0)};
#pragma unroll
      for (int b = 0; b < DE; ++b) y[b] = static_cast<TA>(yreg[b]);
      stsn<DE>(t_s + slot * 4, y);
    }
  }
  __syncthreads();
  // ---- phase 2: u_e = W_e y_p; segmented sums over runs of equal retained
  // variable (runs never cross a window of 32 * EPT edges): sequential within
  // the thread, then a warp-segmented inclusive scan of the carries over as
  // many steps as the warp's longest run needs.
  {
    TA v[EPT][DR];
    int head[EPT];
    bool tail[EPT];
    if constexpr (MODE == 1) {
#pragma unroll
      for (int kb = 0; kb < DR * DE; ++kb) lds_vec<EPT>(Ws + kb * CAP + le0, w[kb]);
    }
#pragma unroll
    for (int j = 0; j < EPT; ++j) {
      const int le = le0 + j;
      const int pos = lane * EPT + j;  // position inside the 32*EPT-edge window
      const bool valid = le < ne;
      const uint32_t m = valid ? meta[le] : 0u;
      head[j] = valid ? (int)((m >> 16) & 63u) : pos;
      tail[j] = valid && ((m >> 22) & 1u);
      TA y[4] = {TA(0), TA(0), TA(0), TA(0)};
      if (valid) ldsn<DE>(t_s + (int)(m & 0xFFFFu) * 4, y);  // y_p at its variable's first edge
      const bool cont = j > 0 && head[j] < pos;  // same run as edge j-1
#pragma unroll
      for (int k = 0; k < DR; ++k) {
        TA u = TA(0);
#pragma unroll
        for (int b = 0; b < DE; ++b) u = fma(static_cast<TA>(w[k * DE + b][j]), y[b], u);
        v[j][k] = cont ? v[j > 0 ? j - 1 : 0][k] + u : u;
      }
    }
    const int hl = head[EPT - 1] / EPT;           // lane holding the start of this thread's last run
    const bool from_left = head[0] < lane * EPT;  // this thread's first run began in an earlier lane
    // lanes any run spans backwards; offsets 1, 2, 4, ... <= span cover it
    const unsigned span = __reduce_max_sync(0xffffffffu, (unsigned)(lane - hl));
    // all DR components advance together, so the shuffle latencies overlap
    TA cval[DR];
#pragma unroll
    for (int k = 0; k < DR; ++k) cval[k] = v[EPT - 1][k];
    for (unsigned off = 1; off <= span; off <<= 1) {
      const bool take = lane - (int)off >= hl;
      TA o[DR];
#pragma unroll
      for (int k = 0; k < DR; ++k) o[k] = __shfl_up_sync(0xffffffffu, cval[k], off);
#pragma unroll
      for (int k = 0; k < DR; ++k)
        if (take) cval[k] += o[k];
    }
    TA prev[DR];
#pragma unroll
    for (int k = 0; k < DR; ++k) prev[k] = __shfl_up_sync(0xffffffffu, cval[k], 1);
#pragma unroll
    for (int j = 0; j < EPT; ++j) {
      if (tail[j]) {
        // only the thread's first run can have begun in an earlier lane
        const bool join = from_left && head[j] == head[0];
        TA* dst = reinterpret_cast<TA*>(a.run_partial) + (int64_t)tpos[le0 + j] * DR;
        bool paired = false;
        if constexpr (sizeof(TA) == 8 && DR % 2 == 0) {
          // float64 partials of even width start on 16-byte boundaries when
          // the buffer does: pairs per store
          paired = (reinterpret_cast<uintptr_t>(a.run_partial) & 15) == 0;
          if (paired) {
#pragma unroll
            for (int k = 0; k < DR; k += 2)
              reinterpret_cast<double2*>(dst)[k / 2] = join ? make_double2(v[j][k] + prev[k], v[j][k + 1] + prev[k + 1])
                                                            : make_double2(v[j][k], v[j][k + 1]);
          }
        }
        if (!paired) {
#pragma unroll
          for (int k = 0; k < DR; ++k) dst[k] = join ? v[j][k] + prev[k] : v[j][k];
        }
      }
    }
  }
  // No barrier here: a caller passes a block barrier before the next chunk's
  // phase 1 rewrites t_s and before its thread 0 refills this stage.
}

// MODE 0: S x partials; MODE 1: reduced rhs. Persistent over chunks: thread 0
// streams chunk slabs with 1-D bulk copies into two shared-memory stages.
template <int DR, int DE, int CAP, int MODE, typename TW, typename TA, bool XS>
__global__ void __launch_bounds__(kChunkThreads, 2) schur_chunk_kernel(tls_schur_args a, const double* __restrict__ x) {
  using S = SlabShape<DR, DE, CAP, TW, TA>;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  TA* t_s = reinterpret_cast<TA*>(smem + 2 * S::kStageBytes);  // [CAP][4]: t_e, then y_p
  TA* x_s = reinterpret_cast<TA*>(smem + S::kBaseSmem);         // [nretained*DR] when XS
  const int tid = threadIdx.x;
  const unsigned char* wsrc = reinterpret_cast<const unsigned char*>(a.w);
  const unsigned char* msrc = reinterpret_cast<const unsigned char*>(a.meta);
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](int c, int stg) {
    unsigned char* base = smem + stg * S::kStageBytes;
    fence_proxy_async();
    mbar_expect_tx(&bar[stg], S::kStageBytes);
    bulk_load(base, wsrc + (size_t)c * S::kWBytes, S::kWBytes, &bar[stg]);
    bulk_load(base + S::kWBytes, msrc + (size_t)c * S::kMetaBytes, S::kMetaBytes, &bar[stg]);
  };
  if (tid == 0 && (int)blockIdx.x < a.nchunks) issue(blockIdx.x, 0);
  if constexpr (XS && MODE == 0) {
    const int nx = a.nretained * DR;
    for (int j = tid; j < nx; j += kChunkThreads) x_s[j] = static_cast<TA>(__ldg(x + j));
    __syncthreads();
  }
  const long long lim = wait_limit(a);
  int it = 0;
  for (int c = blockIdx.x; c < a.nchunks; c += gridDim.x, ++it) {
    const int stg = it & 1;
    const bool next = c + (int)gridDim.x < a.nchunks;
    const bool ok = mbar_wait_bounded(&bar[stg], (it >> 1) & 1, a.err, lim);
    // the block barrier also ends the previous chunk's reads of the other stage and of t_s
    if (__syncthreads_or(!ok)) {  // this stage may be incomplete: leave without reading it
      if (tid == 0) mbar_drain(bar, it, it + 1, a.err);
      return;
    }
    if (tid == 0 && next) issue(c + gridDim.x, stg ^ 1);
    const TW* Ws = reinterpret_cast<const TW*>(smem + stg * S::kStageBytes);
    const int32_t* Ms = reinterpret_cast<const int32_t*>(smem + stg * S::kStageBytes + S::kWBytes);
    chunk_compute<DR, DE, CAP, MODE, TW, TA, XS, false>(a, x, x_s, t_s, Ws, Ms, c);
  }
}

// Sum retained variable i's contiguous run partials (float64, fixed order) and
// finish its rows, with 256 threads:
// MODE 0: out = s U s x + lambda x - sum; returns x_i . out_i to thread 0
// MODE 1: out = b_retained - sum
// COH: x and the run partials are rewritten by this kernel (persistent loop):
// plain loads, not the read-only (.nc) path. They observe this step's values:
// the writers release them through a GPU-scope fence and an atomic before the
// grid barrier, and this CTA acquires them (a fence after the barrier wait,
// then a block barrier) before it reads.
// What gather_one needs before the run partials: retained variable i's run
// range and (MODE 0, threads < DR*DR) its term of s U s x. None of it depends
// on this step's partials, so a persistent kernel loads it ahead of the
// barrier that precedes the gather.
struct GatherPrep {
  int rb, re;
  double ux;
};

template <int DR, int MODE, typename TV>
__device__ __forceinline__ GatherPrep gather_prep(const tls_schur_args& a, const TV* __restrict__ x, int64_t i) {
  const int tid = threadIdx.x;
  GatherPrep g;
  g.rb = __ldg(a.rrun_ptr + i);
  g.re = __ldg(a.rrun_ptr + i + 1);
  g.ux = 0.0;
  if constexpr (MODE == 0) {
    if (tid < DR * DR) {
      const int l = tid % DR;
      const double sl = a.scale ? a.scale[a.retained_offset + i * DR + l] : 1.0;
      const double xl = to_d(x[i * DR + l]);
      g.ux = a.ret_diag[i * DR * DR + tid] * (sl * xl);
    }
  }
  return g;
}

// Run partials each thread keeps in flight per round of gather_one (256
// threads: 1,280 runs per round).
constexpr int kGatherInFlight = 5;

template <int DR, int MODE, typename TV, typename TP, bool COH>
__device__ __forceinline__ double gather_one(const tls_schur_args& a, const TV* __restrict__ x,
                                             const double* __restrict__ b, TV* __restrict__ out, int64_t i,
                                             double (*sm)[DR], double* ux, const GatherPrep& g) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const TP* part = reinterpret_cast<const TP*>(a.run_partial);
  if constexpr (MODE == 0) {
    if (tid < DR * DR) ux[tid] = g.ux;
  }
  double acc[DR];
#pragma unroll
  for (int k = 0; k < DR; ++k) acc[k] = 0.0;
  const int rb = g.rb, re = g.re;
  // kGatherInFlight runs per thread in flight per round; thread t sums runs
  // t, t + 256, t + 512, ... in that order whatever the round size
  constexpr int F = kGatherInFlight;
  for (int j0 = rb + tid; j0 < re; j0 += F * 256) {
    TP v[F][DR];
#pragma unroll
    for (int q = 0; q < F; ++q) {
      const int j = j0 + q * 256;
#pragma unroll
      for (int k = 0; k < DR; ++k) {
        const TP* src = part + (int64_t)j * DR + k;
        v[q][k] = j < re ? *src : TP(0);
      }
    }
#pragma unroll
    for (int q = 0; q < F; ++q)
#pragma unroll
      for (int k = 0; k < DR; ++k) acc[k] += static_cast<double>(v[q][k]);
  }
#pragma unroll
  for (int k = 0; k < DR; ++k) {
    const double v = warp_sum(acc[k]);
    if (lane == 0) sm[warp][k] = v;
  }
  __syncthreads();
  double dot = 0.0;
  if (warp == 0) {
    if (lane < DR) {
      const int k = lane;
      double tot = 0.0;
#pragma unroll
      for (int q = 0; q < 8; ++q) tot += sm[q][k];
      if constexpr (MODE == 0) {
        const double xv = to_d(x[i * DR + k]);
        const double sk = a.scale ? a.scale[a.retained_offset + i * DR + k] : 1.0;
        double v = 0.0;
#pragma unroll
        for (int l = 0; l < DR; ++l) v += ux[k * DR + l];
        v = sk * v + a.damping * xv - tot;
        const TV o = static_cast<TV>(v);
        out[i * DR + k] = o;
        dot = xv * to_d(o);
      } else {
        out[i * DR + k] = static_cast<TV>(b[a.retained_offset + i * DR + k] - tot);
      }
    }
    if constexpr (MODE == 0) dot = warp_sum(dot);
  }
  __syncthreads();  // sm and ux are reused by the caller's next variable
  return dot;
}

// One block per retained variable (gather_one), then for MODE 0 the dot
// partial and the PCG epilogue (curvature and alpha in the last block).
template <int DR, int MODE, typename TV, typename TP>
__global__ void __launch_bounds__(256) schur_gather_kernel(tls_schur_args a, const TV* __restrict__ x,
                                                           const double* __restrict__ b, TV* __restrict__ out,
                                                           double* __restrict__ dot_partials, PcgState* pst) {
  __shared__ double sm[8][DR];
  __shared__ double ux[DR * DR];
  __shared__ double smd[8];
  const GatherPrep g = gather_prep<DR, MODE, TV>(a, x, blockIdx.x);
  const double dot = gather_one<DR, MODE, TV, TP, false>(a, x, b, out, blockIdx.x, sm, ux, g);
  if constexpr (MODE == 0) {
    if (threadIdx.x == 0 && dot_partials) dot_partials[blockIdx.x] = dot;
    if (pst) pcg_operator_epilogue<256>(pst, dot_partials, gridDim.x, smd);
  }
}

// Warp per retained variable, for structures whose variables have few run
// partials each (many small problems merged: a 256-thread block per variable
// would leave most threads idle and take one block per variable). Lanes take
// runs lane, lane + 32, ... (four in flight), a fixed butterfly combines them;
// no dot partials (standalone products only).
template <int DR, int MODE, typename TV, typename TP>
__global__ void __launch_bounds__(256) schur_gather_warp_kernel(tls_schur_args a, const TV* __restrict__ x,
                                                                const double* __restrict__ b,
                                                                TV* __restrict__ out) {
  __shared__ double uxs[8][DR * DR];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t i = (int64_t)blockIdx.x * 8 + warp;
  if (i >= a.nretained) return;
  double* ux = uxs[warp];
  const TP* part = reinterpret_cast<const TP*>(a.run_partial);
  if constexpr (MODE == 0) {
    for (int t = lane; t < DR * DR; t += 32) {
      const int l = t % DR;
      const double sl = a.scale ? a.scale[a.retained_offset + i * DR + l] : 1.0;
      ux[t] = a.ret_diag[i * DR * DR + t] * (sl * to_d(x[i * DR + l]));
    }
  }
  double acc[DR];
#pragma unroll
  for (int k = 0; k < DR; ++k) acc[k] = 0.0;
  const int rb = __ldg(a.rrun_ptr + i), re = __ldg(a.rrun_ptr + i + 1);
  for (int j0 = rb + lane; j0 < re; j0 += 128) {
    TP v[4][DR];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = j0 + q * 32;
#pragma unroll
      for (int k = 0; k < DR; ++k) v[q][k] = j < re ? part[(int64_t)j * DR + k] : TP(0);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int k = 0; k < DR; ++k) acc[k] += static_cast<double>(v[q][k]);
  }
#pragma unroll
  for (int k = 0; k < DR; ++k) acc[k] = warp_sum(acc[k]);
  __syncwarp();
  if (lane < DR) {
    const int k = lane;
    double tot = acc[0];
#pragma unroll
    for (int q = 1; q < DR; ++q)
      if (q == k) tot = acc[q];
    if constexpr (MODE == 0) {
      const double xv = to_d(x[i * DR + k]);
      const double sk = a.scale ? a.scale[a.retained_offset + i * DR + k] : 1.0;
      double v = 0.0;
#pragma unroll
      for (int l = 0; l < DR; ++l) v += ux[k * DR + l];
      out[i * DR + k] = static_cast<TV>(sk * v + a.damping * xv - tot);
    } else {
      out[i * DR + k] = static_cast<TV>(b[a.retained_offset + i * DR + k] - tot);
    }
  }
}

// Warp per retained variable for the preconditioner blocks: lanes take edges
// s0 + lane, s0 + lane + 32, ... of each of the variable's cross runs.
template <int DR, int DE, typename TW>
__global__ void __launch_bounds__(256) schur_precond_warp_kernel(tls_schur_args a, double* __restrict__ out) {
  constexpr int NU = DR * (DR + 1) / 2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t i = (int64_t)blockIdx.x * 8 + warp;
  if (i >= a.nretained) return;
  double sr[DR];
#pragma unroll
  for (int k = 0; k < DR; ++k) sr[k] = a.scale ? a.scale[a.retained_offset + i * DR + k] : 1.0;
  double acc[NU];
#pragma unroll
  for (int k = 0; k < NU; ++k) acc[k] = 0.0;
  const int rb = a.rrun_ptr[i], re = a.rrun_ptr[i + 1];
  for (int j = rb; j < re; ++j) {
    const int64_t s0 = a.crun_start[j];
    const int len = a.crun_len[j];
    for (int64_t s = s0 + lane; s < s0 + len; s += 32) {
      // the whitened block as the operator stores it (lanes read consecutive
      // slab entries: coalesced)
      const TW* ws = reinterpret_cast<const TW*>(a.w) + ((s / a.cap) * (DR * DE)) * a.cap + (s % a.cap);
      double wv[DR][DE];
#pragma unroll
      for (int r = 0; r < DR; ++r)
#pragma unroll
        for (int c = 0; c < DE; ++c) wv[r][c] = to_d(ws[(int64_t)(r * DE + c) * a.cap]);
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
#pragma unroll
  for (int k = 0; k < NU; ++k) acc[k] = warp_sum(acc[k]);
  if (lane != 0) return;
  const double* U = a.ret_diag + i * DR * DR;
  double* o = out + i * DR * DR;
  int idx = 0;
#pragma unroll
  for (int r = 0; r < DR; ++r)
#pragma unroll
    for (int q = r; q < DR; ++q) {
      const double v = sr[r] * U[r * DR + q] * sr[q] - acc[idx++];
      o[r * DR + q] = v;
      o[q * DR + r] = v;
    }
}

// ---------------------------------------------------------------- persistent Schur-PCG
// The whole PCG loop on the reduced system in ONE cooperative launch (all
// CTAs co-resident): per step
//   A  every CTA streams its chunks (Ap partials from p), prefetching the
//      next step's first chunk while B and C run (W does not change)
//   -- grid barrier --
//   B  gather: one retained variable per CTA at a time -> Ap, x.Ap partials
//   -- grid barrier; before releasing, the last CTA to arrive runs --
//   C  curvature and alpha, update x, r, z = M r, the decision and the
//      direction (the same state machine as the multi-kernel path)
// Every wait is bounded (about a second); on timeout the kernel flags a.err
// and every CTA leaves after draining its own bulk copy.
// Grid barrier over all CTAs of a cooperative launch; the last CTA to arrive
// runs `tail()` (all its threads) before releasing the others. Waiters poll
// with a short sleep; false on timeout (about a second).
template <typename F>
__device__ __forceinline__ bool grid_barrier(PcgState* st, int32_t* err, long long limit, F&& tail) {
  __shared__ int ok, last;
  __shared__ uint32_t gen0;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile uint32_t* gen = &st->bar_gen;
    gen0 = *gen;
    __threadfence();
    ok = 1;
    last = atomicAdd(&st->bar_count, 1u) == gridDim.x - 1;
    if (last) __threadfence();
  }
  __syncthreads();
  if (last) {
    tail();
    __syncthreads();
    if (threadIdx.x == 0) {
      st->bar_count = 0;
      __threadfence();
      atomicExch(&st->bar_gen, gen0 + 1u);
    }
  } else if (threadIdx.x == 0) {
    volatile uint32_t* gen = &st->bar_gen;
    const long long t0 = clock64();
    while (*gen == gen0) {
      __nanosleep(64);
      if (clock64() - t0 > limit) {
        if (err) atomicExch(err, 2);
        ok = 0;
        break;
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

template <int DR, int DE, int CAP, typename TW, int D>
__global__ void __launch_bounds__(kChunkThreads, 2) schur_pcg_kernel(tls_schur_args a, PcgLoop q) {
  using TA = double;
  using S = SlabShape<DR, DE, CAP, TW, TA>;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ double sm[8][DR];
  __shared__ double ux[DR * DR];
  __shared__ double smd[kChunkThreads / 32];
  __shared__ int s_action, s_tofinal, s_go;
  __shared__ double s_beta;
  TA* t_s = reinterpret_cast<TA*>(smem + 2 * S::kStageBytes);
  const int tid = threadIdx.x;
  const unsigned char* wsrc = reinterpret_cast<const unsigned char*>(a.w);
  const unsigned char* msrc = reinterpret_cast<const unsigned char*>(a.meta);
  PcgState* st = q.st;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](int c, int stg) {
    unsigned char* base = smem + stg * S::kStageBytes;
    fence_proxy_async();
    mbar_expect_tx(&bar[stg], S::kStageBytes);
    bulk_load(base, wsrc + (size_t)c * S::kWBytes, S::kWBytes, &bar[stg]);
    bulk_load(base + S::kWBytes, msrc + (size_t)c * S::kMetaBytes, S::kMetaBytes, &bar[stg]);
  };
  // this CTA's chunks: blockIdx.x + j * gridDim.x, j < kct, cycled every step
  const int kct = (int)blockIdx.x < a.nchunks ? (a.nchunks - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  auto chunk_of = [&](int j) { return (int)blockIdx.x + (j % kct) * (int)gridDim.x; };
  const long long lim = wait_limit(a);
  int it = 0;  // chunk consumptions so far; the copy for `it` is always in flight
  if (tid == 0 && kct > 0) issue(chunk_of(0), 0);
  for (int step = 0; step < q.steps; ++step) {
    if (tid == 0) {
      const int status = __ldcg(&st->pub.status), mode = __ldcg(&st->pub.mode);
      s_go = status == TLS_PCG_ACTIVE && mode != M_DONE;
    }
    __syncthreads();
    if (!s_go) break;
    // ---- A: chunk partials of A p
    bool failed = false;
    for (int j = 0; j < kct; ++j, ++it) {
      const int stg = it & 1;
      const bool ok = mbar_wait_bounded(&bar[stg], (it >> 1) & 1, a.err, lim);
      // the block barrier also ends the previous chunk's reads of the other stage and of t_s
      if (__syncthreads_or(!ok)) {  // this stage may be incomplete: leave without reading it
        failed = true;
        break;
      }
      if (tid == 0) issue(chunk_of(it + 1), stg ^ 1);
      const TW* Ws = reinterpret_cast<const TW*>(smem + stg * S::kStageBytes);
      const int32_t* Ms = reinterpret_cast<const int32_t*>(smem + stg * S::kStageBytes + S::kWBytes);
      chunk_compute<DR, DE, CAP, 0, TW, TA, false, true>(a, q.p, nullptr, t_s, Ws, Ms, chunk_of(it));
    }
    if (failed) break;
    if (!grid_barrier(st, a.err, lim, [] {})) break;
    // ---- B: gather per retained variable
    for (int64_t i = blockIdx.x; i < a.nretained; i += gridDim.x) {
      const double dot =
          gather_one<DR, 0, double, double, true>(a, q.p, nullptr, q.ap, i, sm, ux, gather_prep<DR, 0>(a, q.p, i));
      if (tid == 0) q.dots[i] = dot;
    }
    // ---- C (the last CTA through the barrier): curvature and alpha, update,
    // preconditioner, decision, direction
    auto phase_c = [&] {
      tls_pcg_control& c = st->pub;
      const int mode = c.mode;
      if (c.status == TLS_PCG_ACTIVE && mode == M_ITER) {
        const double curv = block_sum_cg<kChunkThreads>(q.dots, a.nretained, smd);
        if (tid == 0) {
          const double rz = c.rz;
          c.curvature = curv;
          const bool ok = isfinite(curv) && isfinite(rz) && curv > 0.0 && rz > 0.0;
          st->alpha_ok = ok;
          c.alpha = ok ? rz / curv : 0.0;
        }
        __syncthreads();
      }
      double a0 = 0.0, a1 = 0.0, a2 = 0.0;
      bool work = c.status == TLS_PCG_ACTIVE && mode != M_DONE;
      double alpha = 0.0;
      if (work && mode == M_ITER) {
        if (!st->alpha_ok) work = false;
        else alpha = c.alpha;
      }
      if (work)
        pcg_update_blocks<D, double, true>(q.bs, q.nb, tid, kChunkThreads, mode, alpha, q.rhs, q.x, q.r, q.z, q.p,
                                           q.ap, q.ztrue, a0, a1, a2);
      __shared__ double smd3[3][kChunkThreads / 32];
      block_sum3<kChunkThreads>(a0, a1, a2, smd3);
      const double t0 = a0, t1 = a1, t2 = a2;
      if (tid == 0) {
        pcg_decide(st, t0, t1, t2);
        s_action = st->action;
        s_beta = st->pub.beta;
        s_tofinal = st->pub.mode == M_FINAL && st->action != A_SWAP_TO_X;
      }
      __syncthreads();
      if (s_action != A_NONE)
        pcg_direction_elems<double, true>(q.n, tid, kChunkThreads, s_action, s_beta, s_tofinal != 0, q.x, q.r, q.z,
                                          q.p, q.psave, q.ap, q.ztrue);
    };
    if (!grid_barrier(st, a.err, lim, phase_c)) break;
  }
  // drain this CTA's copies in flight before leaving (bounded)
  if (kct > 0 && tid == 0) mbar_drain(bar, it, it + 1, a.err);  // the copy for `it` is in flight
  __syncthreads();
}

// Variant for small reduced systems: the LAST CTA is a "vector CTA" that
// keeps x, r, z, p and Ap of the PCG in its shared memory (where the other
// CTAs keep chunk slabs), with the preconditioner factors and block columns
// when one thread per block suffices, and runs the whole vector phase; the
// other CTAs stream the chunks and gather. Per step:
//   A  chunk CTAs: chunk partials of A p            -- barrier over chunk CTAs --
//   B  chunk CTAs: gather Ap and x.Ap partials, then arrive at the vector CTA
//   C  vector CTA (after every arrival): curvature and alpha, update,
//      preconditioner, decision, direction in shared memory; publishes p and
//      the control block, then releases the chunk CTAs.
// The arithmetic (and its order) is that of schur_pcg_kernel. Every wait is
// bounded; on timeout the kernel flags a.err and every CTA leaves.
// The vector CTA's per-block work: thread b owns preconditioner block b. Its
// columns (bcol[k * kChunkThreads + b], -1 past the block's size) and its
// packed factor (fac[k * kChunkThreads + b], the diagonal entries replaced by
// their reciprocals) sit in shared memory from the start of the solve, so a
// step reads no kernel parameters, divides nothing and keeps few values live.
// The vector CTA runs this code once per step after a long wait during which
// its SM runs the chunk code, so its instructions are fetched cold: it is kept
// short. The arithmetic and its order are pcg_update_block's.
template <int D>
__device__ __forceinline__ void vc_update_block(int b, int mode, double alpha, const double* __restrict__ rhs,
                                                double* x, double* r, double* z, const double* p, double* ap,
                                                double* ztrue, const double* fac, const int* bcol, bool solve,
                                                double& a0, double& a1, double& a2) {
  int cols[D];
#pragma unroll
  for (int k = 0; k < D; ++k) cols[k] = bcol[k * kChunkThreads + b];
  double rb[D];
  if (mode == M_ITER) {
#pragma unroll
    for (int k = 0; k < D; ++k) {
      rb[k] = 0.0;
      if (cols[k] >= 0) {
        const int c = cols[k];
        x[c] = x[c] + alpha * p[c];
        const double rn = r[c] - alpha * ap[c];
        r[c] = rn;
        rb[k] = rn;
      }
    }
  } else {
#pragma unroll
    for (int k = 0; k < D; ++k) {
      rb[k] = 0.0;
      if (cols[k] >= 0) {
        const int c = cols[k];
        const double t = rhs[c] - ap[c];
        const double rv = r[c];
        ap[c] = t;
        rb[k] = t;
        a0 += t * t;
        const double dr = t - rv;
        a1 += dr * dr;
      }
    }
  }
  if (mode == M_FINAL) return;
  double zb[D];
  if (!solve) {
#pragma unroll
    for (int k = 0; k < D; ++k) zb[k] = rb[k];
  } else {
    auto L = [&](int row, int col) -> double { return fac[(row * (row + 1) / 2 + col) * kChunkThreads + b]; };
    double inv[D];
#pragma unroll
    for (int k = 0; k < D; ++k) inv[k] = (cols[k] >= 0) ? L(k, k) : 0.0;
    double y[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
      double t = rb[k];
#pragma unroll
      for (int m = 0; m < k; ++m) t -= (cols[k] >= 0) ? L(k, m) * y[m] : 0.0;
      y[k] = (cols[k] >= 0) ? t * inv[k] : 0.0;
    }
#pragma unroll
    for (int k = D - 1; k >= 0; --k) {
      double t = y[k];
#pragma unroll
      for (int m = k + 1; m < D; ++m) t -= (cols[m] >= 0) ? L(m, k) * zb[m] : 0.0;
      zb[k] = (cols[k] >= 0) ? t * inv[k] : 0.0;
    }
  }
  double* zdst = (mode == M_ITER) ? z : ztrue;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    if (cols[k] >= 0) {
      zdst[cols[k]] = zb[k];
      if (mode == M_ITER) {
        a0 += rb[k] * rb[k];
        a1 += rb[k] * zb[k];
      } else {
        a2 += rb[k] * zb[k];
      }
    }
  }
}

// pcg_direction_elems over block b's columns, each new p also stored to
// global memory (`pg`, which the chunk CTAs read); one loop per action.
template <int D>
__device__ __forceinline__ void vc_direction_block(int b, int action, double beta, bool to_final, const double* x,
                                                   double* r, const double* z, double* p, double* psave,
                                                   const double* ap, const double* ztrue, const int* bcol,
                                                   double* pg) {
  int cols[D];
#pragma unroll
  for (int k = 0; k < D; ++k) cols[k] = bcol[k * kChunkThreads + b];
  auto put = [&](int i, double pn) {
    if (to_final) pn = x[i];
    p[i] = pn;
    pg[i] = pn;
  };
  if (action == A_DIR) {
#pragma unroll
    for (int k = 0; k < D; ++k)
      if (cols[k] >= 0) put(cols[k], z[cols[k]] + beta * p[cols[k]]);
  } else if (action == A_RESTORE_DIR) {
#pragma unroll
    for (int k = 0; k < D; ++k)
      if (cols[k] >= 0) put(cols[k], z[cols[k]] + beta * psave[cols[k]]);
  } else if (action == A_RESTART) {
#pragma unroll
    for (int k = 0; k < D; ++k)
      if (cols[k] >= 0) {
        r[cols[k]] = ap[cols[k]];
        put(cols[k], ztrue[cols[k]]);
      }
  } else if (action == A_SWAP_TO_X) {
#pragma unroll
    for (int k = 0; k < D; ++k)
      if (cols[k] >= 0) {
        psave[cols[k]] = p[cols[k]];
        put(cols[k], x[cols[k]]);
      }
  }
}

template <int DR, int DE, int CAP, typename TW, int D>
__global__ void __launch_bounds__(kChunkThreads, 2) schur_pcg_vc_kernel(tls_schur_args a, PcgLoop q) {
  using TA = double;
  using S = SlabShape<DR, DE, CAP, TW, TA>;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ double sm[8][DR];
  __shared__ double ux[DR * DR];
  __shared__ double smd[kChunkThreads / 32];
  __shared__ int s_go, s_ok, last;
  __shared__ uint32_t gen0;
  const int tid = threadIdx.x;
  PcgState* st = q.st;
  const int G = (int)gridDim.x - 1;  // chunk CTAs
  const bool vcta = (int)blockIdx.x == G;
  if (vcta) {
    // ---------------- the vector CTA
    const int64_t n = q.n;
    double* x = reinterpret_cast<double*>(smem);
    double* r = x + n;
    double* z = r + n;
    double* p = z + n;
    double* ap = p + n;
    double* psave = q.psave;  // read at residual checks only: global memory
    // one preconditioner block per thread when they fit: its factor (fixed
    // during the solve) is held in shared memory, column-major over threads
    constexpr int LD = D * (D + 1) / 2;
    uint32_t dyn = 0;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
    const bool one_block =
        q.nb <= kChunkThreads && n * 5 * 8 + kChunkThreads * (LD * 8 + D * 4) <= (int64_t)dyn;
    double* fac = ap + n;                                       // [LD][kChunkThreads] when one_block
    int* bcol = reinterpret_cast<int*>(fac + LD * kChunkThreads);  // [D][kChunkThreads] when one_block
    bool have_f = false;
    int bdim = 0;
    if (one_block) {
      if (tid < q.nb) {
        double l[LD];
        have_f = pcg_prefetch_factor<D>(q.bs, tid, M_ITER, l);
        if (have_f) {
#pragma unroll
          for (int k = 0; k < LD; ++k) fac[k * kChunkThreads + tid] = l[k];
#pragma unroll
          for (int k = 0; k < D; ++k) fac[(k * (k + 3) / 2) * kChunkThreads + tid] = 1.0 / l[k * (k + 3) / 2];
        }
        const int gi = find_group(q.bs, tid);
        const tls_block_group& g = q.bs.g[gi];
        int64_t cols[D];
        block_cols<D>(g, tid - q.bs.block_begin[gi], cols);
        bdim = g.dim;
#pragma unroll
        for (int k = 0; k < D; ++k) bcol[k * kChunkThreads + tid] = k < bdim ? (int)cols[k] : -1;
      } else {
#pragma unroll
        for (int k = 0; k < D; ++k) bcol[k * kChunkThreads + tid] = -1;
      }
    }
    // the direction runs per block when the (disjoint) blocks cover every column
    __shared__ int s_block_dir;
    {
      const double cover = block_sum<kChunkThreads>((double)bdim, smd);
      if (tid == 0) s_block_dir = one_block && cover == (double)n;
      __syncthreads();
    }
    const bool block_dir = s_block_dir != 0;
    // The control block lives in this CTA's shared memory during the solve;
    // status and mode are published to global memory every step (the chunk
    // CTAs read them), the rest when the loop ends.
    __shared__ PcgState sst;
    if (tid == 0) sst = *st;
    for (int64_t i = tid; i < n; i += kChunkThreads) {
      x[i] = q.x[i];
      r[i] = q.r[i];
      z[i] = q.z[i];
      p[i] = q.p[i];
    }
    __syncthreads();
    for (int step = 0; step < q.steps; ++step) {
      if (tid == 0) s_go = sst.pub.status == TLS_PCG_ACTIVE && sst.pub.mode != M_DONE;
      __syncthreads();
      if (!s_go) break;
      const int mode = sst.pub.mode;
      // wait until every chunk CTA has gathered its variables
      uint32_t gen_now = 0;  // thread 0: the barrier generation this step releases
      if (tid == 0) {
        s_ok = 1;
        volatile uint32_t* cnt = &st->bar_count2;
        const long long t0 = clock64();
        while (*cnt != (uint32_t)G) {
          __nanosleep(32);
          if (clock64() - t0 > wait_limit(a)) {
            if (a.err) atomicExch(a.err, 2);
            s_ok = 0;
            break;
          }
        }
        __threadfence();
        // stable until this CTA's release (every chunk CTA has passed this
        // step's chunk barrier); read now, used at the release
        gen_now = *reinterpret_cast<volatile uint32_t*>(&st->bar_gen);
      }
      __syncthreads();
      if (!s_ok) break;
      // Ap into shared memory, and the curvature p.Ap in the same pass
      // (eight loads per thread in flight; the sum runs in element order)
      double part = 0.0;
      for (int64_t i0 = tid; i0 < n; i0 += 8 * kChunkThreads) {
        double v[8];
#pragma unroll
        for (int m = 0; m < 8; ++m) {
          const int64_t i = i0 + m * kChunkThreads;
          v[m] = i < n ? __ldcg(q.ap + i) : 0.0;
        }
#pragma unroll
        for (int m = 0; m < 8; ++m) {
          const int64_t i = i0 + m * kChunkThreads;
          if (i < n) {
            ap[i] = v[m];
            part += p[i] * v[m];
          }
        }
      }
      const double curv = block_sum<kChunkThreads>(part, smd);
      tls_pcg_control& c = sst.pub;
      if (tid == 0 && c.status == TLS_PCG_ACTIVE && mode == M_ITER) {
        const double rz = c.rz;
        c.curvature = curv;
        const bool ok = isfinite(curv) && isfinite(rz) && curv > 0.0 && rz > 0.0;
        sst.alpha_ok = ok;
        c.alpha = ok ? rz / curv : 0.0;
      }
      __syncthreads();
      double a0 = 0.0, a1 = 0.0, a2 = 0.0;
      bool work = c.status == TLS_PCG_ACTIVE && mode != M_DONE;
      double alpha = 0.0;
      if (work && mode == M_ITER) {
        if (!sst.alpha_ok) work = false;
        else alpha = c.alpha;
      }
      if (work) {
        if (one_block) {
          if (tid < q.nb)
            vc_update_block<D>(tid, mode, alpha, q.rhs, x, r, z, p, ap, q.ztrue, fac, bcol, have_f, a0, a1, a2);
        } else {
          pcg_update_blocks<D, double, false>(q.bs, q.nb, tid, kChunkThreads, mode, alpha, q.rhs, x, r, z, p, ap,
                                              q.ztrue, a0, a1, a2);
        }
      }
      __shared__ double smd3[3][kChunkThreads / 32];
      block_sum3<kChunkThreads>(a0, a1, a2, smd3);
      const double t0 = a0, t1 = a1, t2 = a2;
      __shared__ int s_action, s_tofinal;
      __shared__ double s_beta;
      if (tid == 0) {
        pcg_decide(&sst, t0, t1, t2);
        s_action = sst.action;
        s_beta = sst.pub.beta;
        s_tofinal = sst.pub.mode == M_FINAL && sst.action != A_SWAP_TO_X;
        st->pub.status = sst.pub.status;  // read by the chunk CTAs at their next step
        st->pub.mode = sst.pub.mode;
      }
      __syncthreads();
      if (block_dir) {
        if (s_action != A_NONE)
          vc_direction_block<D>(tid, s_action, s_beta, s_tofinal != 0, x, r, z, p, psave, ap, q.ztrue, bcol, q.p);
        __syncthreads();
      } else {
        if (s_action != A_NONE)
          pcg_direction_elems<double, false>(n, tid, kChunkThreads, s_action, s_beta, s_tofinal != 0, x, r, z, p,
                                             psave, ap, q.ztrue);
        __syncthreads();
        for (int64_t i = tid; i < n; i += kChunkThreads) q.p[i] = p[i];  // the operator reads p
        __syncthreads();
      }
      if (tid == 0) {
        st->bar_count2 = 0;
        __threadfence();
        atomicExch(&st->bar_gen, gen_now + 1u);
      }
    }
    __syncthreads();
    if (tid == 0) {  // the control block back to global memory (not the barrier words)
      st->pub = sst.pub;
      st->action = sst.action;
      st->pending = sst.pending;
      st->rec = sst.rec;
      st->rec_hit = sst.rec_hit;
      st->periodic_hit = sst.periodic_hit;
      st->alpha_ok = sst.alpha_ok;
    }
    for (int64_t i = tid; i < n; i += kChunkThreads) {
      q.x[i] = x[i];
      q.r[i] = r[i];
      q.z[i] = z[i];
      q.p[i] = p[i];
    }
    return;
  }
  // ---------------- chunk CTAs
  TA* t_s = reinterpret_cast<TA*>(smem + 2 * S::kStageBytes);
  const unsigned char* wsrc = reinterpret_cast<const unsigned char*>(a.w);
  const unsigned char* msrc = reinterpret_cast<const unsigned char*>(a.meta);
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](int c, int stg) {
    unsigned char* base = smem + stg * S::kStageBytes;
    fence_proxy_async();
    mbar_expect_tx(&bar[stg], S::kStageBytes);
    bulk_load(base, wsrc + (size_t)c * S::kWBytes, S::kWBytes, &bar[stg]);
    bulk_load(base + S::kWBytes, msrc + (size_t)c * S::kMetaBytes, S::kMetaBytes, &bar[stg]);
  };
  const int kct = (int)blockIdx.x < a.nchunks ? (a.nchunks - 1 - (int)blockIdx.x) / G + 1 : 0;
  auto chunk_of = [&](int j) { return (int)blockIdx.x + (j % kct) * G; };
  const long long lim = wait_limit(a);
  int it = 0;
  if (tid == 0 && kct > 0) issue(chunk_of(0), 0);
  for (int step = 0; step < q.steps; ++step) {
    if (tid == 0) {
      const int status = __ldcg(&st->pub.status), mode = __ldcg(&st->pub.mode);
      s_go = status == TLS_PCG_ACTIVE && mode != M_DONE;
    }
    __syncthreads();
    if (!s_go) break;
    // ---- A
    bool failed = false;
    for (int j = 0; j < kct; ++j, ++it) {
      const int stg = it & 1;
      const bool ok = mbar_wait_bounded(&bar[stg], (it >> 1) & 1, a.err, lim);
      // the block barrier also ends the previous chunk's reads of the other stage and of t_s
      if (__syncthreads_or(!ok)) {  // this stage may be incomplete: leave without reading it
        failed = true;
        break;
      }
      if (tid == 0) issue(chunk_of(it + 1), stg ^ 1);
      const TW* Ws = reinterpret_cast<const TW*>(smem + stg * S::kStageBytes);
      const int32_t* Ms = reinterpret_cast<const int32_t*>(smem + stg * S::kStageBytes + S::kWBytes);
      chunk_compute<DR, DE, CAP, 0, TW, TA, false, true>(a, q.p, nullptr, t_s, Ws, Ms, chunk_of(it));
    }
    if (failed) break;
    // this CTA's first retained variable: its run range and diagonal term load
    // while the barrier waits
    GatherPrep g0{0, 0, 0.0};
    if ((int64_t)blockIdx.x < a.nretained) g0 = gather_prep<DR, 0>(a, q.p, blockIdx.x);
    // ---- barrier over the chunk CTAs
    __syncthreads();
    if (tid == 0) {
      volatile uint32_t* gen = &st->bar_gen;
      gen0 = *gen;
      __threadfence();
      s_ok = 1;
      last = atomicAdd(&st->bar_count, 1u) == (uint32_t)G - 1;
      if (last) {
        st->bar_count = 0;
        __threadfence();
        atomicExch(&st->bar_gen, gen0 + 1u);
      } else {
        const long long t0 = clock64();
        while (*gen == gen0) {
          __nanosleep(64);
          if (clock64() - t0 > lim) {
            if (a.err) atomicExch(a.err, 2);
            s_ok = 0;
            break;
          }
        }
      }
      __threadfence();
    }
    __syncthreads();
    if (!s_ok) break;
    // ---- B (the vector CTA forms p.Ap itself)
    for (int64_t i = blockIdx.x; i < a.nretained; i += G)
      gather_one<DR, 0, double, double, true>(a, q.p, nullptr, q.ap, i, sm, ux,
                                              i == blockIdx.x ? g0 : gather_prep<DR, 0>(a, q.p, i));
    // ---- arrive at the vector CTA, wait for its release
    __syncthreads();
    if (tid == 0) {
      volatile uint32_t* gen = &st->bar_gen;
      gen0 = *gen;
      __threadfence();
      atomicAdd(&st->bar_count2, 1u);
      const long long t0 = clock64();
      while (*gen == gen0) {
        __nanosleep(64);
        if (clock64() - t0 > lim) {
          if (a.err) atomicExch(a.err, 2);
          s_ok = 0;
          break;
        }
      }
      __threadfence();
    }
    __syncthreads();
    if (!s_ok) break;
  }
  if (kct > 0 && tid == 0) mbar_drain(bar, it, it + 1, a.err);  // the copy for `it` is in flight
  __syncthreads();
}

// W slab index of component k of slab entry s.
template <int DR, int DE>
__device__ __forceinline__ int64_t w_index(int64_t s, int k, int cap) {
  return ((s / cap) * (DR * DE) + k) * cap + (s % cap);
}

// Per eliminated variable: L = chol(s C s + lambda I), store L^-1.
template <int DE>
__global__ void schur_factor_kernel(tls_schur_args a) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.nelim) return;
  double s[DE];
#pragma unroll
  for (int k = 0; k < DE; ++k) s[k] = a.scale ? a.scale[a.elim_offset + p * DE + k] : 1.0;
  if (!eliminated_factor<DE>(a.elim_diag + p * DE * DE, s, a.damping, a.inv_l + p * DE * DE)) atomicAdd(a.bad, 1);
}

// W_e = diag(s_i) E_e diag(s_p) L_p^-T into the slabs; padding entries get 0.
template <int DR, int DE, typename TW>
__global__ void __launch_bounds__(128) schur_whiten_kernel(tls_schur_args a) {
  // The block's cross blocks ([128][DR][DE] float64, contiguous) are staged in
  // shared memory with coalesced loads; each thread then whitens its own.
  constexpr int kW = DR * DE;
  __shared__ double e_s[128 * kW];
  const int64_t s0 = (int64_t)blockIdx.x * blockDim.x;
  const int64_t s = s0 + threadIdx.x;
  const int64_t nslab = (int64_t)a.nchunks * a.cap;
  const int nvalid = (int)((nslab - s0) < 128 ? (nslab - s0) : 128);
  // this thread's edge, its scales and its point's factor: loaded before the
  // staging barrier so that every load of the block is in flight together
  const bool live = s < nslab;
  const int64_t i = live ? a.slab_r[s] : -1;
  const int64_t p = i >= 0 ? a.slab_e[s] : 0;
  double sr[DR], se[DE], Li[DE * DE];
#pragma unroll
  for (int k = 0; k < DR; ++k) sr[k] = (a.scale && i >= 0) ? a.scale[a.retained_offset + i * DR + k] : 1.0;
#pragma unroll
  for (int k = 0; k < DE; ++k) se[k] = (a.scale && i >= 0) ? a.scale[a.elim_offset + p * DE + k] : 1.0;
#pragma unroll
  for (int k = 0; k < DE * DE; ++k) Li[k] = i >= 0 ? a.inv_l[p * DE * DE + k] : 0.0;
  if (a.cross_contrib) {
    // each element is the float64 sum of its entry's contributions in list
    // order (tls_segment_reduce's sums): usually one, so the first one of
    // every element is loaded with all of them in flight, then any further
    // ones in order
    const int ne = nvalid * kW;
    int jb[kW], je[kW], o[kW];
#pragma unroll
    for (int q = 0; q < kW; ++q) {
      const int e = threadIdx.x + q * 128;
      const int64_t t = s0 + e / kW;
      jb[q] = e < ne ? a.cross_ptr[t] : 0;
      je[q] = e < ne ? a.cross_ptr[t + 1] : 0;
    }
#pragma unroll
    for (int q = 0; q < kW; ++q) o[q] = jb[q] < je[q] ? a.cross_src[jb[q]] : -1;
    double v[kW];
#pragma unroll
    for (int q = 0; q < kW; ++q) {
      const int k = (threadIdx.x + q * 128) % kW;
      v[q] = 0.0;
      if (o[q] >= 0) v[q] += a.cross_contrib[(int64_t)o[q] + k];
    }
#pragma unroll
    for (int q = 0; q < kW; ++q) {
      const int k = (threadIdx.x + q * 128) % kW;
      for (int j = jb[q] + 1; j < je[q]; ++j) v[q] += a.cross_contrib[(int64_t)a.cross_src[j] + k];
      if (threadIdx.x + q * 128 < ne) e_s[threadIdx.x + q * 128] = v[q];
    }
  } else if (nvalid == 128) {  // a full block: kW coalesced loads per thread, all in flight
    double v[kW];
#pragma unroll
    for (int q = 0; q < kW; ++q) v[q] = a.cross[s0 * kW + threadIdx.x + q * 128];
#pragma unroll
    for (int q = 0; q < kW; ++q) e_s[threadIdx.x + q * 128] = v[q];
  } else {
    for (int k = threadIdx.x; k < nvalid * kW; k += 128) e_s[k] = a.cross[s0 * kW + k];
  }
  __syncthreads();
  if (!live) return;
  TW* w = reinterpret_cast<TW*>(a.w);
  if (i < 0) {
#pragma unroll
    for (int k = 0; k < kW; ++k) w[w_index<DR, DE>(s, k, a.cap)] = TW(0);
    return;
  }
  const double* E = e_s + threadIdx.x * kW;
#pragma unroll
  for (int r = 0; r < DR; ++r) {
#pragma unroll
    for (int c = 0; c < DE; ++c) {
      double v = 0.0;
#pragma unroll
      for (int k = 0; k < DE; ++k) v += sr[r] * E[r * DE + k] * se[k] * Li[c * DE + k];
      w[w_index<DR, DE>(s, r * DE + c, a.cap)] = static_cast<TW>(v);
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

// delta_p = L_p^-T (y_p - sum_{e in p} W_e^T x_i); the retained part of delta is x
template <int DR, int DE, typename TW, typename TV>
__global__ void schur_backsub_kernel(tls_schur_args a, const TV* __restrict__ xc, double* __restrict__ delta) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nret = (int64_t)a.nretained * DR;
  if (tid < nret) delta[a.retained_offset + tid] = to_d(xc[tid]);
  if (tid >= a.nelim) return;
  const int64_t p = tid;
  const TW* w = reinterpret_cast<const TW*>(a.w);
  double t[DE];
#pragma unroll
  for (int b = 0; b < DE; ++b) t[b] = a.ybuf[p * DE + b];
  const int pb = a.elim_ptr[p], pe = a.elim_ptr[p + 1];
  // unrolled so that several edges' loads are in flight (the subtractions
  // keep their order)
#pragma unroll 4
  for (int j = pb; j < pe; ++j) {
    const int64_t s = a.elim_slab[j];
    const int64_t i = a.slab_r[s];
#pragma unroll
    for (int b = 0; b < DE; ++b) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < DR; ++k) acc += to_d(w[w_index<DR, DE>(s, k * DE + b, a.cap)]) * to_d(xc[i * DR + k]);
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

// out_i = s U s - sum_{e in i} W_e W_e^T (lambda added by the Cholesky), one
// 256-thread block per retained variable, one thread per run of its edges.
// W_e is recomputed in float64 from the cross block and L_p^-1 with the
// whitening kernel's arithmetic (each run's cross blocks are contiguous, so
// the reads are whole sectors; the stored W slab is strided by the chunk cap).
template <int DR, int DE, typename TW>
__global__ void __launch_bounds__(256) schur_precond_kernel(tls_schur_args a, double* __restrict__ out) {
  constexpr int NU = DR * (DR + 1) / 2;
  __shared__ double red[8][NU];
  const int64_t i = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double sr[DR];
#pragma unroll
  for (int k = 0; k < DR; ++k) sr[k] = a.scale ? a.scale[a.retained_offset + i * DR + k] : 1.0;
  double acc[NU];
#pragma unroll
  for (int k = 0; k < NU; ++k) acc[k] = 0.0;
  const int rb = a.rrun_ptr[i], re = a.rrun_ptr[i + 1];
  for (int j = rb + tid; j < re; j += 256) {
    const int64_t s0 = a.crun_start[j];
    const int len = a.crun_len[j];
    for (int64_t s = s0; s < s0 + len; ++s) {
      // the whitened block as the operator stores it (schur_whiten_kernel
      // rounds exactly this product to TW)
      const TW* ws = reinterpret_cast<const TW*>(a.w) + w_index<DR, DE>(s, 0, a.cap);
      double wv[DR][DE];
#pragma unroll
      for (int r = 0; r < DR; ++r)
#pragma unroll
        for (int c = 0; c < DE; ++c) wv[r][c] = to_d(ws[(int64_t)(r * DE + c) * a.cap]);
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
#pragma unroll
  for (int k = 0; k < NU; ++k) {
    const double v = warp_sum(acc[k]);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (tid != 0) return;
  const double* U = a.ret_diag + i * DR * DR;
  double* o = out + i * DR * DR;
  int idx = 0;
#pragma unroll
  for (int r = 0; r < DR; ++r)
#pragma unroll
    for (int q = r; q < DR; ++q) {
      double t = 0.0;
#pragma unroll
      for (int w = 0; w < 8; ++w) t += red[w][idx];
      const double v = sr[r] * U[r * DR + q] * sr[q] - t;
      o[r * DR + q] = v;
      o[q * DR + r] = v;
      ++idx;
    }
}

template <int DR, int DE>
struct SchurOps {
  template <int MODE, typename TW, int CAP, bool XS>
  static int launch_chunks(const tls_schur_args& a, const double* x, int smem, cudaStream_t s) {
    auto k = schur_chunk_kernel<DR, DE, CAP, MODE, TW, double, XS>;
    // resident CTAs per SM x SMs, per device and shared-memory size, per instantiation
    static DeviceGridCache cache;
    int grid_cap = 0;
    const int rc = cache.get(smem, &grid_cap, [&](int dev) -> int {
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      int per_sm = 0, sms = 0;
      if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kChunkThreads, smem);
      if (e != cudaSuccess) return -1;
      return (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
    });
    if (rc) return rc;
    const int grid = a.nchunks < grid_cap ? a.nchunks : grid_cap;
    k<<<grid, kChunkThreads, smem, s>>>(a, x);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  }
  template <int MODE, typename TW, int CAP>
  static int chunks_cap(const tls_schur_args& a, const double* x, cudaStream_t s) {
    using S = SlabShape<DR, DE, CAP, TW, double>;
    if (a.meta_ints != S::kMetaInts) return tls_set_error(TLS_ERR_INVALID, "metadata slab size mismatch");
    if ((reinterpret_cast<uintptr_t>(a.w) & 15) || (reinterpret_cast<uintptr_t>(a.meta) & 15))
      return tls_set_error(TLS_ERR_INVALID, "W and metadata slabs must be 16-byte aligned");
    // Stage x in shared memory when two CTAs per SM still fit (228 KB per SM,
    // 1 KB reserved per CTA, static barriers).
    constexpr int kTwoCtaSmem = (233472 / 2) - 1024 - 64;
    const int xbytes = ((a.nretained * DR * (int)sizeof(double)) + 15) & ~15;
    if constexpr (MODE == 0) {
      if (S::kBaseSmem + xbytes <= kTwoCtaSmem)
        return launch_chunks<MODE, TW, CAP, true>(a, x, S::kBaseSmem + xbytes, s);
    }
    return launch_chunks<MODE, TW, CAP, false>(a, x, S::kBaseSmem, s);
  }
  template <int MODE, typename TW>
  static int chunks(const tls_schur_args& a, const double* x, cudaStream_t s) {
    if (a.nchunks == 0) return TLS_OK;
    if constexpr (sizeof(TW) == 4) {
      if (a.cap != 512) return tls_set_error(TLS_ERR_INVALID, "float32 W uses 512-edge chunk slabs");
      return chunks_cap<MODE, TW, 512>(a, x, s);
    } else {
      if (a.cap != 256) return tls_set_error(TLS_ERR_INVALID, "float64 W uses 256-edge chunk slabs");
      return chunks_cap<MODE, TW, 256>(a, x, s);
    }
  }
  template <typename TW, typename TV, typename TA>
  static int matvec(const tls_schur_args& a, const TV* x, TV* out, double* dots, int* gblocks, PcgState* pst,
                    cudaStream_t s) {
    static_assert(sizeof(TV) == 8, "reduced vectors are float64");
    int rc = chunks<0, TW>(a, reinterpret_cast<const double*>(x), s);
    if (rc) return rc;
    if (gblocks) *gblocks = a.nretained;
    if (a.nretained > 0) {
      if (!dots && !pst && light(a))
        schur_gather_warp_kernel<DR, 0, TV, double><<<(unsigned)((a.nretained + 7) / 8), 256, 0, s>>>(a, x, nullptr,
                                                                                                   out);
      else
        schur_gather_kernel<DR, 0, TV, double><<<a.nretained, 256, 0, s>>>(a, x, nullptr, out, dots, pst);
    }
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  }
  // many retained variables with few run partials each (merged small
  // problems): a warp per variable instead of a block
  static bool light(const tls_schur_args& a) {
    return a.nretained >= 4096 && (int64_t)a.nruns <= (int64_t)a.nretained * 64;
  }
  template <typename TW, typename TV, typename TA>
  static int rhs(const tls_schur_args& a, const double* b, TV* out, cudaStream_t s) {
    if (a.nelim > 0) schur_elim_rhs_kernel<DE><<<(a.nelim + 127) / 128, 128, 0, s>>>(a, b);
    TLS_CHECK_LAUNCH();
    int rc = chunks<1, TW>(a, nullptr, s);
    if (rc) return rc;
    if (a.nretained > 0) {
      if (light(a))
        schur_gather_warp_kernel<DR, 1, TV, double><<<(unsigned)((a.nretained + 7) / 8), 256, 0, s>>>(a, nullptr, b,
                                                                                                   out);
      else
        schur_gather_kernel<DR, 1, TV, double><<<a.nretained, 256, 0, s>>>(a, nullptr, b, out, nullptr, nullptr);
    }
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  }
  template <typename TW, int CAP, int D>
  static int pcg_go(const tls_schur_args& a, const PcgLoop& q, cudaStream_t s) {
    using S = SlabShape<DR, DE, CAP, TW, double>;
    if (a.meta_ints != S::kMetaInts) return tls_set_error(TLS_ERR_INVALID, "metadata slab size mismatch");
    if ((reinterpret_cast<uintptr_t>(a.w) & 15) || (reinterpret_cast<uintptr_t>(a.meta) & 15))
      return tls_set_error(TLS_ERR_INVALID, "W and metadata slabs must be 16-byte aligned");
    // Five float64 vectors of the reduced system in one CTA's shared memory,
    // and with them (one block per thread) the preconditioner factors and
    // block columns when they fit too; the kernel reads which from its
    // dynamic shared-memory size.
    constexpr int LD = D * (D + 1) / 2;
    const int64_t vec = q.n * 5 * (int64_t)sizeof(double);
    const int64_t blocks = (int64_t)kChunkThreads * (LD * (int64_t)sizeof(double) + D * (int64_t)sizeof(int));
    int64_t need = -1;
    if (q.nb <= kChunkThreads && vec + blocks <= kVectorSmemMax) need = vec + blocks;
    else if (vec <= kVectorSmemMax) need = vec;
    if (need >= 0) return pcg_launch<TW, CAP, D, true>(a, q, need > S::kBaseSmem ? (int)need : S::kBaseSmem, s);
    return pcg_launch<TW, CAP, D, false>(a, q, S::kBaseSmem, s);
  }
  template <typename TW, int CAP, int D, bool VC>
  static int pcg_launch(const tls_schur_args& a, const PcgLoop& q, int smem, cudaStream_t s) {
    auto k = VC ? schur_pcg_vc_kernel<DR, DE, CAP, TW, D> : schur_pcg_kernel<DR, DE, CAP, TW, D>;
    // co-resident CTAs (per-SM occupancy x SMs), per device and instantiation;
    // 0 when the device cannot launch cooperatively
    static DeviceGridCache cache;
    int grid = 0;
    const int rc = cache.get(smem, &grid, [&](int dev) -> int {
      // the largest dynamic size this kernel can take, so that the smem of any
      // later call (cached under its own key) stays within the attribute
      cudaFuncAttributes fa{};
      int optin = 0;
      cudaError_t e = cudaFuncGetAttributes(&fa, k);
      if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
      int per_sm = 0, sms = 0, coop = 0;
      if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e == cudaSuccess) e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
      if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kChunkThreads, smem);
      if (e != cudaSuccess) return -1;
      return (coop && per_sm > 0 && sms > 0) ? per_sm * sms : 0;
    });
    if (rc) return rc;
    if (grid <= 0) return tls_set_error(TLS_ERR_UNSUPPORTED, "cooperative launch unavailable");
    tls_schur_args aa = a;
    PcgLoop qq = q;
    void* args[] = {&aa, &qq};
    const cudaError_t e = cudaLaunchCooperativeKernel((const void*)k, dim3(grid), dim3(kChunkThreads), args,
                                                      (size_t)smem, s);
    if (e == cudaErrorCooperativeLaunchTooLarge) {
      cudaGetLastError();  // clear; the caller falls back to the multi-kernel loop
      return tls_set_error(TLS_ERR_UNSUPPORTED, "cooperative grid does not fit");
    }
    if (e != cudaSuccess) return tls_set_error(TLS_ERR_CUDA, cudaGetErrorString(e));
    tls_count_launch();
    return TLS_OK;
  }
  template <typename TW, int D>
  static int pcg_cap(const tls_schur_args& a, const PcgLoop& q, cudaStream_t s) {
    if constexpr (sizeof(TW) == 4) {
      if (a.cap != 512) return tls_set_error(TLS_ERR_INVALID, "float32 W uses 512-edge chunk slabs");
      return pcg_go<TW, 512, D>(a, q, s);
    } else {
      if (a.cap != 256) return tls_set_error(TLS_ERR_INVALID, "float64 W uses 256-edge chunk slabs");
      return pcg_go<TW, 256, D>(a, q, s);
    }
  }
  template <typename TW>
  static int pcg(const tls_schur_args& a, const PcgLoop& q, int maxdim, cudaStream_t s) {
    constexpr int DB = DR <= 3 ? 3 : (DR <= 6 ? 6 : 8);
    if (maxdim <= 1) return pcg_cap<TW, 1>(a, q, s);
    if (maxdim <= DB) return pcg_cap<TW, DB>(a, q, s);
    return tls_set_error(TLS_ERR_UNSUPPORTED, "preconditioner blocks wider than the retained blocks");
  }
  template <typename TW>
  static int damp(const tls_schur_args& a, cudaStream_t s) {
    cudaMemsetAsync(a.bad, 0, sizeof(int32_t), s);
    if (a.err) cudaMemsetAsync(a.err, 0, sizeof(int32_t), s);  // the error word describes this system
    if (a.nelim > 0) schur_factor_kernel<DE><<<(a.nelim + 127) / 128, 128, 0, s>>>(a);
    TLS_CHECK_LAUNCH();
    const int64_t nslab = (int64_t)a.nchunks * a.cap;
    if (nslab > 0) schur_whiten_kernel<DR, DE, TW><<<(unsigned)((nslab + 127) / 128), 128, 0, s>>>(a);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  }
  template <typename TW, typename TV>
  static int backsub(const tls_schur_args& a, const TV* xc, double* delta, cudaStream_t s) {
    const int64_t n = a.nelim > (int64_t)a.nretained * DR ? a.nelim : (int64_t)a.nretained * DR;
    if (n > 0) schur_backsub_kernel<DR, DE, TW, TV><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(a, xc, delta);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  }
  template <typename TW>
  static int precond(const tls_schur_args& a, double* out, cudaStream_t s) {
    if (a.nretained > 0) {
      if (a.nretained >= 4096 && a.nedges <= (int64_t)a.nretained * 1024)
        schur_precond_warp_kernel<DR, DE, TW><<<(unsigned)((a.nretained + 7) / 8), 256, 0, s>>>(a, out);
      else
        schur_precond_kernel<DR, DE, TW><<<a.nretained, 256, 0, s>>>(a, out);
    }
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
  TLS_D(2, 1)
  TLS_D(1, 3)
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

// The whole Schur-PCG loop (up to q.steps state-machine steps) in one
// cooperative launch; TLS_ERR_UNSUPPORTED when the block shapes have no
// persistent instantiation (the caller then runs the multi-kernel loop).
int tls_schur_pcg_launch(const tls_schur_args* a, const PcgLoop& q, int maxdim, cudaStream_t s) {
  if (a->vec_dtype != TLS_F64) return tls_set_error(TLS_ERR_UNSUPPORTED, "reduced Schur vectors are float64");
  if (a->nchunks == 0 || a->nretained == 0) return tls_set_error(TLS_ERR_UNSUPPORTED, "empty Schur system");
  auto go = [&](auto ops) -> int {
    using O = decltype(ops);
    return a->wdtype == TLS_F64 ? O::template pcg<double>(*a, q, maxdim, s) : O::template pcg<float>(*a, q, maxdim, s);
  };
  if (a->dr == 6 && a->de == 3) return go(SchurOps<6, 3>{});
  if (a->dr == 7 && a->de == 3) return go(SchurOps<7, 3>{});
  if (a->dr == 3 && a->de == 3) return go(SchurOps<3, 3>{});
  return tls_set_error(TLS_ERR_UNSUPPORTED, "no persistent Schur-PCG for these block dims");
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
