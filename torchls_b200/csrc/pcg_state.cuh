// Device-side PCG state shared by the PCG driver and the operators' final
// kernels (which finalise the curvature p.Ap in their last block).
#pragma once
#include "common.cuh"

namespace tls {

enum { M_ITER = 0, M_CHECK = 1, M_FINAL = 2, M_DONE = 3 };
enum { A_NONE = 0, A_DIR = 1, A_RESTART = 2, A_RESTORE_DIR = 3, A_SWAP_TO_X = 4 };

// tls_pcg_control first (read by the host), then private fields.
struct PcgState {
  tls_pcg_control pub;
  int32_t action;        // direction-kernel action decided by the update kernel
  int32_t pending;       // reason when the loop broke early
  int32_t op_blocks;     // number of operator dot partials
  int32_t upd_blocks;    // number of update partial blocks
  double rec;            // recurrence norm of the last iteration
  int32_t rec_hit;       // rec <= threshold at the last iteration
  int32_t periodic_hit;  // periodic check due at the last iteration
  int32_t alpha_ok;      // curvature and r.z finite and positive this step
  uint32_t ticket_op;    // last-block-done counters (reset by the last block)
  uint32_t ticket_upd;
  uint32_t bar_count;    // grid barrier of the persistent Schur-PCG kernel
  uint32_t bar_gen;
  uint32_t bar_count2;   // arrivals the vector CTA waits for (persistent kernel)
  uint32_t pad2_;
};

// Deterministic sum of p[0..n) by one block (fixed strided order, fixed tree).
// Loads bypass L1: the values were written by other blocks of this kernel.
// Four strides per round are loaded together; the sum runs in stride order.
template <int BLOCK>
__device__ __forceinline__ double block_sum_cg(const double* p, int n, double* sm) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += 4 * BLOCK) {
    double v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = i + u * BLOCK < n ? __ldcg(p + i + u * BLOCK) : 0.0;
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (i + u * BLOCK < n) acc += v[u];
  }
  return block_sum<BLOCK>(acc, sm);
}

// block_sum_cg of three arrays of n values in one pass: bitwise the three
// calls' results (same strided order per thread, same tree), with four
// strides of all three arrays in flight per round and two barriers instead of
// six. Valid in thread 0.
template <int BLOCK>
__device__ __forceinline__ void block_sum3_cg(const double* p0, const double* p1, const double* p2, int n,
                                              double& s0, double& s1, double& s2, double (*sm)[BLOCK / 32]) {
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int i = threadIdx.x; i < n; i += 4 * BLOCK) {
    double v0[4], v1[4], v2[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int j = i + u * BLOCK;
      v0[u] = j < n ? __ldcg(p0 + j) : 0.0;
      v1[u] = j < n ? __ldcg(p1 + j) : 0.0;
      v2[u] = j < n ? __ldcg(p2 + j) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (i + u * BLOCK < n) {
        a0 += v0[u];
        a1 += v1[u];
        a2 += v2[u];
      }
    }
  }
  block_sum3<BLOCK>(a0, a1, a2, sm);
  s0 = a0;
  s1 = a1;
  s2 = a2;
}

// Called by every block of an operator's final kernel after thread 0 stored
// the block's dot partial. The last block to finish computes the curvature
// p.Ap (the sum of the first `nsum` partials; default: one per block of this
// kernel) and alpha = r.z / p.Ap for the PCG update (threadfence reduction).
template <int BLOCK>
__device__ __forceinline__ void pcg_operator_epilogue(PcgState* st, const double* partials, int nblocks,
                                                      double* sm, int nsum = -1) {
  __shared__ int last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&st->ticket_op, 1u) == (unsigned)(nblocks - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  const double curv = block_sum_cg<BLOCK>(partials, nsum < 0 ? nblocks : nsum, sm);
  if (threadIdx.x == 0) {
    st->ticket_op = 0;
    tls_pcg_control& c = st->pub;
    if (c.status == TLS_PCG_ACTIVE && c.mode == M_ITER) {
      const double rz = c.rz;
      c.curvature = curv;
      const bool ok = isfinite(curv) && isfinite(rz) && curv > 0.0 && rz > 0.0;
      st->alpha_ok = ok;
      c.alpha = ok ? rz / curv : 0.0;
    } else {
      st->alpha_ok = 0;
    }
  }
}

}  // namespace tls
