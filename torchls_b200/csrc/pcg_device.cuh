// Device pieces of the PCG state machine shared by the PCG driver kernels
// (pcg.cu) and the persistent Schur-PCG kernel (schur.cu): preconditioner
// block sets, the per-block update / preconditioner body, the decision and
// the direction update. The control flow mirrors torchls solvers.py:167-256.
#pragma once
#include "blocks.cuh"
#include "common.cuh"
#include "pcg_state.cuh"

namespace tls {

// Vector loads: plain, or L2-coherent (__ldcg) when another CTA of the same
// kernel may have written the value (persistent kernels).
template <bool COH, typename T>
__device__ __forceinline__ T ldv(const T* p) {
  if constexpr (COH) return __ldcg(p);
  else return *p;
}

struct BlockSet {
  int32_t ngroups;
  int32_t identity;                         // no preconditioner: unit blocks
  int64_t block_begin[TLS_MAX_GROUPS + 1];  // prefix of block counts
  tls_block_group g[TLS_MAX_GROUPS];
};

__device__ __forceinline__ int find_group(const BlockSet& bs, int64_t b) {
  int gi = 0;
  while (gi + 1 < bs.ngroups && b >= bs.block_begin[gi + 1]) ++gi;
  return gi;
}

// z = (L L^T)^-1 r for one block of runtime size dim <= D (registers only).
// The lower triangle is loaded into registers first (independent loads, one
// memory latency), then the two substitutions run from registers.
template <int D>
__device__ __forceinline__ void load_tri(const double* __restrict__ L, int dim, double (&l)[D * (D + 1) / 2]) {
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int k = 0; k <= i; ++k) l[i * (i + 1) / 2 + k] = (i < dim) ? __ldg(L + i * dim + k) : 1.0;
}

// z = (L L^T)^-1 r with the packed lower triangle l.
template <int D>
__device__ __forceinline__ void solve_tri(const double (&l)[D * (D + 1) / 2], int dim, const double (&r)[D],
                                          double (&z)[D]) {
  // the diagonal's reciprocals first: independent divisions, off the
  // substitution chains (which then only multiply)
  double inv[D];
#pragma unroll
  for (int i = 0; i < D; ++i) inv[i] = (i < dim) ? 1.0 / l[i * (i + 1) / 2 + i] : 0.0;
  double y[D];
#pragma unroll
  for (int i = 0; i < D; ++i) {
    double t = r[i];
#pragma unroll
    for (int k = 0; k < i; ++k) t -= (i < dim) ? l[i * (i + 1) / 2 + k] * y[k] : 0.0;
    y[i] = (i < dim) ? t * inv[i] : 0.0;
  }
#pragma unroll
  for (int i = D - 1; i >= 0; --i) {
    double t = y[i];
#pragma unroll
    for (int k = i + 1; k < D; ++k) t -= (k < dim) ? l[k * (k + 1) / 2 + i] * z[k] : 0.0;
    z[i] = (i < dim) ? t * inv[i] : 0.0;
  }
}

template <int D>
__device__ __forceinline__ void solve_block(const double* __restrict__ L, int dim, const double (&r)[D],
                                            double (&z)[D]) {
  double l[D * (D + 1) / 2];
  load_tri<D>(L, dim, l);
  solve_tri<D>(l, dim, r, z);
}

template <int D>
__device__ __forceinline__ void block_cols(const tls_block_group& g, int64_t i, int64_t (&cols)[D]) {
  int m = 0, start = 0;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    if (k < g.dim) {
      while (k >= start + g.member_dim[m]) {
        start += g.member_dim[m];
        ++m;
      }
      cols[k] = g.member_offset[m] + i * g.member_dim[m] + (k - start);
    } else {
      cols[k] = 0;
    }
  }
}

// ---------------------------------------------------------------- decision (last update block)
__device__ __forceinline__ void pcg_decide(PcgState* st, double s0, double s1, double s2) {
  tls_pcg_control& c = st->pub;
  st->action = A_NONE;
  if (c.status != TLS_PCG_ACTIVE || c.mode == M_DONE) return;
  const double thr = c.threshold;
  if (c.mode == M_ITER) {
    const double curv = c.curvature;
    const double rz = c.rz;
    const int it = ++c.iterations;
    if (!isfinite(curv) || !isfinite(rz)) {
      st->pending = TLS_PCG_NONFINITE;
      c.mode = M_FINAL;
      st->action = A_SWAP_TO_X;
      return;
    }
    if (curv <= 0.0 || rz <= 0.0) {
      st->pending = TLS_PCG_NONPOSITIVE;
      c.mode = M_FINAL;
      st->action = A_SWAP_TO_X;
      return;
    }
    c.rr = s0;
    c.rz_new = s1;
    const double rec = sqrt(s0);
    st->rec = rec;
    const bool periodic = c.check_interval > 0 && (it % c.check_interval) == 0;
    st->rec_hit = rec <= thr;
    st->periodic_hit = periodic;
    if (rec <= thr || periodic) {
      c.mode = M_CHECK;
      st->action = A_SWAP_TO_X;
      return;
    }
    if (it >= c.max_iterations) {
      c.mode = M_FINAL;
      st->action = A_SWAP_TO_X;
      return;
    }
    c.beta = s1 / rz;
    c.rz = s1;
    c.mode = M_ITER;
    st->action = A_DIR;
    return;
  }
  if (c.mode == M_CHECK) {
    const double tn = sqrt(s0);
    c.checks += 1;
    c.true_rr = s0;
    c.residual_norm = tn;
    if (!isfinite(tn)) {
      c.status = TLS_PCG_NONFINITE;
      c.mode = M_DONE;
      return;
    }
    if (tn <= thr) {
      c.status = TLS_PCG_CONVERGED;
      c.mode = M_DONE;
      return;
    }
    const double drift = sqrt(s1);
    c.drift_rr = s1;
    const bool last = c.iterations >= c.max_iterations;
    if (st->rec_hit || c.periodic || drift > c.drift_tolerance * fmax(tn, thr)) {
      c.rz = s2;
      c.rz_true = s2;
      c.restarts += 1;
      st->action = A_RESTART;
      c.mode = last ? M_FINAL : M_ITER;
      return;
    }
    c.beta = c.rz_new / c.rz;
    c.rz = c.rz_new;
    st->action = A_RESTORE_DIR;
    c.mode = last ? M_FINAL : M_ITER;
    return;
  }
  // M_FINAL
  const double tn = sqrt(s0);
  c.checks += 1;
  c.true_rr = s0;
  c.residual_norm = tn;
  if (isfinite(tn) && tn <= thr) c.status = TLS_PCG_CONVERGED;
  else if (!isfinite(tn)) c.status = TLS_PCG_NONFINITE;
  else c.status = st->pending;
  c.mode = M_DONE;
}

// One block's PCG vector work (block b of the set; `l` holds its packed
// factor when `have_l`, else it is loaded here):
// ITER: x += alpha p, r -= alpha Ap, z = M r; sums r.r, r.z.
// CHECK/FINAL: ap holds A x; true residual tr = rhs - A x (into ap), ztrue = M tr;
// sums tr.tr, (tr - r).(tr - r), tr.ztrue.
template <int D, typename TV, bool COH = false>
__device__ __forceinline__ void pcg_update_block(const BlockSet& bs, int64_t b, int mode, double alpha,
                                                 const TV* __restrict__ rhs, TV* x, TV* r, TV* z, const TV* p,
                                                 TV* ap, TV* ztrue, double (&l)[D * (D + 1) / 2], bool have_l,
                                                 double& a0, double& a1, double& a2) {
  const int gi = find_group(bs, b);
  const int64_t i = b - bs.block_begin[gi];
  const tls_block_group& g = bs.g[gi];
  const int dim = g.dim;
  int64_t cols[D];
  block_cols<D>(g, i, cols);
  // every load of the block before its first store (the stores may alias
  // the loads' arrays, so the compiler would otherwise order them one by one)
  const bool solve = mode != M_FINAL && !(bs.identity || g.factor == nullptr);
  if (solve && !have_l) load_tri<D>(g.factor + i * dim * dim, dim, l);
  double v0[D], v1[D], v2[D], v3[D];
#pragma unroll
  for (int k = 0; k < D; ++k) {
    v0[k] = v1[k] = v2[k] = v3[k] = 0.0;
    if (k < dim) {
      const int64_t col = cols[k];
      if (mode == M_ITER) {
        v0[k] = to_d(ldv<COH>(x + col));
        v1[k] = to_d(ldv<COH>(p + col));
      } else {
        v0[k] = to_d(rhs[col]);
      }
      v2[k] = to_d(ldv<COH>(r + col));
      v3[k] = to_d(ldv<COH>(ap + col));
    }
  }
  double rb[D], zb[D];
  if (mode == M_ITER) {
#pragma unroll
    for (int k = 0; k < D; ++k) {
      rb[k] = 0.0;
      if (k < dim) {
        const int64_t col = cols[k];
        x[col] = static_cast<TV>(v0[k] + alpha * v1[k]);
        const TV rn = static_cast<TV>(v2[k] - alpha * v3[k]);
        r[col] = rn;
        rb[k] = to_d(rn);
      }
    }
  } else {
#pragma unroll
    for (int k = 0; k < D; ++k) {
      rb[k] = 0.0;
      if (k < dim) {
        const int64_t col = cols[k];
        const TV tr = static_cast<TV>(v0[k] - v3[k]);
        ap[col] = tr;
        const double t = to_d(tr);
        rb[k] = t;
        a0 += t * t;
        const double dr = t - v2[k];
        a1 += dr * dr;
      }
    }
  }
  if (mode == M_FINAL) return;
  if (!solve) {
#pragma unroll
    for (int k = 0; k < D; ++k) zb[k] = rb[k];
  } else {
    solve_tri<D>(l, dim, rb, zb);
  }
  TV* zdst = (mode == M_ITER) ? z : ztrue;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    if (k < dim) {
      const TV zk = static_cast<TV>(zb[k]);
      zdst[cols[k]] = zk;
      const double zd = to_d(zk);
      if (mode == M_ITER) {
        a0 += rb[k] * rb[k];
        a1 += rb[k] * zd;
      } else {
        a2 += rb[k] * zd;
      }
    }
  }
}

// The PCG vector work of blocks [b0, nblocks) with stride `step` (see
// pcg_update_block).
template <int D, typename TV, bool COH = false>
__device__ __forceinline__ void pcg_update_blocks(const BlockSet& bs, int64_t nblocks, int64_t b0, int64_t step,
                                                  int mode, double alpha, const TV* __restrict__ rhs, TV* x, TV* r,
                                                  TV* z, const TV* p, TV* ap, TV* ztrue, double& a0, double& a1,
                                                  double& a2) {
  for (int64_t b = b0; b < nblocks; b += step) {
    double l[D * (D + 1) / 2];
    pcg_update_block<D, TV, COH>(bs, b, mode, alpha, rhs, x, r, z, p, ap, ztrue, l, false, a0, a1, a2);
  }
}

// Load block b's packed factor into `l` ahead of its update (false when the
// step's mode solves no block or the set has no factors).
template <int D>
__device__ __forceinline__ bool pcg_prefetch_factor(const BlockSet& bs, int64_t b, int mode,
                                                    double (&l)[D * (D + 1) / 2]) {
  if (mode == M_FINAL || bs.identity) return false;
  const int gi = find_group(bs, b);
  const tls_block_group& g = bs.g[gi];
  if (g.factor == nullptr) return false;
  const int64_t i = b - bs.block_begin[gi];
  load_tri<D>(g.factor + i * g.dim * g.dim, g.dim, l);
  return true;
}

// Direction / restart / swap for elements [i0, n) with stride `step`.
template <typename TV, bool COH = false>
__device__ __forceinline__ void pcg_direction_elems(int64_t n, int64_t i0, int64_t step, int action, double beta,
                                                    bool to_final, const TV* x, TV* r, const TV* z, TV* p, TV* psave,
                                                    const TV* ap, const TV* ztrue) {
  for (int64_t i = i0; i < n; i += step) {
    switch (action) {
      case A_DIR:
        p[i] = static_cast<TV>(to_d(ldv<COH>(z + i)) + beta * to_d(ldv<COH>(p + i)));
        break;
      case A_RESTART:
        r[i] = ldv<COH>(ap + i);
        p[i] = ldv<COH>(ztrue + i);
        break;
      case A_RESTORE_DIR:
        p[i] = static_cast<TV>(to_d(ldv<COH>(z + i)) + beta * to_d(ldv<COH>(psave + i)));
        break;
      case A_SWAP_TO_X:
        psave[i] = ldv<COH>(p + i);
        p[i] = ldv<COH>(x + i);
        break;
    }
    if (to_final) p[i] = ldv<COH>(x + i);
  }
}

// Arguments of the persistent Schur-PCG loop (schur.cu).
struct PcgLoop {
  BlockSet bs;
  int64_t nb;
  int64_t n;
  PcgState* st;
  const double* rhs;
  double* x;
  double* r;
  double* z;
  double* p;
  double* psave;
  double* ap;
  double* ztrue;
  double* dots;  // [nretained] x.Ap partials
  int32_t steps;
};

}  // namespace tls

int tls_schur_pcg_launch(const tls_schur_args* a, const tls::PcgLoop& q, int maxdim, cudaStream_t s);
