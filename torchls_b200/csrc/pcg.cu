// Block-Jacobi factor/apply and the device-resident PCG state machine.
//
// The PCG mirrors torchls solvers.py:167-256 step for step: x0 = 0,
// threshold = max(atol, rtol |b|), stop on nonfinite or nonpositive
// curvature, a true-residual check when the recurrence converges or every
// `check_interval` iterations, restarts on drift (adaptive) or always
// (periodic), and a final true-residual check. Every decision is taken on the
// device from float64 scalars reduced in a fixed order, so a run needs no
// host synchronisation and is bitwise reproducible.
//
// One state-machine step is three kernels:
//   operator   ap = A p; its last block finalises curvature and alpha
//   update     x, r (or the true residual), z = M r, partial norms; its last
//              block takes the step's decision (converged, check, restart...)
//   direction  p = z + beta p, restart, or swap p <-> x for a residual check
// During a true-residual check p temporarily holds x (the operator always
// reads p); the saved direction is restored if the iteration continues.
#include <type_traits>

#include <map>

#include "blocks.cuh"
#include "common.cuh"
#include "pcg_device.cuh"
#include "pcg_state.cuh"

int tls_normal_apply(const tls_normal_args* a, const void* x, void* y, double* dot_partials, int* gather_blocks,
                     void* pcg_state, cudaStream_t st);
int tls_schur_apply(const tls_schur_args* a, const void* x, void* out, double* dot_partials, int* gather_blocks,
                    void* pcg_state, cudaStream_t st);
int tls_normal_gather_blocks(const tls_normal_args* a);
int tls_schur_general_apply(const tls_schur_general_args* a, const double* x, double* out, double* dots,
                            int* gblocks, void* pcg_state, cudaStream_t s);
int tls_schur_general_ret_blocks(const tls_schur_general_args* a);

namespace tls {

constexpr int kUpdThreads = 128;
constexpr int kMaxUpdBlocks = 1024;
// partials layout: [0, kOpPartials) operator dots; update partials at
// kOpPartials + k * kMaxUpdBlocks (k = 0, 1, 2).
constexpr int kOpPartials = 65536;

// ---------------------------------------------------------------- start
template <typename TV>
__global__ void __launch_bounds__(kUpdThreads) pcg_init_kernel(int64_t n, const TV* __restrict__ rhs, TV* x, TV* r,
                                                               double* partials) {
  __shared__ double sm[kUpdThreads / 32];
  double acc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const TV v = rhs[i];
    x[i] = TV(0);
    r[i] = v;
    acc += to_d(v) * to_d(v);
  }
  const double s = block_sum<kUpdThreads>(acc, sm);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void __launch_bounds__(256) pcg_init_finish_kernel(PcgState* st, const double* partials, int blocks,
                                                              double rtol, double atol, int max_it, int interval,
                                                              int periodic, double drift_tol) {
  __shared__ double sm[8];
  double acc = 0.0;
  for (int i = threadIdx.x; i < blocks; i += 256) acc += partials[i];
  const double ss = block_sum<256>(acc, sm);
  if (threadIdx.x != 0) return;
  tls_pcg_control& c = st->pub;
  const double nrm = sqrt(ss);
  c.rhs_norm = nrm;
  c.threshold = fmax(atol, rtol * nrm);
  c.residual_norm = nrm;
  c.iterations = 0;
  c.restarts = 0;
  c.checks = 0;
  c.max_iterations = max_it;
  c.check_interval = interval;
  c.periodic = periodic;
  c.drift_tolerance = drift_tol;
  c.status = TLS_PCG_ACTIVE;
  c.mode = M_ITER;
  st->action = A_NONE;
  st->pending = TLS_PCG_MAX_ITERATIONS;
  st->rec = nrm;
  st->rec_hit = 0;
  st->periodic_hit = 0;
  st->alpha_ok = 0;
  st->ticket_op = 0;
  st->ticket_upd = 0;
  st->bar_count = 0;
  st->bar_count2 = 0;
  if (!isfinite(nrm)) {
    c.status = TLS_PCG_NONFINITE;
    c.mode = M_DONE;
  } else if (nrm <= c.threshold) {
    c.status = TLS_PCG_CONVERGED;
    c.mode = M_DONE;
  }
}

// z = M r, p = z, partial r.z (only while ACTIVE)
template <int D, typename TV>
__global__ void __launch_bounds__(kUpdThreads) pcg_precondition_kernel(BlockSet bs, int64_t nblocks, const PcgState* st,
                                                                       const TV* r, TV* z, TV* p, double* partials) {
  __shared__ double sm[kUpdThreads / 32];
  double acc = 0.0;
  if (st->pub.status == TLS_PCG_ACTIVE) {
    for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nblocks;
         b += (int64_t)gridDim.x * blockDim.x) {
      const int gi = find_group(bs, b);
      const int64_t i = b - bs.block_begin[gi];
      const tls_block_group& g = bs.g[gi];
      int64_t cols[D];
      block_cols<D>(g, i, cols);
      double rb[D], zb[D];
#pragma unroll
      for (int k = 0; k < D; ++k) rb[k] = (k < g.dim) ? to_d(r[cols[k]]) : 0.0;
      if (bs.identity || g.factor == nullptr) {
#pragma unroll
        for (int k = 0; k < D; ++k) zb[k] = rb[k];
      } else {
        solve_block<D>(g.factor + i * g.dim * g.dim, g.dim, rb, zb);
      }
#pragma unroll
      for (int k = 0; k < D; ++k) {
        if (k < g.dim) {
          const TV zk = static_cast<TV>(zb[k]);
          z[cols[k]] = zk;
          p[cols[k]] = zk;
          acc += rb[k] * to_d(zk);
        }
      }
    }
  }
  const double s = block_sum<kUpdThreads>(acc, sm);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void pcg_rz_finish_kernel(PcgState* st, const double* partials, int blocks) {
  if (threadIdx.x != 0) return;
  if (st->pub.status != TLS_PCG_ACTIVE) return;
  double s = 0.0;
  for (int i = 0; i < blocks; ++i) s += partials[i];
  st->pub.rz = s;
}

// ---------------------------------------------------------------- update
// The block update for one preconditioner group of `count` blocks of one
// member, each block D contiguous columns and a D x D factor: the operations
// and order of pcg_update_block, but every vector and factor row is read and
// written in pairs (float2 / double2; the host checks the alignment): half
// the memory instructions and 114 registers instead of 166, so four CTAs fit
// an SM instead of three. Compiled from a different code shape, its results
// differ from the general path's at rounding level (both are deterministic).
template <typename TV>
struct Pair;
template <>
struct Pair<float> {
  using type = float2;
};
template <>
struct Pair<double> {
  using type = double2;
};

template <int D, typename TV>
__device__ __forceinline__ void pcg_update_uniform(const tls_block_group& g, int64_t nblocks, int64_t b0,
                                                   int64_t step, int mode, double alpha, const TV* __restrict__ rhs,
                                                   TV* x, TV* r, TV* z, const TV* p, TV* ap, TV* ztrue, double& a0,
                                                   double& a1, double& a2) {
  static_assert(D % 2 == 0, "pairs");
  using P2 = typename Pair<TV>::type;
  constexpr int H = D / 2, LD = D * (D + 1) / 2;
  for (int64_t b = b0; b < nblocks; b += step) {
    const int64_t base = g.member_offset[0] + b * D;
    double l[LD];
    if (mode != M_FINAL) {
      const double* L = g.factor + b * D * D;
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int c2 = 0; c2 <= i / 2; ++c2) {
          const double2 v = __ldg(reinterpret_cast<const double2*>(L + i * D) + c2);
          l[i * (i + 1) / 2 + 2 * c2] = v.x;
          if (2 * c2 + 1 <= i) l[i * (i + 1) / 2 + 2 * c2 + 1] = v.y;
        }
    }
    double v0[D], v1[D], v2[D], v3[D];
    const P2* src0 = reinterpret_cast<const P2*>((mode == M_ITER ? x : rhs) + base);
#pragma unroll
    for (int h = 0; h < H; ++h) {
      const P2 q0 = src0[h];
      const P2 q2 = reinterpret_cast<const P2*>(r + base)[h];
      const P2 q3 = reinterpret_cast<const P2*>(ap + base)[h];
      v0[2 * h] = to_d(q0.x), v0[2 * h + 1] = to_d(q0.y);
      v2[2 * h] = to_d(q2.x), v2[2 * h + 1] = to_d(q2.y);
      v3[2 * h] = to_d(q3.x), v3[2 * h + 1] = to_d(q3.y);
      if (mode == M_ITER) {
        const P2 q1 = reinterpret_cast<const P2*>(p + base)[h];
        v1[2 * h] = to_d(q1.x), v1[2 * h + 1] = to_d(q1.y);
      } else {
        v1[2 * h] = v1[2 * h + 1] = 0.0;
      }
    }
    // pcg_update_block's arithmetic in its form (guards on the runtime block
    // size included)
    const int dim = g.dim;
    double rb[D], zb[D];
    if (mode == M_ITER) {
      TV xn[D], rn[D];
#pragma unroll
      for (int k = 0; k < D; ++k) {
        rb[k] = 0.0;
        xn[k] = rn[k] = TV(0);
        if (k < dim) {
          xn[k] = static_cast<TV>(v0[k] + alpha * v1[k]);
          rn[k] = static_cast<TV>(v2[k] - alpha * v3[k]);
          rb[k] = to_d(rn[k]);
        }
      }
#pragma unroll
      for (int h = 0; h < H; ++h) {
        reinterpret_cast<P2*>(x + base)[h] = P2{xn[2 * h], xn[2 * h + 1]};
        reinterpret_cast<P2*>(r + base)[h] = P2{rn[2 * h], rn[2 * h + 1]};
      }
    } else {
      TV tr[D];
#pragma unroll
      for (int k = 0; k < D; ++k) {
        rb[k] = 0.0;
        tr[k] = TV(0);
        if (k < dim) {
          tr[k] = static_cast<TV>(v0[k] - v3[k]);
          const double t = to_d(tr[k]);
          rb[k] = t;
          a0 += t * t;
          const double dr = t - v2[k];
          a1 += dr * dr;
        }
      }
#pragma unroll
      for (int h = 0; h < H; ++h) reinterpret_cast<P2*>(ap + base)[h] = P2{tr[2 * h], tr[2 * h + 1]};
    }
    if (mode == M_FINAL) continue;
    solve_tri<D>(l, dim, rb, zb);
    TV zt[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
      zt[k] = TV(0);
      if (k < dim) {
        zt[k] = static_cast<TV>(zb[k]);
        const double zd = to_d(zt[k]);
        if (mode == M_ITER) {
          a0 += rb[k] * rb[k];
          a1 += rb[k] * zd;
        } else {
          a2 += rb[k] * zd;
        }
      }
    }
    TV* zdst = (mode == M_ITER) ? z : ztrue;
#pragma unroll
    for (int h = 0; h < H; ++h) reinterpret_cast<P2*>(zdst + base)[h] = P2{zt[2 * h], zt[2 * h + 1]};
  }
}

template <int D, typename TV, bool UNI>
__global__ void __launch_bounds__(kUpdThreads) pcg_update_kernel(BlockSet bs, int64_t nblocks, PcgState* st,
                                                                 const TV* __restrict__ rhs, TV* x, TV* r, TV* z,
                                                                 const TV* p, TV* ap, TV* ztrue,
                                                                 double* partials) {
  __shared__ double sm3[3][kUpdThreads / 32];
  __shared__ int last;
  const tls_pcg_control& c = st->pub;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  const int mode = c.mode;
  bool work = c.status == TLS_PCG_ACTIVE && mode != M_DONE;
  double alpha = 0.0;
  if (work && mode == M_ITER) {
    if (!st->alpha_ok) work = false;
    else alpha = c.alpha;
  }
  if (work) {
    const int64_t b0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, step = (int64_t)gridDim.x * blockDim.x;
    if constexpr (UNI)
      pcg_update_uniform<D, TV>(bs.g[0], nblocks, b0, step, mode, alpha, rhs, x, r, z, p, ap, ztrue, a0, a1, a2);
    else
      pcg_update_blocks<D, TV>(bs, nblocks, b0, step, mode, alpha, rhs, x, r, z, p, ap, ztrue, a0, a1, a2);
  }
  double* up = partials + kOpPartials;
  block_sum3<kUpdThreads>(a0, a1, a2, sm3);
  if (threadIdx.x == 0) {
    up[blockIdx.x] = a0;
    up[kMaxUpdBlocks + blockIdx.x] = a1;
    up[2 * kMaxUpdBlocks + blockIdx.x] = a2;
  }
  // last block to finish takes the step's decision
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&st->ticket_upd, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  double t0, t1, t2;
  block_sum3_cg<kUpdThreads>(up, up + kMaxUpdBlocks, up + 2 * kMaxUpdBlocks, gridDim.x, t0, t1, t2, sm3);
  if (threadIdx.x == 0) {
    st->ticket_upd = 0;
    pcg_decide(st, t0, t1, t2);
  }
}

// Direction / restart / swap. When the next mode is FINAL after a restart or
// a direction update, p is additionally replaced by x (the operator reads p).
template <typename TV>
__global__ void __launch_bounds__(256) pcg_direction_kernel(int64_t n, const PcgState* st, const TV* x, TV* r,
                                                            const TV* z, TV* p, TV* psave, const TV* ap,
                                                            const TV* ztrue) {
  const int action = st->action;
  if (action == A_NONE) return;
  const bool to_final = st->pub.mode == M_FINAL && action != A_SWAP_TO_X;
  pcg_direction_elems<TV>(n, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x,
                          action, st->pub.beta, to_final, x, r, z, p, psave, ap, ztrue);
}

// Small systems (few preconditioner blocks): the whole post-operator part of a
// PCG step in ONE block -- update, preconditioner, dot products, decision and
// direction -- without grid-wide atomics or a second launch.
constexpr int kSmallThreads = 512;
constexpr int64_t kSmallMaxBlocks = 8192;

template <int D, typename TV>
__global__ void __launch_bounds__(kSmallThreads) pcg_step_small_kernel(BlockSet bs, int64_t nblocks, int64_t n,
                                                                       PcgState* st, const TV* __restrict__ rhs,
                                                                       TV* x, TV* r, TV* z, TV* p, TV* psave, TV* ap,
                                                                       TV* ztrue) {
  __shared__ int s_action, s_tofinal;
  __shared__ double s_beta;
  const tls_pcg_control& c = st->pub;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  const int mode = c.mode;
  bool work = c.status == TLS_PCG_ACTIVE && mode != M_DONE;
  double alpha = 0.0;
  if (work && mode == M_ITER) {
    if (!st->alpha_ok) work = false;
    else alpha = c.alpha;
  }
  if (work)
    pcg_update_blocks<D, TV>(bs, nblocks, threadIdx.x, kSmallThreads, mode, alpha, rhs, x, r, z, p, ap, ztrue, a0,
                             a1, a2);
  __shared__ double sm3[3][kSmallThreads / 32];
  block_sum3<kSmallThreads>(a0, a1, a2, sm3);
  const double t0 = a0, t1 = a1, t2 = a2;
  if (threadIdx.x == 0) {
    pcg_decide(st, t0, t1, t2);
    s_action = st->action;
    s_beta = st->pub.beta;
    s_tofinal = st->pub.mode == M_FINAL && st->action != A_SWAP_TO_X;
  }
  __syncthreads();
  if (s_action == A_NONE) return;
  pcg_direction_elems<TV>(n, threadIdx.x, kSmallThreads, s_action, s_beta, s_tofinal != 0, x, r, z, p, psave, ap,
                          ztrue);
}

__host__ BlockSet make_blocks(const tls_pcg_args* a, int64_t* total, int* maxdim) {
  BlockSet bs{};
  int64_t nb = 0;
  *maxdim = 1;
  if (a->pre == nullptr || a->npre == 0) {
    bs.identity = 1;
    bs.ngroups = 1;
    bs.g[0].count = (int32_t)a->n;
    bs.g[0].dim = 1;
    bs.g[0].nmembers = 1;
    bs.g[0].member_offset[0] = 0;
    bs.g[0].member_dim[0] = 1;
    bs.block_begin[0] = 0;
    bs.block_begin[1] = a->n;
    *total = a->n;
    return bs;
  }
  bs.ngroups = a->npre;
  for (int i = 0; i < a->npre; ++i) {
    bs.g[i] = a->pre[i];
    bs.block_begin[i] = nb;
    nb += a->pre[i].count;
    if (a->pre[i].dim > *maxdim) *maxdim = a->pre[i].dim;
  }
  bs.block_begin[a->npre] = nb;
  *total = nb;
  return bs;
}

// One group of one member, every block D contiguous columns with a D x D
// factor, and every vector and factor row 16-byte aligned: the paired
// update (pcg_update_uniform) applies.
static bool uniform_blocks(const tls_pcg_args* a, const BlockSet& bs, int D) {
  if (bs.identity || bs.ngroups != 1) return false;
  const tls_block_group& g = bs.g[0];
  if (g.nmembers != 1 || g.dim != D || g.member_dim[0] != D || g.factor == nullptr) return false;
  if (g.member_offset[0] % 2 != 0) return false;
  const void* ptrs[] = {a->rhs, a->x, a->r, a->z, a->p, a->ap, a->ztrue, g.factor};
  for (const void* q : ptrs)
    if (reinterpret_cast<uintptr_t>(q) % 16 != 0) return false;
  return true;
}

static int grid_of(int64_t n, int block, int cap) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

template <typename F>
static int with_dim(int maxdim, F&& f) {
  if (maxdim <= 1) return f(std::integral_constant<int, 1>{});
  if (maxdim <= 3) return f(std::integral_constant<int, 3>{});
  if (maxdim <= 6) return f(std::integral_constant<int, 6>{});
  if (maxdim <= 8) return f(std::integral_constant<int, 8>{});
  if (maxdim <= 16) return f(std::integral_constant<int, 16>{});
  return tls_set_error(TLS_ERR_UNSUPPORTED, "preconditioner block dim > 16");
}

template <typename TV>
static int pcg_start_t(const tls_pcg_args* a, double rtol, double atol, int max_it, int interval, int periodic,
                       double drift, cudaStream_t s) {
  PcgState* st = reinterpret_cast<PcgState*>(a->control);
  const int g = grid_of(a->n, kUpdThreads, kMaxUpdBlocks);
  double* scratch = a->partials + kOpPartials;
  pcg_init_kernel<TV><<<g, kUpdThreads, 0, s>>>(a->n, (const TV*)a->rhs, (TV*)a->x, (TV*)a->r, scratch);
  TLS_CHECK_LAUNCH();
  pcg_init_finish_kernel<<<1, 256, 0, s>>>(st, scratch, g, rtol, atol, max_it, interval, periodic, drift);
  TLS_CHECK_LAUNCH();
  int64_t nb;
  int maxdim;
  BlockSet bs = make_blocks(a, &nb, &maxdim);
  const int gb = grid_of(nb, kUpdThreads, kMaxUpdBlocks);
  return with_dim(maxdim, [&](auto dim) -> int {
    constexpr int D = decltype(dim)::value;
    pcg_precondition_kernel<D, TV><<<gb, kUpdThreads, 0, s>>>(bs, nb, st, (const TV*)a->r, (TV*)a->z, (TV*)a->p,
                                                              scratch);
    TLS_CHECK_LAUNCH();
    pcg_rz_finish_kernel<<<1, 32, 0, s>>>(st, scratch, gb);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  });
}

__global__ void set_block_counts_kernel(PcgState* st, int op_blocks, int upd_blocks) {
  st->op_blocks = op_blocks;
  st->upd_blocks = upd_blocks;
}

// Number of dot partials the operator's final kernel writes (one per block).
static int operator_blocks(const tls_pcg_args* a) {
  if (a->op_kind == 0) return tls_normal_gather_blocks(a->normal);
  if (a->op_kind == 2) return tls_schur_general_ret_blocks(a->schur_general);
  return a->schur->nretained;  // one gather block per retained variable
}

// CUDA-graph replay of the queued PCG steps: the steps are recorded on a
// private capture stream of this thread and device, the recording updates the
// thread's executable graph (instantiated again only when the topology
// changes) and the graph is launched on the caller's stream. The kernels and
// their order are exactly those of direct launches. When the caller's stream
// is itself being captured, or recording fails (an API call that cannot be
// captured, such as a first-use attribute setting), the steps are launched
// directly; after repeated failures the thread stops trying. The executable
// graphs live until the process exits.
struct GraphSlot {
  cudaStream_t cap = nullptr;
  cudaGraphExec_t exec = nullptr;
  int failures = 0;
  uint64_t key = 0;      // graph_key the executable graph was recorded for (0: none)
  int steps = -1;        // and its step count
  long long launches = 0;  // this library's kernels in it
};

// `key` nonzero: a call with the slot's key and step count launches the
// recorded graph again (the caller guarantees identical arguments).
template <typename F>
static int replay_steps(F&& enqueue, cudaStream_t s, uint64_t key, int steps) {
  thread_local std::map<int, GraphSlot> slots;
  int dev = 0;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaStreamIsCapturing(s, &cs) != cudaSuccess ||
      cs != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return enqueue(s);
  }
  GraphSlot& g = slots[dev];
  if (g.failures >= 3) return enqueue(s);
  if (key != 0 && g.exec && g.key == key && g.steps == steps) {
    const cudaError_t e = cudaGraphLaunch(g.exec, s);
    if (e != cudaSuccess) return tls_set_cuda_error(e);
    tls_count_launches(g.launches);
    return TLS_OK;
  }
  g.key = 0;
  if (!g.cap && cudaStreamCreateWithFlags(&g.cap, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    g.cap = nullptr;
    g.failures = 3;
    return enqueue(s);
  }
  cudaGraph_t graph = nullptr;
  int rc = TLS_OK;
  const long long launches0 = tls_launches_now();
  cudaError_t e = cudaStreamBeginCapture(g.cap, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    rc = enqueue(g.cap);
    e = cudaStreamEndCapture(g.cap, &graph);
  }
  const long long recorded = tls_launches_now() - launches0;
  if (rc != TLS_OK || e != cudaSuccess || graph == nullptr) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    ++g.failures;
    return enqueue(s);  // the same steps, launched directly
  }
  if (g.exec) {
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(g.exec, graph, &info) != cudaSuccess) {
      cudaGetLastError();
      cudaGraphExecDestroy(g.exec);
      g.exec = nullptr;
    }
  }
  if (!g.exec && cudaGraphInstantiate(&g.exec, graph, 0) != cudaSuccess) {
    cudaGetLastError();
    g.exec = nullptr;
    cudaGraphDestroy(graph);
    ++g.failures;
    return enqueue(s);
  }
  cudaGraphDestroy(graph);
  e = cudaGraphLaunch(g.exec, s);
  if (e != cudaSuccess) return tls_set_cuda_error(e);
  g.failures = 0;
  g.key = key;
  g.steps = steps;
  g.launches = recorded;
  return TLS_OK;
}

template <typename TV>
static int pcg_run_t(const tls_pcg_args* a, int steps, cudaStream_t s) {
  PcgState* st = reinterpret_cast<PcgState*>(a->control);
  int64_t nb;
  int maxdim;
  BlockSet bs = make_blocks(a, &nb, &maxdim);
  const int gb = grid_of(nb, kUpdThreads, kMaxUpdBlocks);
  const int gd = grid_of(a->n, 256, 148 * 8);
  const int op_blocks = operator_blocks(a);
  if (op_blocks > kOpPartials) return tls_set_error(TLS_ERR_UNSUPPORTED, "operator uses too many blocks");
  set_block_counts_kernel<<<1, 1, 0, s>>>(st, op_blocks, gb);
  TLS_CHECK_LAUNCH();
  if constexpr (sizeof(TV) == 8) {
    // small Schur systems: the whole loop in one persistent cooperative launch
    if (a->op_kind == 1 && nb <= kSmallMaxBlocks && steps > 0) {
      PcgLoop q{};
      q.bs = bs;
      q.nb = nb;
      q.n = a->n;
      q.st = st;
      q.rhs = (const double*)a->rhs;
      q.x = (double*)a->x;
      q.r = (double*)a->r;
      q.z = (double*)a->z;
      q.p = (double*)a->p;
      q.psave = (double*)a->psave;
      q.ap = (double*)a->ap;
      q.ztrue = (double*)a->ztrue;
      q.dots = a->partials;
      q.steps = steps;
      const int rc = tls_schur_pcg_launch(a->schur, q, maxdim, s);
      if (rc != TLS_ERR_UNSUPPORTED) return rc;
    }
  }
  // multi-kernel path: at most 16 queued steps per call (the host polls between calls)
  if (steps > 16) steps = 16;
  auto enqueue = [&](cudaStream_t s) -> int {
  return with_dim(maxdim, [&](auto dim) -> int {
    constexpr int D = decltype(dim)::value;
    const bool uni = D % 2 == 0 && uniform_blocks(a, bs, D);  // the paired update
    for (int k = 0; k < steps; ++k) {
      int launched = 0;
      int rc;
      if (a->op_kind == 0) {
        rc = tls_normal_apply(a->normal, a->p, a->ap, a->partials, &launched, st, s);
      } else if (a->op_kind == 2) {
        if (a->vec_dtype != TLS_F64) return tls_set_error(TLS_ERR_UNSUPPORTED, "general Schur vectors are float64");
        rc = tls_schur_general_apply(a->schur_general, (const double*)a->p, (double*)a->ap, a->partials, &launched,
                                     st, s);
      } else {
        rc = tls_schur_apply(a->schur, a->p, a->ap, a->partials, &launched, st, s);
      }
      if (rc) return rc;
      if (launched != op_blocks) return tls_set_error(TLS_ERR_INVALID, "operator block count changed");
      if (nb <= kSmallMaxBlocks) {
        pcg_step_small_kernel<D, TV><<<1, kSmallThreads, 0, s>>>(bs, nb, a->n, st, (const TV*)a->rhs, (TV*)a->x,
                                                                 (TV*)a->r, (TV*)a->z, (TV*)a->p, (TV*)a->psave,
                                                                 (TV*)a->ap, (TV*)a->ztrue);
        TLS_CHECK_LAUNCH();
        continue;
      }
      if (uni)
        pcg_update_kernel<D, TV, (D % 2 == 0)><<<gb, kUpdThreads, 0, s>>>(bs, nb, st, (const TV*)a->rhs,
                                                                          (TV*)a->x, (TV*)a->r, (TV*)a->z,
                                                                          (const TV*)a->p, (TV*)a->ap,
                                                                          (TV*)a->ztrue, a->partials);
      else
        pcg_update_kernel<D, TV, false><<<gb, kUpdThreads, 0, s>>>(bs, nb, st, (const TV*)a->rhs, (TV*)a->x,
                                                                   (TV*)a->r, (TV*)a->z, (const TV*)a->p,
                                                                   (TV*)a->ap, (TV*)a->ztrue, a->partials);
      TLS_CHECK_LAUNCH();
      pcg_direction_kernel<TV><<<gd, 256, 0, s>>>(a->n, st, (const TV*)a->x, (TV*)a->r, (const TV*)a->z, (TV*)a->p,
                                                  (TV*)a->psave, (const TV*)a->ap, (const TV*)a->ztrue);
      TLS_CHECK_LAUNCH();
    }
    return TLS_OK;
  });
  };
  return replay_steps(enqueue, s, a->graph_key, steps);
}

// ---------------------------------------------------------------- block Jacobi
__global__ void block_cholesky_kernel(tls_block_group g, double damping, int32_t* bad) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.count) return;
  const int d = g.dim;
  double A[kMaxBlock * kMaxBlock], L[kMaxBlock * kMaxBlock], s[kMaxBlock];
  for (int k = 0; k < d; ++k) s[k] = g.scale ? g.scale[block_column(g, i, k)] : 1.0;
  for (int a = 0; a < d; ++a)
    for (int b = 0; b < d; ++b) A[a * d + b] = s[a] * g.blocks[i * d * d + a * d + b] * s[b];
  const bool ok = cholesky_block(A, L, d, damping);
  for (int k = 0; k < d * d; ++k) g.factor[i * d * d + k] = L[k];
  if (!ok) atomicAdd(bad, 1);
}

template <int D, typename TV>
__global__ void block_solve_kernel(BlockSet bs, int64_t nblocks, const TV* r, TV* z) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nblocks; b += (int64_t)gridDim.x * blockDim.x) {
    const int gi = find_group(bs, b);
    const int64_t i = b - bs.block_begin[gi];
    const tls_block_group& g = bs.g[gi];
    int64_t cols[D];
    block_cols<D>(g, i, cols);
    double rb[D], zb[D];
#pragma unroll
    for (int k = 0; k < D; ++k) rb[k] = (k < g.dim) ? to_d(r[cols[k]]) : 0.0;
    if (bs.identity || g.factor == nullptr) {
#pragma unroll
      for (int k = 0; k < D; ++k) zb[k] = rb[k];
    } else {
      solve_block<D>(g.factor + i * g.dim * g.dim, g.dim, rb, zb);
    }
#pragma unroll
    for (int k = 0; k < D; ++k)
      if (k < g.dim) z[cols[k]] = static_cast<TV>(zb[k]);
  }
}

}  // namespace tls

using namespace tls;

extern "C" int tls_block_cholesky(const tls_block_group* groups, int32_t ngroups, double damping, int32_t* bad,
                                  tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cudaMemsetAsync(bad, 0, sizeof(int32_t), s);
  for (int i = 0; i < ngroups; ++i) {
    if (groups[i].dim > kMaxBlock) return tls_set_error(TLS_ERR_UNSUPPORTED, "preconditioner block dim > 16");
    if (groups[i].count == 0) continue;
    block_cholesky_kernel<<<(groups[i].count + 127) / 128, 128, 0, s>>>(groups[i], damping, bad);
    TLS_CHECK_LAUNCH();
  }
  return TLS_OK;
}

extern "C" int tls_block_solve(const tls_block_group* groups, int32_t ngroups, const void* r, void* z,
                               int32_t vec_dtype, tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  tls_pcg_args a{};
  a.pre = groups;
  a.npre = ngroups;
  int64_t nb;
  int maxdim;
  BlockSet bs = make_blocks(&a, &nb, &maxdim);
  if (nb == 0) return TLS_OK;
  const int g = grid_of(nb, 128, 148 * 16);
  return with_dim(maxdim, [&](auto dim) -> int {
    constexpr int D = decltype(dim)::value;
    if (vec_dtype == TLS_F64)
      block_solve_kernel<D, double><<<g, 128, 0, s>>>(bs, nb, (const double*)r, (double*)z);
    else
      block_solve_kernel<D, float><<<g, 128, 0, s>>>(bs, nb, (const float*)r, (float*)z);
    TLS_CHECK_LAUNCH();
    return TLS_OK;
  });
}

extern "C" int tls_pcg_start(const tls_pcg_args* a, double rtol, double atol, int32_t max_iterations,
                             int32_t check_interval, int32_t periodic, double drift_tolerance, tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (a->npre > TLS_MAX_GROUPS) return tls_set_error(TLS_ERR_INVALID, "too many preconditioner groups");
  if (a->vec_dtype == TLS_F64)
    return pcg_start_t<double>(a, rtol, atol, max_iterations, check_interval, periodic, drift_tolerance, s);
  return pcg_start_t<float>(a, rtol, atol, max_iterations, check_interval, periodic, drift_tolerance, s);
}

extern "C" int tls_pcg_run(const tls_pcg_args* a, int32_t steps, tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (a->vec_dtype == TLS_F64) return pcg_run_t<double>(a, steps, s);
  return pcg_run_t<float>(a, steps, s);
}

extern "C" int tls_pcg_state_bytes(void) { return (int)sizeof(PcgState); }
