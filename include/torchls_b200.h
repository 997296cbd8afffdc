/*
 * torchls_b200 -- C ABI of the B200 (sm_100a) block-sparse LM/GN inner loop.
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t and
 * returns an int status (TLS_OK = 0). Nothing here allocates device memory:
 * callers pass every buffer and workspace. Calls are asynchronous on `stream`
 * unless stated otherwise; the only global mutable state is the thread-local
 * last-error message and a launch counter.
 *
 * Layout conventions (shared by all calls):
 *   tangent vector   : variable groups in declaration order; group g occupies
 *                      [offset_g, offset_g + count_g * dim_g), variable i at
 *                      offset_g + i * dim_g  (torchls variables.py:100-117).
 *   Jacobian (jac)   : per factor group, structure-of-arrays [r * D][N]:
 *                      element (row i, column c) of factor f at
 *                      (i * D + c) * N + f, columns grouped by slot.
 *   residuals        : per factor group, factor-major [N][r] float64.
 *   contributions    : per factor group, factor-major [N][W] (W = D for
 *                      vectors, sum_s d_s (d_s + 1) / 2 for Gram blocks).
 *   segments         : CSR lists of contribution offsets per target
 *                      (variable or Schur edge); reductions follow list order,
 *                      so every result is deterministic (no atomics).
 */
#ifndef TORCHLS_B200_H
#define TORCHLS_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define TLS_API __attribute__((visibility("default")))
#else
#define TLS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* tls_stream_t; /* == cudaStream_t */

enum {
  TLS_OK = 0,
  TLS_ERR_INVALID = 1,   /* bad argument; maps to ValueError */
  TLS_ERR_CUDA = 2,      /* CUDA launch/runtime error */
  TLS_ERR_UNSUPPORTED = 3,
  TLS_ERR_NOT_PD = 4     /* a damped block is not positive definite; maps to LinAlgError */
};

enum { TLS_F32 = 0, TLS_F64 = 1 };

enum {
  TLS_LOSS_NONE = 0,     /* plain least squares */
  TLS_LOSS_HUBER = 1,    /* Huber on the block squared norm (torchls losses.py:56-107) */
  TLS_LOSS_GENERIC = 2   /* caller supplies rho', rho'' per factor (losses.py:30-50) */
};

enum {
  TLS_RES_PACKED = 0,       /* residual + blocks supplied by the caller (torch.func path) */
  TLS_RES_REPROJECTION = 1, /* depth-guarded normalized pinhole reprojection, r = 2 */
  TLS_RES_SE3_BETWEEN = 2,  /* log(Z^-1 Ti^-1 Tj), r = 6 */
  TLS_RES_SIM3_BETWEEN = 3  /* log(Z^-1 Si^-1 Sj), r = 7 */
};

enum { TLS_KIND_EUCLIDEAN = 0, TLS_KIND_SO3 = 1, TLS_KIND_SE3 = 2, TLS_KIND_SIM3 = 3, TLS_KIND_SE2 = 4 };

#define TLS_MAX_SLOTS 8
#define TLS_MAX_GROUPS 8
#define TLS_MAX_FACTOR_GROUPS 16

typedef struct tls_var_group {
  int64_t offset; /* tangent offset */
  int32_t count;  /* number of variables */
  int32_t dim;    /* tangent dim */
} tls_var_group;

typedef struct tls_factor_group {
  int64_t count;                            /* N factors */
  int32_t rdim;                             /* residual dim r */
  int32_t nslots;                           /* variable slots S */
  int32_t total_dim;                        /* D = sum of slot dims */
  int32_t jac_dtype;                        /* TLS_F32 / TLS_F64 */
  int32_t slot_group[TLS_MAX_SLOTS];        /* variable group per slot */
  int32_t slot_dim[TLS_MAX_SLOTS];
  int32_t slot_col[TLS_MAX_SLOTS];          /* first column of the slot inside D */
  int32_t slot_gram[TLS_MAX_SLOTS];         /* first Gram entry of the slot inside W */
  const int32_t* index[TLS_MAX_SLOTS];      /* [N] variable index (within its group) */
  void* jac;                                /* [r*D][jac_stride] SoA */
  int64_t jac_stride;                       /* leading dimension of jac (0: count) */
} tls_factor_group;

/* A deterministic segmented reduction: target t sums src[ptr[t]..ptr[t+1])
 * blocks of `width` values from a contribution buffer, in list order. */
typedef struct tls_segments {
  int32_t count;       /* targets */
  int32_t width;       /* values per contribution block */
  int32_t lanes;       /* lanes per target: power of two <= 32, or 256 (one block per target) */
  int32_t pad_;
  const int32_t* ptr;  /* [count + 1] */
  const int32_t* src;  /* [nnz] element offset of each block */
} tls_segments;

/* ---------------------------------------------------------------- linearization
 * Replaces: torchls linearization.py:62-128 (vmap(jacrev) + loss transform),
 * problem.py:157-221 (weights, gather) and the per-linearization halves of
 * sparse.py:43-55 (J^T r) and sparse.py:104-121 / warp_diagonal.py:14-66
 * (Gram blocks). One kernel per factor group writes J (SoA, jac_dtype), the
 * model and raw residuals, the per-factor objective, and FP64 per-factor
 * gradient and Gram contributions (aliased slots include their cross terms).
 */
typedef struct tls_linearize_args {
  tls_factor_group fg;
  int32_t residual_kind;      /* TLS_RES_* */
  int32_t loss_kind;          /* TLS_LOSS_* */
  double loss_delta;          /* Huber delta */
  int32_t has_loss;           /* problem-level: any loss or weights (problem.py:264-270) */
  int32_t want_jacobian;      /* 0: residual/objective only (trial evaluation) */
  /* residual inputs; for TLS_RES_PACKED `packed_blocks[s]` are [N][r][d_s] and
   * `packed_residual` is [N][r], in float64 */
  const double* packed_residual;
  const double* packed_blocks[TLS_MAX_SLOTS];
  /* built-in residual arguments: per argument position, a float64 pointer and
   * a per-factor stride in doubles (0 broadcasts one value to every factor);
   * variable arguments point at the group's value storage and use the slot's
   * index array; `arg_slot[a]` is the slot of argument a, or -1 for data. */
  const double* arg_data[4];
  int64_t arg_stride[4];
  int32_t arg_slot[4];
  const double* weights;      /* [N] or NULL */
  const double* rho1;         /* generic loss: rho'(s) per factor */
  const double* rho2;         /* generic loss: rho''(s) per factor */
  /* outputs (any may be NULL when not wanted) */
  double* residual;           /* [N][r] model residual */
  double* raw_residual;       /* [N][r] */
  double* squared_norm;       /* [N] s = |r_raw|^2 */
  double* objective;          /* [N] w * rho(s) (or s) */
  double* grad_contrib;       /* [N][D] */
  double* gram_contrib;       /* [N][W] */
  /* Schur cross blocks J_s^T (sum of eliminated slots) for every retained slot
   * s with slot_cross[s] >= 0, written at cross_contrib[f*cross_width + slot_cross[s]]
   * as a (d_s x elim_dim) row-major block (schur.py:213-224). */
  int32_t elim_mask;          /* bitmask of eliminated slots (0: none) */
  int32_t elim_dim;
  int32_t slot_cross[TLS_MAX_SLOTS];
  int32_t cross_width;
  int32_t pad2_;
  double* cross_contrib;      /* [N][cross_width] or NULL */
} tls_linearize_args;

TLS_API int tls_linearize(const tls_linearize_args* args, tls_stream_t stream);

/* Segmented reduction to dense outputs.
 * mode 0: vector targets, out[t*width + k] (out_dtype).
 * mode 1: packed-upper Gram targets of dimension d -> out[t][d][d] float64,
 *         symmetrised. */
TLS_API int tls_segment_reduce(const tls_segments* seg, const void* contrib, int32_t contrib_dtype,
                       int32_t mode, int32_t dim, void* out, int32_t out_dtype, tls_stream_t stream);

/* ---------------------------------------------------------------- normal operator
 * Replaces: torchls sparse.py:83-84 BlockJacobian.normal_matvec and
 * warp_normal.py:125-294 WarpNormalPlan(J).bind(J).normal_matvec(v, damping).
 * y = diag(s) J^T J diag(s) x + damping * x, deterministic.
 * `contrib` is a caller workspace of sum_k N_k * D_k elements of vec_dtype.
 */

/* Tile plan of the one-pass normal operator, built once per incidence
 * structure by the host (torchls_b200/normal_tiles.py). Factor group k is cut
 * into tiles of tile_factors[k] consecutive factors; CTA c (global numbering)
 * runs tiles [cta_tile[c], cta_tile[c + 1]). For each tile, the x values of
 * its distinct target variables are loaded once into a compact shared buffer,
 * and every factor's per-slot contribution J_s^T J_f x (float64) goes to a
 * shared-memory stage at the offset in pos[k][s * N_k + f]; the stage is
 * ordered by target variable,
 * so each target's contributions in the tile form one contiguous run, summed
 * in order. A run is final (written to y), added to the CTA's shared
 * accumulator, or written to a partial slot; at the end the CTA flushes its
 * accumulator the same way. A last kernel sums each remaining target's
 * partials in list order. Fixed orders throughout: bitwise reproducible. */
typedef struct tls_normal_tiles {
  int32_t ncta;                                /* CTAs over all factor groups */
  int32_t ntiles;
  int32_t stage_doubles;                       /* contribution stage per CTA */
  int32_t acc_doubles;                         /* accumulator per CTA */
  int32_t ntargets;                            /* targets the gather kernel finishes */
  int32_t gather_lanes;                        /* lanes per gather target: power of two <= 32 */
  int32_t xbuf_doubles;                        /* compact per-tile x buffer */
  int32_t nheavy;                              /* the first nheavy targets get a 256-thread block each */
  int32_t tile_factors[TLS_MAX_FACTOR_GROUPS];
  int32_t tile_base[TLS_MAX_FACTOR_GROUPS];    /* first tile of group k */
  int32_t cta_base[TLS_MAX_FACTOR_GROUPS + 1]; /* first CTA of group k's launch */
  const uint32_t* pos[TLS_MAX_FACTOR_GROUPS];  /* [S_k][N_k] stage offset | x-buffer offset << 16 */
  const int32_t* cta_tile;    /* [ncta + 1] */
  const int32_t* tile_run;    /* [ntiles + 1] */
  const int32_t* run_col;     /* first column of the run's target variable */
  const int32_t* run_meta;    /* stage start | length << 14 | (dim - 1) << 27 */
  const int32_t* run_dest;    /* >= 0: partial offset; -1: final; <= -2: accumulator offset -2 - dest */
  const int32_t* run_xoff;    /* offset of the run's x values in the tile's x buffer */
  const int32_t* cta_flush;   /* [ncta + 1] */
  const int32_t* flush_col;
  const int32_t* flush_meta;  /* accumulator offset | (dim - 1) << 16 */
  const int32_t* flush_dest;  /* >= 0: partial offset; -1: final */
  const int32_t* target_col;  /* [ntargets] */
  const int32_t* target_dim;  /* [ntargets] */
  const int32_t* target_ptr;  /* [ntargets + 1] into target_src */
  const int32_t* target_src;  /* partial offsets, in summation order */
  double* partials;           /* workspace of partial slots */
} tls_normal_tiles;

typedef struct tls_normal_args {
  int32_t nfactor_groups;
  int32_t nvar_groups;
  int32_t vec_dtype;          /* x, y, scale dtype */
  int32_t pad_;
  tls_factor_group fg[TLS_MAX_FACTOR_GROUPS];
  int64_t contrib_offset[TLS_MAX_FACTOR_GROUPS];  /* element offset of group k in contrib */
  tls_var_group vg[TLS_MAX_GROUPS];
  tls_segments seg[TLS_MAX_GROUPS];               /* width = dim_g; src offsets into contrib */
  const void* scale;          /* [n] or NULL */
  void* contrib;
  double damping;
  /* one-pass plan for this structure, or NULL (two-pass: factor pass into
   * `contrib`, then a per-variable gather); products other than the normal
   * operator always take the two-pass route */
  const tls_normal_tiles* tiles;
} tls_normal_args;

TLS_API int tls_normal_matvec(const tls_normal_args* args, const void* x, void* y, tls_stream_t stream);

/* dst[r][p] = src[r][perm[p]] (r < rows, p < ncols; src row stride ld_src,
 * dst dense): the SoA Jacobian of a factor group in a tile plan's factor
 * order. A plan may reorder a group's factors (torchls_b200/normal_tiles.py
 * `perm`) so that a tile's factors share variables; the one-pass operator
 * then reads that group's J from this copy (fg[k].jac, jac_stride = N_k).
 * No counterpart in the reference (its operator has no tile plan). */
TLS_API int tls_permute_columns(const void* src, void* dst, int32_t dtype, int64_t rows, int64_t ncols,
                                int64_t ld_src, const int32_t* perm, tls_stream_t stream);

/* J diag(s) x per factor row -> out [rows] (factor groups concatenated,
 * factor-major [N][r]); replaces sparse.py:31-41 BlockJacobian.matvec. */
TLS_API int tls_jacobian_matvec(const tls_normal_args* args, const void* x, void* out_rows, tls_stream_t stream);

/* sum_f |J_f diag(s) x|^2 in float64 (x float64), written to *out (device);
 * replaces sparse.py:57-81 squared_matvec_norm. `partials` holds at least
 * ceil(N_k / 128) doubles for the largest factor group. */
TLS_API int tls_squared_matvec_norm(const tls_normal_args* args, const double* x, double* partials,
                            double* out, tls_stream_t stream);

/* The same |J diag(s) x|^2 for callers that cannot allocate device memory
 * where they need it (inside another framework's memory pool, a binding with
 * no device allocator, a loop where an allocation may block): the block
 * partials live in a 512 KB array inside this library, held on every GPU
 * that loads it until the process exits. No counterpart in the reference.
 * Limit: at most 8,388,608 factors per factor group (65,536 blocks of 128);
 * larger inputs return TLS_ERR_INVALID before any work. The first call on a
 * device looks up the array's device address (make that device current and
 * make the first call before any stream capture). Calls share the array:
 * calls that overlap on the GPU race. Allocates nothing. */
TLS_API int tls_squared_matvec_norm_static(const tls_normal_args* args, const double* x, double* out,
                                   tls_stream_t stream);

/* J^T u (times diag(s) when scale is set) for u in factor-major row layout,
 * through the contribution workspace; replaces sparse.py:43-55 rmatvec. */
TLS_API int tls_jacobian_rmatvec(const tls_normal_args* args, const void* rows, void* out, tls_stream_t stream);

/* ---------------------------------------------------------------- block Jacobi
 * Replaces: solvers.py:259-285 block_jacobi, preconditioning.py:12-17,117-134.
 * A block group is `count` blocks of dimension `dim` whose columns are the
 * concatenation of up to 4 member ranges (joint groups, preconditioning.py:47-88).
 */
typedef struct tls_block_group {
  int32_t count;
  int32_t dim;
  int32_t nmembers;
  int32_t pad_;
  int64_t member_offset[4];   /* tangent offset of each member group */
  int32_t member_dim[4];
  const double* blocks;       /* [count][dim][dim] float64 */
  double* factor;             /* [count][dim][dim] float64 lower Cholesky factor */
  const double* scale;        /* full-vector column scale s: factor of s B s + damping I; or NULL */
} tls_block_group;

/* factor[i] = chol(S blocks[i] S + damping * I), S = diag of `scale` over the
 * block's columns (identity when NULL). Writes the number of blocks that
 * are not positive definite (or non-finite) to *bad (device int32). */
TLS_API int tls_block_cholesky(const tls_block_group* groups, int32_t ngroups, double damping,
                       int32_t* bad, tls_stream_t stream);

/* z = (L L^T)^-1 r per block; r, z of vec_dtype, arithmetic in float64. */
TLS_API int tls_block_solve(const tls_block_group* groups, int32_t ngroups, const void* r, void* z,
                    int32_t vec_dtype, tls_stream_t stream);

/* ---------------------------------------------------------------- PCG
 * Replaces: solvers.py:167-256 pcg and warp_pcg.py:33-214. The state machine
 * mirrors torchls's PCG step for step (true-residual checks, adaptive or
 * periodic restarts, reason codes); all decisions are taken on the device
 * from float64 scalars, so iterations need no host synchronisation.
 */
enum { TLS_PCG_ACTIVE = 0, TLS_PCG_CONVERGED = 1, TLS_PCG_NONFINITE = 2,
       TLS_PCG_NONPOSITIVE = 3, TLS_PCG_MAX_ITERATIONS = 4 };

typedef struct tls_pcg_control {
  /* host-visible result, float64 scalars first */
  double rhs_norm, threshold, residual_norm;
  double rz, curvature, alpha, beta, rz_new, rr, true_rr, drift_rr, rz_true;
  int32_t iterations, status, restarts, checks;
  int32_t mode, stop_at, max_iterations, check_interval;
  int32_t periodic, pad_[3];
  double drift_tolerance;
  uint32_t ticket[4];
} tls_pcg_control;

typedef struct tls_schur_args tls_schur_args;
typedef struct tls_schur_general_args tls_schur_general_args;

typedef struct tls_pcg_args {
  int64_t n;
  int32_t vec_dtype;
  int32_t op_kind;               /* 0: normal operator, 1: Schur reduced operator, 2: general Schur */
  const tls_normal_args* normal; /* op_kind 0 */
  const tls_schur_args* schur;   /* op_kind 1 */
  const tls_block_group* pre;    /* preconditioner blocks, or NULL (identity) */
  int32_t npre;
  int32_t pad_;
  const void* rhs;
  void *x, *r, *z, *p, *ap, *ztrue, *psave;   /* [n] workspaces of vec_dtype */
  double* partials;              /* >= 65536 + 3 * 1024 doubles */
  tls_pcg_control* control;      /* device buffer of tls_pcg_state_bytes() bytes */
  const tls_schur_general_args* schur_general; /* op_kind 2 */
  /* Nonzero: tls_pcg_run calls with this key and the same step count on the
   * same device and host thread launch again the CUDA graph recorded by the
   * first of them instead of recording the steps again. The caller keeps
   * *args and everything it points to unchanged between those calls (a PCG
   * solve's repeated calls; a new solve takes a new key). 0: record every
   * call. */
  uint64_t graph_key;
} tls_pcg_args;

/* Initialise: x = 0, r = rhs, norms, threshold = max(atol, rtol |rhs|),
 * z = M r, p = z, rz. */
TLS_API int tls_pcg_start(const tls_pcg_args* args, double rtol, double atol, int32_t max_iterations,
                  int32_t check_interval, int32_t periodic, double drift_tolerance, tls_stream_t stream);

/* Run up to `steps` state-machine steps (each = one operator application plus
 * its vector updates); steps after termination leave x unchanged. Launches
 * only. Small Schur systems (float64 vectors, <= 8192 preconditioner blocks,
 * retained/eliminated dims 6/3, 7/3 or 3/3) run all `steps` in ONE
 * persistent cooperative kernel that stops at termination; otherwise each
 * step is 2-3 kernels and at most 16 steps are enqueued per call (poll the
 * control block and call again while it is active). */
TLS_API int tls_pcg_run(const tls_pcg_args* args, int32_t steps, tls_stream_t stream);

/* Size in bytes of the device control block (tls_pcg_control first). */
TLS_API int tls_pcg_state_bytes(void);

/* ---------------------------------------------------------------- Schur complement
 * Replaces: schur.py:192-397 (SchurLinearization, DampedSchurSystem) for one
 * retained group of dimension dr <= 8 and an eliminated group of dimension
 * de <= 4. Edges (retained i, eliminated p) are stored in chunks of whole
 * eliminated variables; each chunk owns a fixed-size slab (W and int32
 * metadata) that the matvec kernel streams into shared memory with 1-D bulk
 * copies (TMA), double-buffered, in a persistent grid. Inside a chunk edges
 * are sorted by retained variable and cut into runs that never cross a
 * 32-edge window, so a run is reduced by one warp. Every reduction follows a
 * fixed order (deterministic).
 */
struct tls_schur_args {
  int32_t nedges;
  int32_t nchunks;
  int32_t dr, de;
  int32_t nretained;            /* retained variables */
  int32_t nelim;                /* eliminated variables */
  int32_t wdtype;               /* TLS_F32 / TLS_F64 storage of W */
  int32_t vec_dtype;            /* reduced vectors (float64) */
  int32_t cap;                  /* edges per chunk slab: 512 (float32 W) or 256 (float64 W); runs of
                                   equal retained variable never cross a 32 * cap / 256 edge window */
  int32_t meta_ints;            /* int32 words per chunk metadata slab: 5 * cap + 8 */
  int32_t nruns;
  int32_t pad_;
  int64_t retained_offset;      /* tangent offset of the retained group (full vector) */
  int64_t elim_offset;          /* tangent offset of the eliminated group (full vector) */
  const int32_t* meta;          /* [nchunks][meta_ints]: [ne, np, 0, 0][edge_r][meta][tail pos][pt ptr][pt edges] */
  const int32_t* slab_r;        /* [nchunks*cap] retained variable per slab entry (-1: padding) */
  const int32_t* slab_e;        /* [nchunks*cap] eliminated variable per slab entry */
  const int32_t* elim_ptr;      /* [nelim+1] CSR: slab entries of each eliminated variable */
  const int32_t* elim_slab;     /* [E] slab indices, ascending */
  const int32_t* rrun_ptr;      /* [nretained+1] CSR over retained-major run positions */
  const int32_t* crun_start;    /* [nruns] first slab index of each run (retained-major) */
  const int32_t* crun_len;      /* [nruns] edges in each run */
  const double* cross;          /* [nchunks*cap][dr][de] J_r^T J_e per slab entry (unscaled) */
  const double* elim_diag;      /* [nelim][de][de] eliminated diagonal blocks (unscaled) */
  const double* ret_diag;       /* [nretained][dr][dr] retained diagonal blocks (unscaled) */
  const double* scale;          /* [n_full] column scale or NULL */
  double* inv_l;                /* [nelim][de][de] L^-1, L = chol(s C s + lambda I) */
  void* w;                      /* [nchunks][dr*de][cap] whitened W slabs (wdtype), 16-byte aligned */
  double* run_partial;          /* [nruns][dr] workspace, retained-major */
  double* ybuf;                 /* [nelim][de] workspace: L^-1 b_e */
  double damping;
  int32_t* bad;                 /* device: number of non-PD eliminated blocks */
  int32_t* err;                 /* device: 1 if a bulk-copy wait gave up, 2 if a grid-barrier wait gave
                                   up (never expected); cleared (in stream order) by tls_schur_damp, so
                                   it covers one damped system: its rhs, PCG and back-substitution */
  int64_t wait_cycles;          /* limit of every bounded wait in SM cycles; <= 0: 2^31 (about a second) */
  /* Optional (zero-initialise the struct; NULL: whitening reads `cross`):
   * when cross_contrib is set, `cross` is not read; tls_schur_damp's
   * whitening forms each slab entry's cross block itself from the
   * linearization's per-factor contributions (float64 sums in list order, the
   * sums tls_segment_reduce forms): entry s sums the dr*de values at
   * cross_contrib + cross_src[j] for j in [cross_ptr[s], cross_ptr[s+1]). */
  const double* cross_contrib;
  const int32_t* cross_ptr;     /* [nchunks*cap + 1] */
  const int32_t* cross_src;     /* [contributions] offsets into cross_contrib */
};

/* ---------------------------------------------------------------- general Schur complement
 * Replaces: schur.py:17-397 where the one-group path above does not apply:
 * several retained groups (e.g. cameras and intrinsics), residuals that couple
 * retained variables (camera priors, odometry between cameras; schur.py:41-56,
 * 303-328) and joint preconditioner groups (schur.py:163-189, 330-352).
 * Retained variables are numbered in reduced order (groups in layout order,
 * IDs ascending); each one's edges are contiguous, in the reference's edge
 * order (sorted key r * E + e, schur.py:80, 93). Every sum runs in a fixed
 * order: results are deterministic. Reduced vectors are float64.
 */
struct tls_schur_general_args {
  int32_t de;                   /* eliminated block dim (<= 4) */
  int32_t nelim;                /* eliminated variables */
  int32_t nretained;            /* retained variables over all groups */
  int32_t wdtype;               /* TLS_F32 / TLS_F64 storage of the whitened blocks */
  int64_t nedges;
  int64_t reduced_dim;
  int64_t full_dim;             /* length of the full tangent vector */
  int64_t elim_offset;          /* tangent offset of the eliminated group (full vector) */
  const int32_t* var_dim;       /* [nretained] tangent dim (<= max_dim) */
  const int64_t* var_row;       /* [nretained] offset in the reduced vector */
  const int64_t* var_full;      /* [nretained] offset in the full tangent vector */
  const int64_t* var_diag;      /* [nretained] element offset of its dim x dim block in ret_diag / outputs */
  const int32_t* var_ptr;       /* [nretained + 1] edges of variable v: [var_ptr[v], var_ptr[v+1]) */
  const int32_t* edge_var;      /* [nedges] retained variable of each edge */
  const int32_t* edge_elim;     /* [nedges] eliminated variable of each edge */
  const int64_t* edge_w;        /* [nedges] element offset of its dim x de block in cross and w */
  const int32_t* elim_ptr;      /* [nelim + 1] CSR over the edges of each eliminated variable */
  const int32_t* elim_edge;     /* [nnz] edge ids, in (retained variable, edge) order */
  const double* cross;          /* J_r^T J_e per edge (unscaled) */
  const double* elim_diag;      /* [nelim][de][de] eliminated diagonal blocks (unscaled) */
  const double* ret_diag;       /* retained diagonal blocks at var_diag (unscaled) */
  const double* scale;          /* [n_full] column scale or NULL */
  double* inv_l;                /* [nelim][de][de] L^-1, L = chol(s C s + lambda I) */
  void* w;                      /* whitened blocks (wdtype) at edge_w */
  double* tbuf;                 /* [nelim][de] workspace */
  double* ybuf;                 /* [nelim][de] workspace: L^-1 b_e */
  /* retained couplings: the normal operator of the (column-scaled) full
   * Jacobian with this system's damping, and two full-length float64
   * workspaces; NULL: the base term is the block-diagonal s U s + lambda I */
  const tls_normal_args* normal;
  double* xfull;
  double* yfull;
  double damping;
  int32_t* bad;                 /* device: number of non-PD eliminated blocks */
  int32_t max_dim;              /* largest retained dim (<= 16) */
  int32_t pad2_;
  /* retained couplings with the cached retained normal matrix
   * (cache_retained_matrix, schur.py:225-241, 303-306): base = B x + lambda x
   * from this block-sparse B = (s J_r)^T (s J_r) (yfull is then the base
   * workspace and `normal` may be NULL); like `normal`, a host pointer to a
   * struct of device pointers; NULL: as above */
  const struct tls_retained_matrix* retained;
};

/* The retained normal matrix B = (s J_r)^T (s J_r) of a general Schur system,
 * block-sparse by retained variable: row v's blocks [row_ptr[v], row_ptr[v+1])
 * name their column variable (ascending) and the element offset of a
 * var_dim[v] x var_dim[col] row-major block in `values`. */
typedef struct tls_retained_matrix {
  const int32_t* row_ptr;       /* [nretained + 1] */
  const int32_t* block_col;     /* [nblocks] */
  const int64_t* block_off;     /* [nblocks] */
  const double* values;
} tls_retained_matrix;

/* Factor eliminated blocks and whiten every edge (schur.py:263-283). */
TLS_API int tls_schur_general_damp(const tls_schur_general_args* a, tls_stream_t stream);
/* out = base(x) - W W^T x (schur.py:303-328). */
TLS_API int tls_schur_general_matvec(const tls_schur_general_args* a, const double* x, double* out,
                                     tls_stream_t stream);
/* rhs = b_r - W (L^-1 b_e), y_e = L^-1 b_e kept in ybuf; b full, scaled (schur.py:285-290). */
TLS_API int tls_schur_general_reduced_rhs(const tls_schur_general_args* a, const double* b, double* out,
                                          tls_stream_t stream);
/* delta_e = L^-T (y_e - W^T x); writes the full tangent step (schur.py:292-301). */
TLS_API int tls_schur_general_backsubstitute(const tls_schur_general_args* a, const double* x, double* delta_full,
                                             tls_stream_t stream);
/* out (at var_diag) = s U s - sum_e W_e W_e^T per retained variable, W in float64 (schur.py:353-378). */
TLS_API int tls_schur_general_preconditioner_blocks(const tls_schur_general_args* a, double* out,
                                                    tls_stream_t stream);
/* out[i] (da x db) = sum_k W_{edge_a[k]} W_{edge_b[k]}^T over k in [ptr[i], ptr[i+1]): the Schur
 * cross terms between two members of a joint preconditioner group (schur.py:330-352). */
TLS_API int tls_schur_general_pair_blocks(const tls_schur_general_args* a, int32_t count, const int32_t* ptr,
                                          const int32_t* edge_a, const int32_t* edge_b, int32_t da, int32_t db,
                                          double* out, tls_stream_t stream);

/* Dense reduced matrix S = s U s + lambda I - W W^T (n = nretained * dr, row-major,
 * exactly symmetric) from the slabs (schur.py:380-397): per lower block
 * (target_r[t], target_c[t]) the pairs [ptr[t], ptr[t+1]) of slab entries
 * (pair_a, pair_b) of a shared eliminated variable, summed in a fixed order
 * (the assembly of tls_batched_schur_dense for one problem). */
TLS_API int tls_schur_dense_matrix(const tls_schur_args* a, int64_t ntargets, const int32_t* target_r,
                                   const int32_t* target_c, const int32_t* ptr, const int32_t* pair_a,
                                   const int32_t* pair_b, double* S, tls_stream_t stream);

/* Factor eliminated blocks and whiten every edge (schur.py:263-283). */
TLS_API int tls_schur_damp(const tls_schur_args* a, tls_stream_t stream);
/* out = (s U s + lambda I) x - W W^T x on the reduced vector (schur.py:303-328). */
TLS_API int tls_schur_matvec(const tls_schur_args* a, const void* x, void* out, tls_stream_t stream);
/* rhs_c = b_c - W (L^-1 b_e); stores y_e = L^-1 b_e in a->ybuf (schur.py:285-290).
 * b is the full scaled right-hand side (float64, full tangent layout). */
TLS_API int tls_schur_reduced_rhs(const tls_schur_args* a, const double* b, void* rhs_c, tls_stream_t stream);
/* delta_e = L^-T (y_e - W^T x_c); writes the full tangent step (schur.py:292-301). */
TLS_API int tls_schur_backsubstitute(const tls_schur_args* a, const void* x_c, double* delta_full,
                             tls_stream_t stream);
/* Preconditioner blocks s U s - sum_e W_e W_e^T -> out [nretained][dr][dr]
 * (schur.py:353-363); the damping is added by tls_block_cholesky. */
TLS_API int tls_schur_preconditioner_blocks(const tls_schur_args* a, double* out, tls_stream_t stream);

/* ---------------------------------------------------------------- dense Cholesky
 * Replaces: torch.linalg.cholesky / cholesky_solve at the reference's dense
 * sites (solvers.py:517-518 schur_dense, schur.py:380-397, linear_system.py:61-98).
 * Row-major float64, lower triangle. Blocked right-looking (64-column panels)
 * with the trailing updates on the FP64 tensor cores; deterministic. */
/* In place: A (n x n, leading dimension lda) <- L with zeros above the diagonal;
 * *info (device) = 0, or the 1-based index of the first pivot that is not
 * positive (then L is not usable). */
TLS_API int tls_dense_cholesky(int64_t n, double* A, int64_t lda, int32_t* info, tls_stream_t stream);
/* In place: B (n x nrhs, leading dimension ldb) <- (L L^T)^-1 B; n <= 22,816. */
TLS_API int tls_dense_cholesky_solve(int64_t n, const double* L, int64_t lda, int64_t nrhs, double* B, int64_t ldb,
                                     tls_stream_t stream);

/* ---------------------------------------------------------------- fixed linear systems
 * Replaces: linear_system.py:15-141 (FixedLinearSystem, LinearFactor,
 * least_absolute_deviations) for a sparse m x n matrix A (COO, coalesced):
 * entries in row order with a column-ordered index, and the pairs of entries
 * of each row that meet at normal-matrix element target = c1 * n + c2
 * (sorted targets, pairs in row order). Vectors are float64, row-major
 * [rows][k] for k right-hand sides. */
typedef struct tls_fixed_system {
  int64_t m, n, nnz, ntargets;
  const int32_t* row_ptr;       /* [m + 1] entries of each row */
  const int32_t* row;           /* [nnz] row of each entry */
  const int32_t* col;           /* [nnz] column of each entry */
  const double* val;            /* [nnz] */
  const int32_t* col_ptr;       /* [n + 1] */
  const int32_t* col_entry;     /* [nnz] entries of each column, ascending row */
  const int64_t* target;        /* [ntargets] normal-matrix element c1 * n + c2 */
  const int32_t* target_ptr;    /* [ntargets + 1] */
  const int32_t* pair_left;     /* entry pairs (same row) of each target */
  const int32_t* pair_right;
} tls_fixed_system;

/* y = A x (x [n][k], y [m][k]) (linear_system.py:42-46). */
TLS_API int tls_fixed_matvec(const tls_fixed_system* s, const double* x, int64_t k, double* y, tls_stream_t stream);
/* y = A^T x (x [m][k], y [n][k]) (linear_system.py:48-52). */
TLS_API int tls_fixed_rmatvec(const tls_fixed_system* s, const double* x, int64_t k, double* y, tls_stream_t stream);
/* N (n x n, dense) = A^T diag(w) A + ridge I; weights [m] or NULL (linear_system.py:54-73). */
TLS_API int tls_fixed_normal(const tls_fixed_system* s, const double* weights, double ridge, double* N,
                             tls_stream_t stream);
/* One LAD ADMM update (linear_system.py:126-133) over `count` entries: z <- soft(ax - target + u, kappa),
 * u += ax - z - target, zdiff = z_new - z_old, next = target + z - u (the next least-squares target);
 * out[0..2] = |primal|^2, |ax|^2, |z|^2 (deterministic sums); partials holds >= 3 * 1024 doubles. */
TLS_API int tls_admm_step(int64_t count, const double* ax, const double* target, double* z, double* u,
                          double* zdiff, double* next, double kappa, double* partials, double* out,
                          tls_stream_t stream);

/* ---------------------------------------------------------------- batched independent problems
 * Replaces, per problem, the reduced-system CG of solvers.py:167-256 (pcg)
 * and the LM decisions of solvers.py:597-689 when thousands of independent
 * problems are merged into one block-diagonal system (batched.py). Problem p
 * owns the retained variables [ret_ptr[p], ret_ptr[p+1]) and one dense
 * n_p x n_p reduced matrix (n_p = its variables x dr) at element s_off[p] of S,
 * row-major in the storage type sdtype; diag keeps each variable's dr x dr
 * diagonal block in float64 (the block-Jacobi preconditioner). */
typedef struct tls_batched_systems {
  int32_t nproblems, nretained;
  int32_t dr, sdtype;             /* dr 3, 6 or 7; TLS_F32 / TLS_F64 */
  const int32_t* ret_ptr;         /* [nproblems + 1] */
  const int32_t* ret_problem;     /* [nretained]; NULL (with ret_ptr and s_off): one problem of every variable */
  const int64_t* s_off;           /* [nproblems] */
  void* S;
  double* diag;                   /* [nretained][dr][dr]; may be NULL for the assembly alone */
} tls_batched_systems;

/* S_p = s U s + lambda I - W W^T of every problem from the one-group Schur
 * slabs (schur.py:380-397 per diagonal block of the merged system), the
 * lower blocks (target_r, target_c) and their pairs as for
 * tls_schur_dense_matrix; each entry is summed in float64 in a fixed order
 * (for dr 3 or 6 and de 3: lane l of a block's warp takes pairs l, l + 32, ...
 * and the 32 lane sums are added in lane order; else list order) and rounded
 * once to sdtype, and S_p is exactly symmetric. */
TLS_API int tls_batched_schur_dense(const tls_schur_args* a, const tls_batched_systems* b, int64_t ntargets,
                                    const int32_t* target_r, const int32_t* target_c, const int32_t* ptr,
                                    const int32_t* pair_a, const int32_t* pair_b, tls_stream_t stream);

/* Preconditioned CG of every problem in ONE persistent launch (torchls
 * solvers.py:167-256 per problem: x0 = 0, threshold max(atol, rtol |b_p|),
 * stop on the recurrence residual, on a curvature p.Ap that is not positive
 * and finite, or after max_iterations). The CTAs pull tasks from a work
 * queue (*queue, zeroed by this call): task t is task_size[t] <= task_groups[t]
 * problems order[task_first[t] ...], task_groups[t] in {1, 2, 4, 8} problems
 * sharing one 256-thread CTA (8 / task_groups[t] warps each) and smem_bytes /
 * task_groups[t] bytes of its dynamic shared memory (tls_batched_share_bytes
 * gives a problem's need; with the cache its matrix is read from shared
 * memory). iterations[p] and status[p] (0; 1 when a diagonal block is not
 * positive definite, x_p = 0; 2 when the share is too small, *err = 1) are
 * written for every problem of the tasks. Results do not depend on the tiling. */
typedef struct tls_batched_pcg_args {
  const double* rhs;              /* [sum n_p] reduced right-hand sides */
  double* x;                      /* [sum n_p] solutions */
  int32_t* iterations;            /* [nproblems] */
  int32_t* status;                /* [nproblems] */
  const int32_t* order;
  const int32_t* task_first;
  const int32_t* task_size;
  const int32_t* task_groups;
  int32_t* queue;                 /* one device int32 */
  int32_t* err;                   /* one device int32, set on failure */
  double rtol, atol;
  int32_t ntasks, max_iterations;
  int32_t smem_bytes, pad_;       /* dynamic shared memory per CTA (<= 227 KB) */
} tls_batched_pcg_args;

TLS_API int tls_batched_pcg(const tls_batched_systems* sys, const tls_batched_pcg_args* a, tls_stream_t stream);

/* Shared-memory bytes a problem of `blocks` variables needs in its group's
 * share, without (with_cache = 0) or with its packed matrix. */
TLS_API int64_t tls_batched_share_bytes(int32_t dr, int32_t blocks, int32_t sdtype, int32_t with_cache);

/* Per factor of rows [nfactors][rdim]: obj = 1/2 w rho(|new|^2) and
 * red = 1/2 w (rho(|old|^2) - rho(|new|^2)) with the exact forms of
 * losses.py:92-107 (loss 0: rho(s) = s, difference (old-new).(old+new);
 * loss 1: Huber delta, divided difference across the kink); weights may be NULL. */
TLS_API int tls_factor_terms(int64_t nfactors, int32_t rdim, const double* old_raw, const double* new_raw,
                             int32_t loss, double delta, const double* weights, double* obj, double* red,
                             tls_stream_t stream);
/* out[f] = |rows[f]|^2 for rows [nfactors][rdim]. */
TLS_API int tls_factor_sqnorm(int64_t nfactors, int32_t rdim, const double* rows, double* out,
                              tls_stream_t stream);

enum { TLS_BATCH_MAX_ITERATIONS = 0, TLS_BATCH_GRADIENT_TOLERANCE = 1, TLS_BATCH_COST_TOLERANCE = 2,
       TLS_BATCH_TRIALS_EXHAUSTED = 3 };

/* Per-problem step decision (solvers.py:597-689): gain ratio actual /
 * predicted (-inf when predicted <= 0), acceptance of tried problems (finite
 * new cost, actual > 0, ratio >= step_quality_min), cost update, damping
 * divided by lambda_factor when the ratio is above 0.75 and multiplied on
 * rejection (clamped), step counters, and the cost-tolerance stop
 * (|actual| <= cost_tolerance (cost + actual)), which clears active and sets
 * reason; accepted problems leave pending. */
typedef struct tls_batched_lm {
  int32_t nproblems, pad_;
  double lambda_factor, lambda_min, lambda_max, step_quality_min, cost_tolerance;
  const double *actual, *predicted, *new_cost;
  double *cost, *lam;
  const uint8_t* tried;
  uint8_t *ok, *active, *pending;
  int64_t *accepted, *rejected;
  int32_t* reason;
} tls_batched_lm;

TLS_API int tls_batched_lm_update(const tls_batched_lm* m, tls_stream_t stream);

/* ---------------------------------------------------------------- retraction
 * Replaces: variables.py:153-160 / 242-249 with geometry.py:40-160 retractions.
 * out[i] = values[i] * Exp(delta[i]) (right update) for Lie groups,
 * values + delta for Euclidean. Storage float64: SO3 [3][3], SE3/Sim3 [4][4],
 * SE2 [3]. Optional clamping to [lower, upper] (Euclidean only, bounds.py:61-75)
 * rewrites delta_out with the effective step. */
TLS_API int tls_retract(int32_t kind, int32_t count, int32_t dim, const double* values, const double* delta,
                double* out, const double* lower, const double* upper, double* delta_out,
                tls_stream_t stream);

/* ---------------------------------------------------------------- reductions
 * Deterministic float64 sums used by the LM driver (cost, trial reduction,
 * gradient norms). `partials` holds >= 1024 doubles. */
enum { TLS_SUM_PLAIN = 0, TLS_SUM_SQUARES = 1, TLS_SUM_ABSMAX = 2 };
TLS_API int tls_reduce(const void* x, int32_t dtype, int64_t n, int32_t op, double* partials, double* out,
               tls_stream_t stream);

/* Trial objective and exact reduction per factor group (problem.py:315-348,
 * losses.py:92-107): adds 0.5 * sum w*rho(s_new) and 0.5 * sum w*reduction to
 * out[0], out[1] (device). old/new raw residuals are [N][r] float64. */
TLS_API int tls_trial_terms(int64_t count, int32_t rdim, const double* old_raw, const double* new_raw,
                    int32_t loss_kind, double delta, const double* rho_old, const double* rho_new,
                    const double* weights, int32_t has_loss, double* partials, double* out,
                    tls_stream_t stream);

/* ---------------------------------------------------------------- misc */
/* Number of kernels this library has launched in the process (a relaxed
 * atomic counter; the only global state besides the last-error message). */
TLS_API int64_t tls_launch_count(void);
TLS_API const char* tls_last_error(void);
TLS_API int tls_version(void);
TLS_API int tls_device_init(int32_t device);

#ifdef __cplusplus
}
#endif
#endif /* TORCHLS_B200_H */
