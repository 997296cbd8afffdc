// Fused linearization: residual + Jacobian + robust loss + per-factor
// gradient / Gram / Schur-cross contributions, one thread per factor.
//
// Restates torchls linearization.py:62-112 (values and Jacobians at delta=0
// through the retraction chart), losses.py:30-50 / 88-90 (loss transforms),
// problem.py:177-181 (sqrt(weight) scaling), sparse.py:104-121 (Gram blocks
// with aliased-slot cross terms) and schur.py:213-224 (cross blocks).
#include "common.cuh"
#include "geometry.cuh"

namespace tls {

struct LinParams {
  int64_t n;
  int32_t rdim, nslots, D, W;
  int32_t kind, loss_kind, has_loss, want_jac;
  double delta;
  int32_t slot_dim[TLS_MAX_SLOTS];
  int32_t slot_col[TLS_MAX_SLOTS];
  int32_t slot_gram[TLS_MAX_SLOTS];
  int32_t slot_group[TLS_MAX_SLOTS];
  int32_t slot_cross[TLS_MAX_SLOTS];  // first cross entry of a retained slot, -1 otherwise
  int32_t elim_mask;                  // bitmask of eliminated slots
  int32_t elim_dim;
  int32_t cross_width;
  int32_t stage_w;                    // doubles per lane in the shared-memory output stage
  int8_t col_slot[32];                // slot of each column, -1 past D
  const int32_t* index[TLS_MAX_SLOTS];
  const double* packed_residual;
  const double* packed_blocks[TLS_MAX_SLOTS];
  const double* arg_data[4];
  int64_t arg_stride[4];
  int32_t arg_slot[4];
  const double* weights;
  const double* rho1;
  const double* rho2;
  void* jac;
  int64_t jac_ld;
  double* residual;
  double* raw_residual;
  double* squared_norm;
  double* objective;
  double* grad;
  double* gram;
  double* cross;
};

__device__ __forceinline__ int packed_index(int a, int b, int d) {
  // upper-triangular row-major index of (a, b), a <= b
  return a * d - (a * (a - 1)) / 2 + (b - a);
}

template <int RM, int DM, int KIND, bool CAM, bool PT>
__device__ __forceinline__ void evaluate(const LinParams& p, int64_t f, double (&r)[RM], double (&J)[RM][DM]) {
#pragma unroll
  for (int i = 0; i < RM; ++i) {
    r[i] = 0.0;
#pragma unroll
    for (int c = 0; c < DM; ++c) J[i][c] = 0.0;
  }
  if constexpr (KIND == TLS_RES_PACKED) {
#pragma unroll
    for (int i = 0; i < RM; ++i)
      if (i < p.rdim) r[i] = p.packed_residual[f * p.rdim + i];
    if (p.want_jac) {
#pragma unroll
      for (int c = 0; c < DM; ++c) {
        const int s = p.col_slot[c];
        if (s >= 0) {
          const int j = c - p.slot_col[s];
          const int d = p.slot_dim[s];
          const double* blk = p.packed_blocks[s] + f * p.rdim * d + j;
#pragma unroll
          for (int i = 0; i < RM; ++i)
            if (i < p.rdim) J[i][c] = blk[i * d];
        }
      }
    }
  } else if constexpr (KIND == TLS_RES_REPROJECTION) {
    // args: camera (4x4 world-to-camera), point (3), observation (2)
    const double* cam = CAM ? p.arg_data[0] + (int64_t)p.index[0][f] * 16
                            : p.arg_data[0] + f * p.arg_stride[0];
    const double* pt = PT ? p.arg_data[1] + (int64_t)p.index[CAM ? 1 : 0][f] * 3
                          : p.arg_data[1] + f * p.arg_stride[1];
    const double* uv = p.arg_data[2] + f * p.arg_stride[2];
    double R[9], t[3], X[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
      for (int b = 0; b < 3; ++b) R[a * 3 + b] = cam[a * 4 + b];
      t[a] = cam[a * 4 + 3];
      X[a] = pt[a];
    }
    double xyz[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) xyz[a] = R[a * 3] * X[0] + R[a * 3 + 1] * X[1] + R[a * 3 + 2] * X[2] + t[a];
    const bool valid = xyz[2] > 1e-6;
    const double z = valid ? xyz[2] : 1.0;
    const double iz = 1.0 / z;
    const double u = xyz[0] * iz, v = xyz[1] * iz;
    r[0] = valid ? u - uv[0] : 0.0;
    r[1] = valid ? v - uv[1] : 0.0;
    if (p.want_jac && valid) {
      // d(u,v)/dxyz = [[1/z, 0, -u/z], [0, 1/z, -v/z]]
      double P[2][3] = {{iz, 0.0, -u * iz}, {0.0, iz, -v * iz}};
      double PR[2][3];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int b = 0; b < 3; ++b) PR[i][b] = P[i][0] * R[b] + P[i][1] * R[3 + b] + P[i][2] * R[6 + b];
      if constexpr (CAM) {
        // d xyz / d[t, w] = [R, -R [X]x]  ->  columns 0..2: PR, 3..5: -PR [X]x
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          J[i][0] = PR[i][0];
          J[i][1] = PR[i][1];
          J[i][2] = PR[i][2];
          // -(PR [X]x) : row vector times skew(X)
          // [X]x = [[0,-X2,X1],[X2,0,-X0],[-X1,X0,0]]
          J[i][3] = -(PR[i][1] * X[2] - PR[i][2] * X[1]);
          J[i][4] = -(-PR[i][0] * X[2] + PR[i][2] * X[0]);
          J[i][5] = -(PR[i][0] * X[1] - PR[i][1] * X[0]);
        }
      }
      if constexpr (PT) {
        constexpr int o = CAM ? 6 : 0;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          J[i][o] = PR[i][0];
          J[i][o + 1] = PR[i][1];
          J[i][o + 2] = PR[i][2];
        }
      }
    }
  } else if constexpr (KIND == TLS_RES_SE3_BETWEEN) {
    // args: pose_i (4x4), pose_j (4x4), measurement Z (4x4)
    double Ti[16], Tj[16], Z[16];
    const bool vi = p.arg_slot[0] >= 0, vj = p.arg_slot[1] >= 0;
    const double* pi = vi ? p.arg_data[0] + (int64_t)p.index[p.arg_slot[0]][f] * 16 : p.arg_data[0] + f * p.arg_stride[0];
    const double* pj = vj ? p.arg_data[1] + (int64_t)p.index[p.arg_slot[1]][f] * 16 : p.arg_data[1] + f * p.arg_stride[1];
    const double* pz = p.arg_data[2] + f * p.arg_stride[2];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      Ti[k] = pi[k];
      Tj[k] = pj[k];
      Z[k] = pz[k];
    }
    double jr_inv[36], ad[36];
    se3_between_residual(Ti, Tj, Z, r, p.want_jac ? jr_inv : nullptr, p.want_jac ? ad : nullptr);
    if (p.want_jac) {
      const int ci = vi ? p.slot_col[p.arg_slot[0]] : -1;
      const int cj = vj ? p.slot_col[p.arg_slot[1]] : -1;
#pragma unroll
      for (int c = 0; c < DM; ++c) {
        if (c >= p.D) continue;
        const bool in_i = ci >= 0 && c >= ci && c < ci + 6;
        const bool in_j = cj >= 0 && c >= cj && c < cj + 6;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          double v = 0.0;
          if (in_j) v += jr_inv[i * 6 + (c - cj)];
          if (in_i) {
            double acc = 0.0;
#pragma unroll
            for (int k = 0; k < 6; ++k) acc += jr_inv[i * 6 + k] * ad[k * 6 + (c - ci)];
            v -= acc;
          }
          if (i < RM) J[i][c] = v;
        }
      }
    }
  } else if constexpr (KIND == TLS_RES_SIM3_BETWEEN) {
    // args: pose_i (4x4 [sR t; 0 1]), pose_j (4x4), measurement Z (4x4)
    double Si[16], Sj[16], Z[16];
    const bool vi = p.arg_slot[0] >= 0, vj = p.arg_slot[1] >= 0;
    const double* pi = vi ? p.arg_data[0] + (int64_t)p.index[p.arg_slot[0]][f] * 16 : p.arg_data[0] + f * p.arg_stride[0];
    const double* pj = vj ? p.arg_data[1] + (int64_t)p.index[p.arg_slot[1]][f] * 16 : p.arg_data[1] + f * p.arg_stride[1];
    const double* pz = p.arg_data[2] + f * p.arg_stride[2];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      Si[k] = pi[k];
      Sj[k] = pj[k];
      Z[k] = pz[k];
    }
    double jr_inv[49], ad[49];
    sim3_between_residual(Si, Sj, Z, r, p.want_jac ? jr_inv : nullptr, p.want_jac ? ad : nullptr);
    if (p.want_jac) {
      const int ci = vi ? p.slot_col[p.arg_slot[0]] : -1;
      const int cj = vj ? p.slot_col[p.arg_slot[1]] : -1;
#pragma unroll
      for (int c = 0; c < DM; ++c) {
        if (c >= p.D) continue;
        const bool in_i = ci >= 0 && c >= ci && c < ci + 7;
        const bool in_j = cj >= 0 && c >= cj && c < cj + 7;
#pragma unroll
        for (int i = 0; i < 7; ++i) {
          double v = 0.0;
          if (in_j) v += jr_inv[i * 7 + (c - cj)];
          if (in_i) {
            double acc = 0.0;
#pragma unroll
            for (int k = 0; k < 7; ++k) acc += jr_inv[i * 7 + k] * ad[k * 7 + (c - ci)];
            v -= acc;
          }
          if (i < RM) J[i][c] = v;
        }
      }
    }
  }
}

// The warp's factors are consecutive, so its rows of a factor-major [N][width]
// output form one contiguous range: each lane writes its row into the warp's
// shared-memory buffer, then the warp stores the range with coalesced stores.
__device__ __forceinline__ void warp_flush(const double* buf, int width, double* dst, int64_t f0, int nvalid) {
  __syncwarp();
  const int total = nvalid * width;
  double* d = dst + f0 * width;
  for (int i = threadIdx.x & 31; i < total; i += 32) d[i] = buf[i];
  __syncwarp();
}

template <int RM, int DM, int KIND, bool CAM, bool PT, bool ALIAS, typename TJ>
__global__ void __launch_bounds__(128) linearize_kernel(const LinParams p) {
  extern __shared__ double lin_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t f0 = (int64_t)blockIdx.x * blockDim.x + warp * 32;
  if (f0 >= p.n) return;  // whole warp past the end
  const int nvalid = (int)((p.n - f0) < 32 ? (p.n - f0) : 32);
  const int64_t f = f0 + lane;
  const bool live = lane < nvalid;
  // per-warp stage: lane rows of the width being flushed, contiguous
  double* buf = lin_smem + (size_t)warp * 32 * p.stage_w;
  double* row = buf + lane * p.rdim;
  double r[RM];
  double J[RM][DM];
  if (live) {
    evaluate<RM, DM, KIND, CAM, PT>(p, f, r, J);
  } else {
#pragma unroll
    for (int i = 0; i < RM; ++i) {
      r[i] = 0.0;
#pragma unroll
      for (int c = 0; c < DM; ++c) J[i][c] = 0.0;
    }
  }
  const int R = p.rdim;

  double s = 0.0;
#pragma unroll
  for (int i = 0; i < RM; ++i)
    if (i < R) s += r[i] * r[i];
  if (p.raw_residual) {
#pragma unroll
    for (int i = 0; i < RM; ++i)
      if (i < R) row[i] = r[i];
    warp_flush(buf, R, p.raw_residual, f0, nvalid);
  }
  if (p.squared_norm && live) p.squared_norm[f] = s;

  // --- robust loss / weights (problem-level has_loss, problem.py:264-270)
  double wscale = 1.0, rscale = 1.0, corr = 0.0, obj = s;
  if (p.has_loss && live) {
    if (p.loss_kind == TLS_LOSS_HUBER) {
      const double dl = p.delta;
      const double tiny = 2.2250738585072014e-308;
      const double norm = sqrt(s > tiny ? s : tiny);
      const bool out = s > dl * dl;
      const double first = out ? dl / norm : 1.0;
      obj = out ? dl * (2.0 * norm - dl) : s;
      wscale = sqrt(first);
      rscale = wscale;
    } else if (p.loss_kind == TLS_LOSS_GENERIC) {
      // Triggs / Ceres correction with clamped curvature (losses.py:30-50)
      const double tiny = 2.2250738585072014e-308;
      const double first = p.rho1[f], second = p.rho2[f];
      const bool positive = (s > 0.0) && (second > 0.0);
      const double ratio = positive ? 2.0 * s * second / (first > tiny ? first : tiny) : 0.0;
      const double alpha = -ratio / (1.0 + sqrt(1.0 + ratio));
      corr = alpha / (s > tiny ? s : tiny);
      wscale = sqrt(first);
      rscale = wscale / (1.0 - alpha);
      obj = 0.0;  // objective for generic losses is supplied by the caller
    }
    if (p.weights) {
      const double w = p.weights[f];
      const double sw = sqrt(w);
      wscale *= sw;
      rscale *= sw;
      obj *= w;
    }
    if (p.objective && p.loss_kind != TLS_LOSS_GENERIC) p.objective[f] = obj;
  } else if (p.objective && live && !p.has_loss) {
    p.objective[f] = s;
  }

  if (!p.want_jac) {
    if (p.residual) {
#pragma unroll
      for (int i = 0; i < RM; ++i)
        if (i < R) row[i] = r[i] * rscale;
      warp_flush(buf, R, p.residual, f0, nvalid);
    }
    return;
  }

  if (p.has_loss) {
    if (corr != 0.0) {
#pragma unroll
      for (int c = 0; c < DM; ++c) {
        double rtj = 0.0;
#pragma unroll
        for (int i = 0; i < RM; ++i) rtj += r[i] * J[i][c];
#pragma unroll
        for (int i = 0; i < RM; ++i) J[i][c] = wscale * (J[i][c] - corr * r[i] * rtj);
      }
    } else if (wscale != 1.0) {
#pragma unroll
      for (int c = 0; c < DM; ++c)
#pragma unroll
        for (int i = 0; i < RM; ++i) J[i][c] *= wscale;
    }
#pragma unroll
    for (int i = 0; i < RM; ++i) r[i] *= rscale;
  }
  if (p.residual) {
#pragma unroll
    for (int i = 0; i < RM; ++i)
      if (i < R) row[i] = r[i];
    warp_flush(buf, R, p.residual, f0, nvalid);
  }

  // --- Jacobian store, SoA [r*D][N] (already coalesced: factor index fastest)
  TJ* jac = reinterpret_cast<TJ*>(p.jac);
  if (jac && live) {
#pragma unroll
    for (int i = 0; i < RM; ++i)
#pragma unroll
      for (int c = 0; c < DM; ++c)
        if (i < R && c < p.D) jac[(int64_t)(i * p.D + c) * p.jac_ld + f] = static_cast<TJ>(J[i][c]);
  }
  // --- gradient contributions J^T r (float64)
  if (p.grad) {
    row = buf + lane * p.D;
#pragma unroll
    for (int c = 0; c < DM; ++c) {
      double g = 0.0;
#pragma unroll
      for (int i = 0; i < RM; ++i) g += J[i][c] * r[i];
      if (c < p.D) row[c] = g;
    }
    warp_flush(buf, p.D, p.grad, f0, nvalid);
  }
  // --- Gram contributions per slot (packed upper), with aliased-slot cross terms
  if (p.gram) {
    row = buf + lane * p.W;
#pragma unroll
    for (int c1 = 0; c1 < DM; ++c1) {
#pragma unroll
      for (int c2 = c1; c2 < DM; ++c2) {
        const int s1 = p.col_slot[c1];
        if (s1 >= 0 && s1 == p.col_slot[c2]) {
          double g = 0.0;
#pragma unroll
          for (int i = 0; i < RM; ++i) g += J[i][c1] * J[i][c2];
          const int a = c1 - p.slot_col[s1], b = c2 - p.slot_col[s1];
          row[p.slot_gram[s1] + packed_index(a, b, p.slot_dim[s1])] = g;
        }
      }
    }
    if constexpr (ALIAS) {
      // slot s1 > s2 of the same group and same variable: add J_s1^T J_s2 + J_s2^T J_s1
      if (live) {
#pragma unroll
        for (int c1 = 0; c1 < DM; ++c1) {
#pragma unroll
          for (int c2 = 0; c2 < DM; ++c2) {
            const int s1 = p.col_slot[c1], s2 = p.col_slot[c2];
            if (s1 >= 0 && s2 >= 0 && s2 < s1 && p.slot_group[s1] == p.slot_group[s2] &&
                p.index[s1][f] == p.index[s2][f]) {
              double g = 0.0;
#pragma unroll
              for (int i = 0; i < RM; ++i) g += J[i][c1] * J[i][c2];
              const int a = c1 - p.slot_col[s1], b = c2 - p.slot_col[s2];
              const int lo = a < b ? a : b, hi = a < b ? b : a;
              row[p.slot_gram[s1] + packed_index(lo, hi, p.slot_dim[s1])] += (a == b) ? 2.0 * g : g;
            }
          }
        }
      }
    }
    warp_flush(buf, p.W, p.gram, f0, nvalid);
  }
  // --- Schur cross contributions: retained slot s -> J_s^T (sum of eliminated slots)
  if (p.cross) {
    row = buf + lane * p.cross_width;
    for (int k = 0; k < p.cross_width; ++k) row[k] = 0.0;
#pragma unroll
    for (int c1 = 0; c1 < DM; ++c1) {
      const int s1 = p.col_slot[c1];
      if (s1 < 0 || p.slot_cross[s1] < 0) continue;
      const int a = c1 - p.slot_col[s1];
#pragma unroll
      for (int c2 = 0; c2 < DM; ++c2) {
        const int s2 = p.col_slot[c2];
        if (s2 >= 0 && ((p.elim_mask >> s2) & 1)) {
          double g = 0.0;
#pragma unroll
          for (int i = 0; i < RM; ++i) g += J[i][c1] * J[i][c2];
          row[p.slot_cross[s1] + a * p.elim_dim + (c2 - p.slot_col[s2])] += g;
        }
      }
    }
    warp_flush(buf, p.cross_width, p.cross, f0, nvalid);
  }
}

template <int RM, int DM, int KIND, bool CAM, bool PT, bool ALIAS>
static int launch_lin(const LinParams& p, int jac_dtype, cudaStream_t st) {
  const int block = 128;
  const int64_t grid = (p.n + block - 1) / block;
  if (p.n == 0) return TLS_OK;
  const int smem = block * p.stage_w * (int)sizeof(double);
  if (jac_dtype == TLS_F32) {
    auto k = linearize_kernel<RM, DM, KIND, CAM, PT, ALIAS, float>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k<<<grid, block, smem, st>>>(p);
  } else {
    auto k = linearize_kernel<RM, DM, KIND, CAM, PT, ALIAS, double>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k<<<grid, block, smem, st>>>(p);
  }
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}

template <bool ALIAS>
static int launch_packed(const LinParams& p, int jac_dtype, cudaStream_t st) {
  const int R = p.rdim, D = p.D;
#define TLS_TRY(RM, DM) \
  if (R <= RM && D <= DM) return launch_lin<RM, DM, TLS_RES_PACKED, false, false, ALIAS>(p, jac_dtype, st);
  TLS_TRY(1, 4)
  TLS_TRY(2, 4)
  TLS_TRY(3, 4)
  TLS_TRY(2, 9)
  TLS_TRY(3, 6)
  TLS_TRY(3, 9)
  TLS_TRY(4, 8)
  TLS_TRY(6, 12)
  TLS_TRY(7, 14)
  TLS_TRY(8, 16)
#undef TLS_TRY
  return tls_set_error(TLS_ERR_UNSUPPORTED, "residual dim > 8 or total slot dim > 16 not supported by the CUDA linearizer");
}

}  // namespace tls

using namespace tls;

extern "C" int tls_linearize(const tls_linearize_args* a, tls_stream_t stream) {
  const int32_t elim_mask = a->elim_mask, elim_dim = a->elim_dim, cross_width = a->cross_width;
  const int32_t* slot_cross = a->cross_contrib ? a->slot_cross : nullptr;
  double* cross = a->cross_contrib;
  const tls_factor_group& fg = a->fg;
  if (fg.nslots < 0 || fg.nslots > TLS_MAX_SLOTS || fg.total_dim > 32)
    return tls_set_error(TLS_ERR_INVALID, "bad factor group");
  LinParams p{};
  p.n = fg.count;
  p.rdim = fg.rdim;
  p.nslots = fg.nslots;
  p.D = fg.total_dim;
  p.kind = a->residual_kind;
  p.loss_kind = a->loss_kind;
  p.has_loss = a->has_loss;
  p.want_jac = a->want_jacobian;
  p.delta = a->loss_delta;
  int W = 0;
  bool alias = false;
  for (int c = 0; c < 32; ++c) p.col_slot[c] = -1;
  for (int s = 0; s < fg.nslots; ++s) {
    p.slot_dim[s] = fg.slot_dim[s];
    p.slot_col[s] = fg.slot_col[s];
    p.slot_group[s] = fg.slot_group[s];
    p.slot_gram[s] = fg.slot_gram[s];
    p.index[s] = fg.index[s];
    p.packed_blocks[s] = a->packed_blocks[s];
    p.slot_cross[s] = slot_cross ? slot_cross[s] : -1;
    W += fg.slot_dim[s] * (fg.slot_dim[s] + 1) / 2;
    for (int j = 0; j < fg.slot_dim[s]; ++j) p.col_slot[fg.slot_col[s] + j] = (int8_t)s;
    for (int o = 0; o < s; ++o)
      if (fg.slot_group[o] == fg.slot_group[s]) alias = true;
  }
  p.W = W;
  {
    int sw = fg.rdim > fg.total_dim ? fg.rdim : fg.total_dim;
    if (W > sw) sw = W;
    if (cross && cross_width > sw) sw = cross_width;
    p.stage_w = sw < 1 ? 1 : sw;
  }
  p.elim_mask = elim_mask;
  p.elim_dim = elim_dim;
  p.cross_width = cross_width;
  p.cross = cross;
  p.packed_residual = a->packed_residual;
  for (int k = 0; k < 4; ++k) {
    p.arg_data[k] = a->arg_data[k];
    p.arg_stride[k] = a->arg_stride[k];
    p.arg_slot[k] = a->arg_slot[k];
  }
  p.weights = a->weights;
  p.rho1 = a->rho1;
  p.rho2 = a->rho2;
  p.jac = fg.jac;
  p.jac_ld = fg.jac_stride ? fg.jac_stride : fg.count;
  p.residual = a->residual;
  p.raw_residual = a->raw_residual;
  p.squared_norm = a->squared_norm;
  p.objective = a->objective;
  p.grad = a->grad_contrib;
  p.gram = a->gram_contrib;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  switch (a->residual_kind) {
    case TLS_RES_PACKED:
      return alias ? launch_packed<true>(p, fg.jac_dtype, st) : launch_packed<false>(p, fg.jac_dtype, st);
    case TLS_RES_REPROJECTION: {
      const bool cam = a->arg_slot[0] >= 0, pt = a->arg_slot[1] >= 0;
      if (fg.rdim != 2) return tls_set_error(TLS_ERR_INVALID, "reprojection has r = 2");
      if (cam && pt) return launch_lin<2, 9, TLS_RES_REPROJECTION, true, true, false>(p, fg.jac_dtype, st);
      if (cam) return launch_lin<2, 6, TLS_RES_REPROJECTION, true, false, false>(p, fg.jac_dtype, st);
      if (pt) return launch_lin<2, 3, TLS_RES_REPROJECTION, false, true, false>(p, fg.jac_dtype, st);
      return launch_lin<2, 1, TLS_RES_REPROJECTION, false, false, false>(p, fg.jac_dtype, st);
    }
    case TLS_RES_SE3_BETWEEN: {
      if (fg.rdim != 6) return tls_set_error(TLS_ERR_INVALID, "se3_between has r = 6");
      if (fg.total_dim == 12)
        return alias ? launch_lin<6, 12, TLS_RES_SE3_BETWEEN, false, false, true>(p, fg.jac_dtype, st)
                     : launch_lin<6, 12, TLS_RES_SE3_BETWEEN, false, false, false>(p, fg.jac_dtype, st);
      return launch_lin<6, 6, TLS_RES_SE3_BETWEEN, false, false, false>(p, fg.jac_dtype, st);
    }
    case TLS_RES_SIM3_BETWEEN: {
      if (fg.rdim != 7) return tls_set_error(TLS_ERR_INVALID, "sim3_between has r = 7");
      if (fg.total_dim == 14)
        return alias ? launch_lin<7, 14, TLS_RES_SIM3_BETWEEN, false, false, true>(p, fg.jac_dtype, st)
                     : launch_lin<7, 14, TLS_RES_SIM3_BETWEEN, false, false, false>(p, fg.jac_dtype, st);
      if (fg.total_dim != 7) return tls_set_error(TLS_ERR_INVALID, "sim3_between takes Sim(3) slots");
      return launch_lin<7, 7, TLS_RES_SIM3_BETWEEN, false, false, false>(p, fg.jac_dtype, st);
    }
    default:
      return tls_set_error(TLS_ERR_UNSUPPORTED, "unknown residual kind");
  }
}
