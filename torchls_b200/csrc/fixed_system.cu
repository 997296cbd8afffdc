// Fixed sparse linear least squares (torchls linear_system.py:15-141): the
// products of a COO matrix with one or several right-hand sides, its weighted
// normal matrix A^T diag(w) A + ridge I (dense, for the Cholesky kernels of
// dense.cu) and the fused elementwise step of the LAD ADMM iteration.
//
// Every sum runs in a fixed order (row lists, column lists and normal-matrix
// pair lists built once on the host): results are deterministic.
#include <stdint.h>

#include "common.cuh"

namespace tls {

// y[r][c] = sum_{e in row r} val[e] x[col[e]][c]
__global__ void fixed_matvec_kernel(tls_fixed_system s, const double* __restrict__ x, int64_t k,
                                    double* __restrict__ y) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= s.m * k) return;
  const int64_t r = t / k, c = t % k;
  double acc = 0.0;
  for (int e = s.row_ptr[r]; e < s.row_ptr[r + 1]; ++e) acc += s.val[e] * x[(int64_t)s.col[e] * k + c];
  y[t] = acc;
}

// y[j][c] = sum_{e in column j} val[e] x[row[e]][c] (entries in ascending row)
__global__ void fixed_rmatvec_kernel(tls_fixed_system s, const double* __restrict__ x, int64_t k,
                                     double* __restrict__ y) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= s.n * k) return;
  const int64_t j = t / k, c = t % k;
  double acc = 0.0;
  for (int q = s.col_ptr[j]; q < s.col_ptr[j + 1]; ++q) {
    const int e = s.col_entry[q];
    acc += s.val[e] * x[(int64_t)s.row[e] * k + c];
  }
  y[t] = acc;
}

// N[target[t]] = sum_{q in pairs of t} w[row[left[q]]] val[left[q]] val[right[q]]
// (N zeroed before), then the ridge on the diagonal.
__global__ void fixed_normal_kernel(tls_fixed_system s, const double* __restrict__ w, double* __restrict__ N) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= s.ntargets) return;
  double acc = 0.0;
  for (int q = s.target_ptr[t]; q < s.target_ptr[t + 1]; ++q) {
    const int a = s.pair_left[q], b = s.pair_right[q];
    const double p = s.val[a] * s.val[b];
    acc += w ? w[s.row[a]] * p : p;
  }
  N[s.target[t]] = acc;
}

__global__ void fixed_ridge_kernel(int64_t n, double ridge, double* __restrict__ N) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) N[i * n + i] += ridge;
}

// LAD ADMM, elementwise part (linear_system.py:126-133): v = ax - target + u,
// z_new = sign(v) max(|v| - kappa, 0), primal = ax - z_new - target,
// u += primal, zdiff = z_new - z_old (z <- z_new), next = target + z_new - u
// (the next least-squares target); block partial sums of primal^2, ax^2,
// z_new^2 into partials[3][blocks].
__global__ void __launch_bounds__(256) admm_step_kernel(int64_t count, const double* __restrict__ ax,
                                                        const double* __restrict__ target, double* __restrict__ z,
                                                        double* __restrict__ u, double* __restrict__ zdiff,
                                                        double* __restrict__ next, double kappa,
                                                        double* __restrict__ partials) {
  __shared__ double sm[3][8];
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
    const double axi = ax[i], ti = target[i], zo = z[i];
    const double v = axi - ti + u[i];
    const double mag = fabs(v) - kappa;
    const double zn = mag > 0.0 ? copysign(mag, v) : 0.0;
    const double primal = axi - zn - ti;
    const double un = u[i] + primal;
    u[i] = un;
    zdiff[i] = zn - zo;
    z[i] = zn;
    next[i] = ti + zn - un;
    a0 += primal * primal;
    a1 += axi * axi;
    a2 += zn * zn;
  }
  block_sum3<256>(a0, a1, a2, sm);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = a0;
    partials[gridDim.x + blockIdx.x] = a1;
    partials[2 * gridDim.x + blockIdx.x] = a2;
  }
}

__global__ void __launch_bounds__(256) admm_finish_kernel(const double* __restrict__ partials, int blocks,
                                                          double* __restrict__ out) {
  __shared__ double sm[3][8];
  double a[3] = {0.0, 0.0, 0.0};
  for (int q = 0; q < 3; ++q)
    for (int b = threadIdx.x; b < blocks; b += 256) a[q] += partials[q * blocks + b];
  block_sum3<256>(a[0], a[1], a[2], sm);
  if (threadIdx.x == 0) {
    out[0] = a[0];
    out[1] = a[1];
    out[2] = a[2];
  }
}

}  // namespace tls

using namespace tls;

extern "C" int tls_fixed_matvec(const tls_fixed_system* s, const double* x, int64_t k, double* y, tls_stream_t stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (!s || k < 1) return tls_set_error(TLS_ERR_INVALID, "fixed system matvec: bad arguments");
  const int64_t n = s->m * k;
  if (n > 0) fixed_matvec_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(*s, x, k, y);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}

extern "C" int tls_fixed_rmatvec(const tls_fixed_system* s, const double* x, int64_t k, double* y,
                                 tls_stream_t stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (!s || k < 1) return tls_set_error(TLS_ERR_INVALID, "fixed system rmatvec: bad arguments");
  const int64_t n = s->n * k;
  if (n > 0) fixed_rmatvec_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(*s, x, k, y);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}

extern "C" int tls_fixed_normal(const tls_fixed_system* s, const double* weights, double ridge, double* N,
                                tls_stream_t stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (!s || !N) return tls_set_error(TLS_ERR_INVALID, "fixed system normal matrix: bad arguments");
  cudaError_t e = cudaMemsetAsync(N, 0, (size_t)(s->n * s->n) * sizeof(double), st);
  if (e != cudaSuccess) return tls_set_cuda_error(e);
  if (s->ntargets > 0) fixed_normal_kernel<<<(unsigned)((s->ntargets + 255) / 256), 256, 0, st>>>(*s, weights, N);
  TLS_CHECK_LAUNCH();
  if (ridge != 0.0 && s->n > 0) fixed_ridge_kernel<<<(unsigned)((s->n + 255) / 256), 256, 0, st>>>(s->n, ridge, N);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}

extern "C" int tls_admm_step(int64_t count, const double* ax, const double* target, double* z, double* u,
                             double* zdiff, double* next, double kappa, double* partials, double* out,
                             tls_stream_t stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (count < 0 || !partials || !out) return tls_set_error(TLS_ERR_INVALID, "ADMM step: bad arguments");
  const int blocks = grid_for(count, 256, 1024);
  admm_step_kernel<<<blocks, 256, 0, st>>>(count, ax, target, z, u, zdiff, next, kappa, partials);
  TLS_CHECK_LAUNCH();
  admm_finish_kernel<<<1, 256, 0, st>>>(partials, blocks, out);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}
