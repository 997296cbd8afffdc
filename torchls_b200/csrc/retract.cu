// Retractions X <- X * Exp(delta) per variable group (torchls
// variables.py:153-160, geometry.py:40-160) and projected Euclidean updates
// for box bounds (bounds.py:61-75). Storage is float64.
#include "common.cuh"
#include "geometry.cuh"

namespace tls {

__global__ void retract_kernel(int kind, int count, int dim, const double* __restrict__ values,
                               const double* __restrict__ delta, double* __restrict__ out,
                               const double* __restrict__ lower, const double* __restrict__ upper,
                               double* __restrict__ delta_out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (kind == TLS_KIND_EUCLIDEAN) {
    const int64_t n = (int64_t)count * dim;
    if (i >= n) return;
    double v = values[i] + delta[i];
    if (lower) v = fmax(v, lower[i]);
    if (upper) v = fmin(v, upper[i]);
    out[i] = v;
    if (delta_out) delta_out[i] = v - values[i];
    return;
  }
  if (i >= count) return;
  const double* d = delta + i * dim;
  if (kind == TLS_KIND_SO3) {
    double E[9];
    so3_exp(d, E);
    const double* R = values + i * 9;
    double* o = out + i * 9;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) o[r * 3 + c] = R[r * 3] * E[c] + R[r * 3 + 1] * E[3 + c] + R[r * 3 + 2] * E[6 + c];
  } else if (kind == TLS_KIND_SE3 || kind == TLS_KIND_SIM3) {
    double E[16];
    if (kind == TLS_KIND_SE3) se3_exp(d, E);
    else sim3_exp(d, E);
    const double* T = values + i * 16;
    double* o = out + i * 16;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        double acc = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) acc += T[r * 4 + k] * E[k * 4 + c];
        o[r * 4 + c] = acc;
      }
  } else if (kind == TLS_KIND_SE2) {
    const double* p = values + i * 3;
    const double th = d[2];
    double a, b;
    if (th * th < 1e-4) {
      a = 1.0 - th * th / 6.0;
      b = th / 2.0 - th * th * th / 24.0;
    } else {
      double s, c;
      sincos(th, &s, &c);
      a = s / th;
      b = (1.0 - c) / th;
    }
    const double lx = a * d[0] - b * d[1], ly = b * d[0] + a * d[1];
    double s, c;
    sincos(p[2], &s, &c);
    double* o = out + i * 3;
    o[0] = p[0] + c * lx - s * ly;
    o[1] = p[1] + s * lx + c * ly;
    o[2] = p[2] + th;
  }
}

}  // namespace tls

using namespace tls;

extern "C" int tls_retract(int32_t kind, int32_t count, int32_t dim, const double* values, const double* delta,
                           double* out, const double* lower, const double* upper, double* delta_out,
                           tls_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int64_t n = kind == TLS_KIND_EUCLIDEAN ? (int64_t)count * dim : count;
  if (n == 0) return TLS_OK;
  if ((lower || upper || delta_out) && kind != TLS_KIND_EUCLIDEAN)
    return tls_set_error(TLS_ERR_INVALID, "bounds require a Euclidean group");
  retract_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(kind, count, dim, values, delta, out, lower, upper,
                                                            delta_out);
  TLS_CHECK_LAUNCH();
  return TLS_OK;
}
