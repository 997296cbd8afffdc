// Lie-group maps on the device (float64).
//
// Conventions follow torchls geometry.py: SE(3) tangent [t, w], Sim(3)
// [t, w, log s], right updates X * Exp(delta); the rotation series branch is
// taken below theta^2 = 1e-4 (geometry.py:19-37). The SE(3) log and its right
// Jacobian inverse follow Barfoot, "State Estimation for Robotics" (2017),
// sec. 7.1.5, with Taylor series where the closed forms cancel.
#pragma once
#include <cuda_runtime.h>

namespace tls {

__device__ __forceinline__ void skew3(const double* v, double* S) {
  S[0] = 0.0;   S[1] = -v[2]; S[2] = v[1];
  S[3] = v[2];  S[4] = 0.0;   S[5] = -v[0];
  S[6] = -v[1]; S[7] = v[0];  S[8] = 0.0;
}

__device__ __forceinline__ void mat3_mul(const double* A, const double* B, double* C) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) C[i * 3 + j] = A[i * 3] * B[j] + A[i * 3 + 1] * B[3 + j] + A[i * 3 + 2] * B[6 + j];
}

// A = sin t / t, B = (1 - cos t)/t^2, C = (t - sin t)/t^3 (geometry.py:19-37)
__device__ __forceinline__ void rotation_coefficients(double t2, double& a, double& b, double& c) {
  if (t2 < 1e-4) {
    a = 1.0 - t2 / 6.0 + t2 * t2 / 120.0;
    b = 0.5 - t2 / 24.0 + t2 * t2 / 720.0;
    c = 1.0 / 6.0 - t2 / 120.0 + t2 * t2 / 5040.0;
  } else {
    const double t = sqrt(t2);
    double s, co;
    sincos(t, &s, &co);
    a = s / t;
    b = (1.0 - co) / t2;
    c = (t - s) / (t2 * t);
  }
}

__device__ __forceinline__ void so3_exp(const double* w, double* R) {
  const double t2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  double a, b, c;
  rotation_coefficients(t2, a, b, c);
  double W[9], W2[9];
  skew3(w, W);
  mat3_mul(W, W, W2);
#pragma unroll
  for (int k = 0; k < 9; ++k) R[k] = a * W[k] + b * W2[k];
  R[0] += 1.0; R[4] += 1.0; R[8] += 1.0;
}

// 4x4 row-major SE(3) exponential of [t, w]
__device__ __forceinline__ void se3_exp(const double* xi, double* T) {
  const double* w = xi + 3;
  const double t2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  double a, b, c;
  rotation_coefficients(t2, a, b, c);
  double W[9], W2[9];
  skew3(w, W);
  mat3_mul(W, W, W2);
  double R[9], V[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    R[k] = a * W[k] + b * W2[k];
    V[k] = b * W[k] + c * W2[k];
  }
  R[0] += 1.0; R[4] += 1.0; R[8] += 1.0;
  V[0] += 1.0; V[4] += 1.0; V[8] += 1.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) T[i * 4 + j] = R[i * 3 + j];
    T[i * 4 + 3] = V[i * 3] * xi[0] + V[i * 3 + 1] * xi[1] + V[i * 3 + 2] * xi[2];
  }
  T[12] = 0.0; T[13] = 0.0; T[14] = 0.0; T[15] = 1.0;
}

// Matrix exponential of a 4x4 by scaling and squaring with a degree-16
// Taylor polynomial (Moler & Van Loan, "Nineteen dubious ways", method 3).
// After scaling |A| <= 1/4, the truncation error is below 1e-26.
__device__ __forceinline__ void expm4(const double* A_in, double* E) {
  double A[16];
  double norm = 0.0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    double row = 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) row += fabs(A_in[i * 4 + j]);
    norm = row > norm ? row : norm;
  }
  int sq = 0;
  double scale = 1.0;
  while (norm * scale > 0.25 && sq < 60) {
    scale *= 0.5;
    ++sq;
  }
#pragma unroll
  for (int k = 0; k < 16; ++k) A[k] = A_in[k] * scale;
  // Horner: E = I + A(I + A/2(I + A/3(...)))
  double P[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) P[k] = (k % 5 == 0) ? 1.0 : 0.0;
  for (int n = 16; n >= 1; --n) {
    double Q[16];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) s += A[i * 4 + k] * P[k * 4 + j];
        Q[i * 4 + j] = s / n + ((i == j) ? 1.0 : 0.0);
      }
#pragma unroll
    for (int k = 0; k < 16; ++k) P[k] = Q[k];
  }
  for (int s = 0; s < sq; ++s) {
    double Q[16];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        double acc = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) acc += P[i * 4 + k] * P[k * 4 + j];
        Q[i * 4 + j] = acc;
      }
#pragma unroll
    for (int k = 0; k < 16; ++k) P[k] = Q[k];
  }
#pragma unroll
  for (int k = 0; k < 16; ++k) E[k] = P[k];
}

// Sim(3) exponential of [t, w, sigma] = expm([[w^ + sigma I, t], [0, 0]]) (geometry.py:60-73)
__device__ __forceinline__ void sim3_exp(const double* xi, double* T) {
  double W[9];
  skew3(xi + 3, W);
  double A[16];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) A[i * 4 + j] = W[i * 3 + j] + (i == j ? xi[6] : 0.0);
    A[i * 4 + 3] = xi[i];
  }
  A[12] = A[13] = A[14] = A[15] = 0.0;
  expm4(A, T);
  T[12] = 0.0; T[13] = 0.0; T[14] = 0.0; T[15] = 1.0;
}

// Rotation -> axis-angle via the largest quaternion component (Shepperd 1978).
__device__ __forceinline__ void so3_log(const double* R, double* w) {
  double tr[4] = {1.0 + R[0] + R[4] + R[8], 1.0 + R[0] - R[4] - R[8], 1.0 - R[0] + R[4] - R[8],
                  1.0 - R[0] - R[4] + R[8]};
  int k = 0;
  double best = -1.0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const double m = sqrt(tr[i] > 1e-12 ? tr[i] : 1e-12);
    tr[i] = m;
    if (m > best) {
      best = m;
      k = i;
    }
  }
  const double d21 = R[7] - R[5], d02 = R[2] - R[6], d10 = R[3] - R[1];
  const double s01 = R[1] + R[3], s02 = R[2] + R[6], s12 = R[5] + R[7];
  const double m = tr[k], inv = 1.0 / (2.0 * m);
  double q[4];
  if (k == 0) { q[0] = m * m; q[1] = d21; q[2] = d02; q[3] = d10; }
  else if (k == 1) { q[0] = d21; q[1] = m * m; q[2] = s01; q[3] = s02; }
  else if (k == 2) { q[0] = d02; q[1] = s01; q[2] = m * m; q[3] = s12; }
  else { q[0] = d10; q[1] = s02; q[2] = s12; q[3] = m * m; }
#pragma unroll
  for (int i = 0; i < 4; ++i) q[i] *= inv;
  if (q[0] < 0.0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) q[i] = -q[i];
  }
  double n2 = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  const double n = sqrt(n2 > 1e-24 ? n2 : 1e-24);
  const double f = 2.0 * atan2(n, q[0]) / n;
  w[0] = q[1] * f; w[1] = q[2] * f; w[2] = q[3] * f;
}

// k(t) = (1 - (t/2) cot(t/2)) / t^2, the W^2 coefficient of J_l^{-1}
__device__ __forceinline__ double jinv_coefficient(double t2) {
  if (t2 < 0.25) {
    return 1.0 / 12.0 + t2 * (1.0 / 720.0 + t2 * (1.0 / 30240.0 + t2 * (1.0 / 1209600.0 + t2 / 47900160.0)));
  }
  const double t = sqrt(t2);
  double s, c;
  sincos(0.5 * t, &s, &c);
  return (1.0 - 0.5 * t * c / s) / t2;
}

// log of an SE(3) element given R (3x3) and t -> [rho, phi]
__device__ __forceinline__ void se3_log(const double* R, const double* t, double* xi) {
  double phi[3];
  so3_log(R, phi);
  const double t2 = phi[0] * phi[0] + phi[1] * phi[1] + phi[2] * phi[2];
  const double k = jinv_coefficient(t2);
  double W[9], W2[9];
  skew3(phi, W);
  mat3_mul(W, W, W2);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double acc = t[i];
#pragma unroll
    for (int j = 0; j < 3; ++j) acc += (-0.5 * W[i * 3 + j] + k * W2[i * 3 + j]) * t[j];
    xi[i] = acc;
  }
  xi[3] = phi[0]; xi[4] = phi[1]; xi[5] = phi[2];
}

// Coefficients of Barfoot's Q(rho, phi) with series below theta = 0.5.
__device__ __forceinline__ void q_coefficients(double t2, double& c2, double& c3, double& c4) {
  if (t2 < 0.25) {
    c2 = 1.0 / 6.0 + t2 * (-1.0 / 120.0 + t2 * (1.0 / 5040.0 + t2 * (-1.0 / 362880.0 + t2 / 39916800.0)));
    c3 = 1.0 / 24.0 + t2 * (-1.0 / 720.0 + t2 * (1.0 / 40320.0 + t2 * (-1.0 / 3628800.0 + t2 / 479001600.0)));
    const double d5 = -1.0 / 120.0 + t2 * (1.0 / 5040.0 + t2 * (-1.0 / 362880.0 + t2 * (1.0 / 39916800.0 - t2 / 6227020800.0)));
    c4 = 0.5 * (c3 + 3.0 * d5);
  } else {
    const double t = sqrt(t2);
    double s, c;
    sincos(t, &s, &c);
    c2 = (t - s) / (t2 * t);
    c3 = (0.5 * t2 + c - 1.0) / (t2 * t2);
    const double d5 = (t - s - t2 * t / 6.0) / (t2 * t2 * t);
    c4 = 0.5 * (c3 + 3.0 * d5);
  }
}

// Right Jacobian inverse of SE(3) at xi = [rho, phi]: J_r^{-1}(xi) = J_l^{-1}(-xi).
__device__ __forceinline__ void se3_right_jacobian_inverse(const double* xi, double* out /*6x6*/) {
  const double* rho = xi;
  const double* phi = xi + 3;
  const double t2 = phi[0] * phi[0] + phi[1] * phi[1] + phi[2] * phi[2];
  double P[9], Rh[9], P2[9];
  skew3(phi, P);
  skew3(rho, Rh);
  mat3_mul(P, P, P2);
  const double k = jinv_coefficient(t2);
  double A[9];  // J_l^{-1}(-phi) = I + P/2 + k P^2
#pragma unroll
  for (int i = 0; i < 9; ++i) A[i] = 0.5 * P[i] + k * P2[i];
  A[0] += 1.0; A[4] += 1.0; A[8] += 1.0;
  double c2, c3, c4;
  q_coefficients(t2, c2, c3, c4);
  double PR[9], RP[9], PRP[9], PPR[9], RPP[9], PRPP[9], PPRP[9];
  mat3_mul(P, Rh, PR);
  mat3_mul(Rh, P, RP);
  mat3_mul(PR, P, PRP);
  mat3_mul(P2, Rh, PPR);
  mat3_mul(Rh, P2, RPP);
  mat3_mul(PRP, P, PRPP);
  mat3_mul(P, PRP, PPRP);
  double Q[9];  // Q(-rho, -phi)
#pragma unroll
  for (int i = 0; i < 9; ++i)
    Q[i] = -0.5 * Rh[i] + c2 * (PR[i] + RP[i] - PRP[i]) - c3 * (PPR[i] + RPP[i] - 3.0 * PRP[i]) +
           c4 * (PRPP[i] + PPRP[i]);
  double AQ[9], B[9];
  mat3_mul(A, Q, AQ);
  mat3_mul(AQ, A, B);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      out[i * 6 + j] = A[i * 3 + j];
      out[i * 6 + 3 + j] = -B[i * 3 + j];
      out[(i + 3) * 6 + j] = 0.0;
      out[(i + 3) * 6 + 3 + j] = A[i * 3 + j];
    }
}

// r = log(Z^-1 Ti^-1 Tj); J_j = J_r^{-1}(r), J_i = -J_r^{-1}(r) Ad(Tj^-1 Ti).
// Ti, Tj, Z are row-major 4x4. jr_inv and ad (6x6 row-major) may be null.
__device__ __forceinline__ void se3_between_residual(const double* Ti, const double* Tj, const double* Z,
                                                     double* r, double* jr_inv, double* ad) {
  double Ri[9], Rj[9], Rz[9], ti[3], tj[3], tz[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      Ri[a * 3 + b] = Ti[a * 4 + b];
      Rj[a * 3 + b] = Tj[a * 4 + b];
      Rz[a * 3 + b] = Z[a * 4 + b];
    }
    ti[a] = Ti[a * 4 + 3];
    tj[a] = Tj[a * 4 + 3];
    tz[a] = Z[a * 4 + 3];
  }
  // M = Ti^-1 Tj : R = Ri^T Rj, t = Ri^T (tj - ti)
  double RM[9], tM[3], d[3] = {tj[0] - ti[0], tj[1] - ti[1], tj[2] - ti[2]};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int b = 0; b < 3; ++b) RM[a * 3 + b] = Ri[a] * Rj[b] + Ri[3 + a] * Rj[3 + b] + Ri[6 + a] * Rj[6 + b];
    tM[a] = Ri[a] * d[0] + Ri[3 + a] * d[1] + Ri[6 + a] * d[2];
  }
  // E = Z^-1 M
  double RE[9], tE[3], e[3] = {tM[0] - tz[0], tM[1] - tz[1], tM[2] - tz[2]};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int b = 0; b < 3; ++b) RE[a * 3 + b] = Rz[a] * RM[b] + Rz[3 + a] * RM[3 + b] + Rz[6 + a] * RM[6 + b];
    tE[a] = Rz[a] * e[0] + Rz[3 + a] * e[1] + Rz[6 + a] * e[2];
  }
  se3_log(RE, tE, r);
  if (jr_inv == nullptr) return;
  se3_right_jacobian_inverse(r, jr_inv);
  // Ad(Tj^-1 Ti): Ra = Rj^T Ri, pa = Rj^T (ti - tj); Ad = [[Ra, [pa]x Ra], [0, Ra]]
  double Ra[9], pa[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int b = 0; b < 3; ++b) Ra[a * 3 + b] = Rj[a] * Ri[b] + Rj[3 + a] * Ri[3 + b] + Rj[6 + a] * Ri[6 + b];
    pa[a] = -(Rj[a] * d[0] + Rj[3 + a] * d[1] + Rj[6 + a] * d[2]);
  }
  double Px[9], PRa[9];
  skew3(pa, Px);
  mat3_mul(Px, Ra, PRa);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      ad[a * 6 + b] = Ra[a * 3 + b];
      ad[a * 6 + 3 + b] = PRa[a * 3 + b];
      ad[(a + 3) * 6 + b] = 0.0;
      ad[(a + 3) * 6 + 3 + b] = Ra[a * 3 + b];
    }
}

// ---------------------------------------------------------------- Sim(3) log and between factor
// Forward-mode dual number: a value and its derivative along one direction.
struct Dual {
  double v, d;
};
__device__ __forceinline__ Dual dc(double v) { return {v, 0.0}; }
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  const double q = a.v / b.v;
  return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
  const double r = sqrt(a.v);
  return {r, a.d / (2.0 * r)};
}
__device__ __forceinline__ Dual dlog(Dual a) { return {log(a.v), a.d / a.v}; }
__device__ __forceinline__ Dual dexp(Dual a) {
  const double e = exp(a.v);
  return {e, e * a.d};
}
__device__ __forceinline__ Dual datan2(Dual y, Dual x) {
  return {atan2(y.v, x.v), (x.v * y.d - y.v * x.d) / (x.v * x.v + y.v * y.v)};
}
__device__ __forceinline__ void dsincos(Dual a, Dual& s, Dual& c) {
  double sv, cv;
  sincos(a.v, &sv, &cv);
  s = {sv, cv * a.d};
  c = {cv, -sv * a.d};
}
// max(a, lo) with the derivative of the branch taken (torch clamp_min)
__device__ __forceinline__ Dual dclamp_min(Dual a, double lo) { return a.v < lo ? dc(lo) : a; }

// so3_log (the largest-quaternion-component branch, as the value path) in duals.
__device__ __forceinline__ void so3_log_dual(const Dual* R, Dual* w) {
  Dual tr[4] = {dc(1.0) + R[0] + R[4] + R[8], dc(1.0) + R[0] - R[4] - R[8], dc(1.0) - R[0] + R[4] - R[8],
                dc(1.0) - R[0] - R[4] + R[8]};
  int k = 0;
  double best = -1.0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    tr[i] = dsqrt(dclamp_min(tr[i], 1e-12));
    if (tr[i].v > best) {
      best = tr[i].v;
      k = i;
    }
  }
  const Dual d21 = R[7] - R[5], d02 = R[2] - R[6], d10 = R[3] - R[1];
  const Dual s01 = R[1] + R[3], s02 = R[2] + R[6], s12 = R[5] + R[7];
  const Dual m = tr[k], den = 2.0 * m;
  Dual q[4];
  if (k == 0) { q[0] = m * m; q[1] = d21; q[2] = d02; q[3] = d10; }
  else if (k == 1) { q[0] = d21; q[1] = m * m; q[2] = s01; q[3] = s02; }
  else if (k == 2) { q[0] = d02; q[1] = s01; q[2] = m * m; q[3] = s12; }
  else { q[0] = d10; q[1] = s02; q[2] = s12; q[3] = m * m; }
#pragma unroll
  for (int i = 0; i < 4; ++i) q[i] = q[i] / den;
  if (q[0].v < 0.0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) q[i] = -q[i];
  }
  const Dual n = dsqrt(dclamp_min(q[1] * q[1] + q[2] * q[2] + q[3] * q[3], 1e-24));
  const Dual f = 2.0 * datan2(n, q[0]) / n;
  w[0] = q[1] * f; w[1] = q[2] * f; w[2] = q[3] * f;
}

// Coefficients of W(w, sigma) = int_0^1 exp(s (w^ + sigma I)) ds
//   = a0 I + c1 w^ + c2 w^2,  z = sigma + i theta, theta^2 = |w|^2:
//   a0 = (e^sigma - 1) / sigma, c1 = Im F / theta, c2 = (a0 - Re F) / theta^2,
//   F = (e^z - 1) / z = sum_k z^k / (k+1)!.
// Where |z| <= 4, or theta^2 < 1e-2 and |sigma| <= 10, the series is summed in
// (sigma, theta^2) by the recurrences z^k = a_k + i theta b_k and
// c_k = (sigma^k - a_k) / theta^2 (44 terms reach double precision for
// |z| <= 4, 64 for |z| <= 10); elsewhere the closed forms, which there cancel
// by at most a factor 1 / theta^2 < 100. The torch form of this residual
// (torchls_b200/residuals.py sim3_w_coefficients) uses the same rule.
__device__ __forceinline__ void sim3_w_coefficients(Dual sigma, Dual t2, Dual& a0, Dual& c1, Dual& c2) {
  const double z2 = sigma.v * sigma.v + t2.v;
  if (z2 <= 16.0 || (t2.v < 1e-2 && sigma.v * sigma.v <= 100.0)) {
    const int terms = z2 <= 16.0 ? 44 : 64;
    Dual a = dc(1.0), b = dc(0.0), c = dc(0.0), sp = dc(1.0);
    Dual sa = dc(0.0), sb = dc(0.0), sc = dc(0.0);
    double inv = 1.0;  // 1 / (k+1)!
    for (int k = 0; k < terms; ++k) {
      inv /= (double)(k + 1);
      sa = sa + inv * sp;
      sb = sb + inv * b;
      sc = sc + inv * c;
      const Dual an = sigma * a - t2 * b;
      const Dual bn = a + sigma * b;
      c = sigma * c + b;
      a = an;
      b = bn;
      sp = sp * sigma;
    }
    a0 = sa;
    c1 = sb;
    c2 = sc;
    return;
  }
  const Dual th = dsqrt(t2), es = dexp(sigma);
  Dual sn, cs;
  dsincos(th, sn, cs);
  const Dual den = sigma * sigma + t2;
  a0 = (es - dc(1.0)) / sigma;
  const Dual ref = (sigma * (es * cs - dc(1.0)) + th * es * sn) / den;
  const Dual imf = (sigma * es * sn - th * (es * cs - dc(1.0))) / den;
  c1 = imf / th;
  c2 = (a0 - ref) / t2;
}

// Sim(3) log of [A t; 0 1] (A = sR) -> [u, w, log s], the inverse of sim3_exp:
// s = sqrt(|A|_F^2 / 3), w = so3_log(A / s), u = W(w, log s)^-1 t.
__device__ __forceinline__ void sim3_log_dual(const Dual* A, const Dual* t, Dual* xi) {
  Dual ss = dc(0.0);
#pragma unroll
  for (int k = 0; k < 9; ++k) ss = ss + A[k] * A[k];
  const Dual s = dsqrt(ss / dc(3.0));
  const Dual sigma = dlog(s);
  Dual R[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) R[k] = A[k] / s;
  Dual w[3];
  so3_log_dual(R, w);
  const Dual t2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  Dual a0, c1, c2;
  sim3_w_coefficients(sigma, t2, a0, c1, c2);
  // W = a0 I + c1 w^ + c2 w^2, with w^2 = w w^T - |w|^2 I
  Dual M[9];
  const Dual Wx[9] = {dc(0.0), -w[2], w[1], w[2], dc(0.0), -w[0], -w[1], w[0], dc(0.0)};
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      Dual v = c1 * Wx[i * 3 + j] + c2 * (w[i] * w[j]);
      if (i == j) v = v + a0 - c2 * t2;
      M[i * 3 + j] = v;
    }
  // u = M^-1 t by the adjugate
  const Dual c00 = M[4] * M[8] - M[5] * M[7], c01 = M[5] * M[6] - M[3] * M[8], c02 = M[3] * M[7] - M[4] * M[6];
  const Dual c10 = M[2] * M[7] - M[1] * M[8], c11 = M[0] * M[8] - M[2] * M[6], c12 = M[1] * M[6] - M[0] * M[7];
  const Dual c20 = M[1] * M[5] - M[2] * M[4], c21 = M[2] * M[3] - M[0] * M[5], c22 = M[0] * M[4] - M[1] * M[3];
  const Dual det = M[0] * c00 + M[1] * c01 + M[2] * c02;
  xi[0] = (c00 * t[0] + c10 * t[1] + c20 * t[2]) / det;
  xi[1] = (c01 * t[0] + c11 * t[1] + c21 * t[2]) / det;
  xi[2] = (c02 * t[0] + c12 * t[1] + c22 * t[2]) / det;
  xi[3] = w[0];
  xi[4] = w[1];
  xi[5] = w[2];
  xi[6] = sigma;
}

// Sim(3) inverse of (A = sR, t): A^-1 = A^T / s^2 with s^2 = |A|_F^2 / 3 (exact on the group)
__device__ __forceinline__ void sim3_inverse(const double* A, const double* t, double* Ai, double* ti) {
  double ss = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) ss += A[k] * A[k];
  const double inv = 3.0 / ss;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) Ai[a * 3 + b] = A[b * 3 + a] * inv;
#pragma unroll
  for (int a = 0; a < 3; ++a) ti[a] = -(Ai[a * 3] * t[0] + Ai[a * 3 + 1] * t[1] + Ai[a * 3 + 2] * t[2]);
}

// (A, t) <- (A1, t1) * (A2, t2) for 4x4 similarity matrices
__device__ __forceinline__ void sim3_compose(const double* A1, const double* t1, const double* A2, const double* t2,
                                             double* A, double* t) {
  mat3_mul(A1, A2, A);
#pragma unroll
  for (int a = 0; a < 3; ++a) t[a] = A1[a * 3] * t2[0] + A1[a * 3 + 1] * t2[1] + A1[a * 3 + 2] * t2[2] + t1[a];
}

// r = log(Z^-1 Si^-1 Sj) (7); when jr_inv and ad are set, J_r^{-1}(r) (7x7,
// row-major) and Ad(Sj^-1 Si) (7x7), so that J_j = J_r^{-1} and
// J_i = -J_r^{-1} Ad. Column k of J_r^{-1} is the derivative of log at
// E = exp(r) along E * G_k (G_k the k-th generator), taken in dual numbers.
__device__ __forceinline__ void sim3_between_residual(const double* Si, const double* Sj, const double* Z,
                                                      double* r, double* jr_inv, double* ad) {
  double Ai[9], Aj[9], Az[9], ti[3], tj[3], tz[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      Ai[a * 3 + b] = Si[a * 4 + b];
      Aj[a * 3 + b] = Sj[a * 4 + b];
      Az[a * 3 + b] = Z[a * 4 + b];
    }
    ti[a] = Si[a * 4 + 3];
    tj[a] = Sj[a * 4 + 3];
    tz[a] = Z[a * 4 + 3];
  }
  double Azi[9], tzi[3], Aii[9], tii[3], A1[9], t1[3], AE[9], tE[3];
  sim3_inverse(Az, tz, Azi, tzi);
  sim3_inverse(Ai, ti, Aii, tii);
  sim3_compose(Azi, tzi, Aii, tii, A1, t1);  // (Z^-1 Si^-1) Sj, the order of the torch residual
  sim3_compose(A1, t1, Aj, tj, AE, tE);
  Dual A[9], t[3], xi[7];
  if (jr_inv == nullptr) {
#pragma unroll
    for (int k = 0; k < 9; ++k) A[k] = dc(AE[k]);
#pragma unroll
    for (int k = 0; k < 3; ++k) t[k] = dc(tE[k]);
    sim3_log_dual(A, t, xi);
#pragma unroll
    for (int k = 0; k < 7; ++k) r[k] = xi[k].v;
    return;
  }
  for (int k = 0; k < 7; ++k) {
    // E G_k = [A (w_k^ + sigma_k I), A u_k; 0 0]
    double dA[9], dt[3];
#pragma unroll
    for (int q = 0; q < 9; ++q) dA[q] = 0.0;
#pragma unroll
    for (int q = 0; q < 3; ++q) dt[q] = 0.0;
    if (k < 3) {
#pragma unroll
      for (int a = 0; a < 3; ++a) dt[a] = AE[a * 3 + k];
    } else if (k < 6) {
      double e[3] = {0.0, 0.0, 0.0}, G[9];
      e[k - 3] = 1.0;
      skew3(e, G);
      mat3_mul(AE, G, dA);
    } else {
#pragma unroll
      for (int q = 0; q < 9; ++q) dA[q] = AE[q];
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) A[q] = {AE[q], dA[q]};
#pragma unroll
    for (int q = 0; q < 3; ++q) t[q] = {tE[q], dt[q]};
    sim3_log_dual(A, t, xi);
#pragma unroll
    for (int i = 0; i < 7; ++i) jr_inv[i * 7 + k] = xi[i].d;
    if (k == 0) {
#pragma unroll
      for (int i = 0; i < 7; ++i) r[i] = xi[i].v;
    }
  }
  // X = Sj^-1 Si; Ad_X = [[sR, t^ R, -t], [0, R, 0], [0, 0, 1]]
  double Aji[9], tji[3], AX[9], tX[3];
  sim3_inverse(Aj, tj, Aji, tji);
  sim3_compose(Aji, tji, Ai, ti, AX, tX);
  double ssx = 0.0;
#pragma unroll
  for (int q = 0; q < 9; ++q) ssx += AX[q] * AX[q];
  const double sx = sqrt(ssx / 3.0);
  double RX[9], Tx[9], TR[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) RX[q] = AX[q] / sx;
  skew3(tX, Tx);
  mat3_mul(Tx, RX, TR);
#pragma unroll
  for (int q = 0; q < 49; ++q) ad[q] = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      ad[a * 7 + b] = AX[a * 3 + b];
      ad[a * 7 + 3 + b] = TR[a * 3 + b];
      ad[(a + 3) * 7 + 3 + b] = RX[a * 3 + b];
    }
    ad[a * 7 + 6] = -tX[a];
  }
  ad[48] = 1.0;
}

}  // namespace tls
