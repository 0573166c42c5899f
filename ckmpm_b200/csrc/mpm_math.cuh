// Device math for the CK-MPM substep: 3x3 helpers, the FP32 SVD, the compact
// (CK) kernel weights and the three constitutive models on the hot path.
//
// Matrices are row-major float[9] like the reference's Matrix<float,3,3>
// (AppledoreM/CKMPM include/data_type.cuh:32-425).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ckmpm {

#define CKMPM_DEV __device__ __forceinline__

CKMPM_DEV float det3(const float* a) {
  return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
         a[2] * (a[3] * a[7] - a[4] * a[6]);
}

// Adjugate inverse (include/data_type.cuh:369-386).
CKMPM_DEV void inv3(const float* a, float* r) {
  const float id = 1.0f / det3(a);
  r[0] = id * (a[4] * a[8] - a[5] * a[7]);
  r[1] = id * (a[2] * a[7] - a[1] * a[8]);
  r[2] = id * (a[1] * a[5] - a[2] * a[4]);
  r[3] = id * (a[5] * a[6] - a[3] * a[8]);
  r[4] = id * (a[0] * a[8] - a[2] * a[6]);
  r[5] = id * (a[2] * a[3] - a[0] * a[5]);
  r[6] = id * (a[3] * a[7] - a[4] * a[6]);
  r[7] = id * (a[1] * a[6] - a[0] * a[7]);
  r[8] = id * (a[0] * a[4] - a[1] * a[3]);
}

// Inverse of a symmetric matrix given by its 6 unique entries
// (d00, d11, d22, d01, d02, d12); writes the 6 unique entries of the inverse.
CKMPM_DEV void inv_sym3(float d00, float d11, float d22, float d01, float d02, float d12, float* r) {
  const float c00 = d11 * d22 - d12 * d12;
  const float c01 = d02 * d12 - d01 * d22;
  const float c02 = d01 * d12 - d02 * d11;
  const float det = d00 * c00 + d01 * c01 + d02 * c02;
  const float id = 1.0f / det;
  r[0] = id * c00;
  r[1] = id * (d00 * d22 - d02 * d02);
  r[2] = id * (d00 * d11 - d01 * d01);
  r[3] = id * c01;
  r[4] = id * c02;
  r[5] = id * (d01 * d02 - d00 * d12);
}

CKMPM_DEV void matmul3(const float* a, const float* b, float* r) {
  float t[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) t[i * 3 + j] = a[i * 3] * b[j] + a[i * 3 + 1] * b[3 + j] + a[i * 3 + 2] * b[6 + j];
#pragma unroll
  for (int k = 0; k < 9; ++k) r[k] = t[k];
}

// ------------------------------------------------------------------ SVD
//
// A = U diag(S) V^T with U, V proper rotations, |S0| >= |S1| >= |S2|, S0, S1 >= 0
// and the sign of det(A) on S2 -- the convention of the method of
// McAdams, Selle, Tamstorf, Teran, Sifakis, "Computing the Singular Value
// Decomposition of 3x3 matrices with minimal branching and elementary floating
// point operations", UW-Madison TR1690 (2011), which the reference vendors
// (include/mpm_math.cuh:1-18).  Implemented here from the published outline:
//   1. symmetric eigenproblem of A^T A by cyclic Jacobi (fixed sweep count,
//      exact rotation angles from the 2x2 Schur form).  Three sweeps reach
//      FP32 rounding: in an FP32 emulation of these steps over 4000 random
//      F = R1 diag(s) R2 per family, with s in [0.1, 3] and
//      e^[-2, 2], and I + N(0, 0.5) shears, the singular values agree with an
//      FP64 SVD to 4e-7 relative (max) with three sweeps and with four; the
//      off-diagonal residual of (A V)^T (A V) is ~1.6e-7 at the 99th percentile
//      either way, and up to 6e-6 for about 1 matrix in 1000 with three
//      (2.7e-7 at worst with four); the fourth sweep costs ~2 % of the substep
//      (tests/test_svd_sweeps.py restates these steps and checks the bounds);
//   2. B = A V, columns sorted by decreasing norm (sign flips keep det V = 1);
//   3. Givens QR of B gives U and the diagonal S.

// 1/sqrt(x) from the hardware estimate (up to 2 ulp) with one Newton step: ~1 ulp,
// and exactly 1 for x = 1, so that a pair left unrotated keeps c = 1, s = 0.
CKMPM_DEV float rsqrt_refined(float x) {
  const float r = rsqrtf(x);
  return r * fmaf(-0.5f * x * r, r, 1.5f);
}

// Off-diagonal entries of A^T A below this magnitude are left in place, as the
// reference's SVD leaves a pair unrotated when (a_pq / 2)^2 < 1e-20
// (include/mpm_math.cuh:117-123).  Without it a deformation gradient within
// rounding of the identity (every particle of a rigidly moving or free-falling
// body) has equal diagonal entries and a 1e-11 off-diagonal, which an exact
// Jacobi step rotates by 45 degrees; the re-projected F = U V^T of the
// Drucker-Prager tension branch then carries ~1e-7 of rounding back into F
// every substep.
constexpr float kJacobiNegligible = 2e-10f;

CKMPM_DEV void jacobi_rotate(float& app, float& aqq, float& apq, float& arp, float& arq, float* V, int p, int q) {
  if (!(fabsf(apq) >= kJacobiNegligible)) return;
  // Zero apq.  t = tan(theta) of the smaller rotation solving
  // t^2 + 2 tau t - 1 = 0 with tau = (aqq - app) / (2 apq).
  const float d = aqq - app;
  const float e = 2.0f * apq;
  const float h = sqrtf(d * d + e * e);
  const float den = d + copysignf(h, d);
  float t = den != 0.0f ? e / den : 0.0f;
  const float c = rsqrt_refined(1.0f + t * t);
  const float s = t * c;
  app = app - t * apq;
  aqq = aqq + t * apq;
  apq = 0.0f;
  const float rp = arp, rq = arq;
  arp = c * rp - s * rq;
  arq = s * rp + c * rq;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float vp = V[k * 3 + p], vq = V[k * 3 + q];
    V[k * 3 + p] = c * vp - s * vq;
    V[k * 3 + q] = s * vp + c * vq;
  }
}

// Entries below this are already zero for the QR (the reference's threshold
// for its QR Givens steps, include/mpm_math.cuh:735-741).
constexpr float kQrNegligible = 1e-12f;

CKMPM_DEV void givens_qr_step(float* B, float* U, int p, int q, int col) {
  const float a = B[p * 3 + col], b = B[q * 3 + col];
  float c = a < 0.0f ? -1.0f : 1.0f, s = 0.0f;
  if (fabsf(b) >= kQrNegligible) {
    const float ir = rsqrt_refined(a * a + b * b);
    c = a * ir;
    s = b * ir;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float bp = B[p * 3 + k], bq = B[q * 3 + k];
    B[p * 3 + k] = c * bp + s * bq;
    B[q * 3 + k] = -s * bp + c * bq;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float up = U[k * 3 + p], uq = U[k * 3 + q];
    U[k * 3 + p] = c * up + s * uq;
    U[k * 3 + q] = -s * up + c * uq;
  }
}

CKMPM_DEV void swap_cols(float* V, float& la, float& lb, int a, int b) {
  const float t = la;
  la = lb;
  lb = t;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float va = V[k * 3 + a];
    V[k * 3 + a] = V[k * 3 + b];
    V[k * 3 + b] = -va;
  }
}

template <int kSweeps = 3>
CKMPM_DEV void svd3(const float* A, float* U, float* S, float* V) {
  // M = A^T A (symmetric; 6 unique entries)
  float m00 = A[0] * A[0] + A[3] * A[3] + A[6] * A[6];
  float m11 = A[1] * A[1] + A[4] * A[4] + A[7] * A[7];
  float m22 = A[2] * A[2] + A[5] * A[5] + A[8] * A[8];
  float m01 = A[0] * A[1] + A[3] * A[4] + A[6] * A[7];
  float m02 = A[0] * A[2] + A[3] * A[5] + A[6] * A[8];
  float m12 = A[1] * A[2] + A[4] * A[5] + A[7] * A[8];
#pragma unroll
  for (int k = 0; k < 9; ++k) V[k] = (k & 3) ? 0.0f : 1.0f;
#pragma unroll
  for (int sweep = 0; sweep < kSweeps; ++sweep) {
    jacobi_rotate(m00, m11, m01, m02, m12, V, 0, 1);  // r = 2: (m20, m21)
    jacobi_rotate(m00, m22, m02, m01, m12, V, 0, 2);  // r = 1: (m10, m12)
    jacobi_rotate(m11, m22, m12, m01, m02, V, 1, 2);  // r = 0: (m01, m02)
  }
  float l0 = m00, l1 = m11, l2 = m22;
  if (l0 < l1) swap_cols(V, l0, l1, 0, 1);
  if (l0 < l2) swap_cols(V, l0, l2, 0, 2);
  if (l1 < l2) swap_cols(V, l1, l2, 1, 2);
  float B[9];
  matmul3(A, V, B);
#pragma unroll
  for (int k = 0; k < 9; ++k) U[k] = (k & 3) ? 0.0f : 1.0f;
  givens_qr_step(B, U, 0, 1, 0);
  givens_qr_step(B, U, 0, 2, 0);
  givens_qr_step(B, U, 1, 2, 1);
  S[0] = B[0];
  S[1] = B[4];
  S[2] = B[8];
}

// ------------------------------------------------------------------ CK weights
// w0 = 1 - o + sin(2 pi o) / (2 pi) for offset o in [0, 1); node weights are
// w0 and 1 - w0 along each axis (include/mpm_kernel.cuh:91-114, which also
// evaluates the sine with the __sinf intrinsic).
CKMPM_DEV float ck_w0(float o) {
  const float kTwoPi = 6.283185307179586f;
  const float kInvTwoPi = 0.15915494309189535f;
  return 1.0f - o + kInvTwoPi * __sinf(kTwoPi * o);
}

// ------------------------------------------------------------------ materials
// Numbering of MPMConstitutiveModel (include/mpm_material.cuh:10-18).
enum MaterialKind : int32_t {
  kFixedCorotated = 0,
  kLinear = 1,
  kDruckerPrager = 2,
  kFluid = 3,
  kVonMises = 4,
  kNacc = 5,
};

constexpr int kMaterialParams = 8;

struct MaterialParams {
  int32_t kind;
  // FC / DP / Linear: lambda, mu.  Fluid: bulk, gamma, viscosity, J0.  Von Mises: mu, lambda, yield
  // stress.  NACC: mu, lambda, alpha0, beta, hardening factor, M, hardening on (0 / 1).
  float p[kMaterialParams];
};

// Fixed-corotated Kirchhoff stress, tau = U diag(2 mu s (s - 1) + lambda J (J - 1)) U^T
// (include/mpm_material.cuh:320-357).
CKMPM_DEV void stress_fixed_corotated(float lambda, float mu, const float* F, float* tau) {
  float U[9], S[3], V[9];
  svd3(F, U, S, V);
  const float J = S[0] * S[1] * S[2];
  const float lj = lambda * J * (J - 1.0f);
  float sc[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) sc[i] = 2.0f * mu * S[i] * (S[i] - 1.0f) + lj;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = r; c < 3; ++c) {
      const float v = U[r * 3] * sc[0] * U[c * 3] + U[r * 3 + 1] * sc[1] * U[c * 3 + 1] + U[r * 3 + 2] * sc[2] * U[c * 3 + 2];
      tau[r * 3 + c] = v;
      tau[c * 3 + r] = v;
    }
}

// Drucker-Prager StVK-Hencky return map with the reference's constants:
// zero cohesion, beta = 1, volume correction on, sin(phi) = 0.5
// (include/mpm_material.cuh:362-464).  Updates F and logJp in place.
CKMPM_DEV void stress_drucker_prager(float lambda, float mu, float* F, float& logJp, float* tau) {
  const float kYs = 0.816496580927726f * 2.0f * 0.5f / (3.0f - 0.5f);
  const float smu = 2.0f * mu;
  float U[9], S[3], V[9];
  svd3(F, U, S, V);
  float eps[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) eps[i] = logf(fmaxf(fabsf(S[i]), 1e-4f));
  const float esum = eps[0] + eps[1] + eps[2];
  const float etr = esum + logJp;
  float eh[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) eh[i] = eps[i] - etr / 3.0f;
  const float ehn = sqrtf(eh[0] * eh[0] + eh[1] * eh[1] + eh[2] * eh[2]);
  float ns[3];
  if (etr >= 0.0f) {
    ns[0] = ns[1] = ns[2] = 1.0f;
    logJp = esum + logJp;
  } else {
    logJp = 0.0f;
    const float dg = ehn + (3.0f * lambda + smu) / smu * etr * kYs;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const float H = dg <= 0.0f ? eps[i] : eps[i] - (dg / ehn) * eh[i];
      ns[i] = expf(H);
    }
  }
  // F <- U diag(ns) V^T
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      F[r * 3 + c] = U[r * 3] * ns[0] * V[c * 3] + U[r * 3 + 1] * ns[1] * V[c * 3 + 1] + U[r * 3 + 2] * ns[2] * V[c * 3 + 2];
  // tau = U diag(p) V^T F^T with p = (2 mu log s + lambda tr log s) / s (the reference's order,
  // include/mpm_material.cuh:447-463).  With F = U diag(s) V^T and V orthogonal,
  // V^T F^T = diag(s) U^T, so tau = U diag(2 mu log s + lambda tr log s) U^T: symmetric, and
  // 36 multiply-adds and three divisions fewer per particle (1.7 % of the fused substep on the
  // sand column).  log s is 0 on the tension branch (s = 1), and log(exp(H)) there otherwise.
  float h[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) h[i] = etr >= 0.0f ? 0.0f : logf(ns[i]);
  const float trh = h[0] + h[1] + h[2];
  float sc[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) sc[i] = smu * h[i] + lambda * trh;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = r; c < 3; ++c) {
      const float v = U[r * 3] * sc[0] * U[c * 3] + U[r * 3 + 1] * sc[1] * U[c * 3 + 1] + U[r * 3 + 2] * sc[2] * U[c * 3 + 2];
      tau[r * 3 + c] = v;
      tau[c * 3 + r] = v;
    }
}

// Von Mises plasticity on the Hencky strain of the trial elastic F, then the
// StVK-Hencky stress of the projected F from its own SVD, as the reference
// computes it (include/mpm_algorithm.cuh:404-520, include/mpm_material.cuh:480-518):
//   eps = log S, eps_hat = eps - tr(eps) / 3, f = |eps_hat| - yield / (2 mu);
//   f > 0: S <- exp(eps - f eps_hat / |eps_hat|), Fe <- U diag(S) V^T;
//   tau = U diag((2 mu log S + lambda tr log S) / S) V^T Fe^T.
// Fe holds the trial elastic F on entry and the projected one on exit.
CKMPM_DEV void stress_von_mises(float mu, float lambda, float yield, float* Fe, float* tau) {
  float U[9], S[3], V[9];
  svd3(Fe, U, S, V);
  float eps[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) eps[i] = logf(S[i]);
  const float etr = eps[0] + eps[1] + eps[2];
  float eh[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) eh[i] = eps[i] - etr / 3.0f;
  const float ehn = sqrtf(eh[0] * eh[0] + eh[1] * eh[1] + eh[2] * eh[2]);
  const float yf = ehn - yield / (2.0f * mu);
  if (yf > 0.0f) {
    float ns[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) ns[i] = expf(eps[i] - yf * eh[i] / ehn);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        Fe[r * 3 + c] = U[r * 3] * ns[0] * V[c * 3] + U[r * 3 + 1] * ns[1] * V[c * 3 + 1] + U[r * 3 + 2] * ns[2] * V[c * 3 + 2];
  }
  svd3(Fe, U, S, V);
  float ls[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) ls[i] = logf(S[i]);
  const float lsum = ls[0] + ls[1] + ls[2];
  float ph[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float inv = 1.0f / S[i];
    ph[i] = 2.0f * mu * inv * ls[i] + lambda * lsum * inv;
  }
  float P[9];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      P[r * 3 + c] = U[r * 3] * ph[0] * V[c * 3] + U[r * 3 + 1] * ph[1] * V[c * 3 + 1] + U[r * 3 + 2] * ph[2] * V[c * 3 + 2];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      tau[r * 3 + c] = P[r * 3] * Fe[c * 3] + P[r * 3 + 1] * Fe[c * 3 + 1] + P[r * 3 + 2] * Fe[c * 3 + 2];
}

// Non-associated Cam-clay (include/mpm_material.cuh:520-669, driven from
// include/mpm_algorithm.cuh:330-402), restated step for step, including what
// it does beyond the textbook model, so that results match the reference:
//  * the projected F is U diag(S) V (V itself, not its transpose); the stress
//    only sees F F^T = U S^2 U^T, so V never affects the motion, but the stored
//    F is fixed only up to a rotation on the right;
//  * the hardening update of the yield-surface branch sits in a loop of 9
//    identical iterations, so logJp takes the same increment 9 times;
//  * thresholds written as double literals (1e-4) compare in double.
// Both branches (pressure clamped to [pMin, p0], or the return to the yield
// surface) end in the same stress: mu Je_trial^(-2/3) dev(F F^T) + K/2 (J^2 - 1) I.
// F holds dW F_old on entry and the projected F on exit.
CKMPM_DEV void stress_nacc(const float* prm, float* F, float& logJp, float* tau) {
  const float mu = prm[0], lambda = prm[1], beta = prm[3], xi = prm[4], msq = prm[5] * prm[5];
  const bool hardening = prm[6] != 0.0f;
  const float K = 2.0f * mu / 3.0f + lambda;
  float U[9], S[3], V[9];
  svd3(F, U, S, V);
  const float p0 = K * (1e-5f + sinhf(xi * (-logJp > 0.0f ? -logJp : 0.0f)));
  const float pmin = -beta * p0;
  const float je = S[0] * S[1] * S[2];
  const float bh[3] = {S[0] * S[0], S[1] * S[1], S[2] * S[2]};
  const float btr3 = (bh[0] + bh[1] + bh[2]) / 3.0f;
  const float devf = mu * powf(je, -2.0f / 3.0f);
  const float sh[3] = {devf * (bh[0] - btr3), devf * (bh[1] - btr3), devf * (bh[2] - btr3)};
  const float hydro = K * 0.5f * (je - 1.0f / je);
  const float ptrial = -hydro * je;
  const float ysh = 3.0f / 2.0f * (1.0f + 2.0f * beta);
  const float yph = msq * (ptrial - pmin) * (ptrial - p0);
  const float sn2 = sh[0] * sh[0] + sh[1] * sh[1] + sh[2] * sh[2];
  const float y = ysh * sn2 + yph;
  float Sn[3] = {S[0], S[1], S[2]};
  if (ptrial > p0 || ptrial < pmin) {
    const float pp = ptrial > p0 ? p0 : pmin;
    const float jn = sqrtf(-2.0f * pp / K + 1.0f);
    const float sc = powf(jn, 1.0f / 3.0f);
    Sn[0] = Sn[1] = Sn[2] = sc;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        F[r * 3 + c] = sc * (U[r * 3] * V[c] + U[r * 3 + 1] * V[3 + c] + U[r * 3 + 2] * V[6 + c]);
    if (hardening) logJp += logf(je / jn);
  } else if (static_cast<double>(y) >= 1e-4) {
    const float coef = powf(je, 2.0f / 3.0f) / mu * sqrtf(-yph / ysh) / sqrtf(sn2);
#pragma unroll
    for (int i = 0; i < 3; ++i) Sn[i] = sqrtf(sh[i] * coef + btr3);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        F[r * 3 + c] = U[r * 3] * Sn[0] * V[c] + U[r * 3 + 1] * Sn[1] * V[3 + c] + U[r * 3 + 2] * Sn[2] * V[6 + c];
    if (hardening && static_cast<double>(p0) > 1e-4 && static_cast<double>(ptrial) < static_cast<double>(p0) - 1e-4 &&
        static_cast<double>(ptrial) > 1e-4 + static_cast<double>(pmin)) {
      const float pc = (1.0f - beta) * p0 / 2.0f;
      const float qt = sqrtf(3.0f / 2.0f * sn2);
      float d0 = pc - ptrial, d1 = -qt;
      const float dn = sqrtf(d0 * d0 + d1 * d1);
      d0 /= dn;
      d1 /= dn;
      const float A = msq * d0 * d0 + (1.0f + 2.0f * beta) * d1 * d1;
      const float B = msq * d0 * (2.0f * pc - p0 - pmin);
      const float C = msq * (pc - pmin) * (pc - p0);
      const float disc = B * B - 4.0f * A * C;
      const float l1 = (-B + sqrtf(disc)) / (2.0f * A);
      const float l2 = (-B - sqrtf(disc)) / (2.0f * A);
      const float p1 = pc + l1 * d0, p2 = pc + l2 * d0;
      const float pf = (ptrial - pc) * (p1 - pc) > 0.0f ? p1 : p2;
      const float jsq = -2.0f * pf / K + 1.0f;
      const float jn = sqrtf(jsq > 0.0f ? jsq : -jsq);
      if (static_cast<double>(jn) > 1e-4) {
        const float inc = logf(je / jn);
        for (int it = 0; it < 9; ++it) logJp += inc;
      }
    }
  }
  const float J = Sn[0] * Sn[1] * Sn[2];
  float b[9];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) b[r * 3 + c] = F[r * 3] * F[c * 3] + F[r * 3 + 1] * F[c * 3 + 1] + F[r * 3 + 2] * F[c * 3 + 2];
  const float btr = (b[0] + b[4] + b[8]) / 3.0f;
  const float hc = K * 0.5f * (J * J - 1.0f);
#pragma unroll
  for (int k = 0; k < 9; ++k) tau[k] = devf * (b[k] - ((k & 3) ? 0.0f : btr));
  tau[0] += hc;
  tau[4] += hc;
  tau[8] += hc;
}

// Linear model as the reference updates it (include/mpm_algorithm.cuh:107-191):
// F <- dW F (done by the caller); the stored stress Q <- (Q + 50 (C + C^T - I) dt)
// det(F), with its rows 1 and 2 zeroed; tau = Q.  lambda and mu are not read.
CKMPM_DEV void stress_linear(const float* C, float dt, const float* F, float* Q, float* tau) {
  const float detF = det3(F);
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int k = r * 3 + c;
      const float t = 50.0f * (C[k] + C[c * 3 + r] - ((k & 3) ? 0.0f : 1.0f)) * dt;
      Q[k] = r == 0 ? (Q[k] + t) * detF : 0.0f;
    }
#pragma unroll
  for (int k = 0; k < 9; ++k) tau[k] = Q[k];
}

// J-fluid: J += tr(C) dt J; p = bulk (J^-gamma - 1); tau = J (visc (C + C^T) - p I)
// (include/mpm_algorithm.cuh:528-569, include/mpm_material.cuh:468-477).
CKMPM_DEV void stress_fluid(float bulk, float gamma, float visc, const float* C, float dt, float& J, float* tau) {
  J += (C[0] + C[4] + C[8]) * dt * J;
  const float p = bulk * (powf(J, -gamma) - 1.0f);
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) tau[r * 3 + c] = (C[r * 3 + c] + C[c * 3 + r]) * visc;
  tau[0] -= p;
  tau[4] -= p;
  tau[8] -= p;
#pragma unroll
  for (int k = 0; k < 9; ++k) tau[k] *= J;
}

}  // namespace ckmpm
