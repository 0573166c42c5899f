// Differentiable CK-MPM substep: the per-particle forward of the fixed-corotated
// substep on a dense grid and its hand-written adjoint, generic in the scalar
// type T so that the same source runs on the GPU (T = float) and in double on
// the host for finite-difference checks of the derivation.
//
// Forward (one substep; dt advects, ndt deposits stress, as the substep of
// include/mpm_algorithm.cuh:1367-1845 with currentDt / nextDt):
//   G2P at x:   v = 1/2 sum_i w_i v_i,  B = sum_i w_i v_i r_i^T,  C = B D^-1
//   x' = x + dt v;   F' = (I + dt C) F
//   tau = 2 mu (F' - R) F'^T + lambda J (J - 1) I        (R = U V^T, F' = U S V^T)
//   P2G at x':  m_i += m w'_i,  mv_i += m w'_i (v + A r'_i),  A = C - ndt V/m M tau,
//               M = (0.5 (D + D'))^-1 (the reference adds D' at x' onto the G2P D at x
//               and inverts half the sum, include/mpm_algorithm.cuh:1524,1604,1729-1732)
// with r_i = (d - o) dx the node offset from the particle, w_i the tensor
// product of CK weights w0(o) = 1 - o + sin(2 pi o) / (2 pi) (include/mpm_kernel.cuh:91-114),
// and D = sum_i w_i r_i r_i^T over both staggered grids (g = -1/4, +1/4 dx).
//
// Adjoint (reverse of the above, per particle; the grid adjoint of the
// deposit is gathered, the grid adjoint of G2P is scattered):
//   P2G:  vbar += m sum w' mvbar_i;  Abar = m sum w' mvbar_i r'_i^T;
//         x'bar from dw'/dx', from dr'/dx' = -I and from D'(x')
//   A:    Cbar += Abar;  (M tau)bar = -ndt V/m Abar;  Mbar = (M tau)bar tau^T;
//         taubar = M (M tau)bar;  Dbar' = Dbar(M) = -1/2 M Mbar M
//   tau:  Fbar' += 2 mu (taubar F' + taubar (F' - R)) + polar term of Rbar = -2 mu taubar F'
//         + lambda (2J - 1) tr(taubar) cof(F');  mubar, lambdabar for the parameters
//         polar term: Q = U^T Rbar V, Mbar_ij = (Q_ij - Q_ji) / (s_i + s_j), Fbar += U Mbar V^T
//   F:    Fbar = (I + dt C)^T Fbar';  Cbar += dt Fbar' F^T
//   x:    xbar += x'bar;  vbar += dt x'bar
//   C:    Bbar = Cbar D^-1;  Dbar = -D^-1 B^T Cbar D^-1 + Dbar(M)
//   G2P:  vibar_i += 1/2 w_i vbar + w_i Bbar r_i;  xbar from dw/dx, dr/dx, D(x)
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define CKD __host__ __device__ __forceinline__
#define CKD_UNROLL _Pragma("unroll")
#define CKD_ROLLED _Pragma("unroll 1")
#else
#define CKD inline
#define CKD_UNROLL
#define CKD_ROLLED
#endif

#include <cmath>

namespace ckmpm {
namespace diff {

template <class T>
CKD T dsin(T a) {
#if defined(__CUDA_ARCH__)
  if constexpr (sizeof(T) == 4) return __sinf(a);  // as the substep's weights (include/mpm_kernel.cuh:109)
  else return sin(a);
#else
  return std::sin(a);
#endif
}

template <class T>
CKD T dcos(T a) {
#if defined(__CUDA_ARCH__)
  if constexpr (sizeof(T) == 4) return __cosf(a);
  else return cos(a);
#else
  return std::cos(a);
#endif
}

// ------------------------------------------------------------------ 3x3 helpers (row-major)
template <class T>
CKD void mm(const T* a, const T* b, T* r) {  // r = a b (r may alias neither)
  CKD_UNROLL
  for (int i = 0; i < 3; ++i)
    CKD_UNROLL
    for (int j = 0; j < 3; ++j) r[i * 3 + j] = a[i * 3] * b[j] + a[i * 3 + 1] * b[3 + j] + a[i * 3 + 2] * b[6 + j];
}

template <class T>
CKD void mmt(const T* a, const T* b, T* r) {  // r = a b^T
  CKD_UNROLL
  for (int i = 0; i < 3; ++i)
    CKD_UNROLL
    for (int j = 0; j < 3; ++j) r[i * 3 + j] = a[i * 3] * b[j * 3] + a[i * 3 + 1] * b[j * 3 + 1] + a[i * 3 + 2] * b[j * 3 + 2];
}

template <class T>
CKD void mtm(const T* a, const T* b, T* r) {  // r = a^T b
  CKD_UNROLL
  for (int i = 0; i < 3; ++i)
    CKD_UNROLL
    for (int j = 0; j < 3; ++j) r[i * 3 + j] = a[i] * b[j] + a[3 + i] * b[3 + j] + a[6 + i] * b[6 + j];
}

template <class T>
CKD void sym_full(const T* s6, T* f) {  // (00, 11, 22, 01, 02, 12) -> full
  f[0] = s6[0];
  f[4] = s6[1];
  f[8] = s6[2];
  f[1] = f[3] = s6[3];
  f[2] = f[6] = s6[4];
  f[5] = f[7] = s6[5];
}

template <class T>
CKD void inv_sym(const T* d, T* r) {  // inverse of a symmetric 3x3 (6 entries in, 6 out)
  const T c00 = d[1] * d[2] - d[5] * d[5];
  const T c01 = d[4] * d[5] - d[3] * d[2];
  const T c02 = d[3] * d[5] - d[4] * d[1];
  const T det = d[0] * c00 + d[3] * c01 + d[4] * c02;
  const T id = T(1) / det;
  r[0] = id * c00;
  r[1] = id * (d[0] * d[2] - d[4] * d[4]);
  r[2] = id * (d[0] * d[1] - d[3] * d[3]);
  r[3] = id * c01;
  r[4] = id * c02;
  r[5] = id * (d[3] * d[4] - d[0] * d[5]);
}

template <class T>
CKD void cofactor(const T* a, T* c) {  // cof(A) = det(A) A^-T
  c[0] = a[4] * a[8] - a[5] * a[7];
  c[1] = a[5] * a[6] - a[3] * a[8];
  c[2] = a[3] * a[7] - a[4] * a[6];
  c[3] = a[2] * a[7] - a[1] * a[8];
  c[4] = a[0] * a[8] - a[2] * a[6];
  c[5] = a[1] * a[6] - a[0] * a[7];
  c[6] = a[1] * a[5] - a[2] * a[4];
  c[7] = a[2] * a[3] - a[0] * a[5];
  c[8] = a[0] * a[4] - a[1] * a[3];
}

// ------------------------------------------------------------------ stencil
// One axis of one grid: base cell, offset o in [0,1), w0(o) and dw0/do.
template <class T>
struct Axis {
  int base;
  T o, w0, dw0;
};

// Both grids (index 0: -dx/4, 1: +dx/4), three axes, at scaled position xs = x / dx.
template <class T>
struct Stencil {
  Axis<T> a[2][3];
};

template <class T>
CKD void make_stencil(const T* x, T inv_dx, Stencil<T>& st) {
  const T kTwoPi = T(6.283185307179586);
  const T kInvTwoPi = T(0.15915494309189535);
  CKD_UNROLL
  for (int g = 0; g < 2; ++g) {
    const T shift = g == 0 ? T(-0.25) : T(0.25);
    CKD_UNROLL
    for (int a = 0; a < 3; ++a) {
      const T xs = x[a] * inv_dx;
      Axis<T>& s = st.a[g][a];
      s.base = static_cast<int>(xs - shift);
      s.o = (xs - static_cast<T>(s.base)) - shift;
      s.w0 = T(1) - s.o + kInvTwoPi * dsin(kTwoPi * s.o);
      s.dw0 = T(-1) + dcos(kTwoPi * s.o);
    }
  }
}

// Weight of node d (bits dx dy dz) of grid g and its gradient in x (world units).
template <class T>
CKD T node_weight(const Stencil<T>& st, int g, int n, T inv_dx, T* grad) {
  T w[3], dw[3];
  CKD_UNROLL
  for (int a = 0; a < 3; ++a) {
    const int d = (n >> (2 - a)) & 1;
    const Axis<T>& s = st.a[g][a];
    w[a] = d ? T(1) - s.w0 : s.w0;
    dw[a] = (d ? -s.dw0 : s.dw0) * inv_dx;
  }
  if (grad) {
    grad[0] = dw[0] * w[1] * w[2];
    grad[1] = w[0] * dw[1] * w[2];
    grad[2] = w[0] * w[1] * dw[2];
  }
  return w[0] * w[1] * w[2];
}

// D = sum over both grids' 16 nodes of w r r^T (6 entries), from per-axis moments
// m1 = (w1 - o) dx and m2 = (w0 o^2 + w1 (1 - o)^2) dx^2: D_aa = sum_g m2, D_ab = sum_g m1_a m1_b.
template <class T>
CKD void d_moments(const Axis<T>& s, T dx, T& m1, T& m2, T& dm1, T& dm2) {
  const T w1 = T(1) - s.w0, o = s.o, q = T(1) - o;
  m1 = (w1 - o) * dx;
  m2 = (s.w0 * o * o + w1 * q * q) * dx * dx;
  dm1 = (-s.dw0 - T(1)) * dx;                                              // d m1 / d o
  dm2 = (s.dw0 * o * o + T(2) * s.w0 * o - s.dw0 * q * q - T(2) * w1 * q) * dx * dx;  // d m2 / d o
}

template <class T>
CKD void d_matrix(const Stencil<T>& st, T dx, T* D6) {
  T m1[2][3], m2[2][3], u, v;
  CKD_UNROLL
  for (int g = 0; g < 2; ++g)
    CKD_UNROLL
    for (int a = 0; a < 3; ++a) d_moments(st.a[g][a], dx, m1[g][a], m2[g][a], u, v);
  D6[0] = m2[0][0] + m2[1][0];
  D6[1] = m2[0][1] + m2[1][1];
  D6[2] = m2[0][2] + m2[1][2];
  D6[3] = m1[0][0] * m1[0][1] + m1[1][0] * m1[1][1];
  D6[4] = m1[0][0] * m1[0][2] + m1[1][0] * m1[1][2];
  D6[5] = m1[0][1] * m1[0][2] + m1[1][1] * m1[1][2];
}

// xbar += dL/dx given Dbar (full 3x3 adjoint of the symmetric D).
template <class T>
CKD void d_matrix_adjoint(const Stencil<T>& st, T dx, T inv_dx, const T* Dbar, T* xbar) {
  T m1[2][3], m2[2][3], dm1[2][3], dm2[2][3];
  CKD_UNROLL
  for (int g = 0; g < 2; ++g)
    CKD_UNROLL
    for (int a = 0; a < 3; ++a) d_moments(st.a[g][a], dx, m1[g][a], m2[g][a], dm1[g][a], dm2[g][a]);
  CKD_UNROLL
  for (int a = 0; a < 3; ++a) {
    T acc = T(0);
    CKD_UNROLL
    for (int g = 0; g < 2; ++g) {
      acc += Dbar[a * 3 + a] * dm2[g][a];
      CKD_UNROLL
      for (int b = 0; b < 3; ++b)
        if (b != a) acc += (Dbar[a * 3 + b] + Dbar[b * 3 + a]) * m1[g][b] * dm1[g][a];
    }
    xbar[a] += acc * inv_dx;
  }
}

// ------------------------------------------------------------------ fixed-corotated stress
// tau = U diag(2 mu s (s - 1) + lambda J (J - 1)) U^T from an SVD F = U diag(S) V^T
// (include/mpm_material.cuh:320-357).
template <class T>
CKD void fc_tau(const T* U, const T* S, T lambda, T mu, T* tau) {
  const T J = S[0] * S[1] * S[2];
  const T lj = lambda * J * (J - T(1));
  T sc[3];
  CKD_UNROLL
  for (int i = 0; i < 3; ++i) sc[i] = T(2) * mu * S[i] * (S[i] - T(1)) + lj;
  CKD_UNROLL
  for (int r = 0; r < 3; ++r)
    CKD_UNROLL
    for (int c = 0; c < 3; ++c)
      tau[r * 3 + c] = U[r * 3] * sc[0] * U[c * 3] + U[r * 3 + 1] * sc[1] * U[c * 3 + 1] + U[r * 3 + 2] * sc[2] * U[c * 3 + 2];
}

// Adjoint of tau(F) = 2 mu (F - R) F^T + lambda J (J - 1) I at F = U diag(S) V^T:
// Fbar += dL/dF, mubar / lambdabar += dL/dmu, dL/dlambda, for taubar (any 3x3).
template <class T>
CKD void fc_tau_adjoint(const T* F, const T* U, const T* S, const T* V, T lambda, T mu, const T* taubar_in, T* Fbar,
                        T& mubar, T& lambdabar) {
  T tb[9];
  CKD_UNROLL
  for (int r = 0; r < 3; ++r)
    CKD_UNROLL
    for (int c = 0; c < 3; ++c) tb[r * 3 + c] = T(0.5) * (taubar_in[r * 3 + c] + taubar_in[c * 3 + r]);
  T R[9], X[9];
  mmt(U, V, R);  // R = U V^T
  CKD_UNROLL
  for (int k = 0; k < 9; ++k) X[k] = F[k] - R[k];
  // tau1 = 2 mu X F^T: Xbar = 2 mu tb F and Fbar += 2 mu tb X; then X = F - R
  // gives Fbar += Xbar and Rbar = -Xbar.
  T tbF[9], tbX[9];
  mm(tb, F, tbF);
  mm(tb, X, tbX);
  T Rbar[9];
  CKD_UNROLL
  for (int k = 0; k < 9; ++k) {
    Fbar[k] += T(2) * mu * (tbF[k] + tbX[k]);
    Rbar[k] = -T(2) * mu * tbF[k];
  }
  // polar rotation: Q = U^T Rbar V; Mbar_ij = (Q_ij - Q_ji) / (s_i + s_j); Fbar += U Mbar V^T
  T t1[9], Q[9];
  mtm(U, Rbar, t1);
  mm(t1, V, Q);
  T Mb[9];
  CKD_UNROLL
  for (int i = 0; i < 3; ++i)
    CKD_UNROLL
    for (int j = 0; j < 3; ++j) {
      if (i == j) {
        Mb[i * 3 + j] = T(0);
      } else {
        const T den = S[i] + S[j];
        Mb[i * 3 + j] = den != T(0) ? (Q[i * 3 + j] - Q[j * 3 + i]) / den : T(0);
      }
    }
  T t2[9], t3[9];
  mm(U, Mb, t2);
  mmt(t2, V, t3);
  CKD_UNROLL
  for (int k = 0; k < 9; ++k) Fbar[k] += t3[k];
  // lambda J (J - 1) I
  const T J = S[0] * S[1] * S[2];
  const T tr = tb[0] + tb[4] + tb[8];
  T cof[9];
  cofactor(F, cof);
  const T cj = lambda * (T(2) * J - T(1)) * tr;
  CKD_UNROLL
  for (int k = 0; k < 9; ++k) Fbar[k] += cj * cof[k];
  // parameters
  T XFt[9];
  mmt(X, F, XFt);
  T s = T(0);
  CKD_UNROLL
  for (int k = 0; k < 9; ++k) s += tb[k] * XFt[k];
  mubar += T(2) * s;
  lambdabar += J * (J - T(1)) * tr;
}

// ------------------------------------------------------------------ grid update
// Node velocity from mass and momentum (include/mpm_algorithm.cuh:739-869):
// v = mv / m + g dt e_y when m > clamp and the node's block is not within two
// blocks of the domain edge (sticky, boundary 0) or, with the slip floor
// (boundary 1), sticky x/z walls and ceiling and v_y >= 0 below floor_cells.
struct DenseGrid {
  int n[3];          // cells per axis
  int nb[3];         // blocks per axis (n / 4)
  float gravity, mass_clamp, floor_cells;
  int boundary;
};

CKD bool node_active_block(const DenseGrid& G, int cx, int cy, int cz) {
  const int bx = cx >> 2, by = cy >> 2, bz = cz >> 2;
  if (G.boundary == 0)
    return !(bx < 2 || bx + 2 >= G.nb[0] || by < 2 || by + 2 >= G.nb[1] || bz < 2 || bz + 2 >= G.nb[2]);
  return !(bx < 2 || bx + 2 >= G.nb[0] || bz < 2 || bz + 2 >= G.nb[2] || by + 2 >= G.nb[1]);
}

CKD int64_t node_index(const DenseGrid& G, int g, int cx, int cy, int cz) {
  return ((static_cast<int64_t>(g) * G.n[0] + cx) * G.n[1] + cy) * G.n[2] + cz;
}

CKD bool node_in_grid(const DenseGrid& G, int cx, int cy, int cz) {
  return cx >= 0 && cy >= 0 && cz >= 0 && cx < G.n[0] && cy < G.n[1] && cz < G.n[2];
}

// ------------------------------------------------------------------ particle forward / adjoint
template <class T>
struct Particle {
  T x[3], F[9];
};

// Everything the adjoint needs from the forward of one particle.
template <class T>
struct Fwd {
  Stencil<T> st, stn;       // stencils at x and at x'
  T v[3], B[9], C[9], Di[9];  // G2P result, D^-1
  T xn[3], Fn[9];
  T tau[9], M[9], A[9];     // M = (0.5 (D + D'))^-1, A per unit mass
};

// G2P + x, F update + stress + affine term.  vel(g, cx, cy, cz, T* v) returns
// the node velocity after the grid update; svd(F, U, S, V) any SVD.
template <class T, class Vel, class Svd>
CKD void particle_forward(const Particle<T>& p, T lambda, T mu, T vol_over_mass, T dt, T ndt, T dx, T inv_dx,
                          Vel vel, Svd svd, Fwd<T>& f, T* U, T* S, T* V) {
  make_stencil(p.x, inv_dx, f.st);
  CKD_UNROLL
  for (int k = 0; k < 9; ++k) f.B[k] = T(0);
  CKD_UNROLL
  for (int a = 0; a < 3; ++a) f.v[a] = T(0);
  CKD_UNROLL
  for (int g = 0; g < 2; ++g)
    CKD_UNROLL
    for (int n = 0; n < 8; ++n) {
      const T w = node_weight(f.st, g, n, inv_dx, static_cast<T*>(nullptr));
      int c[3];
      T r[3];
      CKD_UNROLL
      for (int a = 0; a < 3; ++a) {
        const int d = (n >> (2 - a)) & 1;
        c[a] = f.st.a[g][a].base + d;
        r[a] = (static_cast<T>(d) - f.st.a[g][a].o) * dx;
      }
      T vi[3];
      vel(g, c[0], c[1], c[2], vi);
      CKD_UNROLL
      for (int i = 0; i < 3; ++i) {
        f.v[i] += w * vi[i];
        CKD_UNROLL
        for (int a = 0; a < 3; ++a) f.B[i * 3 + a] += w * vi[i] * r[a];
      }
    }
  CKD_UNROLL
  for (int i = 0; i < 3; ++i) f.v[i] *= T(0.5);
  T D6[6], Di6[6];
  d_matrix(f.st, dx, D6);
  inv_sym(D6, Di6);
  sym_full(Di6, f.Di);
  mm(f.B, f.Di, f.C);
  CKD_UNROLL
  for (int a = 0; a < 3; ++a) f.xn[a] = p.x[a] + dt * f.v[a];
  T dW[9];
  CKD_UNROLL
  for (int k = 0; k < 9; ++k) dW[k] = f.C[k] * dt + ((k & 3) ? T(0) : T(1));
  mm(dW, p.F, f.Fn);
  svd(f.Fn, U, S, V);
  fc_tau(U, S, lambda, mu, f.tau);
  make_stencil(f.xn, inv_dx, f.stn);
  T Dn6[6], M6[6];
  d_matrix(f.stn, dx, Dn6);
  CKD_UNROLL
  for (int k = 0; k < 6; ++k) Dn6[k] = T(0.5) * (D6[k] + Dn6[k]);
  inv_sym(Dn6, M6);
  sym_full(M6, f.M);
  T Mt[9];
  mm(f.M, f.tau, Mt);
  const T sA = ndt * vol_over_mass;
  CKD_UNROLL
  for (int k = 0; k < 9; ++k) f.A[k] = f.C[k] - sA * Mt[k];
}

// Deposit of one particle (per unit mass) to each of its 16 nodes at x':
// emit(g, cx, cy, cz, w, wv[3]) with node mass w and momentum w (v + A r).
template <class T, class Emit>
CKD void particle_deposit(const Fwd<T>& f, T dx, T inv_dx, Emit emit) {
  CKD_UNROLL
  for (int g = 0; g < 2; ++g)
    CKD_UNROLL
    for (int n = 0; n < 8; ++n) {
      const T w = node_weight(f.stn, g, n, inv_dx, static_cast<T*>(nullptr));
      int c[3];
      T r[3];
      CKD_UNROLL
      for (int a = 0; a < 3; ++a) {
        const int d = (n >> (2 - a)) & 1;
        c[a] = f.stn.a[g][a].base + d;
        r[a] = (static_cast<T>(d) - f.stn.a[g][a].o) * dx;
      }
      T wv[3];
      CKD_UNROLL
      for (int i = 0; i < 3; ++i) wv[i] = w * (f.v[i] + f.A[i * 3] * r[0] + f.A[i * 3 + 1] * r[1] + f.A[i * 3 + 2] * r[2]);
      emit(g, c[0], c[1], c[2], w, wv);
    }
}

// Adjoint of one particle's substep.  In: the forward record, the particle
// mass m, xnbar / Fnbar (adjoints of x', F'), gadj(g, cx, cy, cz, T* mbar_mvbar4)
// (adjoint of the deposited grid).  Out: xbar, Fbar (adjoints of x, F),
// mubar / lambdabar accumulated, and vscatter(g, cx, cy, cz, T* vibar3) for the
// adjoint of the node velocities read by G2P.
template <class T, class Vel, class GAdj, class VScatter>
CKD void particle_adjoint(const Particle<T>& p, const Fwd<T>& f, const T* U, const T* S, const T* V, T m, T lambda,
                          T mu, T vol_over_mass, T dt, T ndt, T dx, T inv_dx, Vel vel, GAdj gadj, VScatter vscatter,
                          const T* xnbar_in, const T* Fnbar_in, T* xbar, T* Fbar, T& mubar, T& lambdabar) {
  T xnb[3], Fnb[9], vb[3] = {T(0), T(0), T(0)}, Ab[9];
  CKD_UNROLL
  for (int a = 0; a < 3; ++a) xnb[a] = xnbar_in[a];
  CKD_UNROLL
  for (int k = 0; k < 9; ++k) {
    Fnb[k] = Fnbar_in[k];
    Ab[k] = T(0);
  }
  // P2G at x' (gather of the grid adjoint).  The two node loops of the adjoint
  // stay rolled: unrolled, the kernel's code outgrew the instruction cache
  // (ncu: a third of the stall samples waiting for instructions), and rolled
  // with 3 CTAs per SM the adjoint substep measured 8 % faster.
  CKD_UNROLL
  for (int g = 0; g < 2; ++g)
    CKD_ROLLED
    for (int n = 0; n < 8; ++n) {
      T gw[3];
      const T w = node_weight(f.stn, g, n, inv_dx, gw);
      int c[3];
      T r[3];
      CKD_UNROLL
      for (int a = 0; a < 3; ++a) {
        const int d = (n >> (2 - a)) & 1;
        c[a] = f.stn.a[g][a].base + d;
        r[a] = (static_cast<T>(d) - f.stn.a[g][a].o) * dx;
      }
      T gb[4];
      gadj(g, c[0], c[1], c[2], gb);  // mbar, mvbar x/y/z
      T q[3];  // v + A r
      CKD_UNROLL
      for (int i = 0; i < 3; ++i) q[i] = f.v[i] + f.A[i * 3] * r[0] + f.A[i * 3 + 1] * r[1] + f.A[i * 3 + 2] * r[2];
      T dLdw = m * gb[0];
      CKD_UNROLL
      for (int i = 0; i < 3; ++i) {
        dLdw += m * gb[1 + i] * q[i];
        vb[i] += m * w * gb[1 + i];
        CKD_UNROLL
        for (int a = 0; a < 3; ++a) Ab[i * 3 + a] += m * w * gb[1 + i] * r[a];
      }
      CKD_UNROLL
      for (int a = 0; a < 3; ++a) {
        // dr/dx' = -I: -(m w A^T mvbar)_a
        T atm = T(0);
        CKD_UNROLL
        for (int i = 0; i < 3; ++i) atm += f.A[i * 3 + a] * gb[1 + i];
        xnb[a] += dLdw * gw[a] - m * w * atm;
      }
    }
  // A = C - ndt V/m M tau
  T Cb[9];
  CKD_UNROLL
  for (int k = 0; k < 9; ++k) Cb[k] = Ab[k];
  const T sA = ndt * vol_over_mass;
  T MTb[9];
  CKD_UNROLL
  for (int k = 0; k < 9; ++k) MTb[k] = -sA * Ab[k];
  T Mb[9], taub[9];
  mmt(MTb, f.tau, Mb);   // Mbar = (M tau)bar tau^T
  mm(f.M, MTb, taub);    // taubar = M^T (M tau)bar, M symmetric
  // M = X^-1, X = (D + D') / 2: Xbar = -M Mbar M; D'bar = Dbar(old) = Xbar / 2
  T t1[9], Dnb[9];
  mm(f.M, Mb, t1);
  mm(t1, f.M, Dnb);
  CKD_UNROLL
  for (int k = 0; k < 9; ++k) Dnb[k] *= T(-0.5);
  d_matrix_adjoint(f.stn, dx, inv_dx, Dnb, xnb);
  // tau(F')
  fc_tau_adjoint(f.Fn, U, S, V, lambda, mu, taub, Fnb, mubar, lambdabar);
  // F' = (I + dt C) F
  T dW[9];
  CKD_UNROLL
  for (int k = 0; k < 9; ++k) dW[k] = f.C[k] * dt + ((k & 3) ? T(0) : T(1));
  mtm(dW, Fnb, Fbar);  // Fbar = dW^T Fnbar
  T FnbFt[9];
  mmt(Fnb, p.F, FnbFt);
  CKD_UNROLL
  for (int k = 0; k < 9; ++k) Cb[k] += dt * FnbFt[k];
  // x' = x + dt v
  CKD_UNROLL
  for (int a = 0; a < 3; ++a) {
    xbar[a] = xnb[a];
    vb[a] += dt * xnb[a];
  }
  // C = B D^-1
  T Bb[9], t2[9], t3[9], Db[9];
  mm(Cb, f.Di, Bb);
  mtm(f.B, Cb, t2);     // B^T Cbar
  mm(f.Di, t2, t3);
  mm(t3, f.Di, Db);
  CKD_UNROLL
  for (int k = 0; k < 9; ++k) Db[k] = Dnb[k] - Db[k];
  d_matrix_adjoint(f.st, dx, inv_dx, Db, xbar);
  // G2P at x: v = 1/2 sum w v_i, B = sum w v_i r^T
  CKD_UNROLL
  for (int g = 0; g < 2; ++g)
    CKD_ROLLED
    for (int n = 0; n < 8; ++n) {
      T gw[3];
      const T w = node_weight(f.st, g, n, inv_dx, gw);
      int c[3];
      T r[3];
      CKD_UNROLL
      for (int a = 0; a < 3; ++a) {
        const int d = (n >> (2 - a)) & 1;
        c[a] = f.st.a[g][a].base + d;
        r[a] = (static_cast<T>(d) - f.st.a[g][a].o) * dx;
      }
      T vi[3];
      vel(g, c[0], c[1], c[2], vi);
      T vib[3];
      T dLdw = T(0);
      CKD_UNROLL
      for (int i = 0; i < 3; ++i) {
        const T br = Bb[i * 3] * r[0] + Bb[i * 3 + 1] * r[1] + Bb[i * 3 + 2] * r[2];
        vib[i] = w * (T(0.5) * vb[i] + br);
        dLdw += vi[i] * (T(0.5) * vb[i] + br);
      }
      vscatter(g, c[0], c[1], c[2], vib);
      CKD_UNROLL
      for (int a = 0; a < 3; ++a) {
        T btv = T(0);
        CKD_UNROLL
        for (int i = 0; i < 3; ++i) btv += Bb[i * 3 + a] * vi[i];
        xbar[a] += dLdw * gw[a] - w * btv;
      }
    }
}

// Adjoint of the initial rasterisation m_i += m w_i, mv_i += m w_i v0 at x0.
template <class T, class GAdj>
CKD void raster_adjoint(const T* x, const T* v0, T m, T inv_dx, GAdj gadj, T* xbar, T* v0bar) {
  Stencil<T> st;
  make_stencil(x, inv_dx, st);
  CKD_UNROLL
  for (int g = 0; g < 2; ++g)
    CKD_UNROLL
    for (int n = 0; n < 8; ++n) {
      T gw[3];
      const T w = node_weight(st, g, n, inv_dx, gw);
      int c[3];
      CKD_UNROLL
      for (int a = 0; a < 3; ++a) c[a] = st.a[g][a].base + ((n >> (2 - a)) & 1);
      T gb[4];
      gadj(g, c[0], c[1], c[2], gb);
      T dLdw = m * gb[0];
      CKD_UNROLL
      for (int i = 0; i < 3; ++i) {
        dLdw += m * gb[1 + i] * v0[i];
        v0bar[i] += m * w * gb[1 + i];
      }
      CKD_UNROLL
      for (int a = 0; a < 3; ++a) xbar[a] += dLdw * gw[a];
    }
}

// Grid update of one node and its adjoint.  In: m, mv; out: v (zero when the
// node is inactive).  The adjoint maps vbar to (mbar, mvbar).
template <class T>
CKD bool node_update(const DenseGrid& G, int cx, int cy, int cz, T m, const T* mv, T dt, T* v) {
  v[0] = v[1] = v[2] = T(0);
  if (!(m > static_cast<T>(G.mass_clamp)) || !node_active_block(G, cx, cy, cz)) return false;
  CKD_UNROLL
  for (int i = 0; i < 3; ++i) v[i] = mv[i] / m;
  v[1] += static_cast<T>(G.gravity) * dt;
  if (G.boundary == 1 && static_cast<T>(cy) < static_cast<T>(G.floor_cells) && v[1] < T(0)) v[1] = T(0);
  return true;
}

template <class T>
CKD void node_update_adjoint(const DenseGrid& G, int cx, int cy, int cz, T m, const T* v, T dt, const T* vbar,
                             T* out4) {
  out4[0] = out4[1] = out4[2] = out4[3] = T(0);
  if (!(m > static_cast<T>(G.mass_clamp)) || !node_active_block(G, cx, cy, cz)) return;
  T vb[3] = {vbar[0], vbar[1], vbar[2]};
  // slip floor clamp: v_y = max(u_y + g dt, 0) passes no gradient where it clamped
  if (G.boundary == 1 && static_cast<T>(cy) < static_cast<T>(G.floor_cells) && v[1] == T(0)) vb[1] = T(0);
  // u = mv / m = v - g dt e_y (where not clamped)
  const T u[3] = {v[0], v[1] - static_cast<T>(G.gravity) * dt, v[2]};
  out4[0] = -(vb[0] * u[0] + vb[1] * u[1] + vb[2] * u[2]) / m;
  CKD_UNROLL
  for (int i = 0; i < 3; ++i) out4[1 + i] = vb[i] / m;
}

}  // namespace diff
}  // namespace ckmpm
