// TEST INFRASTRUCTURE ONLY — the FP64 CPU oracle for the CK-MPM substep.
//
// This file is the checker, never the product: only tests/, __graft_entry__.smoke()
// and bench.py's cpu_baseline leg may load it.  It restates, in double precision and
// in plain serial C++, the algorithm of the reference engine's substep
// (AppledoreM/CKMPM, include/mpm_engine.cuh:519-876 and the kernels it launches in
// include/mpm_algorithm.cuh), so that the CUDA path can be compared against it
// particle by particle.  Parity is pinned by the golden fixtures under tests/golden/
// (outputs of the reference CUDA build run on a B200, see oracle/Makefile) and by the
// analytic identities the tests check (partition of unity, conservation, SVD
// reconstruction).
//
// Semantics restated here, with the reference lines they follow:
//  * CK dual-grid weights: two staggered grids at -dx/4 and +dx/4,
//    base = int(x/dx - g/4), o = x/dx - base - g/4, w0 = 1 - o + sin(2 pi o)/(2 pi),
//    node weights w0 / 1-w0 per axis (mpm_kernel.cuh:91-114, mpm_algorithm.cuh:60-67).
//  * Grid update: v = mv/m (+ g dt on y) when m > mass clamp, else 0; block-granular
//    sticky walls two blocks deep (mpm_algorithm.cuh:739-869).
//  * G2P / APIC: v = 1/2 sum w v_i, B = sum v_i (w (x_i - x_p))^T,
//    D = sum w (x_i-x_p)(x_i-x_p)^T over both grids, C = B D^-1, x += dt v
//    (mpm_algorithm.cuh:1555-1638).
//  * Constitutive: fixed-corotated (mpm_algorithm.cuh:193-254, mpm_material.cuh:320-357),
//    Drucker-Prager StVK-Hencky with sin(phi)=0.5 (mpm_algorithm.cuh:261-327,
//    mpm_material.cuh:362-464), J-fluid (mpm_algorithm.cuh:528-569, mpm_material.cuh:468-477).
//  * P2G: A = C m - dt_next V M tau with M = (1/2 (D_old + D_new))^-1, D_old the G2P D of the
//    old position (the reference never resets D between its G2P and P2G loops and inverts
//    half the sum, mpm_algorithm.cuh:1524,1604,1729-1736); m_i += w m;
//    mv_i += w (m v + A (x_i - x_p)) (mpm_algorithm.cuh:1687-1792).
//  * A particle whose new cell leaves the (1..6) window of its block is skipped in P2G
//    (mpm_algorithm.cuh:1670-1683); block of a particle = (int(x/dx + 1/4) - 2) / 4
//    (mpm_algorithm.cuh:595-600, mpm_particle.cuh:337-340).
//  * The first substep after setup advects with dt = 0 (mpm_engine.cuh:479-480,870).
//  * Initial grid: mass and momentum only (mpm_algorithm.cuh:872-947).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

namespace {

constexpr double kPi = 3.14159265358979323846;

struct SceneDesc {
  double dx;
  int32_t dims[3];       // domain extent in 4^3-cell blocks
  double gravity;        // acceleration on y
  double mass_clamp;     // grid nodes with m <= clamp get v = 0
  int32_t boundary;      // 0: sticky blocks (reference default), 1: slip floor, 2: per-cell rules
  double floor_cells;    // slip floor height in cells (boundary == 1)
  std::vector<uint8_t> rule;   // boundary == 2: rule per cell (0 free, 1 fixed, 2 slip, 3 velocity, 4 separate)
  std::vector<double> param;   // boundary == 2: normal or velocity per cell (3 each)
};

struct GridBlock {
  double a[4][2][64];  // [m, mvx, mvy, mvz][grid -1/+1][cell i*16+j*4+k]
};

struct Model {
  int kind = 0;           // 0 fixed-corotated, 2 Drucker-Prager, 3 J-fluid
  // FC / DP / linear: lambda, mu; fluid: bulk, gamma, viscosity, J0; von Mises: mu,
  // lambda, yield stress; NACC: mu, lambda, alpha0, beta, hardening factor, M, hardening on.
  double p[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double mass = 0, vol = 0;
  int n = 0;
  std::vector<double> x, F, aux;  // aux: J (fluid), logJp (DP, NACC) or the rigid flag (von Mises)
  std::vector<double> Q;          // the linear model's stored stress (9 per particle)
  std::vector<double> v0;         // initial velocities (n or 1 entries of 3)
  std::vector<double> plam, pmu;  // optional per-particle Lame parameters (fixed-corotated)
  std::vector<uint8_t> alive;
  std::vector<uint8_t> skipped;   // P2G skipped in the last step (window escape)
};

struct Scene {
  SceneDesc d;
  std::vector<Model> models;
  std::unordered_map<int64_t, GridBlock> grid;
  double current_dt = 0.0;
  int64_t steps = 0;
  int64_t lost = 0, window_skips = 0;
  std::vector<double> dt_log;
  // Rigid particles (mpm_config.h:92-106 GetExistRigidParticle / GetRigidParticleCount /
  // GetRigidParticleVelocity): the first rigid_count particles of every von Mises
  // model start rigid (mpm_algorithm.cuh:1063-1069).
  bool rigid = false;
  int rigid_count = 0;
  double rigid_v[3] = {0, 0, 0};
};

// The attribute the reference's G2P2G tests for rigidity when rigid particles
// are on: bucket attribute 3 (mpm_algorithm.cuh:1540-1543), which is F00 for
// fixed-corotated, Drucker-Prager and linear, J for the fluid, logJp for NACC
// and the rigid flag for von Mises.
inline double attribute3(const Model& m, int p) {
  return (m.kind == 3 || m.kind == 4 || m.kind == 5) ? m.aux[p] : m.F[9 * p];
}

inline void init_rigid_flags(const Scene& s, Model& m) {
  if (m.kind != 4) return;
  for (int p = 0; p < m.n; ++p) m.aux[p] = (s.rigid && p < s.rigid_count) ? 0.0 : 1.0;
}

inline int64_t flat_key(const Scene& s, int bx, int by, int bz) {
  return (static_cast<int64_t>(bx) * s.d.dims[1] + by) * s.d.dims[2] + bz;
}

inline bool in_domain(const Scene& s, int bx, int by, int bz) {
  return bx >= 0 && by >= 0 && bz >= 0 && bx < s.d.dims[0] && by < s.d.dims[1] && bz < s.d.dims[2];
}

// ---------------------------------------------------------------- 3x3 helpers
inline double det3(const double* a) {
  return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
         a[2] * (a[3] * a[7] - a[4] * a[6]);
}

// Adjugate inverse, data_type.cuh:369-386.
inline void inv3(const double* a, double* r) {
  const double id = 1.0 / det3(a);
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

inline void matmul3(const double* a, const double* b, double* r) {
  double t[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) t[i * 3 + j] = a[i * 3] * b[j] + a[i * 3 + 1] * b[3 + j] + a[i * 3 + 2] * b[6 + j];
  std::memcpy(r, t, sizeof(t));
}

inline void transpose3(const double* a, double* r) {
  double t[9] = {a[0], a[3], a[6], a[1], a[4], a[7], a[2], a[5], a[8]};
  std::memcpy(r, t, sizeof(t));
}

// SVD A = U diag(S) V^T with U, V proper rotations, S sorted by decreasing
// magnitude and the sign of det(A) carried by S[2] (the convention of the
// McAdams et al. 2011 TR1690 method the reference vendors, mpm_math.cuh:1-18).
// Computed here by cyclic Jacobi on A^T A run to convergence in double, then a
// Givens QR of A V.
void svd3(const double* A, double* U, double* S, double* V) {
  double M[9];
  double At[9];
  transpose3(A, At);
  matmul3(At, A, M);
  double Vm[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int sweep = 0; sweep < 60; ++sweep) {
    const double off = M[1] * M[1] + M[2] * M[2] + M[5] * M[5];
    const double diag = M[0] * M[0] + M[4] * M[4] + M[8] * M[8];
    if (off <= 1e-34 * diag || off == 0.0) break;
    for (auto& pq : pairs) {
      const int p = pq[0], q = pq[1];
      const double apq = M[p * 3 + q];
      if (apq == 0.0) continue;
      const double app = M[p * 3 + p], aqq = M[q * 3 + q];
      const double theta = (aqq - app) / (2.0 * apq);
      const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
      const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
      // M <- J^T M J with J the (p,q) rotation [[c, s], [-s, c]].
      for (int k = 0; k < 3; ++k) {
        const double mkp = M[k * 3 + p], mkq = M[k * 3 + q];
        M[k * 3 + p] = c * mkp - s * mkq;
        M[k * 3 + q] = s * mkp + c * mkq;
      }
      for (int k = 0; k < 3; ++k) {
        const double mpk = M[p * 3 + k], mqk = M[q * 3 + k];
        M[p * 3 + k] = c * mpk - s * mqk;
        M[q * 3 + k] = s * mpk + c * mqk;
      }
      for (int k = 0; k < 3; ++k) {
        const double vkp = Vm[k * 3 + p], vkq = Vm[k * 3 + q];
        Vm[k * 3 + p] = c * vkp - s * vkq;
        Vm[k * 3 + q] = s * vkp + c * vkq;
      }
    }
  }
  double lam[3] = {M[0], M[4], M[8]};
  // Sort eigenpairs by decreasing eigenvalue, keeping det(V) = +1.
  auto swapcols = [&](int i, int j) {
    std::swap(lam[i], lam[j]);
    for (int k = 0; k < 3; ++k) {
      std::swap(Vm[k * 3 + i], Vm[k * 3 + j]);
      Vm[k * 3 + j] = -Vm[k * 3 + j];
    }
  };
  if (lam[0] < lam[1]) swapcols(0, 1);
  if (lam[0] < lam[2]) swapcols(0, 2);
  if (lam[1] < lam[2]) swapcols(1, 2);
  if (det3(Vm) < 0) for (int k = 0; k < 3; ++k) Vm[k * 3 + 2] = -Vm[k * 3 + 2];
  double B[9];
  matmul3(A, Vm, B);
  // Givens QR of B: B = U R, U a rotation, R upper triangular.
  double Um[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  auto givens = [&](int p, int q, int col) {
    const double a = B[p * 3 + col], b = B[q * 3 + col];
    const double r = std::sqrt(a * a + b * b);
    double c = 1.0, s = 0.0;
    if (r > 0.0) { c = a / r; s = b / r; }
    for (int k = 0; k < 3; ++k) {  // rows p, q of B <- G B
      const double bp = B[p * 3 + k], bq = B[q * 3 + k];
      B[p * 3 + k] = c * bp + s * bq;
      B[q * 3 + k] = -s * bp + c * bq;
    }
    for (int k = 0; k < 3; ++k) {  // U <- U G^T
      const double up = Um[k * 3 + p], uq = Um[k * 3 + q];
      Um[k * 3 + p] = c * up + s * uq;
      Um[k * 3 + q] = -s * up + c * uq;
    }
  };
  givens(0, 1, 0);
  givens(0, 2, 0);
  givens(1, 2, 1);
  std::memcpy(U, Um, sizeof(Um));
  std::memcpy(V, Vm, sizeof(Vm));
  S[0] = B[0];
  S[1] = B[4];
  S[2] = B[8];
}

// CK compact kernel, mpm_kernel.cuh:91-114 (exact sine in place of __sinf).
inline double ck_w0(double o) { return 1.0 - o + std::sin(2.0 * kPi * o) / (2.0 * kPi); }

struct Stencil {
  int base[3];
  double o[3];
  double w0[3];
};

inline Stencil stencil(const double* x, double invdx, int g) {
  Stencil st;
  for (int a = 0; a < 3; ++a) {
    const double s = x[a] * invdx;
    st.base[a] = static_cast<int>(s - 0.25 * g);
    st.o[a] = s - st.base[a] - 0.25 * g;
    st.w0[a] = ck_w0(st.o[a]);
  }
  return st;
}

inline double node_w(const Stencil& st, int dx, int dy, int dz) {
  const double wx = dx ? 1.0 - st.w0[0] : st.w0[0];
  const double wy = dy ? 1.0 - st.w0[1] : st.w0[1];
  const double wz = dz ? 1.0 - st.w0[2] : st.w0[2];
  return wx * wy * wz;
}

// Grid velocity at (grid gi, node cell c) after the grid update of
// mpm_algorithm.cuh:739-869 with timestep dt.
void node_velocity(const Scene& s, int gi, const int* c, double dt, double* v) {
  v[0] = v[1] = v[2] = 0.0;
  if (c[0] < 0 || c[1] < 0 || c[2] < 0) return;
  const int bx = c[0] / 4, by = c[1] / 4, bz = c[2] / 4;
  if (!in_domain(s, bx, by, bz)) return;
  auto it = s.grid.find(flat_key(s, bx, by, bz));
  if (it == s.grid.end()) return;
  const int cell = (c[0] % 4) * 16 + (c[1] % 4) * 4 + (c[2] % 4);
  const GridBlock& b = it->second;
  const double m = b.a[0][gi][cell];
  if (!(m > s.d.mass_clamp)) return;
  for (int k = 0; k < 3; ++k) v[k] = b.a[1 + k][gi][cell] / m;
  v[1] += s.d.gravity * dt;
  const int K[3] = {bx, by, bz};
  if (s.d.boundary == 0) {
    bool out = false;
    for (int a = 0; a < 3; ++a) out |= (K[a] < 2 || K[a] + 2 >= s.d.dims[a]);
    if (out) v[0] = v[1] = v[2] = 0.0;
  } else if (s.d.boundary == 2) {
    // Per-cell rules: the scene's irregular-boundary hook (mpm_algorithm.cuh:795-799)
    // evaluated into data; both staggered grids of a cell take its rule.
    const int64_t ci = (static_cast<int64_t>(c[0]) * (4 * s.d.dims[1]) + c[1]) * (4 * s.d.dims[2]) + c[2];
    const int r = s.d.rule.empty() ? 0 : s.d.rule[ci];
    if (r == 1) {
      v[0] = v[1] = v[2] = 0.0;
    } else if (r >= 2 && r <= 4) {
      const double* p = &s.d.param[3 * ci];
      if (r == 3) {
        for (int k = 0; k < 3; ++k) v[k] = p[k];
      } else {
        const double d = p[0] * v[0] + p[1] * v[1] + p[2] * v[2];
        if (r == 2 || d < 0.0)
          for (int k = 0; k < 3; ++k) v[k] -= d * p[k];
      }
    }
  } else {
    // Slip floor: sticky walls on x, z and the ceiling, and v_y >= 0 below the floor.
    bool out = (K[0] < 2 || K[0] + 2 >= s.d.dims[0]) || (K[2] < 2 || K[2] + 2 >= s.d.dims[2]) ||
               (K[1] + 2 >= s.d.dims[1]);
    if (out) {
      v[0] = v[1] = v[2] = 0.0;
    } else if (c[1] < s.d.floor_cells) {
      v[1] = std::max(v[1], 0.0);
    }
  }
}

inline int trunc_div4(int a) { return a / 4; }  // C++ division truncates toward zero

void particle_block(const double* x, double invdx, int* K) {
  for (int a = 0; a < 3; ++a) K[a] = trunc_div4(static_cast<int>(x[a] * invdx + 0.25) - 2);
}

// D = sum_nodes w (x_i - x_p)(x_i - x_p)^T over both grids, in world units.
void d_matrix(const double* x, double invdx, double dx, double* D) {
  std::fill(D, D + 9, 0.0);
  for (int g = -1; g <= 1; g += 2) {
    const Stencil st = stencil(x, invdx, g);
    for (int n = 0; n < 8; ++n) {
      const int d[3] = {(n >> 2) & 1, (n >> 1) & 1, n & 1};
      const double w = node_w(st, d[0], d[1], d[2]);
      double r[3];
      for (int a = 0; a < 3; ++a) r[a] = (d[a] - st.o[a]) * dx;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) D[i * 3 + j] += w * r[i] * r[j];
    }
  }
}

// G2P at position x: returns v (already halved) and C = B D^-1.
void g2p(const Scene& s, const double* x, double dt, double* v, double* C) {
  const double dx = s.d.dx, invdx = 1.0 / dx;
  double B[9] = {0}, D[9] = {0}, vs[3] = {0, 0, 0};
  for (int g = -1; g <= 1; g += 2) {
    const int gi = g < 0 ? 0 : 1;
    const Stencil st = stencil(x, invdx, g);
    for (int n = 0; n < 8; ++n) {
      const int d[3] = {(n >> 2) & 1, (n >> 1) & 1, n & 1};
      const double w = node_w(st, d[0], d[1], d[2]);
      const int c[3] = {st.base[0] + d[0], st.base[1] + d[1], st.base[2] + d[2]};
      double vi[3];
      node_velocity(s, gi, c, dt, vi);
      double r[3];
      for (int a = 0; a < 3; ++a) r[a] = (d[a] - st.o[a]) * dx;
      for (int i = 0; i < 3; ++i) {
        vs[i] += w * vi[i];
        for (int j = 0; j < 3; ++j) {
          B[i * 3 + j] += vi[i] * w * r[j];
          D[i * 3 + j] += w * r[i] * r[j];
        }
      }
    }
  }
  double Di[9];
  inv3(D, Di);
  matmul3(B, Di, C);
  for (int i = 0; i < 3; ++i) v[i] = 0.5 * vs[i];
}

// Fixed-corotated Kirchhoff stress tau = U diag(2 mu s (s-1) + lambda J (J-1)) U^T,
// mpm_material.cuh:320-357.
void stress_fc(double lambda, double mu, const double* F, double* tau) {
  double U[9], S[3], V[9];
  svd3(F, U, S, V);
  const double J = S[0] * S[1] * S[2];
  double sc[3];
  for (int i = 0; i < 3; ++i) sc[i] = 2.0 * mu * S[i] * (S[i] - 1.0) + lambda * J * (J - 1.0);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double acc = 0;
      for (int k = 0; k < 3; ++k) acc += U[r * 3 + k] * sc[k] * U[c * 3 + k];
      tau[r * 3 + c] = acc;
    }
}

// Drucker-Prager (StVK-Hencky) return map with the reference's hard-coded
// friction sin(phi) = 0.5, zero cohesion, volume correction on,
// mpm_material.cuh:362-464.  Updates F and logJp in place.
void stress_dp(double lambda, double mu, double* F, double* logJp, double* tau) {
  const double ys = 0.816496580927726 * 2.0 * 0.5 / (3.0 - 0.5);
  const double smu = 2.0 * mu;
  double U[9], S[3], V[9];
  svd3(F, U, S, V);
  double eps[3];
  for (int i = 0; i < 3; ++i) eps[i] = std::log(std::max(std::fabs(S[i]), 1e-4));
  const double esum = eps[0] + eps[1] + eps[2];
  const double etr = esum + *logJp;
  double eh[3];
  for (int i = 0; i < 3; ++i) eh[i] = eps[i] - etr / 3.0;
  const double ehn = std::sqrt(eh[0] * eh[0] + eh[1] * eh[1] + eh[2] * eh[2]);
  double ns[3];
  if (etr >= 0.0) {
    ns[0] = ns[1] = ns[2] = 1.0;
    *logJp = esum + *logJp;
  } else {
    *logJp = 0.0;
    const double dg = ehn + (3.0 * lambda + smu) / smu * etr * ys;
    for (int i = 0; i < 3; ++i) {
      const double H = dg <= 0.0 ? eps[i] : eps[i] - (dg / ehn) * eh[i];
      ns[i] = std::exp(H);
    }
  }
  // F <- U diag(ns) V^T
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double acc = 0;
      for (int k = 0; k < 3; ++k) acc += U[r * 3 + k] * ns[k] * V[c * 3 + k];
      F[r * 3 + c] = acc;
    }
  // tau = U diag((2 mu log s + lambda tr log s) / s) V^T F^T
  double ph[3];
  const double tr = std::log(ns[0]) + std::log(ns[1]) + std::log(ns[2]);
  for (int i = 0; i < 3; ++i) ph[i] = (smu * std::log(ns[i]) + lambda * tr) / ns[i];
  double P[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double acc = 0;
      for (int k = 0; k < 3; ++k) acc += U[r * 3 + k] * ph[k] * V[c * 3 + k];
      P[r * 3 + c] = acc;
    }
  double Ft[9];
  transpose3(F, Ft);
  matmul3(P, Ft, tau);
}

// Von Mises plasticity on the Hencky strain of the trial elastic F, then the
// StVK-Hencky stress of the projected F from its own SVD,
// mpm_algorithm.cuh:404-520 and mpm_material.cuh:480-518.  F in/out.
void stress_vm(double mu, double lambda, double yield, double* F, double* tau) {
  double U[9], S[3], V[9];
  svd3(F, U, S, V);
  double eps[3];
  for (int i = 0; i < 3; ++i) eps[i] = std::log(S[i]);
  const double etr = eps[0] + eps[1] + eps[2];
  double eh[3];
  for (int i = 0; i < 3; ++i) eh[i] = eps[i] - etr / 3.0;
  const double ehn = std::sqrt(eh[0] * eh[0] + eh[1] * eh[1] + eh[2] * eh[2]);
  const double yf = ehn - yield / (2.0 * mu);
  if (yf > 0.0) {
    double ns[3];
    for (int i = 0; i < 3; ++i) ns[i] = std::exp(eps[i] - yf * eh[i] / ehn);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        double acc = 0;
        for (int k = 0; k < 3; ++k) acc += U[r * 3 + k] * ns[k] * V[c * 3 + k];
        F[r * 3 + c] = acc;
      }
  }
  svd3(F, U, S, V);
  double ls[3];
  for (int i = 0; i < 3; ++i) ls[i] = std::log(S[i]);
  const double lsum = ls[0] + ls[1] + ls[2];
  double P[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double acc = 0;
      for (int k = 0; k < 3; ++k) acc += U[r * 3 + k] * ((2.0 * mu * ls[k] + lambda * lsum) / S[k]) * V[c * 3 + k];
      P[r * 3 + c] = acc;
    }
  double Ft[9];
  transpose3(F, Ft);
  matmul3(P, Ft, tau);
}

// Non-associated Cam-clay, mpm_material.cuh:520-669 (driven from
// mpm_algorithm.cuh:330-402), restated step for step: the projected F is
// U diag(S) V (V, not its transpose); the hardening increment of the
// yield-surface branch is applied 9 times (it sits in a loop of 9 identical
// iterations); both branches end in the same stress from the projected F
// (:649-667).  F in/out; tau out.
void stress_nacc(const double* prm, double* F, double* logJp, double* tau) {
  const double mu = prm[0], lambda = prm[1], beta = prm[3], xi = prm[4], msq = prm[5] * prm[5];
  const bool hardening = prm[6] != 0.0;
  const double K = 2.0 * mu / 3.0 + lambda;
  double U[9], S[3], V[9];
  svd3(F, U, S, V);
  const double p0 = K * (1e-5 + std::sinh(xi * std::max(-*logJp, 0.0)));
  const double pmin = -beta * p0;
  const double je = S[0] * S[1] * S[2];
  const double bh[3] = {S[0] * S[0], S[1] * S[1], S[2] * S[2]};
  const double btr3 = (bh[0] + bh[1] + bh[2]) / 3.0;
  const double devf = mu * std::pow(je, -2.0 / 3.0);
  double sh[3];
  for (int i = 0; i < 3; ++i) sh[i] = devf * (bh[i] - btr3);
  const double ptrial = -K * 0.5 * (je - 1.0 / je) * je;
  const double ysh = 1.5 * (1.0 + 2.0 * beta);
  const double yph = msq * (ptrial - pmin) * (ptrial - p0);
  const double sn2 = sh[0] * sh[0] + sh[1] * sh[1] + sh[2] * sh[2];
  const double y = ysh * sn2 + yph;
  auto u_diag_v = [&](const double* d) {  // F = U diag(d) V
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        double acc = 0;
        for (int k = 0; k < 3; ++k) acc += U[r * 3 + k] * d[k] * V[k * 3 + c];
        F[r * 3 + c] = acc;
      }
  };
  double Sn[3] = {S[0], S[1], S[2]};
  if (ptrial > p0 || ptrial < pmin) {
    const double pp = ptrial > p0 ? p0 : pmin;
    const double jn = std::sqrt(-2.0 * pp / K + 1.0);
    const double sc = std::cbrt(jn);
    Sn[0] = Sn[1] = Sn[2] = sc;
    u_diag_v(Sn);
    if (hardening) *logJp += std::log(je / jn);
  } else if (y >= 1e-4) {
    const double coef = std::pow(je, 2.0 / 3.0) / mu * std::sqrt(-yph / ysh) / std::sqrt(sn2);
    for (int i = 0; i < 3; ++i) Sn[i] = std::sqrt(sh[i] * coef + btr3);
    u_diag_v(Sn);
    if (hardening && p0 > 1e-4 && ptrial < p0 - 1e-4 && ptrial > 1e-4 + pmin) {
      const double pc = (1.0 - beta) * p0 / 2.0;
      const double qt = std::sqrt(1.5 * sn2);
      double d0 = pc - ptrial, d1 = -qt;
      const double dn = std::sqrt(d0 * d0 + d1 * d1);
      d0 /= dn;
      d1 /= dn;
      const double A = msq * d0 * d0 + (1.0 + 2.0 * beta) * d1 * d1;
      const double B = msq * d0 * (2.0 * pc - p0 - pmin);
      const double C = msq * (pc - pmin) * (pc - p0);
      const double disc = B * B - 4.0 * A * C;
      const double l1 = (-B + std::sqrt(disc)) / (2.0 * A), l2 = (-B - std::sqrt(disc)) / (2.0 * A);
      const double p1 = pc + l1 * d0, p2 = pc + l2 * d0;
      const double pf = (ptrial - pc) * (p1 - pc) > 0.0 ? p1 : p2;
      const double jsq = -2.0 * pf / K + 1.0;
      const double jn = std::sqrt(std::fabs(jsq));
      if (jn > 1e-4)
        for (int it = 0; it < 9; ++it) *logJp += std::log(je / jn);
    }
  }
  const double J = Sn[0] * Sn[1] * Sn[2];
  double b[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) b[r * 3 + c] = F[r * 3] * F[c * 3] + F[r * 3 + 1] * F[c * 3 + 1] + F[r * 3 + 2] * F[c * 3 + 2];
  const double btr = (b[0] + b[4] + b[8]) / 3.0;
  const double hc = K * 0.5 * (J * J - 1.0);
  for (int k = 0; k < 9; ++k) tau[k] = devf * (b[k] - ((k & 3) ? 0.0 : btr)) + ((k & 3) ? 0.0 : hc);
}

// Linear model as the reference updates it, mpm_algorithm.cuh:107-191: with
// F already dW F, the stored stress Q <- (Q + 50 (C + C^T - I) dt) det(F) with
// rows 1 and 2 zeroed; tau = Q.
void stress_linear(const double* C, double dt, const double* F, double* Q, double* tau) {
  const double d = det3(F);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      const int k = r * 3 + c;
      Q[k] = r == 0 ? (Q[k] + 50.0 * (C[k] + C[c * 3 + r] - ((k & 3) ? 0.0 : 1.0)) * dt) * d : 0.0;
    }
  for (int k = 0; k < 9; ++k) tau[k] = Q[k];
}

// J-fluid: J += tr(C) dt J; p = bulk (J^-gamma - 1); tau = J (visc (C + C^T) - p I),
// mpm_algorithm.cuh:528-569 and mpm_material.cuh:468-477.
void stress_fluid(const double* prm, const double* C, double dt, double* J, double* tau) {
  *J += (C[0] + C[4] + C[8]) * dt * (*J);
  const double p = prm[0] * (std::pow(*J, -prm[1]) - 1.0);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) tau[r * 3 + c] = (C[r * 3 + c] + C[c * 3 + r]) * prm[2];
  tau[0] -= p;
  tau[4] -= p;
  tau[8] -= p;
  for (int k = 0; k < 9; ++k) tau[k] *= *J;
}

GridBlock& grid_block(std::unordered_map<int64_t, GridBlock>& g, int64_t key) {
  auto it = g.find(key);
  if (it == g.end()) {
    GridBlock b;
    std::memset(&b, 0, sizeof(b));
    it = g.emplace(key, b).first;
  }
  return it->second;
}

// Scatter mass and momentum of one particle at x with affine matrix A (world units).
void p2g(Scene& s, std::unordered_map<int64_t, GridBlock>& out, const double* x, double mass, const double* v,
         const double* A) {
  const double dx = s.d.dx, invdx = 1.0 / dx;
  for (int g = -1; g <= 1; g += 2) {
    const int gi = g < 0 ? 0 : 1;
    const Stencil st = stencil(x, invdx, g);
    for (int n = 0; n < 8; ++n) {
      const int d[3] = {(n >> 2) & 1, (n >> 1) & 1, n & 1};
      const double w = node_w(st, d[0], d[1], d[2]);
      const int c[3] = {st.base[0] + d[0], st.base[1] + d[1], st.base[2] + d[2]};
      if (c[0] < 0 || c[1] < 0 || c[2] < 0) continue;
      const int bx = c[0] / 4, by = c[1] / 4, bz = c[2] / 4;
      if (!in_domain(s, bx, by, bz)) continue;
      GridBlock& b = grid_block(out, flat_key(s, bx, by, bz));
      const int cell = (c[0] % 4) * 16 + (c[1] % 4) * 4 + (c[2] % 4);
      double r[3];
      for (int a = 0; a < 3; ++a) r[a] = (d[a] - st.o[a]) * dx;
      b.a[0][gi][cell] += w * mass;
      for (int i = 0; i < 3; ++i) {
        const double ar = A[i * 3] * r[0] + A[i * 3 + 1] * r[1] + A[i * 3 + 2] * r[2];
        b.a[1 + i][gi][cell] += w * (mass * v[i] + ar);
      }
    }
  }
}

void substep(Scene& s, double next_dt) {
  const double dt = s.current_dt;
  const double dx = s.d.dx, invdx = 1.0 / dx;
  std::unordered_map<int64_t, GridBlock> out;
  out.reserve(s.grid.size() * 2 + 16);
  for (Model& m : s.models) {
    for (int p = 0; p < m.n; ++p) {
      m.skipped[p] = 0;
      if (!m.alive[p]) continue;
      double* x = &m.x[3 * p];
      int K[3];
      particle_block(x, invdx, K);
      double v[3], C[9];
      g2p(s, x, dt, v, C);
      // A rigid particle moves with the scene's rigid velocity and carries no
      // velocity, no affine field and no G2P D (mpm_algorithm.cuh:1609-1618).
      const bool rigid = s.rigid && attribute3(m, p) == 0.0;
      if (rigid)
        for (int k = 0; k < 9; ++k) C[k] = 0.0;
      double xn[3], xold[3];
      for (int a = 0; a < 3; ++a) {
        xold[a] = x[a];
        if (rigid) v[a] = 0.0;
        xn[a] = x[a] + dt * (rigid ? s.rigid_v[a] : v[a]);
      }
      double tau[9];
      if (m.kind == 3) {
        stress_fluid(m.p, C, dt, &m.aux[p], tau);
      } else {
        double dW[9];
        for (int k = 0; k < 9; ++k) dW[k] = C[k] * dt + ((k & 3) ? 0.0 : 1.0);
        double* F = &m.F[9 * p];
        matmul3(dW, F, F);
        if (m.kind == 0)
          stress_fc(m.plam.empty() ? m.p[0] : m.plam[p], m.pmu.empty() ? m.p[1] : m.pmu[p], F, tau);
        else if (m.kind == 2)
          stress_dp(m.p[0], m.p[1], F, &m.aux[p], tau);
        else if (m.kind == 4)
          stress_vm(m.p[0], m.p[1], m.p[2], F, tau);
        else if (m.kind == 5)
          stress_nacc(m.p, F, &m.aux[p], tau);
        else
          stress_linear(C, dt, F, &m.Q[9 * p], tau);
      }
      for (int a = 0; a < 3; ++a) x[a] = xn[a];
      // Advection: new block must be a neighbour inside the domain.
      int Kn[3];
      particle_block(xn, invdx, Kn);
      bool ok = in_domain(s, Kn[0], Kn[1], Kn[2]);
      for (int a = 0; a < 3; ++a) ok &= std::abs(Kn[a] - K[a]) <= 1;
      // Window check against the source block (mpm_algorithm.cuh:1670-1683).
      bool win = true;
      for (int a = 0; a < 3; ++a) {
        const int lc = static_cast<int>(xn[a] * invdx + 0.25) - 4 * K[a];
        win &= (lc > 0 && lc < 7);
      }
      if (!ok) {
        m.alive[p] = 0;
        ++s.lost;
      }
      if (!win) {
        m.skipped[p] = 1;
        ++s.window_skips;
        continue;
      }
      // The reference's P2G adds the new position's D onto the G2P D of the old
      // position (it is never reset in between, mpm_algorithm.cuh:1524,1604,1729)
      // and inverts half the sum (:1732).
      double D[9], Dold[9], Di[9], halfD[9];
      d_matrix(xn, invdx, dx, D);
      d_matrix(xold, invdx, dx, Dold);
      for (int k = 0; k < 9; ++k) halfD[k] = 0.5 * (D[k] + (rigid ? 0.0 : Dold[k]));
      inv3(halfD, Di);
      double DT[9];
      matmul3(Di, tau, DT);
      double A[9];
      for (int k = 0; k < 9; ++k) A[k] = C[k] * m.mass - next_dt * m.vol * DT[k];
      p2g(s, out, xn, m.mass, v, A);
    }
  }
  s.grid.swap(out);
  s.current_dt = next_dt;
  ++s.steps;
}

}  // namespace

extern "C" {

void* oracle_create(double dx, const int32_t* dims, double gravity, double mass_clamp, int32_t boundary,
                    double floor_cells) {
  Scene* s = new Scene();
  s->d.dx = dx;
  for (int a = 0; a < 3; ++a) s->d.dims[a] = dims[a];
  s->d.gravity = gravity;
  s->d.mass_clamp = mass_clamp;
  s->d.boundary = boundary;
  s->d.floor_cells = floor_cells;
  return s;
}

void oracle_destroy(void* h) { delete static_cast<Scene*>(h); }

// Per-cell boundary rules of a boundary-2 scene: rule[cells], param[3 cells]
// (NULL: all zero), cells x-major over the domain's 4 * dims cells per axis.
int oracle_set_boundary_field(void* h, const uint8_t* rule, const double* param) {
  Scene* s = static_cast<Scene*>(h);
  if (s->d.boundary != 2 || !rule) return -1;
  const size_t cells = static_cast<size_t>(s->d.dims[0]) * s->d.dims[1] * s->d.dims[2] * 64;
  s->d.rule.assign(rule, rule + cells);
  s->d.param.assign(3 * cells, 0.0);
  if (param) s->d.param.assign(param, param + 3 * cells);
  return 0;
}

// kind: 0 fixed-corotated (params lambda, mu), 2 Drucker-Prager (lambda, mu),
// 3 J-fluid (bulk, gamma, viscosity, J0).  v holds nv = 1 or n velocities.
int oracle_add_model(void* h, int kind, const double* params, int n, const float* x, const float* v, int nv,
                     double mass, double vol) {
  Scene* s = static_cast<Scene*>(h);
  Model m;
  m.kind = kind;
  for (int k = 0; k < 8; ++k) m.p[k] = params[k];
  m.mass = mass;
  m.vol = vol;
  m.n = n;
  m.x.assign(x, x + 3 * static_cast<size_t>(n));
  m.F.assign(9 * static_cast<size_t>(n), 0.0);
  for (int p = 0; p < n; ++p) m.F[9 * p] = m.F[9 * p + 4] = m.F[9 * p + 8] = 1.0;
  m.aux.assign(n, kind == 3 ? params[3] : (kind == 5 ? params[2] : 0.0));
  init_rigid_flags(*s, m);
  if (kind == 1) m.Q.assign(9 * static_cast<size_t>(n), 0.0);
  m.v0.assign(v, v + 3 * static_cast<size_t>(nv));
  m.alive.assign(n, 1);
  m.skipped.assign(n, 0);
  // Particles outside the domain never bin (mpm_algorithm.cuh:586-626 would index out of range).
  const double invdx = 1.0 / s->d.dx;
  for (int p = 0; p < n; ++p) {
    int K[3];
    double xp[3] = {m.x[3 * p], m.x[3 * p + 1], m.x[3 * p + 2]};
    particle_block(xp, invdx, K);
    if (!in_domain(*s, K[0], K[1], K[2]) || xp[0] < 0 || xp[1] < 0 || xp[2] < 0) m.alive[p] = 0;
  }
  s->models.push_back(std::move(m));
  return static_cast<int>(s->models.size()) - 1;
}

// Initial grid: mass and momentum only (mpm_algorithm.cuh:872-947); first dt is 0.
// Per-particle Lame parameters of a fixed-corotated model (the differentiable
// form's per-particle Young's modulus); NULL restores the model's own.
int oracle_set_lame(void* h, int model, const double* lam, const double* mu) {
  Scene* s = static_cast<Scene*>(h);
  if (model < 0 || model >= static_cast<int>(s->models.size())) return -1;
  Model& m = s->models[model];
  if (!lam || !mu) {
    m.plam.clear();
    m.pmu.clear();
    return 0;
  }
  m.plam.assign(lam, lam + m.n);
  m.pmu.assign(mu, mu + m.n);
  return 0;
}

// Initial velocities in double precision (nv = 1 or n rows), before oracle_setup.
int oracle_set_velocity(void* h, int model, const double* v, int nv) {
  Scene* s = static_cast<Scene*>(h);
  if (model < 0 || model >= static_cast<int>(s->models.size())) return -1;
  Model& m = s->models[model];
  if (nv != 1 && nv != m.n) return -1;
  m.v0.assign(v, v + 3 * static_cast<size_t>(nv));
  return 0;
}

// Rigid particles on (enable != 0) with rigid_count leading rigid particles per
// von Mises model and the rigid velocity v; call before oracle_setup.
int oracle_set_rigid(void* h, int enable, int rigid_count, const double* v) {
  Scene* s = static_cast<Scene*>(h);
  if (rigid_count < 0 || !v) return -1;
  s->rigid = enable != 0;
  s->rigid_count = rigid_count;
  for (int a = 0; a < 3; ++a) s->rigid_v[a] = v[a];
  for (Model& m : s->models) init_rigid_flags(*s, m);
  return 0;
}

// The rigid velocity of the following substeps (the reference evaluates its
// hook once per frame, mpm_algorithm.cuh:1614).
int oracle_set_rigid_velocity(void* h, const double* v) {
  Scene* s = static_cast<Scene*>(h);
  if (!v) return -1;
  for (int a = 0; a < 3; ++a) s->rigid_v[a] = v[a];
  return 0;
}

int oracle_setup(void* h) {
  Scene* s = static_cast<Scene*>(h);
  s->grid.clear();
  const double Z[9] = {0};
  for (Model& m : s->models) {
    const bool per = m.v0.size() == 3 * static_cast<size_t>(m.n);
    for (int p = 0; p < m.n; ++p) {
      if (!m.alive[p]) continue;
      const double* v = per ? &m.v0[3 * p] : &m.v0[0];
      p2g(*s, s->grid, &m.x[3 * p], m.mass, v, Z);
    }
  }
  s->current_dt = 0.0;
  s->steps = 0;
  return 0;
}

// One frame with the reference's adaptive rule (include/mpm_engine.cuh:514-557):
// every substep takes next = min(dt_max, frame end - time, dx cfl / max|v|),
// max|v| over all grid nodes after the grid update with the current dt.
// Returns the number of substeps taken.
int oracle_step_frame(void* h, double dt_max, double cfl, double frame_time, double* time) {
  Scene* s = static_cast<Scene*>(h);
  const double end = *time + frame_time;
  int taken = 0;
  while (*time < end) {
    double vmax2 = 0.0;
    for (auto& kv : s->grid) {
      const int64_t k = kv.first;
      const int bz = static_cast<int>(k % s->d.dims[2]);
      const int by = static_cast<int>((k / s->d.dims[2]) % s->d.dims[1]);
      const int bx = static_cast<int>(k / (static_cast<int64_t>(s->d.dims[2]) * s->d.dims[1]));
      for (int gi = 0; gi < 2; ++gi)
        for (int cell = 0; cell < 64; ++cell) {
          const int c[3] = {bx * 4 + (cell >> 4), by * 4 + ((cell >> 2) & 3), bz * 4 + (cell & 3)};
          double v[3];
          node_velocity(*s, gi, c, s->current_dt, v);
          vmax2 = std::max(vmax2, v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        }
    }
    double next = std::min(dt_max, end - *time);
    const double vmax = std::sqrt(vmax2);
    if (vmax > 0.0) next = std::min(next, s->d.dx * cfl / vmax);
    substep(*s, next);
    *time += next;
    ++taken;
    s->dt_log.push_back(next);
  }
  return taken;
}

// The dt of every adaptive substep taken so far (up to cap entries); returns the count.
int oracle_dt_log(void* h, double* out, int cap) {
  Scene* s = static_cast<Scene*>(h);
  const int n = static_cast<int>(s->dt_log.size());
  for (int i = 0; i < n && i < cap; ++i) out[i] = s->dt_log[i];
  return n;
}

int oracle_step(void* h, int nsteps, double dt) {
  Scene* s = static_cast<Scene*>(h);
  for (int i = 0; i < nsteps; ++i) substep(*s, dt);
  return 0;
}

// Per-particle state in input (ID) order.  v is the velocity the next G2P
// would interpolate at the current position (the quantity the reference's
// conservation probe reads, mpm_algorithm.cuh:1306-1331), using the current dt.
int oracle_get_state(void* h, int model, double* x, double* v, double* F, double* aux, uint8_t* alive) {
  Scene* s = static_cast<Scene*>(h);
  if (model < 0 || model >= static_cast<int>(s->models.size())) return -1;
  const Model& m = s->models[model];
  for (int p = 0; p < m.n; ++p) {
    if (x) for (int a = 0; a < 3; ++a) x[3 * p + a] = m.x[3 * p + a];
    if (F) for (int k = 0; k < 9; ++k) F[9 * p + k] = m.F[9 * p + k];
    if (aux) aux[p] = m.aux[p];
    if (alive) alive[p] = m.alive[p];
    if (v) {
      double C[9];
      g2p(*s, &m.x[3 * p], s->current_dt, &v[3 * p], C);
      if (s->rigid && attribute3(m, p) == 0.0) v[3 * p] = v[3 * p + 1] = v[3 * p + 2] = 0.0;  // :1316-1325
    }
  }
  return m.n;
}

// Overwrite one model's state (x, F, aux), in input order; NULL leaves a field.
int oracle_set_state(void* h, int model, const double* x, const double* F, const double* aux) {
  Scene* s = static_cast<Scene*>(h);
  if (model < 0 || model >= static_cast<int>(s->models.size())) return -1;
  Model& m = s->models[model];
  if (x) std::memcpy(m.x.data(), x, sizeof(double) * 3 * m.n);
  if (F) std::memcpy(m.F.data(), F, sizeof(double) * 9 * m.n);
  if (aux) std::memcpy(m.aux.data(), aux, sizeof(double) * m.n);
  return 0;
}

int64_t oracle_counter(void* h, int which) {
  Scene* s = static_cast<Scene*>(h);
  switch (which) {
    case 0: return s->steps;
    case 1: return s->lost;
    case 2: return s->window_skips;
    case 3: return static_cast<int64_t>(s->grid.size());
    default: return -1;
  }
}

double oracle_current_dt(void* h) { return static_cast<Scene*>(h)->current_dt; }

// Dense dump of the grid: for each stored block (sorted by flat key) writes
// the key and 4 x 2 x 64 doubles.  Returns the number of blocks (or the
// number needed when cap is too small).
int oracle_get_grid(void* h, int64_t* keys, double* data, int cap) {
  Scene* s = static_cast<Scene*>(h);
  std::vector<int64_t> ks;
  ks.reserve(s->grid.size());
  for (auto& kv : s->grid) ks.push_back(kv.first);
  std::sort(ks.begin(), ks.end());
  const int n = static_cast<int>(ks.size());
  if (cap < n) return n;
  for (int i = 0; i < n; ++i) {
    keys[i] = ks[i];
    std::memcpy(data + static_cast<size_t>(i) * 512, &s->grid[ks[i]].a[0][0][0], sizeof(double) * 512);
  }
  return n;
}

// Canonical block sets.  which = 0: blocks holding live particles of `model`
// (or of any model when model < 0), lexicographically sorted, with per-block
// particle counts; which = 1: those plus their {0,1}^3 neighbours (the grid
// block set, mpm_algorithm.cuh:658-695 Neighbor policy); which = 2: plus the
// {-1,0,1}^3 neighbours (Exterior policy).  Keys are written as int32 triples.
int oracle_get_blocks(void* h, int model, int which, int32_t* keys, uint32_t* counts, int cap) {
  Scene* s = static_cast<Scene*>(h);
  const double invdx = 1.0 / s->d.dx;
  std::unordered_map<int64_t, uint32_t> pb;
  for (int mi = 0; mi < static_cast<int>(s->models.size()); ++mi) {
    if (model >= 0 && mi != model) continue;
    const Model& m = s->models[mi];
    for (int p = 0; p < m.n; ++p) {
      if (!m.alive[p]) continue;
      int K[3];
      particle_block(&m.x[3 * p], invdx, K);
      pb[flat_key(*s, K[0], K[1], K[2])] += 1;
    }
  }
  std::unordered_map<int64_t, uint32_t> set = pb;
  if (s->steps == 0) {
    // Right after setup the partition also holds the block of each particle's
    // cell on the +dx/4 grid (ActivateBlocksWithParticles activates both
    // staggered grids' blocks, mpm_algorithm.cuh:713-736), with no particles.
    for (int mi = 0; mi < static_cast<int>(s->models.size()); ++mi) {
      if (model >= 0 && mi != model) continue;
      const Model& m = s->models[mi];
      for (int p = 0; p < m.n; ++p) {
        if (!m.alive[p]) continue;
        int K[3];
        for (int a = 0; a < 3; ++a) K[a] = trunc_div4(static_cast<int>(m.x[3 * p + a] * invdx - 0.25) - 2);
        if (in_domain(*s, K[0], K[1], K[2])) set.emplace(flat_key(*s, K[0], K[1], K[2]), 0u);
      }
    }
  }
  if (which >= 1) {
    const int lo = which == 1 ? 0 : -1;
    const std::unordered_map<int64_t, uint32_t> na = set;
    for (auto& kv : na) {
      const int64_t k = kv.first;
      const int bz = static_cast<int>(k % s->d.dims[2]);
      const int by = static_cast<int>((k / s->d.dims[2]) % s->d.dims[1]);
      const int bx = static_cast<int>(k / (static_cast<int64_t>(s->d.dims[2]) * s->d.dims[1]));
      for (int i = lo; i <= 1; ++i)
        for (int j = lo; j <= 1; ++j)
          for (int l = lo; l <= 1; ++l)
            if (in_domain(*s, bx + i, by + j, bz + l)) set.emplace(flat_key(*s, bx + i, by + j, bz + l), 0u);
    }
  }
  std::vector<int64_t> ks;
  for (auto& kv : set) ks.push_back(kv.first);
  std::sort(ks.begin(), ks.end());
  const int n = static_cast<int>(ks.size());
  if (cap < n) return n;
  for (int i = 0; i < n; ++i) {
    const int64_t k = ks[i];
    keys[3 * i + 2] = static_cast<int32_t>(k % s->d.dims[2]);
    keys[3 * i + 1] = static_cast<int32_t>((k / s->d.dims[2]) % s->d.dims[1]);
    keys[3 * i + 0] = static_cast<int32_t>(k / (static_cast<int64_t>(s->d.dims[2]) * s->d.dims[1]));
    if (counts) counts[i] = set[k];
  }
  return n;
}

// ---- unit-level entry points used by the tests ----
void oracle_svd3(const double* A, double* U, double* S, double* V) { svd3(A, U, S, V); }

double oracle_ck_w0(double o) { return ck_w0(o); }

// One constitutive update exactly as the substep applies it: dW = I + dt C,
// F <- dW F (FC/DP), stress tau; aux is logJp (DP) or J (fluid).
void oracle_constitutive(int kind, const double* params, const double* C, double dt, double* F, double* aux,
                         double* tau) {
  if (kind == 3) {
    stress_fluid(params, C, dt, aux, tau);
    return;
  }
  double dW[9];
  for (int k = 0; k < 9; ++k) dW[k] = C[k] * dt + ((k & 3) ? 0.0 : 1.0);
  matmul3(dW, F, F);
  if (kind == 0)
    stress_fc(params[0], params[1], F, tau);
  else if (kind == 2)
    stress_dp(params[0], params[1], F, aux, tau);
  else if (kind == 4)
    stress_vm(params[0], params[1], params[2], F, tau);
  else if (kind == 5)
    stress_nacc(params, F, aux, tau);
}

}  // extern "C"
