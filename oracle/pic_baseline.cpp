// TEST INFRASTRUCTURE / CPU BASELINE ONLY.
//
// C++/OpenMP restatement of the reference's CPU-runnable demo form, the PIC
// CK-MPM substep of python-src/python_demo.py (substep() :101-215), used as the
// timed CPU baseline.  The original is a Taichi program (absent here, and it
// targets ti.cuda); its constants (python_demo.py:7-23) become parameters.
//
//  * P2G (:108-143): on both staggered grids, base = int(x n - s/4),
//    offset = x n - (base + s/4), stencil w0 = 1 - o + sin(2 pi o)/(2 pi)
//    (compact_kernel_stencil :60-67); m_i += w m;
//    mv_i += w m v + dt PF grad_w, PF = -V (2 mu (F - R) F^T + lambda (J-1) J I)
//    (compute_fixed_corotated :84-91), grad from compact_kernel_gradient :69-74.
//  * Grid update (:146-164): v = mv / m when m > 1e-8 m_p, v_y += dt g, zero
//    within `wall` cells of the domain edge.
//  * G2P (:167-192): v = 1/2 sum w v_i, x += dt v, F <- (I + dt/2 sum v_i grad^T) F.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr double kPi = 3.14159265358979323846;

// Symmetric Jacobi SVD in float (U, V rotations, sign on the last value).
void svd3f(const float* A, float* U, float* S, float* V) {
  double M[9], Vm[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) M[i * 3 + j] = A[i] * A[j] + A[3 + i] * A[3 + j] + A[6 + i] * A[6 + j];
  const int pr[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int sw = 0; sw < 8; ++sw)
    for (auto& pq : pr) {
      const int p = pq[0], q = pq[1];
      const double apq = M[p * 3 + q];
      if (std::fabs(apq) < 1e-30) continue;
      const double th = (M[q * 3 + q] - M[p * 3 + p]) / (2 * apq);
      const double t = (th >= 0 ? 1 : -1) / (std::fabs(th) + std::sqrt(th * th + 1));
      const double c = 1 / std::sqrt(t * t + 1), s = t * c;
      for (int k = 0; k < 3; ++k) {
        const double a = M[k * 3 + p], b = M[k * 3 + q];
        M[k * 3 + p] = c * a - s * b;
        M[k * 3 + q] = s * a + c * b;
      }
      for (int k = 0; k < 3; ++k) {
        const double a = M[p * 3 + k], b = M[q * 3 + k];
        M[p * 3 + k] = c * a - s * b;
        M[q * 3 + k] = s * a + c * b;
      }
      for (int k = 0; k < 3; ++k) {
        const double a = Vm[k * 3 + p], b = Vm[k * 3 + q];
        Vm[k * 3 + p] = c * a - s * b;
        Vm[k * 3 + q] = s * a + c * b;
      }
    }
  double l[3] = {M[0], M[4], M[8]};
  auto sw = [&](int i, int j) {
    std::swap(l[i], l[j]);
    for (int k = 0; k < 3; ++k) {
      std::swap(Vm[k * 3 + i], Vm[k * 3 + j]);
      Vm[k * 3 + j] = -Vm[k * 3 + j];
    }
  };
  if (l[0] < l[1]) sw(0, 1);
  if (l[0] < l[2]) sw(0, 2);
  if (l[1] < l[2]) sw(1, 2);
  double B[9], Um[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) B[i * 3 + j] = A[i * 3] * Vm[j] + A[i * 3 + 1] * Vm[3 + j] + A[i * 3 + 2] * Vm[6 + j];
  auto giv = [&](int p, int q, int col) {
    const double a = B[p * 3 + col], b = B[q * 3 + col], r = std::sqrt(a * a + b * b);
    const double c = r > 0 ? a / r : 1, s = r > 0 ? b / r : 0;
    for (int k = 0; k < 3; ++k) {
      const double bp = B[p * 3 + k], bq = B[q * 3 + k];
      B[p * 3 + k] = c * bp + s * bq;
      B[q * 3 + k] = -s * bp + c * bq;
      const double up = Um[k * 3 + p], uq = Um[k * 3 + q];
      Um[k * 3 + p] = c * up + s * uq;
      Um[k * 3 + q] = -s * up + c * uq;
    }
  };
  giv(0, 1, 0);
  giv(0, 2, 0);
  giv(1, 2, 1);
  for (int k = 0; k < 9; ++k) {
    U[k] = static_cast<float>(Um[k]);
    V[k] = static_cast<float>(Vm[k]);
  }
  S[0] = static_cast<float>(B[0]);
  S[1] = static_cast<float>(B[4]);
  S[2] = static_cast<float>(B[8]);
}

struct Params {
  int n_grid;
  float dx, mass, vol, mu, lam, gravity, dt;
  int wall;
};

struct Grid {
  int n;
  std::vector<float> m;  // [i][j][k][2]
  std::vector<float> mv; // [i][j][k][2][3]
  explicit Grid(int n_) : n(n_), m(static_cast<size_t>(n_) * n_ * n_ * 2), mv(static_cast<size_t>(n_) * n_ * n_ * 6) {}
  size_t idx(int i, int j, int k, int w) const { return ((static_cast<size_t>(i) * n + j) * n + k) * 2 + w; }
};

inline void stencil(float x, float n, int sign, int& base, float& o, float (&st)[2]) {
  base = static_cast<int>(x * n - sign * 0.25f);
  o = x * n - (static_cast<float>(base) + 0.25f * sign);
  st[0] = 1.f - o + std::sin(2.f * static_cast<float>(kPi) * o) / (2.f * static_cast<float>(kPi));
  st[1] = 1.f - st[0];
}

inline float grad1(float dw) { return (dw > 0 ? 1.f : (dw < 0 ? -1.f : 0.f)) * (std::cos(2.f * static_cast<float>(kPi) * std::fabs(dw)) - 1.f); }

void substep(const Params& P, Grid& g, int np, float* x, float* v, float* F, int lo[3], int hi[3]) {
  const float nf = static_cast<float>(P.n_grid);
  // Clear the active box.
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = lo[0]; i < hi[0]; ++i)
    for (int j = lo[1]; j < hi[1]; ++j)
      for (int k = lo[2]; k < hi[2]; ++k)
        for (int w = 0; w < 2; ++w) {
          const size_t id = g.idx(i, j, k, w);
          g.m[id] = 0.f;
          g.mv[3 * id] = g.mv[3 * id + 1] = g.mv[3 * id + 2] = 0.f;
        }
  // P2G
#pragma omp parallel for schedule(static)
  for (int p = 0; p < np; ++p) {
    const float* Fp = F + 9 * p;
    float U[9], S[3], V[9];
    svd3f(Fp, U, S, V);
    float R[9];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) R[i * 3 + j] = U[i * 3] * V[j * 3] + U[i * 3 + 1] * V[j * 3 + 1] + U[i * 3 + 2] * V[j * 3 + 2];
    const float J = S[0] * S[1] * S[2];
    float PF[9];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        float acc = 0.f;
        for (int k = 0; k < 3; ++k) acc += (Fp[i * 3 + k] - R[i * 3 + k]) * Fp[j * 3 + k];
        PF[i * 3 + j] = -P.vol * (2.f * P.mu * acc + (i == j ? P.lam * (J - 1.f) * J : 0.f));
      }
    for (int w = 0; w < 2; ++w) {
      const int sign = w == 0 ? -1 : 1;
      int base[3];
      float o[3], st[3][2];
      for (int a = 0; a < 3; ++a) stencil(x[3 * p + a], nf, sign, base[a], o[a], st[a]);
      for (int c = 0; c < 8; ++c) {
        const int I[3] = {(c >> 2) & 1, (c >> 1) & 1, c & 1};
        const float kx = st[0][I[0]], ky = st[1][I[1]], kz = st[2][I[2]];
        const float wgt = kx * ky * kz;
        const float gr[3] = {nf * ky * kz * grad1(o[0] - I[0]), nf * kx * kz * grad1(o[1] - I[1]),
                             nf * kx * ky * grad1(o[2] - I[2])};
        const size_t id = g.idx(base[0] + I[0], base[1] + I[1], base[2] + I[2], w);
        const float wm = wgt * P.mass;
#pragma omp atomic
        g.m[id] += wm;
        for (int r = 0; r < 3; ++r) {
          const float f = wm * v[3 * p + r] + P.dt * (PF[r * 3] * gr[0] + PF[r * 3 + 1] * gr[1] + PF[r * 3 + 2] * gr[2]);
#pragma omp atomic
          g.mv[3 * id + r] += f;
        }
      }
    }
  }
  // Grid update
  const int n = P.n_grid;
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = lo[0]; i < hi[0]; ++i)
    for (int j = lo[1]; j < hi[1]; ++j)
      for (int k = lo[2]; k < hi[2]; ++k)
        for (int w = 0; w < 2; ++w) {
          const size_t id = g.idx(i, j, k, w);
          float vv[3] = {0.f, 0.f, 0.f};
          if (g.m[id] > P.mass * 1e-8f)
            for (int r = 0; r < 3; ++r) vv[r] = g.mv[3 * id + r] / g.m[id];
          vv[1] += P.dt * P.gravity;
          const bool out = i < P.wall || i >= n - P.wall || j < P.wall || j >= n - P.wall || k < P.wall || k >= n - P.wall;
          for (int r = 0; r < 3; ++r) g.mv[3 * id + r] = out ? 0.f : vv[r];
        }
  // G2P
#pragma omp parallel for schedule(static)
  for (int p = 0; p < np; ++p) {
    float vel[3] = {0, 0, 0}, Cv[9] = {0};
    for (int w = 0; w < 2; ++w) {
      const int sign = w == 0 ? -1 : 1;
      int base[3];
      float o[3], st[3][2];
      for (int a = 0; a < 3; ++a) stencil(x[3 * p + a], nf, sign, base[a], o[a], st[a]);
      for (int c = 0; c < 8; ++c) {
        const int I[3] = {(c >> 2) & 1, (c >> 1) & 1, c & 1};
        const float kx = st[0][I[0]], ky = st[1][I[1]], kz = st[2][I[2]];
        const float wgt = kx * ky * kz;
        const float gr[3] = {nf * ky * kz * grad1(o[0] - I[0]), nf * kx * kz * grad1(o[1] - I[1]),
                             nf * kx * ky * grad1(o[2] - I[2])};
        const size_t id = g.idx(base[0] + I[0], base[1] + I[1], base[2] + I[2], w);
        for (int r = 0; r < 3; ++r) {
          const float gv = g.mv[3 * id + r];
          vel[r] += wgt * gv;
          for (int a = 0; a < 3; ++a) Cv[r * 3 + a] += gv * gr[a];
        }
      }
    }
    float dW[9];
    for (int k = 0; k < 9; ++k) dW[k] = 0.5f * P.dt * Cv[k] + ((k & 3) ? 0.f : 1.f);
    float Fn[9];
    float* Fp = F + 9 * p;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) Fn[i * 3 + j] = dW[i * 3] * Fp[j] + dW[i * 3 + 1] * Fp[3 + j] + dW[i * 3 + 2] * Fp[6 + j];
    std::memcpy(Fp, Fn, sizeof(Fn));
    for (int r = 0; r < 3; ++r) {
      v[3 * p + r] = 0.5f * vel[r];
      x[3 * p + r] += P.dt * v[3 * p + r];
    }
  }
}

}  // namespace

extern "C" {

// Runs nsteps PIC substeps on np particles; x (3np) is updated in place, v0 holds
// nv = 1 or np initial velocities.  Returns the wall time of the step loop in
// seconds (setup excluded) and writes the thread count used to *threads_out.
double pic_run(int np, float* x, const float* v0, int nv, int n_grid, double E, double nu, double rho, double gravity,
               int wall, double dt, int nsteps, int threads, int* threads_out) {
  if (threads > 0) omp_set_num_threads(threads);
  Params P;
  P.n_grid = n_grid;
  P.dx = 1.f / n_grid;
  P.vol = P.dx * P.dx * P.dx / 8.f;
  P.mass = static_cast<float>(rho) * P.vol;
  P.mu = static_cast<float>(E / (2 * (1 + nu)));
  P.lam = static_cast<float>(E * nu / ((1 + nu) * (1 - 2 * nu)));
  P.gravity = static_cast<float>(gravity);
  P.dt = static_cast<float>(dt);
  P.wall = wall;
  Grid g(n_grid);
  std::vector<float> v(3 * static_cast<size_t>(np)), F(9 * static_cast<size_t>(np), 0.f);
  for (int p = 0; p < np; ++p) {
    for (int r = 0; r < 3; ++r) v[3 * p + r] = nv == 1 ? v0[r] : v0[3 * p + r];
    F[9 * p] = F[9 * p + 4] = F[9 * p + 8] = 1.f;
  }
  int used = 1;
#pragma omp parallel
  {
#pragma omp single
    used = omp_get_num_threads();
  }
  if (threads_out) *threads_out = used;
  const double t0 = omp_get_wtime();
  for (int s = 0; s < nsteps; ++s) {
    int lo[3] = {n_grid, n_grid, n_grid}, hi[3] = {0, 0, 0};
    for (int p = 0; p < np; ++p)
      for (int a = 0; a < 3; ++a) {
        const int c = static_cast<int>(x[3 * p + a] * n_grid);
        lo[a] = std::min(lo[a], c - 2);
        hi[a] = std::max(hi[a], c + 3);
      }
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::max(lo[a], 0);
      hi[a] = std::min(hi[a], n_grid);
    }
    substep(P, g, np, x, v.data(), F.data(), lo, hi);
  }
  return omp_get_wtime() - t0;
}

}  // extern "C"
