// Test harness (host only, double precision): runs the differentiable
// fixed-corotated CK-MPM rollout of ckmpm_b200/csrc/diff_math.cuh on a dense
// grid -- the same generic forward and adjoint code the GPU kernels
// instantiate with float -- so that tests/test_diff_cpu.py can check the
// hand-written adjoint against central finite differences of this forward.
//
// diff_rollout(): forward of nsteps substeps from (x0, v0, logE) and, if
// gxT != NULL, the gradient of L = <gxT, xT> + <gFT, FT> with respect to x0,
// v0 and logE.  First substep advects with dt = 0 (currentDt / nextDt pair).
#include <cmath>
#include <cstring>
#include <vector>

#include "../../ckmpm_b200/csrc/diff_math.cuh"

using namespace ckmpm::diff;

namespace {

// One-sided Jacobi SVD (Hestenes) of a 3x3 with det > 0: F = U diag(S) V^T.
void svd_jacobi(const double* F, double* U, double* S, double* V) {
  double A[9];
  std::memcpy(A, F, sizeof(A));
  for (int k = 0; k < 9; ++k) V[k] = (k & 3) ? 0.0 : 1.0;
  for (int sweep = 0; sweep < 40; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        double a = 0, b = 0, c = 0;
        for (int i = 0; i < 3; ++i) {
          a += A[i * 3 + p] * A[i * 3 + p];
          b += A[i * 3 + q] * A[i * 3 + q];
          c += A[i * 3 + p] * A[i * 3 + q];
        }
        off += c * c;
        if (std::fabs(c) < 1e-300) continue;
        const double zeta = (b - a) / (2 * c);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1 + zeta * zeta));
        const double cs = 1 / std::sqrt(1 + t * t), sn = cs * t;
        for (int i = 0; i < 3; ++i) {
          const double ap = A[i * 3 + p], aq = A[i * 3 + q];
          A[i * 3 + p] = cs * ap - sn * aq;
          A[i * 3 + q] = sn * ap + cs * aq;
          const double vp = V[i * 3 + p], vq = V[i * 3 + q];
          V[i * 3 + p] = cs * vp - sn * vq;
          V[i * 3 + q] = sn * vp + cs * vq;
        }
      }
    if (off < 1e-60) break;
  }
  for (int j = 0; j < 3; ++j) {
    double s = 0;
    for (int i = 0; i < 3; ++i) s += A[i * 3 + j] * A[i * 3 + j];
    S[j] = std::sqrt(s);
    for (int i = 0; i < 3; ++i) U[i * 3 + j] = S[j] > 0 ? A[i * 3 + j] / S[j] : (i == j ? 1.0 : 0.0);
  }
}

struct Grid {
  DenseGrid G;
  std::vector<double> a;  // [node][4]: m, mv
  explicit Grid(const DenseGrid& g) : G(g), a(static_cast<size_t>(2) * g.n[0] * g.n[1] * g.n[2] * 4, 0.0) {}
  double* at(int g, int cx, int cy, int cz) { return &a[4 * node_index(G, g, cx, cy, cz)]; }
};

}  // namespace

extern "C" int diff_rollout(int n, const double* x0, const double* v0, const double* logE, double nu, double mass,
                            double vol, int nsteps, double dt, int ncells, double gravity, double* xT, double* FT,
                            const double* gxT, const double* gFT, double* gx0, double* gv0, double* glogE) {
  DenseGrid G{};
  for (int a = 0; a < 3; ++a) {
    G.n[a] = ncells;
    G.nb[a] = ncells / 4;
  }
  G.gravity = static_cast<float>(gravity);
  G.mass_clamp = 0.f;
  G.floor_cells = 0.f;
  G.boundary = 0;
  const double dx = 1.0 / ncells, inv_dx = static_cast<double>(ncells);
  const double vom = vol / mass;
  std::vector<double> lam(n), mu(n);
  for (int p = 0; p < n; ++p) {
    const double E = std::exp(logE[p]);
    mu[p] = E / (2 * (1 + nu));
    lam[p] = E * nu / ((1 + nu) * (1 - 2 * nu));
  }
  int bad = 0;
  auto svd = [](const double* F, double* U, double* S, double* V) { svd_jacobi(F, U, S, V); };
  // Rasterisation.
  Grid g0(G);
  for (int p = 0; p < n; ++p) {
    Stencil<double> st;
    make_stencil(&x0[3 * p], inv_dx, st);
    for (int g = 0; g < 2; ++g)
      for (int k = 0; k < 8; ++k) {
        const double w = node_weight(st, g, k, inv_dx, static_cast<double*>(nullptr));
        int c[3];
        for (int a = 0; a < 3; ++a) c[a] = st.a[g][a].base + ((k >> (2 - a)) & 1);
        if (!node_in_grid(G, c[0], c[1], c[2])) {
          bad = 1;
          continue;
        }
        double* q = g0.at(g, c[0], c[1], c[2]);
        q[0] += mass * w;
        for (int i = 0; i < 3; ++i) q[1 + i] += mass * w * v0[3 * p + i];
      }
  }
  // Forward, keeping every substep's inputs.
  std::vector<Grid> grids;           // grids[s]: sums read by substep s
  std::vector<std::vector<double>> vels;  // node velocities after the update of substep s
  std::vector<std::vector<Particle<double>>> parts;
  grids.push_back(g0);
  std::vector<Particle<double>> cur(n);
  for (int p = 0; p < n; ++p) {
    for (int a = 0; a < 3; ++a) cur[p].x[a] = x0[3 * p + a];
    for (int k = 0; k < 9; ++k) cur[p].F[k] = (k & 3) ? 0.0 : 1.0;
  }
  const size_t nn = static_cast<size_t>(2) * ncells * ncells * ncells;
  for (int s = 0; s < nsteps; ++s) {
    const double cdt = s == 0 ? 0.0 : dt, ndt = dt;
    std::vector<double> vel(3 * nn, 0.0);
    Grid& gr = grids[s];
    for (int g = 0; g < 2; ++g)
      for (int cx = 0; cx < ncells; ++cx)
        for (int cy = 0; cy < ncells; ++cy)
          for (int cz = 0; cz < ncells; ++cz) {
            const double* q = gr.at(g, cx, cy, cz);
            node_update(G, cx, cy, cz, q[0], q + 1, cdt, &vel[3 * node_index(G, g, cx, cy, cz)]);
          }
    vels.push_back(vel);
    parts.push_back(cur);
    Grid next(G);
    auto velf = [&](int g, int cx, int cy, int cz, double* v) {
      if (!node_in_grid(G, cx, cy, cz)) {
        bad = 1;
        v[0] = v[1] = v[2] = 0;
        return;
      }
      const double* q = &vel[3 * node_index(G, g, cx, cy, cz)];
      v[0] = q[0];
      v[1] = q[1];
      v[2] = q[2];
    };
    for (int p = 0; p < n; ++p) {
      Fwd<double> f;
      double U[9], S[3], V[9];
      particle_forward(cur[p], lam[p], mu[p], vom, cdt, ndt, dx, inv_dx, velf, svd, f, U, S, V);
      particle_deposit(f, dx, inv_dx, [&](int g, int cx, int cy, int cz, double w, const double* wv) {
        if (!node_in_grid(G, cx, cy, cz)) {
          bad = 1;
          return;
        }
        double* q = next.at(g, cx, cy, cz);
        q[0] += mass * w;
        for (int i = 0; i < 3; ++i) q[1 + i] += mass * wv[i];
      });
      for (int a = 0; a < 3; ++a) cur[p].x[a] = f.xn[a];
      for (int k = 0; k < 9; ++k) cur[p].F[k] = f.Fn[k];
    }
    grids.push_back(next);
  }
  for (int p = 0; p < n; ++p) {
    if (xT)
      for (int a = 0; a < 3; ++a) xT[3 * p + a] = cur[p].x[a];
    if (FT)
      for (int k = 0; k < 9; ++k) FT[9 * p + k] = cur[p].F[k];
  }
  if (!gxT) return bad;

  // Reverse.
  std::vector<double> xb(3 * n), Fb(9 * n), mub(n, 0.0), lamb(n, 0.0);
  for (int p = 0; p < n; ++p) {
    for (int a = 0; a < 3; ++a) xb[3 * p + a] = gxT[3 * p + a];
    for (int k = 0; k < 9; ++k) Fb[9 * p + k] = gFT ? gFT[9 * p + k] : 0.0;
  }
  std::vector<double> gadj(4 * nn, 0.0);  // adjoint of grids[s + 1] (none for the last)
  for (int s = nsteps - 1; s >= 0; --s) {
    const double cdt = s == 0 ? 0.0 : dt, ndt = dt;
    const std::vector<double>& vel = vels[s];
    std::vector<double> vbar(3 * nn, 0.0);
    auto velf = [&](int g, int cx, int cy, int cz, double* v) {
      const double* q = &vel[3 * node_index(G, g, cx, cy, cz)];
      v[0] = q[0];
      v[1] = q[1];
      v[2] = q[2];
    };
    auto gadjf = [&](int g, int cx, int cy, int cz, double* out) {
      const double* q = &gadj[4 * node_index(G, g, cx, cy, cz)];
      for (int i = 0; i < 4; ++i) out[i] = q[i];
    };
    auto vscat = [&](int g, int cx, int cy, int cz, const double* vb) {
      double* q = &vbar[3 * node_index(G, g, cx, cy, cz)];
      for (int i = 0; i < 3; ++i) q[i] += vb[i];
    };
    for (int p = 0; p < n; ++p) {
      const Particle<double>& pp = parts[s][p];
      Fwd<double> f;
      double U[9], S[3], V[9];
      particle_forward(pp, lam[p], mu[p], vom, cdt, ndt, dx, inv_dx, velf, svd, f, U, S, V);
      double xo[3], Fo[9];
      particle_adjoint(pp, f, U, S, V, mass, lam[p], mu[p], vom, cdt, ndt, dx, inv_dx, velf, gadjf, vscat,
                       &xb[3 * p], &Fb[9 * p], xo, Fo, mub[p], lamb[p]);
      for (int a = 0; a < 3; ++a) xb[3 * p + a] = xo[a];
      for (int k = 0; k < 9; ++k) Fb[9 * p + k] = Fo[k];
    }
    // grid-update adjoint of grids[s]
    Grid& gr = grids[s];
    for (int g = 0; g < 2; ++g)
      for (int cx = 0; cx < ncells; ++cx)
        for (int cy = 0; cy < ncells; ++cy)
          for (int cz = 0; cz < ncells; ++cz) {
            const int64_t id = node_index(G, g, cx, cy, cz);
            const double* q = gr.at(g, cx, cy, cz);
            node_update_adjoint(G, cx, cy, cz, q[0], &vel[3 * id], cdt, &vbar[3 * id], &gadj[4 * id]);
          }
  }
  // Rasterisation adjoint and parameter gradients.
  for (int p = 0; p < n; ++p) {
    double xo[3] = {xb[3 * p], xb[3 * p + 1], xb[3 * p + 2]}, vo[3] = {0, 0, 0};
    raster_adjoint(&x0[3 * p], &v0[3 * p], mass, inv_dx,
                   [&](int g, int cx, int cy, int cz, double* out) {
                     const double* q = &gadj[4 * node_index(G, g, cx, cy, cz)];
                     for (int i = 0; i < 4; ++i) out[i] = q[i];
                   },
                   xo, vo);
    for (int a = 0; a < 3; ++a) {
      gx0[3 * p + a] = xo[a];
      gv0[3 * p + a] = vo[a];
    }
    glogE[p] = mub[p] * mu[p] + lamb[p] * lam[p];
  }
  return bad;
}
