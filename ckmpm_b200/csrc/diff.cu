// Differentiable form: a rollout of the fixed-corotated CK-MPM substep with
// per-particle Young's modulus, its hand-written adjoint (diff_math.cuh), and
// substep checkpointing with recomputation.  No counterpart in the reference.
//
// Device layout (cells per axis n_c, nodes nn = 2 n_c^3 over both staggered grids):
//  * gsum[2]: int64 fixed-point node sums [node][m, mvx, mvy, mvz] per unit
//    particle mass (2^36 scale, as the substep's P2G tile), double-buffered;
//    exact, so a recomputed segment reproduces the forward bit for bit;
//  * vel: float4 per node (v after the grid update, m);
//  * bbox[s]: node-coordinate box of what substep s reads (min x,y,z, max x,y,z);
//    the dense passes run over that box only, and every box is zeroed after use;
//  * particles SoA (x[3][n], F[9][n]); checkpoints every K substeps hold x, F
//    and the node velocities of that substep (the forward writes those states
//    straight into their checkpoint slots); the backward recomputes one segment
//    at a time into a tape of the segment's other K - 1 substeps, then runs the
//    adjoint.  With K = 1 every substep is a checkpoint and the backward is the
//    adjoint alone (about 2.2 GB for 50k particles, 200 substeps and a 64^3
//    grid: HBM, not recomputation, holds the rollout);
//  * vbar: the node-velocity adjoint the particle adjoints scatter, as exact
//    int64 fixed-point sums like the forward's, so gradients are bitwise
//    reproducible too.  Its unit is set on the device at the start of each
//    backward from the largest incoming adjoint (the backward is linear in its
//    seed): 2^-40 of that largest component.
#include <climits>

#include "diff_math.cuh"

namespace ckmpm {
namespace diffk {

using diff::DenseGrid;
using diff::Fwd;
using diff::Particle;

constexpr int kThreads = 128;
constexpr float kScale = 68719476736.0f;  // 2^36
constexpr float kMaxValue = 131072.0f;    // 2^17
constexpr uint32_t kErrOutside = 1u, kErrRange = 2u;
constexpr float kAdjUnits = 1099511627776.0f;  // 2^40 fixed-point units per largest seed component
constexpr float kAdjMaxUnits = 4.6e18f;        // |contribution| bound in units (< 2^62)

struct Box {
  int lo[3], hi[3];
};

struct Dev {
  DenseGrid G;
  uint32_t n;
  float dx, inv_dx, mass, vol_over_mass, unit;  // unit = mass * 2^-36
  uint32_t* status;
  float* adj_scale;  // [0]: fixed-point units per adjoint unit, [1]: its inverse; [2]: max |seed| (bits)
};

__device__ __forceinline__ void box_reset(int* b) {
  b[0] = b[1] = b[2] = INT_MAX;
  b[3] = b[4] = b[5] = INT_MIN;
}

// Block-reduce a node box and merge it into b.
__device__ __forceinline__ void box_merge(int* b, int lo0, int lo1, int lo2, int hi0, int hi1, int hi2) {
  __shared__ int s[6];
  if (threadIdx.x < 3) s[threadIdx.x] = INT_MAX;
  else if (threadIdx.x < 6) s[threadIdx.x] = INT_MIN;
  __syncthreads();
  if (lo0 <= hi0) {
    atomicMin(&s[0], lo0);
    atomicMin(&s[1], lo1);
    atomicMin(&s[2], lo2);
    atomicMax(&s[3], hi0);
    atomicMax(&s[4], hi1);
    atomicMax(&s[5], hi2);
  }
  __syncthreads();
  if (threadIdx.x == 0 && s[0] <= s[3]) {
    atomicMin(&b[0], s[0]);
    atomicMin(&b[1], s[1]);
    atomicMin(&b[2], s[2]);
    atomicMax(&b[3], s[3]);
    atomicMax(&b[4], s[4]);
    atomicMax(&b[5], s[5]);
  }
}

__device__ __forceinline__ void fixed_add64(unsigned long long* p, float v) {
  atomicAdd(p, static_cast<unsigned long long>(__float2ll_rn(v * kScale)));
}

// Deposit nodes of one particle (per unit mass) into gsum; returns its node box.
__device__ __forceinline__ void deposit(const Dev& d, const Fwd<float>& f, unsigned long long* gsum, int* lo, int* hi) {
  diff::particle_deposit(f, d.dx, d.inv_dx, [&](int g, int cx, int cy, int cz, float w, const float* wv) {
    if (!diff::node_in_grid(d.G, cx, cy, cz)) {
      atomicOr(d.status, kErrOutside);
      return;
    }
    if (!(fabsf(wv[0]) < kMaxValue && fabsf(wv[1]) < kMaxValue && fabsf(wv[2]) < kMaxValue)) {
      atomicOr(d.status, kErrRange);
      return;
    }
    unsigned long long* q = gsum + 4 * diff::node_index(d.G, g, cx, cy, cz);
    fixed_add64(q, w);
    fixed_add64(q + 1, wv[0]);
    fixed_add64(q + 2, wv[1]);
    fixed_add64(q + 3, wv[2]);
    lo[0] = min(lo[0], cx);
    lo[1] = min(lo[1], cy);
    lo[2] = min(lo[2], cz);
    hi[0] = max(hi[0], cx);
    hi[1] = max(hi[1], cy);
    hi[2] = max(hi[2], cz);
  });
}

// AoS inputs -> SoA state; lambda / mu from log E; F = I.
__global__ void init_kernel(Dev d, const float* __restrict__ x0, const float* __restrict__ logE, float nu,
                            float* __restrict__ x, float* __restrict__ F, float* __restrict__ lam,
                            float* __restrict__ mu) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= d.n) return;
  for (int a = 0; a < 3; ++a) x[a * d.n + p] = x0[3 * p + a];
  for (int k = 0; k < 9; ++k) F[k * d.n + p] = (k & 3) ? 0.f : 1.f;
  const float E = expf(logE[p]);
  mu[p] = E / (2.f * (1.f + nu));
  lam[p] = E * nu / ((1.f + nu) * (1.f - 2.f * nu));
}

__global__ void raster_kernel(Dev d, const float* __restrict__ x, const float* __restrict__ v0,
                              unsigned long long* __restrict__ gsum, int* box) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
  if (p < d.n) {
    Fwd<float> f;
    const float xp[3] = {x[p], x[d.n + p], x[2 * d.n + p]};
    for (int a = 0; a < 3; ++a) {
      f.xn[a] = xp[a];
      f.v[a] = v0[3 * p + a];
    }
    for (int k = 0; k < 9; ++k) f.A[k] = 0.f;
    diff::make_stencil(xp, d.inv_dx, f.stn);
    deposit(d, f, gsum, lo, hi);
  }
  box_merge(box, lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]);
}

// Every substep's box starts empty; deposits widen it.  A recomputed segment
// deposits exactly what the forward did, so its boxes are unchanged.
__global__ void box_init_kernel(int* boxes, uint32_t count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) box_reset(boxes + 6 * i);
}

// Grid update over box b: int64 sums -> float4 (v, m); zero the sums read.
__global__ void grid_kernel(Dev d, unsigned long long* __restrict__ gsum, const int* __restrict__ b, float dt,
                            float4* __restrict__ vel) {
  if (b[0] > b[3]) return;
  const int ex = b[3] - b[0] + 1, ey = b[4] - b[1] + 1, ez = b[5] - b[2] + 1;
  const int64_t total = 2ll * ex * ey * ez;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int z = static_cast<int>(t % ez), y = static_cast<int>((t / ez) % ey);
    const int x = static_cast<int>((t / (static_cast<int64_t>(ez) * ey)) % ex);
    const int g = static_cast<int>(t / (static_cast<int64_t>(ez) * ey * ex));
    const int cx = b[0] + x, cy = b[1] + y, cz = b[2] + z;
    const int64_t id = diff::node_index(d.G, g, cx, cy, cz);
    ulonglong2* q = reinterpret_cast<ulonglong2*>(gsum + 4 * id);
    const ulonglong2 s01 = q[0], s23 = q[1];
    q[0] = make_ulonglong2(0ull, 0ull);
    q[1] = make_ulonglong2(0ull, 0ull);
    const float m = __ll2float_rn(static_cast<long long>(s01.x)) * d.unit;
    const float mv[3] = {__ll2float_rn(static_cast<long long>(s01.y)) * d.unit,
                         __ll2float_rn(static_cast<long long>(s23.x)) * d.unit,
                         __ll2float_rn(static_cast<long long>(s23.y)) * d.unit};
    float v[3];
    diff::node_update(d.G, cx, cy, cz, m, mv, dt, v);
    vel[id] = make_float4(v[0], v[1], v[2], m);
  }
}

struct VelReader {
  const DenseGrid* G;
  const float4* vel;
  uint32_t* status;
  __device__ void operator()(int g, int cx, int cy, int cz, float* v) const {
    if (!diff::node_in_grid(*G, cx, cy, cz)) {
      atomicOr(status, kErrOutside);
      v[0] = v[1] = v[2] = 0.f;
      return;
    }
    const float4 q = vel[diff::node_index(*G, g, cx, cy, cz)];
    v[0] = q.x;
    v[1] = q.y;
    v[2] = q.z;
  }
};

struct Svd {
  __device__ void operator()(const float* F, float* U, float* S, float* V) const { svd3(F, U, S, V); }
};

__device__ __forceinline__ void load_particle(const Dev& d, const float* x, const float* F, uint32_t p,
                                              Particle<float>& pp) {
  for (int a = 0; a < 3; ++a) pp.x[a] = x[a * d.n + p];
  for (int k = 0; k < 9; ++k) pp.F[k] = F[k * d.n + p];
}

// Forward substep of every particle: G2P at x, x and F update, stress,
// deposit at x' into gsum_next; new state to (xo, Fo).
__global__ void __launch_bounds__(kThreads) particle_kernel(Dev d, const float* __restrict__ x,
                                                            const float* __restrict__ F, const float* __restrict__ lam,
                                                            const float* __restrict__ mu, const float4* __restrict__ vel,
                                                            float dt, float ndt, unsigned long long* __restrict__ gsum,
                                                            int* bnext, float* __restrict__ xo, float* __restrict__ Fo) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
  if (p < d.n) {
    Particle<float> pp;
    load_particle(d, x, F, p, pp);
    Fwd<float> f;
    float U[9], S[3], V[9];
    VelReader vr{&d.G, vel, d.status};
    diff::particle_forward(pp, lam[p], mu[p], d.vol_over_mass, dt, ndt, d.dx, d.inv_dx, vr, Svd{}, f, U, S, V);
    deposit(d, f, gsum, lo, hi);
    for (int a = 0; a < 3; ++a) xo[a * d.n + p] = f.xn[a];
    for (int k = 0; k < 9; ++k) Fo[k * d.n + p] = f.Fn[k];
  }
  box_merge(bnext, lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]);
}

// Adjoint of one substep for every particle.  xb / Fb hold the adjoints of the
// substep's outputs on entry and of its inputs on exit.
// The fixed-point unit of the velocity adjoint: the largest |component| of the
// incoming adjoints (x and F at the end of the rollout), then 2^40 units per it.
__global__ void adj_seed_max_kernel(uint32_t n, const float* __restrict__ xb, const float* __restrict__ Fb,
                                    float* adj_scale) {
  float m = 0.f;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 12 * n; i += gridDim.x * blockDim.x)
    m = fmaxf(m, fabsf(i < 3 * n ? xb[i] : Fb[i - 3 * n]));
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  // non-negative floats order like their bit patterns
  if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(reinterpret_cast<unsigned*>(adj_scale + 2), __float_as_uint(m));
}

__global__ void adj_scale_kernel(float* adj_scale) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    const float m = adj_scale[2];
    adj_scale[0] = m > 0.f ? __fdiv_rn(kAdjUnits, m) : 1.f;
    adj_scale[1] = m > 0.f ? __fdiv_rn(m, kAdjUnits) : 1.f;
  }
}

__global__ void __launch_bounds__(kThreads, 3) particle_adjoint_kernel(
    Dev d, const float* __restrict__ x, const float* __restrict__ F, const float* __restrict__ lam,
    const float* __restrict__ mu, const float4* __restrict__ vel, float dt, float ndt, const float4* __restrict__ gadj,
    float* __restrict__ xb, float* __restrict__ Fb, float* __restrict__ mub, float* __restrict__ lamb,
    unsigned long long* __restrict__ vbar) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= d.n) return;
  Particle<float> pp;
  load_particle(d, x, F, p, pp);
  Fwd<float> f;
  float U[9], S[3], V[9];
  VelReader vr{&d.G, vel, d.status};
  diff::particle_forward(pp, lam[p], mu[p], d.vol_over_mass, dt, ndt, d.dx, d.inv_dx, vr, Svd{}, f, U, S, V);
  const DenseGrid& G = d.G;
  auto ga = [&](int g, int cx, int cy, int cz, float* out) {
    if (!gadj || !diff::node_in_grid(G, cx, cy, cz)) {
      out[0] = out[1] = out[2] = out[3] = 0.f;
      return;
    }
    const float4 q = gadj[diff::node_index(G, g, cx, cy, cz)];
    out[0] = q.x;
    out[1] = q.y;
    out[2] = q.z;
    out[3] = q.w;
  };
  const float units = d.adj_scale[0];
  auto vs = [&](int g, int cx, int cy, int cz, const float* vb) {
    if (!diff::node_in_grid(G, cx, cy, cz)) return;
    unsigned long long* q = vbar + 3 * diff::node_index(G, g, cx, cy, cz);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float u = vb[c] * units;
      if (!(fabsf(u) < kAdjMaxUnits)) {
        atomicOr(d.status, kErrRange);
        continue;
      }
      atomicAdd(q + c, static_cast<unsigned long long>(__float2ll_rn(u)));
    }
  };
  float xnb[3], Fnb[9], xo[3], Fo[9];
  for (int a = 0; a < 3; ++a) xnb[a] = xb[a * d.n + p];
  for (int k = 0; k < 9; ++k) Fnb[k] = Fb[k * d.n + p];
  float mb = mub[p], lb = lamb[p];
  diff::particle_adjoint(pp, f, U, S, V, d.mass, lam[p], mu[p], d.vol_over_mass, dt, ndt, d.dx, d.inv_dx, vr, ga, vs,
                         xnb, Fnb, xo, Fo, mb, lb);
  for (int a = 0; a < 3; ++a) xb[a * d.n + p] = xo[a];
  for (int k = 0; k < 9; ++k) Fb[k * d.n + p] = Fo[k];
  mub[p] = mb;
  lamb[p] = lb;
}

// Grid-update adjoint over box b: node velocity adjoint -> (mbar, mvbar); zeroes vbar.
__global__ void grid_adjoint_kernel(Dev d, const int* __restrict__ b, const float4* __restrict__ vel, float dt,
                                    unsigned long long* __restrict__ vbar, float4* __restrict__ gadj) {
  if (b[0] > b[3]) return;
  const int ex = b[3] - b[0] + 1, ey = b[4] - b[1] + 1, ez = b[5] - b[2] + 1;
  const int64_t total = 2ll * ex * ey * ez;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int z = static_cast<int>(t % ez), y = static_cast<int>((t / ez) % ey);
    const int x = static_cast<int>((t / (static_cast<int64_t>(ez) * ey)) % ex);
    const int g = static_cast<int>(t / (static_cast<int64_t>(ez) * ey * ex));
    const int cx = b[0] + x, cy = b[1] + y, cz = b[2] + z;
    const int64_t id = diff::node_index(d.G, g, cx, cy, cz);
    unsigned long long* vb = vbar + 3 * id;
    const float inv_units = d.adj_scale[1];
    const float vbv[3] = {__ll2float_rn(static_cast<long long>(vb[0])) * inv_units,
                          __ll2float_rn(static_cast<long long>(vb[1])) * inv_units,
                          __ll2float_rn(static_cast<long long>(vb[2])) * inv_units};
    vb[0] = vb[1] = vb[2] = 0ull;
    const float4 q = vel[id];
    const float v[3] = {q.x, q.y, q.z};
    float out[4];
    diff::node_update_adjoint(d.G, cx, cy, cz, q.w, v, dt, vbv, out);
    gadj[id] = make_float4(out[0], out[1], out[2], out[3]);
  }
}

// Rasterisation adjoint and the outputs: gx0 (AoS), gv0 (AoS), glogE.
__global__ void finish_kernel(Dev d, const float* __restrict__ x, const float* __restrict__ v0,
                              const float4* __restrict__ gadj, const float* __restrict__ xb,
                              const float* __restrict__ lam, const float* __restrict__ mu,
                              const float* __restrict__ mub, const float* __restrict__ lamb, float* __restrict__ gx0,
                              float* __restrict__ gv0, float* __restrict__ glogE) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= d.n) return;
  const float xp[3] = {x[p], x[d.n + p], x[2 * d.n + p]};
  const float vp[3] = {v0[3 * p], v0[3 * p + 1], v0[3 * p + 2]};
  float xo[3] = {xb[p], xb[d.n + p], xb[2 * d.n + p]}, vo[3] = {0.f, 0.f, 0.f};
  const DenseGrid& G = d.G;
  diff::raster_adjoint(xp, vp, d.mass, d.inv_dx,
                       [&](int g, int cx, int cy, int cz, float* out) {
                         if (!diff::node_in_grid(G, cx, cy, cz)) {
                           out[0] = out[1] = out[2] = out[3] = 0.f;
                           return;
                         }
                         const float4 q = gadj[diff::node_index(G, g, cx, cy, cz)];
                         out[0] = q.x;
                         out[1] = q.y;
                         out[2] = q.z;
                         out[3] = q.w;
                       },
                       xo, vo);
  for (int a = 0; a < 3; ++a) {
    gx0[3 * p + a] = xo[a];
    gv0[3 * p + a] = vo[a];
  }
  glogE[p] = mub[p] * mu[p] + lamb[p] * lam[p];
}

// SoA <-> AoS for the outputs and the incoming adjoints.
__global__ void soa_to_aos_kernel(uint32_t n, int w, const float* __restrict__ soa, float* __restrict__ aos) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  for (int k = 0; k < w; ++k) aos[static_cast<size_t>(w) * p + k] = soa[static_cast<size_t>(k) * n + p];
}

__global__ void aos_to_soa_kernel(uint32_t n, int w, const float* __restrict__ aos, float* __restrict__ soa) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  for (int k = 0; k < w; ++k) soa[static_cast<size_t>(k) * n + p] = aos ? aos[static_cast<size_t>(w) * p + k] : 0.f;
}

}  // namespace diffk
}  // namespace ckmpm

// ------------------------------------------------------------------ host side
struct ckmpm_diff {
  ckmpm::diffk::Dev d{};
  int device = 0;
  uint32_t nsteps = 0, every = 20, nseg = 0;
  float dt = 0.f, nu = 0.3f;
  size_t nn = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr, t0 = nullptr, t1 = nullptr;
  std::vector<std::pair<void*, size_t>> allocs;
  // inputs / outputs (internal, fixed addresses for the graphs)
  float *x0 = nullptr, *v0 = nullptr, *logE = nullptr, *xT = nullptr, *FT = nullptr;
  float *gxT = nullptr, *gFT = nullptr, *gx0 = nullptr, *gv0 = nullptr, *glogE = nullptr;
  float *lam = nullptr, *mu = nullptr;
  float* xs[2] = {nullptr, nullptr};  // forward ping-pong (SoA x: 3n, F: 9n in one array of 12n)
  float* ck = nullptr;                // checkpoints: nseg x 12n
  float4* ckvel = nullptr;            // nseg x nn
  float* tape = nullptr;              // max(every - 1, 1) x 12n: substeps s0 + 1 .. s1 - 1 of a segment
  float4* tapevel = nullptr;          // every x nn
  float4* vel = nullptr;              // scratch node velocities (forward pass)
  unsigned long long* gsum[2] = {nullptr, nullptr};
  int* box = nullptr;                 // (nsteps + 1) x 6
  float *xb = nullptr, *Fb = nullptr, *mub = nullptr, *lamb = nullptr;
  unsigned long long* vbar = nullptr;
  float4* gadj = nullptr;
  cudaGraphExec_t gfwd = nullptr, gbwd = nullptr;
  uint64_t generation = 0;
  bool have_forward = false;
  float ms_fwd = 0.f, ms_bwd = 0.f;
  std::string err;
};

namespace {

thread_local std::string g_diff_error;

ckmpm_status dfail(ckmpm_diff* h, ckmpm_status code, const std::string& msg) {
  if (h) h->err = msg;
  else g_diff_error = msg;
  return code;
}

#define DK_CUDA(h, call)                                                                        \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      return dfail((h), CKMPM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
  } while (0)

template <typename T>
cudaError_t dk_alloc(ckmpm_diff* h, T** p, size_t count) {
  void* q = nullptr;
  const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e == cudaSuccess) h->allocs.emplace_back(q, bytes);
  *p = static_cast<T*>(q);
  return e;
}

using namespace ckmpm::diffk;

unsigned blocks_for(uint32_t n) { return (n + kThreads - 1) / kThreads; }

int grid_ctas(const ckmpm_diff* h) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
  return sms * 8;
}

}  // namespace

extern "C" {

ckmpm_status ckmpm_diff_create(const ckmpm_scene_desc* desc, uint32_t n, float mass, float volume, float nu,
                               uint32_t nsteps, float dt, uint32_t checkpoint_every, ckmpm_diff** out) {
  if (!desc || !out) return dfail(nullptr, CKMPM_ERR_INVALID, "null argument");
  *out = nullptr;
  if (n == 0 || nsteps == 0 || checkpoint_every == 0) return dfail(nullptr, CKMPM_ERR_INVALID, "empty rollout");
  if (!(mass > 0.f) || !(volume > 0.f) || !(dt >= 0.f) || !(nu > -1.f && nu < 0.5f))
    return dfail(nullptr, CKMPM_ERR_INVALID, "bad mass, volume, dt or nu");
  if (!(desc->dx > 0.f)) return dfail(nullptr, CKMPM_ERR_INVALID, "dx must be positive");
  for (int a = 0; a < 3; ++a)
    if (desc->domain_blocks[a] < 5 || desc->domain_blocks[a] > 64)
      return dfail(nullptr, CKMPM_ERR_INVALID, "domain_blocks must be 5..64 for the dense differentiable grid");
  if (desc->boundary != CKMPM_BOUNDARY_STICKY_BLOCKS && desc->boundary != CKMPM_BOUNDARY_SLIP_FLOOR)
    return dfail(nullptr, CKMPM_ERR_INVALID, "unknown boundary kind");
  if (cudaSetDevice(desc->device) != cudaSuccess) return dfail(nullptr, CKMPM_ERR_CUDA, "cudaSetDevice failed");
  ckmpm_diff* h = new ckmpm_diff();
  auto bail = [&](ckmpm_status st) {
    g_diff_error = h->err;
    ckmpm_diff_destroy(h);
    return st;
  };
  h->device = desc->device;
  h->nsteps = nsteps;
  h->every = std::min(checkpoint_every, nsteps);
  h->nseg = (nsteps + h->every - 1) / h->every;
  h->dt = dt;
  h->nu = nu;
  Dev& d = h->d;
  for (int a = 0; a < 3; ++a) {
    d.G.nb[a] = desc->domain_blocks[a];
    d.G.n[a] = 4 * desc->domain_blocks[a];
  }
  d.G.gravity = desc->gravity;
  d.G.mass_clamp = desc->mass_clamp;
  d.G.floor_cells = desc->floor_cells;
  d.G.boundary = desc->boundary;
  d.n = n;
  d.dx = desc->dx;
  d.inv_dx = static_cast<float>(1.0 / static_cast<double>(desc->dx));
  d.mass = mass;
  d.vol_over_mass = volume / mass;
  d.unit = mass * 1.4551915228366852e-11f;  // 2^-36
  h->nn = static_cast<size_t>(2) * d.G.n[0] * d.G.n[1] * d.G.n[2];
  const size_t nn = h->nn;
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_in, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_out, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreate(&h->t0) != cudaSuccess || cudaEventCreate(&h->t1) != cudaSuccess)
    return bail(dfail(h, CKMPM_ERR_CUDA, "stream / event creation failed"));
  bool ok = dk_alloc(h, &d.status, 1) == cudaSuccess && dk_alloc(h, &h->x0, 3 * n) == cudaSuccess &&
            dk_alloc(h, &h->v0, 3 * n) == cudaSuccess && dk_alloc(h, &h->logE, n) == cudaSuccess &&
            dk_alloc(h, &h->xT, 3 * n) == cudaSuccess && dk_alloc(h, &h->FT, 9 * n) == cudaSuccess &&
            dk_alloc(h, &h->gxT, 3 * n) == cudaSuccess && dk_alloc(h, &h->gFT, 9 * n) == cudaSuccess &&
            dk_alloc(h, &h->gx0, 3 * n) == cudaSuccess && dk_alloc(h, &h->gv0, 3 * n) == cudaSuccess &&
            dk_alloc(h, &h->glogE, n) == cudaSuccess && dk_alloc(h, &h->lam, n) == cudaSuccess &&
            dk_alloc(h, &h->mu, n) == cudaSuccess && dk_alloc(h, &h->xs[0], 12 * n) == cudaSuccess &&
            dk_alloc(h, &h->xs[1], 12 * n) == cudaSuccess &&
            dk_alloc(h, &h->ck, static_cast<size_t>(h->nseg) * 12 * n) == cudaSuccess &&
            dk_alloc(h, &h->ckvel, static_cast<size_t>(h->nseg) * nn) == cudaSuccess &&
            dk_alloc(h, &h->tape, static_cast<size_t>(std::max<uint32_t>(h->every, 2) - 1) * 12 * n) == cudaSuccess &&
            dk_alloc(h, &h->tapevel, static_cast<size_t>(h->every) * nn) == cudaSuccess &&
            dk_alloc(h, &h->vel, nn) == cudaSuccess && dk_alloc(h, &h->gsum[0], 4 * nn) == cudaSuccess &&
            dk_alloc(h, &h->gsum[1], 4 * nn) == cudaSuccess &&
            dk_alloc(h, &h->box, 6 * static_cast<size_t>(nsteps + 1)) == cudaSuccess &&
            dk_alloc(h, &h->xb, 3 * n) == cudaSuccess && dk_alloc(h, &h->Fb, 9 * n) == cudaSuccess &&
            dk_alloc(h, &h->mub, n) == cudaSuccess && dk_alloc(h, &h->lamb, n) == cudaSuccess &&
            dk_alloc(h, &h->vbar, 3 * nn) == cudaSuccess && dk_alloc(h, &h->gadj, nn) == cudaSuccess &&
            dk_alloc(h, &h->d.adj_scale, 4) == cudaSuccess;
  if (!ok) return bail(dfail(h, CKMPM_ERR_CUDA, "device allocation failed"));
  // Sums and velocity adjoints start (and are always left) at zero inside every box.
  if (cudaMemsetAsync(h->gsum[0], 0, 32 * nn, h->stream) != cudaSuccess ||
      cudaMemsetAsync(h->gsum[1], 0, 32 * nn, h->stream) != cudaSuccess ||
      cudaMemsetAsync(h->vbar, 0, 24 * nn, h->stream) != cudaSuccess ||
      cudaMemsetAsync(h->d.adj_scale, 0, 4 * sizeof(float), h->stream) != cudaSuccess ||
      cudaMemsetAsync(h->vel, 0, 16 * nn, h->stream) != cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess)
    return bail(dfail(h, CKMPM_ERR_CUDA, "initialisation failed"));
  *out = h;
  return CKMPM_OK;
}

const char* ckmpm_diff_last_error(const ckmpm_diff* h) { return h ? h->err.c_str() : g_diff_error.c_str(); }

ckmpm_status ckmpm_diff_destroy(ckmpm_diff* h) {
  if (!h) return CKMPM_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->gfwd) cudaGraphExecDestroy(h->gfwd);
  if (h->gbwd) cudaGraphExecDestroy(h->gbwd);
  for (auto& p : h->allocs) cudaFree(p.first);
  if (h->ev_in) cudaEventDestroy(h->ev_in);
  if (h->ev_out) cudaEventDestroy(h->ev_out);
  if (h->t0) cudaEventDestroy(h->t0);
  if (h->t1) cudaEventDestroy(h->t1);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return CKMPM_OK;
}

}  // extern "C"

namespace {

// The whole forward rollout: init, rasterise, nsteps substeps; checkpoint k
// (x, F and node velocities of substep k * every) on the way; outputs xT, FT.
cudaError_t enqueue_rollout(ckmpm_diff* h) {
  const Dev& d = h->d;
  const uint32_t n = d.n;
  const size_t nn = h->nn;
  const int ctas = grid_ctas(h);
  cudaStream_t st = h->stream;
  cudaError_t e = cudaMemsetAsync(d.status, 0, sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  // State of substep s: its checkpoint slot when it has one, else a ping-pong buffer.
  auto state = [&](uint32_t s) -> float* {
    return (s < h->nsteps && s % h->every == 0) ? h->ck + static_cast<size_t>(s / h->every) * 12 * n
                                                 : h->xs[s & 1];
  };
  init_kernel<<<blocks_for(n), kThreads, 0, st>>>(d, h->x0, h->logE, h->nu, state(0), state(0) + 3 * n, h->lam,
                                                  h->mu);
  box_init_kernel<<<(h->nsteps + 1 + 127) / 128, 128, 0, st>>>(h->box, h->nsteps + 1);
  raster_kernel<<<blocks_for(n), kThreads, 0, st>>>(d, state(0), h->v0, h->gsum[0], h->box);
  for (uint32_t s = 0; s < h->nsteps; ++s) {
    const float cdt = s == 0 ? 0.f : h->dt, ndt = h->dt;
    const bool ck = (s % h->every) == 0;
    const uint32_t k = s / h->every;
    float4* vs = ck ? h->ckvel + static_cast<size_t>(k) * nn : h->vel;
    // grid update of substep s (reads gsum[s & 1] in box s; resets box s + 1)
    grid_kernel<<<ctas, 256, 0, st>>>(d, h->gsum[s & 1], h->box + 6 * s, cdt, vs);
    float* in = state(s);
    float* outp = state(s + 1);
    particle_kernel<<<blocks_for(n), kThreads, 0, st>>>(d, in, in + 3 * n, h->lam, h->mu, vs, cdt, ndt,
                                                        h->gsum[(s + 1) & 1], h->box + 6 * (s + 1), outp,
                                                        outp + 3 * n);
  }
  // Leave the last deposit's sums at zero (they are never read).
  grid_kernel<<<ctas, 256, 0, st>>>(d, h->gsum[h->nsteps & 1], h->box + 6 * h->nsteps, h->dt, h->vel);
  const float* fin = state(h->nsteps);
  soa_to_aos_kernel<<<blocks_for(n), kThreads, 0, st>>>(n, 3, fin, h->xT);
  soa_to_aos_kernel<<<blocks_for(n), kThreads, 0, st>>>(n, 9, fin + 3 * n, h->FT);
  return cudaGetLastError();
}

// The whole backward: for each segment from the last, recompute its substeps
// from the checkpoint into the tape, then run the adjoint in reverse.
cudaError_t enqueue_backward(ckmpm_diff* h) {
  const Dev& d = h->d;
  const uint32_t n = d.n;
  const size_t nn = h->nn;
  const int ctas = grid_ctas(h);
  cudaStream_t st = h->stream;
  aos_to_soa_kernel<<<blocks_for(n), kThreads, 0, st>>>(n, 3, h->gxT, h->xb);
  aos_to_soa_kernel<<<blocks_for(n), kThreads, 0, st>>>(n, 9, h->gFT, h->Fb);
  cudaError_t e = cudaMemsetAsync(h->d.adj_scale + 2, 0, sizeof(float), st);
  if (e != cudaSuccess) return e;
  adj_seed_max_kernel<<<ctas, 256, 0, st>>>(n, h->xb, h->Fb, h->d.adj_scale);
  adj_scale_kernel<<<1, 32, 0, st>>>(h->d.adj_scale);
  e = cudaMemsetAsync(h->mub, 0, sizeof(float) * n, st);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(h->lamb, 0, sizeof(float) * n, st);
  if (e != cudaSuccess) return e;
  bool first = true;  // the last substep's deposit has no adjoint
  for (int k = static_cast<int>(h->nseg) - 1; k >= 0; --k) {
    const uint32_t s0 = static_cast<uint32_t>(k) * h->every;
    const uint32_t s1 = std::min(h->nsteps, s0 + h->every);
    // recompute: the segment's first state is its checkpoint, state s0 + j (j >= 1)
    // tape slot j - 1; tapevel slot j holds the node velocities of substep s0 + j
    auto statep = [&](uint32_t s) -> float* {
      return s == s0 ? h->ck + static_cast<size_t>(k) * 12 * n : h->tape + static_cast<size_t>(s - s0 - 1) * 12 * n;
    };
    auto velp = [&](uint32_t s) -> float4* {
      return s == s0 ? h->ckvel + static_cast<size_t>(k) * nn : h->tapevel + static_cast<size_t>(s - s0) * nn;
    };
    for (uint32_t s = s0; s < s1; ++s) {
      const float cdt = s == 0 ? 0.f : h->dt, ndt = h->dt;
      float* in = statep(s);
      if (s > s0)
        grid_kernel<<<ctas, 256, 0, st>>>(d, h->gsum[s & 1], h->box + 6 * s, cdt, velp(s));
      if (s + 1 < s1) {
        float* outp = statep(s + 1);
        particle_kernel<<<blocks_for(n), kThreads, 0, st>>>(d, in, in + 3 * n, h->lam, h->mu, velp(s), cdt, ndt,
                                                            h->gsum[(s + 1) & 1], h->box + 6 * (s + 1), outp,
                                                            outp + 3 * n);
      }
    }
    // reverse through the segment
    for (int s = static_cast<int>(s1) - 1; s >= static_cast<int>(s0); --s) {
      const float cdt = s == 0 ? 0.f : h->dt, ndt = h->dt;
      const float* in = statep(static_cast<uint32_t>(s));
      particle_adjoint_kernel<<<blocks_for(n), kThreads, 0, st>>>(d, in, in + 3 * n, h->lam, h->mu, velp(s), cdt, ndt,
                                                                  first ? nullptr : h->gadj, h->xb, h->Fb, h->mub,
                                                                  h->lamb, h->vbar);
      first = false;
      grid_adjoint_kernel<<<ctas, 256, 0, st>>>(d, h->box + 6 * s, velp(s), cdt, h->vbar, h->gadj);
    }
  }
  finish_kernel<<<blocks_for(n), kThreads, 0, st>>>(d, h->ck, h->v0, h->gadj, h->xb, h->lam, h->mu, h->mub, h->lamb,
                                                    h->gx0, h->gv0, h->glogE);
  return cudaGetLastError();
}

cudaError_t capture(ckmpm_diff* h, bool fwd, cudaGraphExec_t* exec) {
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  e = fwd ? enqueue_rollout(h) : enqueue_backward(h);
  cudaError_t e2 = cudaStreamEndCapture(h->stream, &g);
  if (e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return e;
  }
  if (e2 != cudaSuccess) return e2;
  e = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  return e;
}

ckmpm_status check_status(ckmpm_diff* h) {
  uint32_t s = 0;
  DK_CUDA(h, cudaMemcpyAsync(&s, h->d.status, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
  DK_CUDA(h, cudaStreamSynchronize(h->stream));
  if (s & kErrOutside) return dfail(h, CKMPM_ERR_CAPACITY, "a particle's stencil left the dense grid");
  if (s & kErrRange) return dfail(h, CKMPM_ERR_NUMERIC, "out-of-range P2G contribution");
  return CKMPM_OK;
}

}  // namespace

extern "C" {

ckmpm_status ckmpm_diff_forward(ckmpm_diff* h, const float* x0, const float* v0, const float* logE, float* xT,
                                float* FT, void* cuda_stream) {
  if (!h || !x0 || !v0 || !logE) return dfail(h, CKMPM_ERR_INVALID, "null argument");
  DK_CUDA(h, cudaSetDevice(h->device));
  cudaStream_t user = static_cast<cudaStream_t>(cuda_stream);
  const uint32_t n = h->d.n;
  DK_CUDA(h, cudaEventRecord(h->ev_in, user));
  DK_CUDA(h, cudaStreamWaitEvent(h->stream, h->ev_in, 0));
  DK_CUDA(h, cudaMemcpyAsync(h->x0, x0, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, h->stream));
  DK_CUDA(h, cudaMemcpyAsync(h->v0, v0, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, h->stream));
  DK_CUDA(h, cudaMemcpyAsync(h->logE, logE, sizeof(float) * n, cudaMemcpyDeviceToDevice, h->stream));
  if (!h->gfwd) DK_CUDA(h, capture(h, true, &h->gfwd));
  DK_CUDA(h, cudaEventRecord(h->t0, h->stream));
  DK_CUDA(h, cudaGraphLaunch(h->gfwd, h->stream));
  DK_CUDA(h, cudaEventRecord(h->t1, h->stream));
  if (xT) DK_CUDA(h, cudaMemcpyAsync(xT, h->xT, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, h->stream));
  if (FT) DK_CUDA(h, cudaMemcpyAsync(FT, h->FT, sizeof(float) * 9 * n, cudaMemcpyDeviceToDevice, h->stream));
  ckmpm_status st = check_status(h);
  cudaEventElapsedTime(&h->ms_fwd, h->t0, h->t1);
  if (st != CKMPM_OK) return st;
  DK_CUDA(h, cudaEventRecord(h->ev_out, h->stream));
  DK_CUDA(h, cudaStreamWaitEvent(user, h->ev_out, 0));
  h->have_forward = true;
  ++h->generation;
  return CKMPM_OK;
}

ckmpm_status ckmpm_diff_backward(ckmpm_diff* h, const float* gxT, const float* gFT, float* gx0, float* gv0,
                                 float* glogE, void* cuda_stream) {
  if (!h) return dfail(h, CKMPM_ERR_INVALID, "null argument");
  if (!h->have_forward) return dfail(h, CKMPM_ERR_INVALID, "ckmpm_diff_forward has not run");
  DK_CUDA(h, cudaSetDevice(h->device));
  cudaStream_t user = static_cast<cudaStream_t>(cuda_stream);
  const uint32_t n = h->d.n;
  DK_CUDA(h, cudaEventRecord(h->ev_in, user));
  DK_CUDA(h, cudaStreamWaitEvent(h->stream, h->ev_in, 0));
  if (gxT) DK_CUDA(h, cudaMemcpyAsync(h->gxT, gxT, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, h->stream));
  else DK_CUDA(h, cudaMemsetAsync(h->gxT, 0, sizeof(float) * 3 * n, h->stream));
  if (gFT) DK_CUDA(h, cudaMemcpyAsync(h->gFT, gFT, sizeof(float) * 9 * n, cudaMemcpyDeviceToDevice, h->stream));
  else DK_CUDA(h, cudaMemsetAsync(h->gFT, 0, sizeof(float) * 9 * n, h->stream));
  if (!h->gbwd) DK_CUDA(h, capture(h, false, &h->gbwd));
  DK_CUDA(h, cudaEventRecord(h->t0, h->stream));
  DK_CUDA(h, cudaGraphLaunch(h->gbwd, h->stream));
  DK_CUDA(h, cudaEventRecord(h->t1, h->stream));
  if (gx0) DK_CUDA(h, cudaMemcpyAsync(gx0, h->gx0, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, h->stream));
  if (gv0) DK_CUDA(h, cudaMemcpyAsync(gv0, h->gv0, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, h->stream));
  if (glogE) DK_CUDA(h, cudaMemcpyAsync(glogE, h->glogE, sizeof(float) * n, cudaMemcpyDeviceToDevice, h->stream));
  ckmpm_status st = check_status(h);
  cudaEventElapsedTime(&h->ms_bwd, h->t0, h->t1);
  if (st != CKMPM_OK) return st;
  DK_CUDA(h, cudaEventRecord(h->ev_out, h->stream));
  DK_CUDA(h, cudaStreamWaitEvent(user, h->ev_out, 0));
  return CKMPM_OK;
}

ckmpm_status ckmpm_diff_timing(ckmpm_diff* h, float* ms_out2, uint64_t* generation) {
  if (!h || !ms_out2) return dfail(h, CKMPM_ERR_INVALID, "null argument");
  ms_out2[0] = h->ms_fwd;
  ms_out2[1] = h->ms_bwd;
  if (generation) *generation = h->generation;
  return CKMPM_OK;
}

}  // extern "C"
