// Device kernels of the CK-MPM substep.
//
// Data layout (per scene; a batch stacks `nstack` identical domains, scene w
// owning table entries [w * blocks, (w + 1) * blocks), and no stencil, flush or
// rebin ever crosses from one stacked domain into another):
//  * grid[2]: dense over every 4^3 block of the domain, 4 KB per block of
//    exact 64-bit fixed-point sums (2^-36 of a particle mass per unit):
//    [m, mvx, mvy, mvz][grid -dx/4, +dx/4][cell i*16 + j*4 + k], the per-block
//    SoA of the reference's MPMGridBlock (include/mpm_grid.cuh:18-67) but
//    addressed directly by block coordinate instead of through a partition
//    slot.  grid[s&1] is read by substep s, grid[(s+1)&1] written by it with
//    integer reductions, so the sums do not depend on the order they arrive in.
//  * stamp[2]: per block, the epoch for which it was last zeroed; a block whose
//    stamp is stale reads as empty.  Only the blocks a substep deposits into
//    are zeroed, by zero_windows_kernel before that substep.
//  * per model, particle state SoA (x[3], F[9], aux, Q[9] for the linear
//    model, id) double-buffered and sorted by particle block; the block list
//    (keys, start, count) in colour-major key order; a dense block table; 28
//    outgoing-direction prefix counts per block and a u16 per-particle index
//    list that records, for each block, which of its particles leave in which
//    of the 27 directions.
//
// Every substep is: one fused kernel per model (grid update + G2P + F update,
// SVD, return map + rebin record + P2G, flushed as exact integer sums), then
// the colour-major compaction that builds the next block list and the zeroing
// of the blocks the next substep deposits into.  No host sync.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mpm_math.cuh"

namespace ckmpm {

constexpr int kMaxParticlesPerBlock = 4096;  // u16 in-block index, 64 per cell x 64 cells as in the reference
// P2G tile rows: the 8x8 (y, z) nodes of one x plane take 64 words plus 4 of
// padding, so a node's bank is (4 x + 8 y + z) mod 32 and lanes whose nodes
// differ only in x no longer share a bank: the expected worst bank load of a
// warp's atomics on particles at random positions in a block drops from 4.7
// to 3.5 words (3.5 is the balls-into-bins figure for 32 random banks), and
// the fused substep measured 3.5 % faster on the sand column.
constexpr int kTileRow = 68;
constexpr int kTileNodes = 2 * 8 * kTileRow;  // 2 grids x 8 x planes around a particle block
constexpr int kCompactThreads = 256;
constexpr int kCompactPerThread = 4;
constexpr int kCompactTile = kCompactThreads * kCompactPerThread;
constexpr float kFixScale = 68719476736.0f;        // 2^36: P2G fixed-point scale (per unit particle mass)
constexpr float kFixInvScale = 1.4551915228366852e-11f;  // 2^-36
constexpr float kFixMaxValue = 131072.0f;          // |contribution| bound per unit mass (2^17)

enum StatusBits : uint32_t {
  kStatusCapacity = 1u,
  kStatusNumeric = 2u,
  kStatusTimeout = 4u,  // no device code waits any more; kept so status words keep their meaning
  kStatusConsistency = 8u,
  kStatusOutsideBlock = 32u,
};

struct SceneDev {
  float dx, inv_dx;
  int32_t dims[3];       // blocks per axis of one domain
  float gravity, mass_clamp;
  int32_t boundary;
  float floor_cells;
  uint32_t cbase[9];     // colour-major traversal: first index of each colour class (all stacked domains)
  int32_t cdims[8][3];   // sub-lattice extent of each colour class in one domain
  uint32_t ccount[8];    // blocks of each colour class in one domain
  uint32_t nstack;       // stacked domains (1 for a single scene, the scene count for a batch)
  uint32_t nblocks_domain;  // table entries over all stacked domains
  float grid_unit;       // single scene: mass of one fixed-point unit (heaviest model's mass x 2^-36)
  int32_t rigid;         // rigid particles on (the velocity is Scalars::rigid_v)
  const uint8_t* brule;  // boundary == 2: per-cell rule (ckmpm_cell_rule), x-major over the domain's cells
  const float* bparam;   // boundary == 2: per-cell normal or velocity, 3 floats per cell
};

// Per-scene material of a batch (one model per stacked domain).
struct SceneMat {
  int32_t kind;
  float p[kMaterialParams];
  float vol_over_mass;  // V_p / m_p
  float unit;           // m_p * 2^-36: mass of one fixed-point unit of the scene's grid
  float aux0;           // initial logJp (0; alpha0 for NACC) or J (J0)
};

constexpr int kMixed = 7;  // material kind read per work item from the scene's SceneMat

struct Scalars {
  int32_t step;        // substeps taken; epoch of the grid that the next substep reads
  float cur_dt;        // dt the next substep advects with
  float next_dt;       // dt the next substep deposits stress with
  uint32_t status;     // StatusBits
  uint32_t lost;       // particles that left the domain
  uint32_t window_skips;
  uint32_t timeouts;    // always 0: the substep has no bounded waits (kept for the counters ABI)
  uint32_t maxv2_bits; // max |v|^2 on the grid (float bits), adaptive dt
  double time;         // simulated time: sum of the dt each substep advanced with
  double frame_end;    // adaptive dt: end of the current frame
  double cur_dt_d;     // cur_dt / next_dt in double, as the reference keeps its clock
  double next_dt_d;
  float rigid_v[3];    // velocity of rigid particles (when SceneDev::rigid)
};

struct BlockListDev {
  int4* keys;           // block coordinate and colour
  uint32_t* start;      // first particle of the block in the state arrays
  uint32_t* count;      // particles in the block
  int32_t* table;       // dense: block -> slot, -1 when inactive
  uint32_t* prefix28;   // per slot: prefix counts of outgoing directions (written by the fused kernel)
  uint16_t* idx;        // per particle: in-block position, grouped by outgoing direction
  uint32_t* nblocks;    // device scalar: active particle blocks
  uint32_t* nparticles; // device scalar: particles in the list
};

struct StateDev {
  float* x[3];
  float* F[9];
  float* aux;    // logJp (Drucker-Prager, NACC) or J (fluid)
  float* Q[9];   // the linear model's stored stress
  uint32_t* id;
};

// Which per-particle arrays a material keeps.
__host__ __device__ __forceinline__ bool material_has_F(int kind) { return kind != kFluid; }
// aux: logJp (Drucker-Prager, NACC), J (fluid) or the rigid flag (von Mises:
// 1 deformable, 0 rigid; include/mpm_algorithm.cuh:1063-1069).
__host__ __device__ __forceinline__ bool material_has_aux(int kind) {
  return kind == kDruckerPrager || kind == kFluid || kind == kNacc || kind == kVonMises;
}

// With rigid particles on, the reference's G2P2G treats a particle as rigid
// when its bucket attribute 3 is exactly zero (include/mpm_algorithm.cuh:1540-1543,
// 1611): that attribute is F00 for fixed-corotated, Drucker-Prager and linear,
// J for the fluid, logJp for NACC and the rigid flag for von Mises.
__host__ __device__ __forceinline__ float rigid_attribute(int kind, const float* F, float aux) {
  return (kind == kFluid || kind == kVonMises || kind == kNacc) ? aux : F[0];
}

struct ModelDev {
  StateDev st[2];
  BlockListDev bl[2];
  uint32_t* dense_total;  // per domain block: particles binned into it (zero between uses)
  uint32_t* tile_sums;    // compaction partials
  uint32_t* ticket;       // work counter of the fused kernel
  float* vel_in;          // setup: sorted initial velocities
  uint32_t cap_slots;
  uint32_t cap_particles;
  uint32_t max_per_block;
  int32_t track_ids;
  MaterialParams mat;
  float mass, vol;
  double flush_ratio;       // single scene: this model's particle mass / the grid unit's mass (1 for one model)
  const SceneMat* smat;     // batch: per stacked domain; null for a single scene
  const uint32_t* sstart;   // batch setup: first input particle of each scene (nstack + 1)
};

struct GridDev {
  long long* grid[2];
  int32_t* stamp[2];
};

// Colour classes of the traversal over `nstack` stacked domains of sc.dims
// blocks: class c holds the blocks whose coordinate parities are the bits of c.
inline void init_colour_classes(SceneDev& sc, uint32_t nstack) {
  sc.nstack = nstack;
  sc.nblocks_domain = nstack * static_cast<uint32_t>(sc.dims[0]) * sc.dims[1] * sc.dims[2];
  uint32_t base = 0;
  for (int c = 0; c < 8; ++c) {
    const int par[3] = {(c >> 2) & 1, (c >> 1) & 1, c & 1};
    for (int a = 0; a < 3; ++a) sc.cdims[c][a] = (sc.dims[a] - par[a] + 1) / 2;
    sc.ccount[c] = static_cast<uint32_t>(sc.cdims[c][0]) * sc.cdims[c][1] * sc.cdims[c][2];
    sc.cbase[c] = base;
    base += nstack * sc.ccount[c];
  }
  sc.cbase[8] = base;
}

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ bool in_domain(const SceneDev& sc, int x, int y, int z) {
  return (unsigned)x < (unsigned)sc.dims[0] && (unsigned)y < (unsigned)sc.dims[1] && (unsigned)z < (unsigned)sc.dims[2];
}

__device__ __forceinline__ int64_t flat_block(const SceneDev& sc, int w, int x, int y, int z) {
  return ((static_cast<int64_t>(w) * sc.dims[0] + x) * sc.dims[1] + y) * sc.dims[2] + z;
}

// Scene of input particle i from the batch's scene offsets (binary search).
__device__ __forceinline__ int scene_of(const uint32_t* sstart, uint32_t nstack, uint32_t i) {
  int lo = 0, hi = static_cast<int>(nstack);
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (sstart[mid] <= i)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int colour_of(int x, int y, int z) { return ((x & 1) << 2) | ((y & 1) << 1) | (z & 1); }

__device__ __forceinline__ int trunc_div4(int a) { return a / 4; }  // truncation toward zero, as the reference

__device__ __forceinline__ void set_status(Scalars* s, uint32_t bits) { atomicOr(&s->status, bits); }

// Grid update of one node (include/mpm_algorithm.cuh:739-869): v = mv / m,
// gravity on y, boundary rule; zero when m <= mass clamp.  The block holds
// fixed-point sums; unit is the mass of one unit.
__device__ __forceinline__ float4 node_velocity(const SceneDev& sc, const long long* blk, float unit, int cell, int bx,
                                                int by, int bz, int cell_y, float dt) {
  float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
  const float m = __ll2float_rn(__ldcg(blk + cell)) * unit;
  if (m > sc.mass_clamp) {
    const float inv = __frcp_rn(m);  // IEEE-rounded 1/m, as the reference's invMass (the build approximates 1/x)
    v.x = __ll2float_rn(__ldcg(blk + 128 + cell)) * unit * inv;
    v.y = __ll2float_rn(__ldcg(blk + 256 + cell)) * unit * inv;
    v.z = __ll2float_rn(__ldcg(blk + 384 + cell)) * unit * inv;
    v.y += sc.gravity * dt;
    if (sc.boundary == 0) {
      const bool out = (bx < 2 || bx + 2 >= sc.dims[0]) || (by < 2 || by + 2 >= sc.dims[1]) ||
                       (bz < 2 || bz + 2 >= sc.dims[2]);
      if (out) v = make_float4(0.f, 0.f, 0.f, 0.f);
    } else if (sc.boundary == 2) {
      // Per-cell rule (the scene's irregular-boundary hook evaluated into data).
      const int cx = bx * 4 + ((cell >> 4) & 3), cy = by * 4 + ((cell >> 2) & 3), cz = bz * 4 + (cell & 3);
      const int64_t c = (static_cast<int64_t>(cx) * (sc.dims[1] * 4) + cy) * (sc.dims[2] * 4) + cz;
      const int rule = sc.brule[c];
      if (rule == 1) {
        v = make_float4(0.f, 0.f, 0.f, 0.f);
      } else if (rule >= 2 && rule <= 4) {
        const float3 p = make_float3(__ldg(sc.bparam + 3 * c), __ldg(sc.bparam + 3 * c + 1), __ldg(sc.bparam + 3 * c + 2));
        if (rule == 3) {
          v = make_float4(p.x, p.y, p.z, 0.f);
        } else {
          const float d = p.x * v.x + p.y * v.y + p.z * v.z;
          if (rule == 2 || d < 0.f) {
            v.x -= d * p.x;
            v.y -= d * p.y;
            v.z -= d * p.z;
          }
        }
      }
    } else {
      const bool out = (bx < 2 || bx + 2 >= sc.dims[0]) || (bz < 2 || bz + 2 >= sc.dims[2]) || (by + 2 >= sc.dims[1]);
      if (out) {
        v = make_float4(0.f, 0.f, 0.f, 0.f);
      } else if (static_cast<float>(cell_y) < sc.floor_cells) {
        v.y = fmaxf(v.y, 0.f);
      }
    }
  }
  return v;
}

// Velocity tile around particle block `key`.  A particle of the block has its
// grid -dx/4 base cell at local 2..5 and its grid +dx/4 base cell at local
// 1..5 (block of a particle = (cell - 2) / 4), so G2P reaches only local nodes
// 2..6 of grid 0 (5^3) and 1..6 of grid 1 (6^3): 341 nodes, stored as
// g0: (lx-2)*25 + (ly-2)*5 + (lz-2) and g1: 125 + (lx-1)*36 + (ly-1)*6 + (lz-1).
constexpr int kVelNodes = 125 + 216;

__device__ __forceinline__ int vtile_index(int g, int lx, int ly, int lz) {
  return g == 0 ? (lx - 2) * 25 + (ly - 2) * 5 + (lz - 2) : 125 + (lx - 1) * 36 + (ly - 1) * 6 + (lz - 1);
}

// s_blk[e] (e = 0..7 over the 2x2x2 window) holds the flat index of each
// window block when it carries this epoch's grid, else -1; filled by
// window_blocks() before the tile load.
__device__ __forceinline__ void window_blocks(const SceneDev& sc, const int32_t* __restrict__ stin, int32_t read_epoch,
                                              int4 key, int64_t* s_blk, int e) {
  const int bx = key.x + (e >> 2), by = key.y + ((e >> 1) & 1), bz = key.z + (e & 1);
  int64_t fb = -1;
  if (in_domain(sc, bx, by, bz)) {
    const int64_t f = flat_block(sc, key.w, bx, by, bz);
    if (stin[f] == read_epoch) fb = f;
  }
  s_blk[e] = fb;
}

// Loads the velocity tile, applying the grid update on the fly.
template <int NT>
__device__ __forceinline__ void load_velocity_tile(const SceneDev& sc, const long long* __restrict__ gin,
                                                   const int64_t* s_blk, int4 key, float unit, float dt,
                                                   float4* vtile) {
  for (int i = threadIdx.x; i < kVelNodes; i += NT) {
    int g, lx, ly, lz;
    if (i < 125) {
      g = 0;
      lx = 2 + i / 25;
      ly = 2 + (i / 5) % 5;
      lz = 2 + i % 5;
    } else {
      const int j = i - 125;
      g = 1;
      lx = 1 + j / 36;
      ly = 1 + (j / 6) % 6;
      lz = 1 + j % 6;
    }
    const int e = ((lx >> 2) << 2) | ((ly >> 2) << 1) | (lz >> 2);
    const int64_t fb = s_blk[e];
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (fb >= 0) {
      const int cell = g * 64 + (lx & 3) * 16 + (ly & 3) * 4 + (lz & 3);
      v = node_velocity(sc, gin + fb * 512, unit, cell, key.x + (lx >> 2), key.y + (ly >> 2), key.z + (lz >> 2),
                        (key.y + (ly >> 2)) * 4 + (ly & 3), dt);
    }
    vtile[i] = v;
  }
}

// Per-axis stencil of one grid at scaled position xs (= x / dx): base cell,
// offset o in [0,1) and weight w0 (include/mpm_algorithm.cuh:60-67,
// include/mpm_kernel.cuh:91-114).  g = -1 or +1.
struct AxisStencil {
  int base;
  float o, w0;
};

template <int G>
__device__ __forceinline__ AxisStencil axis_stencil(float xs) {
  AxisStencil s;
  s.base = static_cast<int>(xs - 0.25f * G);
  const float local = xs - static_cast<float>(s.base);
  s.o = local - 0.25f * G;
  s.w0 = ck_w0(s.o);
  return s;
}


// First and second weighted moments of one grid along one axis (world units):
// m1 = sum_d w_d (d - o) dx, m2 = sum_d w_d (d - o)^2 dx^2.  With a tensor
// product kernel whose 1-D weights sum to one, D = sum_nodes w r r^T has
// D_aa = m2_a and D_ab = m1_a m1_b for each grid.
__device__ __forceinline__ void axis_moments(const AxisStencil& s, float dx, float& m1, float& m2) {
  const float w1 = 1.0f - s.w0;
  m1 = (w1 - s.o) * dx;
  const float a = s.o, b = 1.0f - s.o;
  m2 = (s.w0 * a * a + w1 * b * b) * dx * dx;
}

// D (symmetric, 6 entries: 00, 11, 22, 01, 02, 12) summed over both grids.
__device__ __forceinline__ void d_matrix(const AxisStencil (&st)[2][3], float dx, float* D6) {
  float m1[2][3], m2[2][3];
#pragma unroll
  for (int g = 0; g < 2; ++g)
#pragma unroll
    for (int a = 0; a < 3; ++a) axis_moments(st[g][a], dx, m1[g][a], m2[g][a]);
  D6[0] = m2[0][0] + m2[1][0];
  D6[1] = m2[0][1] + m2[1][1];
  D6[2] = m2[0][2] + m2[1][2];
  D6[3] = m1[0][0] * m1[0][1] + m1[1][0] * m1[1][1];
  D6[4] = m1[0][0] * m1[0][2] + m1[1][0] * m1[1][2];
  D6[5] = m1[0][1] * m1[0][2] + m1[1][1] * m1[1][2];
}

__device__ __forceinline__ void sym_to_full(const float* s6, float* f) {
  f[0] = s6[0];
  f[4] = s6[1];
  f[8] = s6[2];
  f[1] = f[3] = s6[3];
  f[2] = f[6] = s6[4];
  f[5] = f[7] = s6[5];
}

// G2P on both grids (include/mpm_algorithm.cuh:1555-1638): returns the
// halved interpolated velocity and C = B D^-1, where B = sum v_i (w r_i)^T
// and D = sum w r_i r_i^T with r_i = x_i - x_p, both over the 16 nodes, and
// D itself (6 entries) in D6.
// B is accumulated through the separable sums S = sum w v and
// T_a = sum over nodes with d_a = 1 of w v:  B[r][a] = dx (T_a[r] - o_a S[r]).
__device__ __forceinline__ void g2p(const float4* __restrict__ vtile, const float (&xs)[3], int4 key, float dx,
                                    float* v, float* C, bool& inside, float* D6) {
  AxisStencil st[2][3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    st[0][a] = axis_stencil<-1>(xs[a]);
    st[1][a] = axis_stencil<1>(xs[a]);
  }
  float B[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) B[k] = 0.f;
  float vs[3] = {0.f, 0.f, 0.f};
  const int kb[3] = {key.x * 4, key.y * 4, key.z * 4};
#pragma unroll
  for (int g = 0; g < 2; ++g) {
    int l[3];
    const int lo = g == 0 ? 2 : 1;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      l[a] = st[g][a].base - kb[a];
      if (l[a] < lo || l[a] > 5) {
        inside = false;
        l[a] = min(max(l[a], lo), 5);
      }
    }
    const float wx[2] = {st[g][0].w0, 1.f - st[g][0].w0};
    const float wy[2] = {st[g][1].w0, 1.f - st[g][1].w0};
    const float wz[2] = {st[g][2].w0, 1.f - st[g][2].w0};
    float S[3] = {0.f, 0.f, 0.f}, T[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r) T[r][0] = T[r][1] = T[r][2] = 0.f;
    const int sx = g == 0 ? 25 : 36, sy = g == 0 ? 5 : 6;
    const float4* base = vtile + vtile_index(g, l[0], l[1], l[2]);
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      const int dxn = (n >> 2) & 1, dyn = (n >> 1) & 1, dzn = n & 1;
      const float w = wx[dxn] * wy[dyn] * wz[dzn];
      const float4 vi = base[dxn * sx + dyn * sy + dzn];
      const float wv[3] = {w * vi.x, w * vi.y, w * vi.z};
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        S[r] += wv[r];
        if (dxn) T[r][0] += wv[r];
        if (dyn) T[r][1] += wv[r];
        if (dzn) T[r][2] += wv[r];
      }
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      vs[r] += S[r];
#pragma unroll
      for (int a = 0; a < 3; ++a) B[r * 3 + a] += dx * (T[r][a] - st[g][a].o * S[r]);
    }
  }
  float Di6[6], Di[9];
  d_matrix(st, dx, D6);
  inv_sym3(D6[0], D6[1], D6[2], D6[3], D6[4], D6[5], Di6);
  sym_to_full(Di6, Di);
  matmul3(B, Di, C);
#pragma unroll
  for (int r = 0; r < 3; ++r) v[r] = 0.5f * vs[r];
}

// The P2G tile holds 4 channels x kTileNodes nodes of exact 64-bit sums as two
// planes of 32-bit words: the low words first, the high words kTilePlane
// words later.  With the halves in separate planes, the low-word atomics of a
// warp spread over all 32 banks (interleaved 64-bit words would put every low
// word in an even bank); measured 5 % faster on the sand column and 9 % on
// small batched scenes.
constexpr int kTilePlane = kTileNodes * 4;

// Exact 64-bit integer add into the tile with two native 32-bit shared
// atomics: the low word's returned old value gives the carry into the high
// word.  Integer addition is associative, so the final 64-bit value is the
// exact sum whatever order the adds arrive in (64-bit shared atomics are not
// native on this part and measured 1.7x slower as a whole kernel).
// The carry comes from an add with carry-out of the returned old word and the
// addend (two instructions; the compare-and-select form took three and the
// fused kernel ran 2.5 % slower on the sand column).
__device__ __forceinline__ void fixed_add(unsigned* lo_word, long long v) {
  const unsigned lo = static_cast<unsigned>(v);
  const unsigned old = atomicAdd(lo_word, lo);
  unsigned hi;
  asm("{\n\t.reg .u32 t;\n\tadd.cc.u32 t, %1, %2;\n\taddc.u32 %0, %3, 0;\n\t}"
      : "=r"(hi)
      : "r"(old), "r"(lo), "r"(static_cast<unsigned>(v >> 32)));
  atomicAdd(lo_word + kTilePlane, hi);
}

// The 64-bit sum of tile word i (node index + channel * kTileNodes).
__device__ __forceinline__ unsigned long long tile_sum(const unsigned* tile, int i) {
  return static_cast<unsigned long long>(tile[i]) | (static_cast<unsigned long long>(tile[i + kTilePlane]) << 32);
}

// Scatter one particle's mass and momentum into the fixed-point tile.  The
// tile is channel-major, [m, mvx, mvy, mvz][grid][8 x planes of kTileRow words]
// in each plane, so lanes of a warp that update different nodes of one channel
// fall in different banks (measured 17 % faster than node-major for the whole
// kernel).
// Per unit particle mass: node mass w, node momentum w (v + Ah (d - o)) with
// Ah = A dx / m (A the reference's affine contribution).  Integer atomics make
// the tile sum independent of the order in which particles arrive.
__device__ __forceinline__ void p2g_scatter(unsigned* __restrict__ ptile, const AxisStencil (&st)[2][3],
                                            const int (&lbase)[2][3], const float* v, const float* Ah) {
#pragma unroll
  for (int g = 0; g < 2; ++g) {
    float Q[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
      Q[r] = v[r] - (Ah[r * 3] * st[g][0].o + Ah[r * 3 + 1] * st[g][1].o + Ah[r * 3 + 2] * st[g][2].o);
    const float wx[2] = {st[g][0].w0 * kFixScale, (1.f - st[g][0].w0) * kFixScale};
    const float wy[2] = {st[g][1].w0, 1.f - st[g][1].w0};
    const float wz[2] = {st[g][2].w0, 1.f - st[g][2].w0};
    unsigned* base = ptile + ((g * 8 + lbase[g][0]) * kTileRow + lbase[g][1] * 8 + lbase[g][2]);
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      const int dxn = (n >> 2) & 1, dyn = (n >> 1) & 1, dzn = n & 1;
      const float w = wx[dxn] * wy[dyn] * wz[dzn];
      float val[3];
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        val[r] = Q[r];
        if (dxn) val[r] += Ah[r * 3];
        if (dyn) val[r] += Ah[r * 3 + 1];
        if (dzn) val[r] += Ah[r * 3 + 2];
      }
      unsigned* node = base + (dxn * kTileRow + dyn * 8 + dzn);
      const long long fx[4] = {__float2ll_rn(w), __float2ll_rn(w * val[0]), __float2ll_rn(w * val[1]),
                               __float2ll_rn(w * val[2])};
#pragma unroll
      for (int c = 0; c < 4; ++c) fixed_add(node + c * kTileNodes, fx[c]);
    }
  }
}

// Epilogue shared by the substep and the initial rasterisation: add this
// block's tile into the 2x2x2 grid blocks it covers with 64-bit integer
// reductions, one node (4 channels) per thread, skipping nodes nothing touched,
// and leave the tile zero for the CTA's next block (each node's words are
// cleared as they are read; the padding words are never written, and the
// kernels zero the whole tile once before their first block).
// Integer addition is associative, so the grid sums are bitwise deterministic
// whatever order the up to 8 covering particle blocks flush in, and no block
// waits for another (the reference adds floats with atomicAdd,
// include/mpm_algorithm.cuh:1799-1844).  The target blocks were zeroed and
// stamped before the launch; ratio rescales a model's per-unit-mass sums to
// the grid's unit (1 when the scene has one particle mass).
template <int NT>
__device__ __forceinline__ void flush_tile(const SceneDev& sc, int4 key, unsigned* __restrict__ ptile,
                                           double ratio, long long* __restrict__ gout) {
  int64_t fb[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const int x = key.x + (e >> 2), y = key.y + ((e >> 1) & 1), z = key.z + (e & 1);
    fb[e] = in_domain(sc, x, y, z) ? flat_block(sc, key.w, x, y, z) : -1;
  }
  for (int i = threadIdx.x; i < 8 * 128; i += NT) {
    const int e = i >> 7;
    int64_t f = fb[0];
#pragma unroll
    for (int k = 1; k < 8; ++k)
      if (e == k) f = fb[k];
    const int w = i & 127;
    const int gi = w >> 6, cell = w & 63;
    const int lx = (e >> 2) * 4 + (cell >> 4), ly = ((e >> 1) & 1) * 4 + ((cell >> 2) & 3), lz = (e & 1) * 4 + (cell & 3);
    const int node = (gi * 8 + lx) * kTileRow + ly * 8 + lz;
    unsigned long long v[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) v[c] = tile_sum(ptile, node + c * kTileNodes);
    if ((v[0] | v[1] | v[2] | v[3]) == 0ull) continue;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      ptile[node + c * kTileNodes] = 0u;
      ptile[node + c * kTileNodes + kTilePlane] = 0u;
    }
    if (f < 0) continue;
    if (ratio != 1.0) {
#pragma unroll
      for (int c = 0; c < 4; ++c)
        v[c] = static_cast<unsigned long long>(__double2ll_rn(__ll2double_rn(static_cast<long long>(v[c])) * ratio));
    }
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(gout + f * 512 + gi * 64 + cell);
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (v[c]) atomicAdd(dst + c * 128, v[c]);
  }
}

// Zero the grid blocks that the next substep deposits into -- the 2x2x2
// window of every block of `list` -- and stamp them with `epoch`, each block
// once (the first warp to swap its stamp zeroes it).  One warp per (block,
// window corner).  Runs after every kernel that reads the buffer.
__global__ void zero_windows_kernel(SceneDev sc, BlockListDev list, long long* __restrict__ g, int32_t* stamp,
                                    const Scalars* __restrict__ scal, int32_t epoch_offset) {
  const uint32_t nb = *list.nblocks;
  const int32_t epoch = scal->step + epoch_offset;
  const int lane = threadIdx.x & 31;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nb * 8u; t += nwarps) {
    const int4 key = list.keys[t >> 3];
    const int e = static_cast<int>(t & 7u);
    const int x = key.x + (e >> 2), y = key.y + ((e >> 1) & 1), z = key.z + (e & 1);
    if (!in_domain(sc, x, y, z)) continue;
    const int64_t f = flat_block(sc, key.w, x, y, z);
    int won = 0;
    if (lane == 0) won = atomicExch(stamp + f, epoch) != epoch ? 1 : 0;
    won = __shfl_sync(0xffffffffu, won, 0);
    if (!won) continue;
    longlong2* p = reinterpret_cast<longlong2*>(g + f * 512);
    for (int i = lane; i < 256; i += 32) p[i] = make_longlong2(0, 0);
  }
}

// Incoming particle groups of block `key` (run by warp 0): for each of the
// 27 directions d (source = key + dir(d)), the source block's group of
// particles that moved here.  s_off: exclusive prefix over directions (28),
// s_idx: where the group's in-block indices start in prev.idx, s_src: the
// source block's first particle in the state arrays.
__device__ __forceinline__ void incoming_groups(const SceneDev& sc, const BlockListDev& prev, int4 key, uint32_t* s_off,
                                                uint32_t* s_idx, uint32_t* s_src) {
  const int lane = threadIdx.x & 31;
  uint32_t c = 0, ib = 0, ss = 0;
  if (lane < 27) {
    const int x = key.x + lane / 9 - 1, y = key.y + (lane / 3) % 3 - 1, z = key.z + lane % 3 - 1;
    if (in_domain(sc, x, y, z)) {
      const int32_t s = prev.table[flat_block(sc, key.w, x, y, z)];
      if (s >= 0) {
        const uint32_t a = prev.prefix28[s * 28 + lane], b = prev.prefix28[s * 28 + lane + 1];
        c = b - a;
        ss = prev.start[s];
        ib = ss + a;
      }
    }
  }
  uint32_t incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane < 27) {
    s_off[lane] = incl - c;
    s_idx[lane] = ib;
    s_src[lane] = ss;
  }
  if (lane == 26) s_off[27] = incl;
}

__device__ __forceinline__ int find_group(const uint32_t* s_off, uint32_t q) {
  int lo = 0, hi = 27;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (s_off[mid] <= q)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// Output slot of the q-th particle of a block that starts at `start`.
__device__ __forceinline__ uint32_t o_slot(uint32_t start, uint32_t q) { return start + q; }

struct SharedSmall {
  int64_t blk[8];
  uint32_t item;
  uint32_t off[28];
  uint32_t idx[27];
  uint32_t src[27];
};

constexpr size_t kSmemVTile = sizeof(float4) * 344;                      // 5.5 KB (341 nodes)
constexpr size_t kSmemPTile = sizeof(unsigned) * 2 * kTilePlane;            // 34 KB, two planes
constexpr size_t kSmemCodes = kMaxParticlesPerBlock;                     // 4 KB
constexpr size_t kSmemFused = kSmemVTile + kSmemPTile + kSmemCodes;

// ------------------------------------------------------------------ fused substep
//
// One CTA per particle block at a time (persistent, blocks dequeued in
// colour-major order).  Replaces the reference's G2P2G
// (include/mpm_algorithm.cuh:1367-1845) together with the grid update
// (:739-869), the advection record (mpm_particle.cuh:333-371) and the
// per-block list build (:629-649, :1868-1918).  KIND is the material, or
// kMixed for a batch, where each work item reads its scene's material (one
// scene per stacked domain, so the kind is uniform across the CTA).  RIGID
// compiles the rigid-particle test in (scenes with rigid particles on; the
// test alone cost 1.7 % on the sand column).  Register
// budget: 64 per thread at 256 threads (4 CTAs per SM); at 128 threads the
// shared-memory footprint allows 5 CTAs per SM, so up to 102 registers; at
// 1024 threads one CTA fills the SM (for small scenes, where a few hundred
// blocks cannot fill 148 SMs and the fullest block sets the launch's length).
template <int NT>
constexpr int fused_min_ctas() { return NT == 128 ? 5 : 1024 / NT; }

// Per-warp direction counts of the rebin ranking.
template <int NT>
struct RankCounts {
  uint32_t wcnt[NT / 32][28];
};

template <int KIND, int NT, bool RIGID = false>
__global__ void __launch_bounds__(NT, fused_min_ctas<NT>())
    g2p2g_kernel(SceneDev sc, ModelDev md, GridDev gd, Scalars* __restrict__ scal) {
  static_assert(NT % 32 == 0 && NT / 32 <= 32 && NT >= 64, "block size");
  extern __shared__ __align__(16) unsigned char smem[];
  float4* vtile = reinterpret_cast<float4*>(smem);
  unsigned* ptile = reinterpret_cast<unsigned*>(smem + kSmemVTile);
  uint8_t* dcode = smem + kSmemVTile + kSmemPTile;
  __shared__ SharedSmall sh;
  __shared__ RankCounts<NT> rk;

  const int32_t step = scal->step;
  const int parity = step & 1;
  const int32_t read_epoch = step;
  const float dt = scal->cur_dt, ndt = scal->next_dt;
  const BlockListDev cur = md.bl[parity];
  const BlockListDev prev = md.bl[parity ^ 1];
  const StateDev sin = md.st[parity];
  const StateDev sout = md.st[parity ^ 1];
  const long long* __restrict__ gin = gd.grid[parity];
  long long* __restrict__ gout = gd.grid[parity ^ 1];
  const int32_t* __restrict__ stin = gd.stamp[parity];
  const uint32_t nb = *cur.nblocks;
  const float dx = sc.dx, inv_dx = sc.inv_dx;
  const uint32_t maxp = min(md.max_per_block, static_cast<uint32_t>(kMaxParticlesPerBlock));

  for (int i = threadIdx.x; i < 2 * kTilePlane / 4; i += NT)
    reinterpret_cast<uint4*>(ptile)[i] = make_uint4(0u, 0u, 0u, 0u);
  for (;;) {
    if (threadIdx.x == 0) sh.item = atomicAdd(md.ticket, 1u);
    __syncthreads();
    const uint32_t item = sh.item;
    if (item >= nb) break;
    const int4 key = cur.keys[item];
    const uint32_t start = cur.start[item];
    uint32_t n = cur.count[item];
    int kind = KIND;
    float mp0 = md.mat.p[0], mp1 = md.mat.p[1], mp2 = md.mat.p[2];
    // Rounded division: the same bits as the host's V / m that a batched
    // scene carries in its SceneMat (the build's fast division may differ by
    // an ulp), so both forms start from the same constants.
    float vol_over_mass = __fdiv_rn(md.vol, md.mass), unit = sc.grid_unit;
    double ratio = md.flush_ratio;
    if (KIND == kMixed) {
      const SceneMat& sm = md.smat[key.w];
      kind = sm.kind;
      mp0 = sm.p[0];
      mp1 = sm.p[1];
      mp2 = sm.p[2];
      vol_over_mass = sm.vol_over_mass;
      unit = sm.unit;
      ratio = 1.0;
    }

    if (threadIdx.x < 32)
      incoming_groups(sc, prev, key, sh.off, sh.idx, sh.src);
    else if (threadIdx.x < 40)
      window_blocks(sc, stin, read_epoch, key, sh.blk, threadIdx.x - 32);
    for (int i = threadIdx.x; i < static_cast<int>(sizeof(rk.wcnt) / sizeof(uint32_t)); i += NT)
      (&rk.wcnt[0][0])[i] = 0u;
    __syncthreads();
    load_velocity_tile<NT>(sc, gin, sh.blk, key, unit, dt, vtile);
    __syncthreads();
    // The block's output slots [start, start + n) must lie in the state arrays;
    // counts that say otherwise are flagged and clamped, never written past.
    const uint32_t room = start < md.cap_particles ? md.cap_particles - start : 0u;
    if (threadIdx.x == 0) {
      uint32_t flags = 0;
      if (sh.off[27] != n || n > room) flags |= kStatusConsistency;
      if (n > maxp) flags |= kStatusCapacity;
      if (flags) set_status(scal, flags);
    }
    n = min(min(min(n, sh.off[27]), maxp), room);

    for (uint32_t q = threadIdx.x; q < n; q += NT) {
      const int d = find_group(sh.off, q);
      const uint32_t ii = sh.idx[d] + (q - sh.off[d]);
      uint32_t iin = ii < md.cap_particles ? sh.src[d] + prev.idx[ii] : 0xFFFFFFFFu;
      if (iin >= md.cap_particles) {  // corrupted rebin record: flag, never read out of range
        set_status(scal, kStatusConsistency);
        iin = 0;
      }
      float x[3] = {sin.x[0][iin], sin.x[1][iin], sin.x[2][iin]};
      float F[9];
      float aux = 0.f;
      if (material_has_F(kind)) {
#pragma unroll
        for (int k = 0; k < 9; ++k) F[k] = sin.F[k][iin];
      }
      if (material_has_aux(kind)) aux = sin.aux[iin];
      float xs[3] = {x[0] * inv_dx, x[1] * inv_dx, x[2] * inv_dx};
      bool inside = true;
      float v[3], C[9], Dold[6];
      g2p(vtile, xs, key, dx, v, C, inside, Dold);
      float adv[3] = {v[0], v[1], v[2]};
      if (RIGID && rigid_attribute(kind, F, aux) == 0.f) {
        // Rigid: moves with the scene's rigid velocity and carries no velocity,
        // no affine field and no G2P D (include/mpm_algorithm.cuh:1609-1618).
#pragma unroll
        for (int k = 0; k < 9; ++k) C[k] = 0.f;
#pragma unroll
        for (int k = 0; k < 6; ++k) Dold[k] = 0.f;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          v[a] = 0.f;
          adv[a] = scal->rigid_v[a];
        }
      }
#pragma unroll
      for (int a = 0; a < 3; ++a) x[a] += dt * adv[a];

      float tau[9];
      if (kind == kFluid) {
        stress_fluid(mp0, mp1, mp2, C, dt, aux, tau);
      } else {
        float dW[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) dW[k] = C[k] * dt + ((k & 3) ? 0.f : 1.f);
        matmul3(dW, F, F);
        if (kind == kFixedCorotated) {
          stress_fixed_corotated(mp0, mp1, F, tau);
        } else if (kind == kDruckerPrager) {
          stress_drucker_prager(mp0, mp1, F, aux, tau);
        } else if (kind == kVonMises) {
          stress_von_mises(mp0, mp1, mp2, F, tau);
        } else if (kind == kNacc) {
          float prm[kMaterialParams];
#pragma unroll
          for (int k = 0; k < kMaterialParams; ++k) prm[k] = KIND == kMixed ? md.smat[key.w].p[k] : md.mat.p[k];
          stress_nacc(prm, F, aux, tau);
        } else {  // kLinear
          float Q[9];
#pragma unroll
          for (int k = 0; k < 9; ++k) Q[k] = sin.Q[k][iin];
          stress_linear(C, dt, F, Q, tau);
#pragma unroll
          for (int k = 0; k < 9; ++k) sout.Q[k][o_slot(start, q)] = Q[k];
        }
      }

      const uint32_t o = o_slot(start, q);
      sout.x[0][o] = x[0];
      sout.x[1][o] = x[1];
      sout.x[2][o] = x[2];
      if (material_has_F(kind)) {
#pragma unroll
        for (int k = 0; k < 9; ++k) sout.F[k][o] = F[k];
      }
      if (material_has_aux(kind)) sout.aux[o] = aux;
      if (md.track_ids) sout.id[o] = sin.id[iin];

      // Rebin record: direction code of (old block - new block), 27 = lost.
#pragma unroll
      for (int a = 0; a < 3; ++a) xs[a] = x[a] * inv_dx;
      int cn[3], sh3[3];
      bool win = true, ok = true;
      const int kk[3] = {key.x, key.y, key.z};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        cn[a] = static_cast<int>(xs[a] + 0.25f);
        const int nbk = trunc_div4(cn[a] - 2);
        sh3[a] = kk[a] - nbk;
        ok &= (sh3[a] >= -1 && sh3[a] <= 1);
        const int lc = cn[a] - 4 * kk[a];
        win &= (lc > 0 && lc < 7);
      }
      ok &= in_domain(sc, kk[0] - sh3[0], kk[1] - sh3[1], kk[2] - sh3[2]);
      const int code = ok ? (sh3[0] + 1) * 9 + (sh3[1] + 1) * 3 + (sh3[2] + 1) : 27;
      dcode[q] = static_cast<uint8_t>(code);
      if (!inside) set_status(scal, kStatusOutsideBlock);
      if (!win) {
        atomicAdd(&scal->window_skips, 1u);
        continue;
      }

      // P2G at the new position (include/mpm_algorithm.cuh:1687-1792):
      // A = C m - ndt V M tau, scaled here per unit mass and by dx.  The
      // reference adds the new position's D onto the G2P D of the old position
      // (it never resets it, :1524,1604,1729) and inverts half the sum (:1732),
      // so M = (0.5 (D_old + D_new))^-1.
      AxisStencil st[2][3];
      int lb[2][3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        st[0][a] = axis_stencil<-1>(xs[a]);
        st[1][a] = axis_stencil<1>(xs[a]);
        lb[0][a] = st[0][a].base - 4 * kk[a];
        lb[1][a] = st[1][a].base - 4 * kk[a];
      }
      float D6[6], Di6[6], Di[9], DT[9];
      d_matrix(st, dx, D6);
#pragma unroll
      for (int k = 0; k < 6; ++k) D6[k] = 0.5f * (Dold[k] + D6[k]);
      inv_sym3(D6[0], D6[1], D6[2], D6[3], D6[4], D6[5], Di6);
      sym_to_full(Di6, Di);
      matmul3(Di, tau, DT);
      float Ah[9];
      bool finite = true;
      const float sA = ndt * vol_over_mass;
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        Ah[k] = (C[k] - sA * DT[k]) * dx;
        finite &= fabsf(Ah[k]) < kFixMaxValue;
      }
#pragma unroll
      for (int r = 0; r < 3; ++r) finite &= fabsf(v[r]) < kFixMaxValue;
      if (!finite) {
        set_status(scal, kStatusNumeric);
        continue;
      }
      p2g_scatter(ptile, st, lb, v, Ah);
    }
    __syncthreads();

    // Rebin epilogue: stable ranks of the particles within their outgoing
    // direction groups, in two passes over warp-contiguous ranges (per-warp
    // group counts, then prefix over warps and directions, then ranks), the
    // index list, this block's 28 group prefixes and the next step's per-block
    // totals.
    {
      constexpr int kWarps = NT / 32;
      const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
      const uint32_t span = ((n + kWarps * 32 - 1) / (kWarps * 32)) * 32;
      const uint32_t q0 = wid * span, q1 = min(q0 + span, n);
      const uint32_t lt = (1u << lane) - 1u;
      for (uint32_t b = q0; b < q1; b += 32) {
        const uint32_t q = b + lane;
        const int code = q < q1 ? dcode[q] : 255;
        const uint32_t mask = __match_any_sync(0xffffffffu, code);
        if (code < 28 && lane == 31 - __clz(mask)) rk.wcnt[wid][code] += __popc(mask);
        __syncwarp();
      }
      __syncthreads();
      if (threadIdx.x < 32) {
        uint32_t c = 0;
        if (lane < 28) {
#pragma unroll
          for (int w = 0; w < kWarps; ++w) {
            const uint32_t t = rk.wcnt[w][lane];
            rk.wcnt[w][lane] = c;
            c += t;
          }
        }
        const uint32_t cv = lane < 27 ? c : 0u;
        uint32_t incl = cv;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += t;
        }
        if (lane < 27) {
          const uint32_t pre = incl - cv;
#pragma unroll
          for (int w = 0; w < kWarps; ++w) rk.wcnt[w][lane] += pre;
          cur.prefix28[item * 28 + lane] = pre;
          if (c > 0) {
            const int x = key.x - (lane / 9 - 1), y = key.y - ((lane / 3) % 3 - 1), z = key.z - (lane % 3 - 1);
            atomicAdd(md.dense_total + flat_block(sc, key.w, x, y, z), c);
          }
        }
        if (lane == 26) cur.prefix28[item * 28 + 27] = incl;
        if (lane == 27 && c > 0) atomicAdd(&scal->lost, c);
      }
      __syncthreads();
      for (uint32_t b = q0; b < q1; b += 32) {
        const uint32_t q = b + lane;
        const int code = q < q1 ? dcode[q] : 255;
        const uint32_t mask = __match_any_sync(0xffffffffu, code);
        if (code < 27) {
          const uint32_t r = rk.wcnt[wid][code] + __popc(mask & lt);
          if (start + r < md.cap_particles) cur.idx[start + r] = static_cast<uint16_t>(q);
        }
        __syncwarp();
        if (code < 27 && lane == 31 - __clz(mask)) rk.wcnt[wid][code] += __popc(mask);
        __syncwarp();
      }
    }
    flush_tile<NT>(sc, key, ptile, ratio, gout);
  }
}

// ------------------------------------------------------------------ initial rasterisation
// Mass and momentum of the sorted initial particles into grid[0] with epoch 0
// (include/mpm_algorithm.cuh:872-947, here with the same deterministic tile
// flush as the substep).
template <int NT>
__global__ void __launch_bounds__(NT, 2) rasterize_kernel(SceneDev sc, ModelDev md, GridDev gd, Scalars* scal) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned* ptile = reinterpret_cast<unsigned*>(smem + kSmemVTile);
  __shared__ SharedSmall sh;
  const BlockListDev cur = md.bl[0];
  const StateDev s0 = md.st[0];
  const uint32_t nb = *cur.nblocks;
  const float inv_dx = sc.inv_dx;
  const float Z[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = threadIdx.x; i < 2 * kTilePlane / 4; i += NT)
    reinterpret_cast<uint4*>(ptile)[i] = make_uint4(0u, 0u, 0u, 0u);
  for (;;) {
    if (threadIdx.x == 0) sh.item = atomicAdd(md.ticket, 1u);
    __syncthreads();
    const uint32_t item = sh.item;
    if (item >= nb) break;
    const int4 key = cur.keys[item];
    const uint32_t start = cur.start[item];
    const uint32_t n = cur.count[item];
    const int kk[3] = {key.x, key.y, key.z};
    for (uint32_t q = threadIdx.x; q < n; q += NT) {
      const uint32_t i = start + q;
      const float xs[3] = {s0.x[0][i] * inv_dx, s0.x[1][i] * inv_dx, s0.x[2][i] * inv_dx};
      const float v[3] = {md.vel_in[3 * i], md.vel_in[3 * i + 1], md.vel_in[3 * i + 2]};
      AxisStencil st[2][3];
      int lb[2][3];
      bool ok = true;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        st[0][a] = axis_stencil<-1>(xs[a]);
        st[1][a] = axis_stencil<1>(xs[a]);
        lb[0][a] = st[0][a].base - 4 * kk[a];
        lb[1][a] = st[1][a].base - 4 * kk[a];
        ok &= lb[0][a] >= 0 && lb[0][a] <= 6 && lb[1][a] >= 0 && lb[1][a] <= 6;
      }
      bool finite = fabsf(v[0]) < kFixMaxValue && fabsf(v[1]) < kFixMaxValue && fabsf(v[2]) < kFixMaxValue;
      if (!ok) set_status(scal, kStatusOutsideBlock);
      if (!finite) set_status(scal, kStatusNumeric);
      if (ok && finite) p2g_scatter(ptile, st, lb, v, Z);
    }
    __syncthreads();
    flush_tile<NT>(sc, key, ptile, md.smat ? 1.0 : md.flush_ratio, gd.grid[0]);
  }
}

// ------------------------------------------------------------------ compaction
// The next block list from the per-block totals: a scan over the domain in
// colour-major order (colour class, then lexicographic key), so slots come out
// grouped by colour and sorted by key within a colour.  Replaces
// MarkActiveParticleBlocks + ExclusiveScan + InverseExclusiveScan +
// UpdatePartition + UpdateBucket + ComputeBinCount
// (include/mpm_algorithm.cuh:26-45,573-582,1868-1918, include/mpm_engine.cuh:659-787).
// Traversal index -> block key (x, y, z, stacked domain).  Order: colour
// class, then stacked domain, then lexicographic within the class.
__device__ __forceinline__ int4 traversal_key(const SceneDev& sc, uint32_t t) {
  int c = 0;
#pragma unroll
  for (int k = 1; k < 8; ++k) c += (t >= sc.cbase[k]) ? 1 : 0;
  uint32_t loc = t - sc.cbase[c];
  const uint32_t w = loc / sc.ccount[c];
  loc -= w * sc.ccount[c];
  const uint32_t nz = sc.cdims[c][2], ny = sc.cdims[c][1];
  const int k = loc % nz;
  const int j = (loc / nz) % ny;
  const int i = loc / (nz * ny);
  return make_int4(2 * i + ((c >> 2) & 1), 2 * j + ((c >> 1) & 1), 2 * k + (c & 1), static_cast<int>(w));
}

__device__ __forceinline__ uint32_t block_reduce_sum(uint32_t v, uint32_t* scratch) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) scratch[w] = v;
  __syncthreads();
  uint32_t r = 0;
  if (threadIdx.x < 32) {
    r = threadIdx.x < (blockDim.x >> 5) ? scratch[threadIdx.x] : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    if (threadIdx.x == 0) scratch[0] = r;
  }
  __syncthreads();
  r = scratch[0];
  __syncthreads();
  return r;
}

// Exclusive block scan of two values (blockDim = kCompactThreads).
__device__ __forceinline__ void block_scan2(uint32_t a, uint32_t b, uint32_t& ea, uint32_t& eb, uint32_t* scratch) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t ia = a, ib = b;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t ta = __shfl_up_sync(0xffffffffu, ia, o);
    const uint32_t tb = __shfl_up_sync(0xffffffffu, ib, o);
    if (lane >= o) {
      ia += ta;
      ib += tb;
    }
  }
  __syncthreads();
  if (lane == 31) {
    scratch[w] = ia;
    scratch[32 + w] = ib;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int nw = blockDim.x >> 5;
    uint32_t xa = lane < nw ? scratch[lane] : 0u, xb = lane < nw ? scratch[32 + lane] : 0u;
    uint32_t ya = xa, yb = xb;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t ta = __shfl_up_sync(0xffffffffu, ya, o);
      const uint32_t tb = __shfl_up_sync(0xffffffffu, yb, o);
      if (lane >= o) {
        ya += ta;
        yb += tb;
      }
    }
    scratch[64 + lane] = ya - xa;
    scratch[96 + lane] = yb - xb;
  }
  __syncthreads();
  ea = scratch[64 + w] + ia - a;
  eb = scratch[96 + w] + ib - b;
  __syncthreads();
}

__global__ void __launch_bounds__(kCompactThreads) compact_reduce_kernel(SceneDev sc, const uint32_t* __restrict__ total,
                                                                          uint32_t* __restrict__ tile_sums) {
  __shared__ uint32_t scratch[128];
  const uint32_t t0 = blockIdx.x * kCompactTile + threadIdx.x * kCompactPerThread;
  uint32_t nblk = 0, npart = 0;
  for (int k = 0; k < kCompactPerThread; ++k) {
    const uint32_t t = t0 + k;
    if (t >= sc.nblocks_domain) break;
    const int4 key = traversal_key(sc, t);
    const uint32_t c = total[flat_block(sc, key.w, key.x, key.y, key.z)];
    nblk += c > 0 ? 1u : 0u;
    npart += c;
  }
  nblk = block_reduce_sum(nblk, scratch);
  npart = block_reduce_sum(npart, scratch);
  if (threadIdx.x == 0) {
    tile_sums[2 * blockIdx.x] = nblk;
    tile_sums[2 * blockIdx.x + 1] = npart;
  }
}

__global__ void __launch_bounds__(kCompactThreads)
    compact_scatter_kernel(SceneDev sc, uint32_t* __restrict__ total, const uint32_t* __restrict__ tile_sums,
                           BlockListDev out, uint32_t cap_slots, uint32_t* ticket, Scalars* scal) {
  __shared__ uint32_t scratch[128];
  uint32_t pb = 0, pp = 0;
  for (uint32_t t = threadIdx.x; t < blockIdx.x; t += blockDim.x) {
    pb += tile_sums[2 * t];
    pp += tile_sums[2 * t + 1];
  }
  pb = block_reduce_sum(pb, scratch);
  pp = block_reduce_sum(pp, scratch);
  const uint32_t t0 = blockIdx.x * kCompactTile + threadIdx.x * kCompactPerThread;
  uint32_t c[kCompactPerThread];
  int64_t fb[kCompactPerThread];
  int4 keys[kCompactPerThread];
  uint32_t nblk = 0, npart = 0;
#pragma unroll
  for (int k = 0; k < kCompactPerThread; ++k) {
    const uint32_t t = t0 + k;
    c[k] = 0;
    fb[k] = -1;
    if (t < sc.nblocks_domain) {
      keys[k] = traversal_key(sc, t);
      fb[k] = flat_block(sc, keys[k].w, keys[k].x, keys[k].y, keys[k].z);
      c[k] = total[fb[k]];
      nblk += c[k] > 0 ? 1u : 0u;
      npart += c[k];
    }
  }
  uint32_t eb, ep;
  block_scan2(nblk, npart, eb, ep, scratch);
  uint32_t slot = pb + eb, part = pp + ep;
  bool overflow = false;
#pragma unroll
  for (int k = 0; k < kCompactPerThread; ++k) {
    if (fb[k] < 0) continue;
    if (c[k] > 0) {
      if (slot < cap_slots) {
        out.keys[slot] = keys[k];
        out.start[slot] = part;
        out.count[slot] = c[k];
        out.table[fb[k]] = static_cast<int32_t>(slot);
      } else {
        out.table[fb[k]] = -1;
        overflow = true;
      }
      ++slot;
      part += c[k];
      total[fb[k]] = 0;
    } else {
      out.table[fb[k]] = -1;
    }
  }
  if (overflow) set_status(scal, kStatusCapacity);
  if (blockIdx.x == gridDim.x - 1) {
    const uint32_t tb = block_reduce_sum(nblk, scratch), tp = block_reduce_sum(npart, scratch);
    if (threadIdx.x == 0) {
      *out.nblocks = min(pb + tb, cap_slots);
      *out.nparticles = pp + tp;
      *ticket = 0;
    }
  }
}

// Exclusive prefix sum of n 32-bit values in three launches: per-tile sums,
// one CTA scanning the tile sums in place, then each tile scanned from its
// offset.  The export in input order uses it to place each live id.
constexpr int kScanThreads = kCompactThreads;
constexpr int kScanPerThread = 8;
constexpr uint32_t kScanTile = kScanThreads * kScanPerThread;

__host__ __device__ constexpr uint32_t scan_tiles(uint32_t n) { return (n + kScanTile - 1) / kScanTile; }

__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const uint32_t* __restrict__ in, uint32_t n,
                                                                    uint32_t* __restrict__ sums) {
  __shared__ uint32_t scratch[128];
  const uint32_t t0 = blockIdx.x * kScanTile + threadIdx.x * kScanPerThread;
  uint32_t v = 0;
#pragma unroll
  for (int k = 0; k < kScanPerThread; ++k)
    if (t0 + k < n) v += in[t0 + k];
  v = block_reduce_sum(v, scratch);
  if (threadIdx.x == 0) sums[blockIdx.x] = v;
}

__global__ void __launch_bounds__(kScanThreads) scan_sums_kernel(uint32_t* __restrict__ sums, uint32_t ntiles) {
  __shared__ uint32_t scratch[128];
  uint32_t carry = 0;
  for (uint32_t b = 0; b < ntiles; b += kScanThreads) {
    const uint32_t i = b + threadIdx.x;
    const uint32_t v = i < ntiles ? sums[i] : 0u;
    uint32_t e, unused;
    block_scan2(v, 0u, e, unused, scratch);
    const uint32_t total = block_reduce_sum(v, scratch);
    if (i < ntiles) sums[i] = carry + e;
    carry += total;
  }
}

__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const uint32_t* __restrict__ in, uint32_t n,
                                                                   const uint32_t* __restrict__ offsets,
                                                                   uint32_t* __restrict__ out) {
  __shared__ uint32_t scratch[128];
  const uint32_t t0 = blockIdx.x * kScanTile + threadIdx.x * kScanPerThread;
  uint32_t v[kScanPerThread], sum = 0;
#pragma unroll
  for (int k = 0; k < kScanPerThread; ++k) {
    v[k] = t0 + k < n ? in[t0 + k] : 0u;
    sum += v[k];
  }
  uint32_t e, unused;
  block_scan2(sum, 0u, e, unused, scratch);
  uint32_t run = offsets[blockIdx.x] + e;
#pragma unroll
  for (int k = 0; k < kScanPerThread; ++k) {
    if (t0 + k < n) out[t0 + k] = run;
    run += v[k];
  }
}

// Advance the substep counter and roll the dt pair: currentDt = nextDt, then
// the clock advances by it (include/mpm_engine.cuh:869-871).
// End of setup: the particles dropped while binning and the rigid velocity.
// The other fields keep what setup's kernels left (zero, and any status bits
// they raised: a non-finite initial velocity, a full block).
__global__ void finish_setup_kernel(Scalars* scal, uint32_t lost, float rx, float ry, float rz) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    scal->lost += lost;
    scal->rigid_v[0] = rx;
    scal->rigid_v[1] = ry;
    scal->rigid_v[2] = rz;
  }
}

__global__ void end_substep_kernel(Scalars* scal) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    scal->step += 1;
    scal->cur_dt = scal->next_dt;
    scal->cur_dt_d = scal->next_dt_d;
    scal->time += scal->cur_dt_d;
  }
}

// Adaptive dt, part 1: max |v|^2 over every grid node the next substep reads,
// after the grid update with the current dt (include/mpm_algorithm.cuh:739-869,
// the max-velocity query of UpdateGridVelocityAndQueryMax).  One warp per
// domain block; blocks whose stamp is stale are empty.  NaN counts as +inf.
// Nodes lighter than mass_floor are left out: the grid sums are fixed point
// with 2^-36 of a particle mass as unit, so at a few units v = mv / m is a
// ratio of two rounded small integers (e.g. 8/1 where the field moves at 6).
// Such a node's weight in G2P is of the same 2^-36 order, so it never moves
// a particle, but it would set the CFL bound.  The host passes
// mass_floor = 2^-16 x the lightest particle mass (>= 2^20 units, v to ~1e-6).
__global__ void grid_maxv_kernel(SceneDev sc, GridDev gd, Scalars* scal, float mass_floor) {
  sc.mass_clamp = fmaxf(sc.mass_clamp, mass_floor);
  const int32_t step = scal->step;
  const int parity = step & 1;
  const long long* g = gd.grid[parity];
  const int32_t* stamp = gd.stamp[parity];
  const float dt = scal->cur_dt;
  const int lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  float vmax2 = 0.f;
  for (uint32_t b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < sc.nblocks_domain; b += warps) {
    if (stamp[b] != step) continue;
    const int bz = static_cast<int>(b % sc.dims[2]);
    const int by = static_cast<int>((b / sc.dims[2]) % sc.dims[1]);
    const int bx = static_cast<int>((b / (static_cast<uint32_t>(sc.dims[2]) * sc.dims[1])) % sc.dims[0]);
    for (int node = lane; node < 128; node += 32) {
      const float4 v = node_velocity(sc, g + static_cast<int64_t>(b) * 512, sc.grid_unit, node, bx, by, bz,
                                     by * 4 + ((node >> 2) & 3), dt);
      float n2 = v.x * v.x + v.y * v.y + v.z * v.z;
      if (isnan(n2)) n2 = __int_as_float(0x7f800000);
      vmax2 = fmaxf(vmax2, n2);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) vmax2 = fmaxf(vmax2, __shfl_xor_sync(0xffffffffu, vmax2, o));
  if (lane == 0 && vmax2 > 0.f) atomicMax(&scal->maxv2_bits, __float_as_uint(vmax2));
}

// Adaptive dt, part 2 (one thread): nextDt = min(dt_max, frame end - time,
// dx * cfl / max|v|) (include/mpm_engine.cuh:552-557).  An infinite max|v|
// is the reference's "velocity reached infinity" stop: status NUMERIC.
__global__ void adaptive_dt_kernel(Scalars* scal, float dx, float cfl, float dt_max) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double next = fmin(static_cast<double>(dt_max), scal->frame_end - scal->time);
  const float v2 = __uint_as_float(scal->maxv2_bits);
  scal->maxv2_bits = 0u;
  if (isinf(v2)) scal->status |= kStatusNumeric;
  // IEEE-rounded square root and division (the library builds with the
  // approximate ones): the reference takes this bound on the host in FP32
  // (include/mpm_engine.cuh:540,556), and the dt sequence should match it.
  const float vmax = __fsqrt_rn(v2);
  if (vmax > 0.f) next = fmin(next, static_cast<double>(__fdiv_rn(dx * cfl, vmax)));
  if (next < 0.0) next = 0.0;
  scal->next_dt_d = next;
  scal->next_dt = static_cast<float>(next);
}

// ------------------------------------------------------------------ setup
// Initial binning of every particle: its block's flat index in the dense
// table (0xFFFFFFFF outside the domain or not finite), and the per-block
// count.  With the compaction, setup_place_kernel and setup_order_kernel it
// replaces ActivateBlocksWithParticles + BuildParticleCellBucket
// (include/mpm_algorithm.cuh:586-626,713-736).
__global__ void setup_bin_kernel(SceneDev sc, uint32_t n, const float* __restrict__ x, const uint32_t* __restrict__ sstart,
                                 uint32_t* __restrict__ flat, uint32_t* __restrict__ total) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float px = x[3 * i], py = x[3 * i + 1], pz = x[3 * i + 2];
  const int cx = static_cast<int>(px * sc.inv_dx + 0.25f), cy = static_cast<int>(py * sc.inv_dx + 0.25f),
            cz = static_cast<int>(pz * sc.inv_dx + 0.25f);
  const int bx = trunc_div4(cx - 2), by = trunc_div4(cy - 2), bz = trunc_div4(cz - 2);
  uint32_t f = 0xFFFFFFFFu;
  const bool finite = isfinite(px) && isfinite(py) && isfinite(pz) && px >= 0.f && py >= 0.f && pz >= 0.f;
  if (finite && in_domain(sc, bx, by, bz)) {
    const int w = sstart ? scene_of(sstart, sc.nstack, i) : 0;
    f = static_cast<uint32_t>(flat_block(sc, w, bx, by, bz));
    atomicAdd(total + f, 1u);
  }
  flat[i] = f;
}

// Setup placement: after the compaction has laid out the block list (colour-
// major, each block's range [start, start + count)), particle i takes the next
// free position of its block's range.  Inputs usually arrive in spatial order,
// so the lanes of a warp mostly share a block: one atomic per distinct block of
// the warp takes the positions of all its lanes.  The order the atomics hand
// positions out in is not deterministic; setup_order_kernel removes it.
__global__ void setup_place_kernel(uint32_t n, const uint32_t* __restrict__ flat, BlockListDev list,
                                   uint32_t* __restrict__ cursor, uint32_t* __restrict__ perm) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  int32_t slot = -1;
  if (i < n) {
    const uint32_t f = flat[i];
    if (f != 0xFFFFFFFFu) slot = list.table[f];
  }
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t group = __match_any_sync(0xffffffffu, slot);
  const uint32_t leader = __ffs(group) - 1u;
  uint32_t base = 0;
  if (slot >= 0 && lane == leader) base = atomicAdd(cursor + slot, static_cast<uint32_t>(__popc(group)));
  base = __shfl_sync(0xffffffffu, base, static_cast<int>(leader));
  if (slot >= 0) perm[list.start[slot] + base + __popc(group & ((1u << lane) - 1u))] = i;
}

// Bitonic sort of m (a power of two, <= kMaxParticlesPerBlock) 32-bit values in
// shared memory, ascending; every thread of the CTA takes part, one
// compare-exchange pair per thread and stage (m / 2 pairs).
template <int NT>
__device__ __forceinline__ void block_bitonic_sort(uint32_t* v, uint32_t m) {
  for (uint32_t k = 2; k <= m; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      const uint32_t lj = 31u - __clz(j);
      for (uint32_t p = threadIdx.x; p < (m >> 1); p += NT) {
        const uint32_t i = ((p >> lj) << (lj + 1)) | (p & (j - 1u));
        const uint32_t l = i | j;
        const uint32_t a = v[i], b = v[l];
        if ((a > b) == ((i & k) == 0)) {
          v[i] = b;
          v[l] = a;
        }
      }
      __syncthreads();
    }
  }
}

// Sort keys of the setup order for n particles whose cells (0..63) are cell[0..n):
// key[j] = ((r * 64 + cell[j]) << 12) | j, r the number of i < j in the same
// cell, and key[j] = 0xFFFFFFFF for n <= j < m.  Ranks are taken NT particles
// at a time in order of j: within a warp from the lanes of the same cell
// (__match_any_sync), across the warps of a chunk and across chunks from
// per-cell counters.  wcnt holds NT / 32 x 64 counters, base 64.
template <int NT>
__device__ __forceinline__ void cell_order_keys(const uint8_t* cell, uint32_t n, uint32_t m, uint32_t* key,
                                                uint32_t* wcnt, uint32_t* base) {
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  if (threadIdx.x < 64) base[threadIdx.x] = 0u;
  for (uint32_t i = n + threadIdx.x; i < m; i += NT) key[i] = 0xFFFFFFFFu;
  for (uint32_t b0 = 0; b0 < n; b0 += NT) {
    for (uint32_t i = threadIdx.x; i < (NT / 32) * 64; i += NT) wcnt[i] = 0u;
    __syncthreads();
    const uint32_t j = b0 + threadIdx.x;
    const uint32_t c = j < n ? cell[j] : 64u + lane;  // lanes past the end match nobody
    const uint32_t mask = __match_any_sync(0xffffffffu, c);
    const uint32_t below = __popc(mask & ((1u << lane) - 1u));
    if (j < n && below == 0u) wcnt[w * 64 + c] = __popc(mask);
    __syncthreads();
    if (threadIdx.x < 64) {
      uint32_t run = base[threadIdx.x];
#pragma unroll
      for (int q = 0; q < NT / 32; ++q) {
        const uint32_t t = wcnt[q * 64 + threadIdx.x];
        wcnt[q * 64 + threadIdx.x] = run;
        run += t;
      }
      base[threadIdx.x] = run;
    }
    __syncthreads();
    if (j < n) key[j] = (((wcnt[w * 64 + c] + below) * 64u + c) << 12) | j;
    __syncthreads();  // every key read its counter before the next chunk clears them
  }
}

// Setup ordering of each block's range, in two sorts in shared memory:
//  1. by input index, so nothing depends on the order the placement's atomics
//     ran in;
//  2. by (rank of the particle within its cell in that order, cell), with the
//     block's 64 cells numbered x-major (16 x + 4 y + z): 32 consecutive
//     particles then lie in the 32 different cells of one half block (2 x 4 x 4
//     cells), one per cell as far as the counts allow.
// The fused substep hands a warp 32 consecutive particles of a block, and each
// of them adds to 16 nodes of the P2G tile with shared atomics; with the tile's
// 68-word x planes the 32 cells of a half block fall in 32 different banks, while
// particles stored in input (lattice) order put several lanes of a warp in the
// same cell and serialise their atomics on the same words.  The substep's
// rebinning keeps each block's particles in their order, so the layout persists
// while particles stay in their blocks.  Results do not depend on the order (the
// grid sums are exact integers).  A block above kMaxParticlesPerBlock particles
// cannot be held and is reported as a capacity overflow.
template <int NT>
__global__ void __launch_bounds__(NT) setup_order_kernel(SceneDev sc, BlockListDev list, const float* __restrict__ x,
                                                         uint32_t* __restrict__ perm, Scalars* scal) {
  __shared__ uint32_t s[kMaxParticlesPerBlock];
  __shared__ uint32_t t[kMaxParticlesPerBlock];
  __shared__ uint8_t cell[kMaxParticlesPerBlock];
  __shared__ uint32_t wcnt[(NT / 32) * 64];
  __shared__ uint32_t base[64];
  const uint32_t nb = *list.nblocks;
  for (uint32_t slot = blockIdx.x; slot < nb; slot += gridDim.x) {
    const uint32_t n = list.count[slot], start = list.start[slot];
    if (n > static_cast<uint32_t>(kMaxParticlesPerBlock)) {
      if (threadIdx.x == 0) set_status(scal, kStatusCapacity);
      continue;
    }
    const int4 key = list.keys[slot];
    uint32_t m = 1;
    while (m < n) m <<= 1;
    for (uint32_t i = threadIdx.x; i < m; i += NT) s[i] = i < n ? perm[start + i] : 0xFFFFFFFFu;
    __syncthreads();
    block_bitonic_sort<NT>(s, m);
    // Cell of each particle within the block (the binning's +dx/4 cell).
    for (uint32_t i = threadIdx.x; i < n; i += NT) {
      const uint32_t p = s[i];
      const int lx = (static_cast<int>(x[3 * p] * sc.inv_dx + 0.25f) - 2 - 4 * key.x) & 3;
      const int ly = (static_cast<int>(x[3 * p + 1] * sc.inv_dx + 0.25f) - 2 - 4 * key.y) & 3;
      const int lz = (static_cast<int>(x[3 * p + 2] * sc.inv_dx + 0.25f) - 2 - 4 * key.z) & 3;
      cell[i] = static_cast<uint8_t>(lx * 16 + ly * 4 + lz);
    }
    __syncthreads();
    cell_order_keys<NT>(cell, n, m, t, wcnt, base);
    block_bitonic_sort<NT>(t, m);
    for (uint32_t i = threadIdx.x; i < n; i += NT) perm[start + i] = s[t[i] & 4095u];
    __syncthreads();
  }
}

// Re-layout of a model's particles between two substeps.  The setup order
// (setup_order_kernel) puts the 32 particles a warp handles in 32 different
// cells of a half block; the rebinning keeps each block's particles in their
// order, but as particles change cells and blocks the layout fades (on the
// sand column the fused substep's advantage over input order went from 7 % to
// none between 800 and 1600 substeps).  Every so many substeps the host runs
// this kernel before the next substep, whose block list is `parity`: each
// block gathers its incoming particles (through the previous substep's
// rebinning records, as the fused kernel does) into the other state buffer at
// its own range, in the setup order -- by rank within its cell in incoming
// order, then cell -- and the host copies that buffer back and makes the
// previous-step lists the identity, as after setup.  Values are moved, never
// changed; the simulation does not depend on the order.
template <int NT>
__global__ void __launch_bounds__(NT, 4) reorder_gather_kernel(SceneDev sc, ModelDev md, int parity, Scalars* scal) {
  __shared__ uint32_t src_of[kMaxParticlesPerBlock];
  __shared__ uint32_t key[kMaxParticlesPerBlock];
  __shared__ uint8_t cell[kMaxParticlesPerBlock];
  __shared__ uint32_t wcnt[(NT / 32) * 64];
  __shared__ uint32_t base[64];
  __shared__ SharedSmall sh;
  const BlockListDev cur = md.bl[parity];
  const BlockListDev prev = md.bl[parity ^ 1];
  const StateDev sin = md.st[parity];
  const StateDev sdst = md.st[parity ^ 1];
  const uint32_t nb = *cur.nblocks;
  for (uint32_t slot = blockIdx.x; slot < nb; slot += gridDim.x) {
    const int4 k4 = cur.keys[slot];
    const uint32_t start = cur.start[slot];
    if (threadIdx.x < 32) incoming_groups(sc, prev, k4, sh.off, sh.idx, sh.src);
    __syncthreads();
    const uint32_t room = start < md.cap_particles ? md.cap_particles - start : 0u;
    const uint32_t n = min(min(cur.count[slot], sh.off[27]), room);
    if (n > static_cast<uint32_t>(kMaxParticlesPerBlock)) {
      if (threadIdx.x == 0) set_status(scal, kStatusCapacity);
      __syncthreads();
      continue;
    }
    for (uint32_t j = threadIdx.x; j < n; j += NT) {
      const int d = find_group(sh.off, j);
      const uint32_t ii = sh.idx[d] + (j - sh.off[d]);
      uint32_t iin = ii < md.cap_particles ? sh.src[d] + prev.idx[ii] : 0xFFFFFFFFu;
      if (iin >= md.cap_particles) {  // corrupted record: flag, never read out of range
        set_status(scal, kStatusConsistency);
        iin = 0;
      }
      src_of[j] = iin;
      // the cell within the block, as setup_order_kernel numbers it ((c - 2) mod 4 per axis)
      const int lx = (static_cast<int>(sin.x[0][iin] * sc.inv_dx + 0.25f) - 2) & 3;
      const int ly = (static_cast<int>(sin.x[1][iin] * sc.inv_dx + 0.25f) - 2) & 3;
      const int lz = (static_cast<int>(sin.x[2][iin] * sc.inv_dx + 0.25f) - 2) & 3;
      cell[j] = static_cast<uint8_t>(lx * 16 + ly * 4 + lz);
    }
    __syncthreads();
    uint32_t m = 1;
    while (m < n) m <<= 1;
    cell_order_keys<NT>(cell, n, m, key, wcnt, base);
    block_bitonic_sort<NT>(key, m);
    // Replace each key by the source index it selects, then move one array at a
    // time (few registers, many loads in flight).
    for (uint32_t k = threadIdx.x; k < n; k += NT) key[k] = src_of[key[k] & 4095u];
    __syncthreads();
    for (int a = 0; a < 23; ++a) {
      const float* from = a < 3 ? sin.x[a] : a < 12 ? sin.F[a - 3] : a == 12 ? sin.aux : a < 22 ? sin.Q[a - 13]
                                                                               : reinterpret_cast<const float*>(sin.id);
      float* to = a < 3 ? sdst.x[a] : a < 12 ? sdst.F[a - 3] : a == 12 ? sdst.aux : a < 22 ? sdst.Q[a - 13]
                                                                      : reinterpret_cast<float*>(sdst.id);
      if (!from) continue;
      for (uint32_t k = threadIdx.x; k < n; k += NT) to[start + k] = from[key[k]];
    }
    __syncthreads();
  }
}

// Sorted initial state: x from the input, F = I, aux = logJp0 (0), alpha0,
// J0 or the rigid flag (0 for the first rigid_count input particles, else
// aux0 = 1), id = input index, velocities gathered for the rasterisation
// (include/mpm_algorithm.cuh:974-1081).
// n bounds the binned count; n_dev, when given, is the binned count on the
// device (setup launches before it is known on the host).
__global__ void setup_gather_kernel(ModelDev md, uint32_t nstack, uint32_t n, const uint32_t* __restrict__ perm,
                                    const float* __restrict__ x, const float* __restrict__ v, uint32_t nv, float aux0,
                                    uint32_t rigid_count, const uint32_t* __restrict__ n_dev = nullptr) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || (n_dev && i >= *n_dev)) return;
  const uint32_t s = perm[i];
  if (s >= md.cap_particles) return;  // a position the placement never filled
  StateDev st = md.st[0];
  st.x[0][i] = x[3 * s];
  st.x[1][i] = x[3 * s + 1];
  st.x[2][i] = x[3 * s + 2];
  if (st.F[0]) {
#pragma unroll
    for (int k = 0; k < 9; ++k) st.F[k][i] = (k & 3) ? 0.f : 1.f;
  }
  if (st.aux) st.aux[i] = md.smat ? md.smat[scene_of(md.sstart, nstack, s)].aux0 : (s < rigid_count ? 0.f : aux0);
  if (st.Q[0]) {
#pragma unroll
    for (int k = 0; k < 9; ++k) st.Q[k][i] = 0.f;
  }
  if (st.id) st.id[i] = s;
  const uint32_t vs = nv == 1 ? 0u : s;
  md.vel_in[3 * i] = v[3 * vs];
  md.vel_in[3 * i + 1] = v[3 * vs + 1];
  md.vel_in[3 * i + 2] = v[3 * vs + 2];
}

// Identity "previous step" for the first substep: every particle stays in
// its block (direction 13), index list = in-block position
// (include/mpm_algorithm.cuh:950-964 InitializeAdvectionBucket).
// One CTA per block of the list, grid-strided (the block count is read on the
// device).
__global__ void setup_identity_kernel(BlockListDev cur, BlockListDev prev) {
  const uint32_t nb = *cur.nblocks;
  for (uint32_t slot = blockIdx.x; slot < nb; slot += gridDim.x) {
    const uint32_t n = cur.count[slot], start = cur.start[slot];
    if (threadIdx.x < 28) prev.prefix28[slot * 28 + threadIdx.x] = threadIdx.x <= 13 ? 0u : n;
    for (uint32_t q = threadIdx.x; q < n; q += blockDim.x) prev.idx[start + q] = static_cast<uint16_t>(q);
  }
}

// Setup: the particles of a model that binning dropped (outside the domain).
__global__ void count_lost_kernel(Scalars* scal, uint32_t n, const uint32_t* __restrict__ binned) {
  if (threadIdx.x == 0 && blockIdx.x == 0) scal->lost += n - *binned;
}

// ------------------------------------------------------------------ decomposed scene
// One scene split over ranks by particle ownership (no counterpart in the
// reference, which runs on one GPU): every rank keeps the whole dense grid,
// deposits only its own particles, and before the next substep the ranks sum
// the blocks that more than one of them deposited into.  The sums are exact
// 64-bit integers, so every rank then reads the grid a single GPU would hold.

// mask[b] = 1 when block b of the grid the next substep reads holds this
// rank's deposits (its stamp is the read epoch), else 0.
__global__ void dd_mark_kernel(const int32_t* __restrict__ stamp, int32_t epoch, uint32_t nbd, int32_t* mask) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nbd; b += gridDim.x * blockDim.x)
    mask[b] = stamp[b] == epoch ? 1 : 0;
}

// Copies the listed blocks (512 sums each) into buf; a block without this
// rank's deposits contributes zeros.  One warp per block.
__global__ void dd_pack_kernel(const long long* __restrict__ g, const int32_t* __restrict__ stamp, int32_t epoch,
                               const int32_t* __restrict__ list, uint32_t n, uint32_t nbd,
                               longlong2* __restrict__ buf) {
  const int lane = threadIdx.x & 31;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < n; t += nwarps) {
    const int32_t b = list[t];
    const bool own = b >= 0 && static_cast<uint32_t>(b) < nbd && stamp[b] == epoch;
    const longlong2* src = reinterpret_cast<const longlong2*>(g + static_cast<int64_t>(own ? b : 0) * 512);
    for (int i = lane; i < 256; i += 32) buf[static_cast<size_t>(t) * 256 + i] = own ? src[i] : make_longlong2(0, 0);
  }
}

// Writes the summed blocks back and stamps them with the read epoch.
__global__ void dd_unpack_kernel(long long* __restrict__ g, int32_t* __restrict__ stamp, int32_t epoch,
                                 const int32_t* __restrict__ list, uint32_t n, uint32_t nbd,
                                 const longlong2* __restrict__ buf) {
  const int lane = threadIdx.x & 31;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < n; t += nwarps) {
    const int32_t b = list[t];
    if (b < 0 || static_cast<uint32_t>(b) >= nbd) continue;
    longlong2* dst = reinterpret_cast<longlong2*>(g + static_cast<int64_t>(b) * 512);
    for (int i = lane; i < 256; i += 32) dst[i] = buf[static_cast<size_t>(t) * 256 + i];
    if (lane == 0) stamp[b] = epoch;
  }
}

// ------------------------------------------------------------------ probe / export
// Gathers the current state (x, F, aux, id) and interpolates v at each
// particle from the current grid with the grid update applied, as the next
// G2P will (include/mpm_algorithm.cuh:1306-1331).  Output slot: block order,
// or dest[id] when dest is given (ids tracked).  Materials without F write
// the identity, without aux zero (per scene in a batch).
template <int NT>
__global__ void __launch_bounds__(NT) probe_kernel(SceneDev sc, ModelDev md, GridDev gd, Scalars* scal, float* ox,
                                                  float* ov, float* oF, float* oaux, uint32_t* oid,
                                                  const uint32_t* __restrict__ dest) {
  extern __shared__ __align__(16) unsigned char smem[];
  float4* vtile = reinterpret_cast<float4*>(smem);
  __shared__ SharedSmall sh;
  const int32_t step = scal->step;
  const int parity = step & 1;
  const BlockListDev cur = md.bl[parity];
  const BlockListDev prev = md.bl[parity ^ 1];
  const StateDev sin = md.st[parity];
  const uint32_t nb = *cur.nblocks;
  const float dt = scal->cur_dt;
  for (uint32_t item = blockIdx.x; item < nb; item += gridDim.x) {
    const int4 key = cur.keys[item];
    const uint32_t start = cur.start[item];
    const uint32_t n = cur.count[item];
    const int kind = md.smat ? md.smat[key.w].kind : md.mat.kind;
    if (threadIdx.x < 32)
      incoming_groups(sc, prev, key, sh.off, sh.idx, sh.src);
    else if (threadIdx.x < 40)
      window_blocks(sc, gd.stamp[parity], step, key, sh.blk, threadIdx.x - 32);
    __syncthreads();
    if (ov) load_velocity_tile<NT>(sc, gd.grid[parity], sh.blk, key, md.smat ? md.smat[key.w].unit : sc.grid_unit, dt,
                                   vtile);
    __syncthreads();
    const uint32_t nn = min(min(n, sh.off[27]), start < md.cap_particles ? md.cap_particles - start : 0u);
    for (uint32_t q = threadIdx.x; q < nn; q += NT) {
      const int d = find_group(sh.off, q);
      const uint32_t ii = sh.idx[d] + (q - sh.off[d]);
      uint32_t iin = ii < md.cap_particles ? sh.src[d] + prev.idx[ii] : 0xFFFFFFFFu;
      if (iin >= md.cap_particles) {
        set_status(scal, kStatusConsistency);
        iin = 0;
      }
      const uint32_t pid = sin.id ? sin.id[iin] : start + q;
      const uint32_t o = dest ? dest[pid] : start + q;
      const float x[3] = {sin.x[0][iin], sin.x[1][iin], sin.x[2][iin]};
      if (ox) {
        ox[3 * o] = x[0];
        ox[3 * o + 1] = x[1];
        ox[3 * o + 2] = x[2];
      }
      if (oF) {
        const bool hasF = material_has_F(kind) && sin.F[0];
#pragma unroll
        for (int k = 0; k < 9; ++k) oF[9 * o + k] = hasF ? sin.F[k][iin] : ((k & 3) ? 0.f : 1.f);
      }
      if (oaux) oaux[o] = (material_has_aux(kind) && sin.aux) ? sin.aux[iin] : 0.f;
      if (oid) oid[o] = pid;
      if (ov) {
        const float xs[3] = {x[0] * sc.inv_dx, x[1] * sc.inv_dx, x[2] * sc.inv_dx};
        float v[3], C[9], D6[6];
        bool inside = true;
        g2p(vtile, xs, key, sc.dx, v, C, inside, D6);
        if (sc.rigid) {  // rigid particles report zero velocity (include/mpm_algorithm.cuh:1316-1325)
          const float f0 = (material_has_F(kind) && sin.F[0]) ? sin.F[0][iin] : 1.f;
          const float a = (material_has_aux(kind) && sin.aux) ? sin.aux[iin] : 1.f;
          if (rigid_attribute(kind, &f0, a) == 0.f) v[0] = v[1] = v[2] = 0.f;
        }
        ov[3 * o] = v[0];
        ov[3 * o + 1] = v[1];
        ov[3 * o + 2] = v[2];
      }
    }
    __syncthreads();
  }
}

// Input-order export: flag[id] = 1 for every live particle (ids from the
// block-order probe); an exclusive scan of the flags gives each live id its
// position among the live particles in input order.
// Marks the live ids (the first n of ids, or the first *n_dev when given: an
// export enqueued without reading the live count back).
__global__ void mark_ids_kernel(uint32_t n, const uint32_t* __restrict__ ids, uint32_t* __restrict__ flag,
                               uint32_t cap, const uint32_t* __restrict__ n_dev) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t live = n_dev ? min(n, *n_dev) : n;
  if (i < live && ids[i] < cap) flag[ids[i]] = 1u;
}

// ------------------------------------------------------------------ debug hook
__global__ void debug_constitutive_kernel(MaterialParams mat, uint32_t n, const float* C, float dt, float* F,
                                          float* aux, float* tau, float* U, float* S, float* V) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float c[9], f[9], t[9];
  for (int k = 0; k < 9; ++k) c[k] = C[9 * i + k];
  float a = aux ? aux[i] : 0.f;
  if (mat.kind == kFluid) {
    stress_fluid(mat.p[0], mat.p[1], mat.p[2], c, dt, a, t);
  } else {
    for (int k = 0; k < 9; ++k) f[k] = F[9 * i + k];
    float dW[9];
    for (int k = 0; k < 9; ++k) dW[k] = c[k] * dt + ((k & 3) ? 0.f : 1.f);
    matmul3(dW, f, f);
    if (U || S || V) {
      float u[9], s[3], v[9];
      svd3(f, u, s, v);
      for (int k = 0; k < 9; ++k) {
        if (U) U[9 * i + k] = u[k];
        if (V) V[9 * i + k] = v[k];
      }
      if (S)
        for (int k = 0; k < 3; ++k) S[3 * i + k] = s[k];
    }
    if (mat.kind == kFixedCorotated)
      stress_fixed_corotated(mat.p[0], mat.p[1], f, t);
    else if (mat.kind == kDruckerPrager)
      stress_drucker_prager(mat.p[0], mat.p[1], f, a, t);
    else if (mat.kind == kVonMises)
      stress_von_mises(mat.p[0], mat.p[1], mat.p[2], f, t);
    else
      stress_nacc(mat.p, f, a, t);
    for (int k = 0; k < 9; ++k) F[9 * i + k] = f[k];
  }
  if (aux) aux[i] = a;
  for (int k = 0; k < 9; ++k) tau[9 * i + k] = t[k];
}

}  // namespace ckmpm
