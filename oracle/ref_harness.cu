// TEST INFRASTRUCTURE ONLY: driver of the reference CUDA build (AppledoreM/CKMPM).
//
// Compiled (oracle/Makefile, target `ref`) against the reference's own headers
// where they lie; its output binaries go to oracle/_ref/ and are never part of
// the product.  It drives the reference through its public API exactly as the
// reference's scene executables do (tests/fluid_dam_break/test_fluid_dam_break.cu:5-18):
// MPMEngine::Initialize -> InitializeParticle -> InitialSetup -> Simulate, with
// a scene configuration class of our own (the reference takes scene constants
// from compile-time CRTP classes, include/mpm_config.h:12-124).
//
// One binary per grid family (cell size, domain extent, gravity, boundary rule):
//   CKMPM_HARNESS_SCENE_JELLY : dx = 1/64,  16^3 blocks, g = -9.8, sticky walls (the built-in rule)
//   CKMPM_HARNESS_SCENE_SAND  : dx = 1/256, 64^3 blocks, g = -9.8, slip floor at 8 cells
//   CKMPM_HARNESS_SCENE_SLIP  : dx = 1/64,  16^3 blocks, g = -9.8, slip floor at 8 cells
//   CKMPM_HARNESS_SCENE_DAM   : dx = 1/512, 128^3 blocks, g = -9.8, sticky walls
//   CKMPM_HARNESS_SCENE_FIELD : the JELLY grid with an irregular-boundary hook: v = 0 in the cell
//                               box [24,32) x [0,14) x [24,32), elsewhere the slip walls of
//                               tests/fluid_with_two_longs (cells within 8 of a face lose the
//                               velocity component along the normalised sum of the face normals)
//   CKMPM_HARNESS_SCENE_RIGID : the JELLY grid with rigid particles on (GetExistRigidParticle):
//                               the first 2048 particles of every von Mises model are rigid and
//                               move with (2, 0.5 frame - 1, -1) in frame `frame` (every value
//                               exact in float)
// The slip floor is installed through the reference's irregular-boundary hook
// (GetExistIrregularBoundary / ProcessGridCellVelocity, include/mpm_algorithm.cuh:795-799):
// sticky x/z walls and ceiling two blocks deep, v_y >= 0 in cells below the floor.
//
// Usage: ref_<scene> <manifest> <fps> <frames> <dt> <outdir> <mode> [<K1,K2,...>]
//   manifest: one model per line: <material> <p0> ... <p7> <mass> <volume> <x.bin> <v.bin>
//   material and parameters, in the field order of each MaterialParameter_
//   (include/mpm_material.cuh:24-257): fc | dp | linear: lambda mu; fluid: bulk
//   gamma viscosity J0; vm: mu lambda yield; nacc: mu lambda alpha0 beta
//   hardeningFactor M hardeningOn
//   x.bin / v.bin: float32 xyz triples (v.bin holds 1 or n velocities)
//   mode 0: export raw positions every frame (outdir/model_0_particle_frame_<k>.txt)
//   mode 1: profile mode, no export; the reference prints its MPMBenchmark statistics, and the
//           harness prints "HARNESS e2e <seconds>": a host timer from before Initialize to the end
//           of Simulate's frame loop (the CUDA context exists before the timer starts)
//   mode 2: state dump after K1, K2, ... substeps (0 = right after InitialSetup), then exit:
//           outdir/sets_k<K>.bin and outdir/state_m<model>_k<K>.bin (formats at dump::write_sets
//           and dump::write_state).  Particle identity is carried through the reference's own
//           advection records; see namespace dump.
#include <algorithm>
#include <any>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <limits>
#include <map>
#include <mutex>
#include <numbers>
#include <numeric>
#include <random>
#include <span>
#include <sstream>
#include <string>
#include <string_view>
#include <thread>
#include <tuple>
#include <type_traits>
#include <typeinfo>
#include <utility>
#include <variant>
#include <vector>

#include <cooperative_groups.h>
#include <cuda.h>
#include <cuda/atomic>
#include <cuda_profiler_api.h>
#include <cuda_runtime.h>
#include <thrust/device_ptr.h>
#include <thrust/device_vector.h>
#include <thrust/execution_policy.h>
#include <thrust/fill.h>
#include <thrust/scan.h>

#include <nlohmann/json.hpp>

#include "Partio.h"
#include "PartioAttribute.h"
#include "spdlog/spdlog.h"

// The state dump reads the engine's partitions, particle buffers and grids,
// which MPMEngine keeps private.  Every system and third-party header is
// included above, so only the reference's own headers see this definition.
#define private public
#include "mpm_engine.cuh"
#undef private

namespace harness {
void on_substep();
}

namespace harness {

#if defined(CKMPM_HARNESS_SCENE_DAM)
constexpr float kDx = 1.f / 512.f;
constexpr int kBlocks = 128;
constexpr bool kSlipFloor = false;
constexpr uint32_t kMaxBlocks = 650000;
#elif defined(CKMPM_HARNESS_SCENE_SAND)
constexpr float kDx = 1.f / 256.f;
constexpr int kBlocks = 64;
constexpr bool kSlipFloor = true;
constexpr uint32_t kMaxBlocks = 60000;
#elif defined(CKMPM_HARNESS_SCENE_SLIP)
constexpr float kDx = 1.f / 64.f;
constexpr int kBlocks = 16;
constexpr bool kSlipFloor = true;
constexpr uint32_t kMaxBlocks = 4096;
#else
constexpr float kDx = 1.f / 64.f;
constexpr int kBlocks = 16;
constexpr bool kSlipFloor = false;
constexpr uint32_t kMaxBlocks = 4096;
#endif
#if defined(CKMPM_HARNESS_SCENE_RIGID)
constexpr bool kRigid = true;
#else
constexpr bool kRigid = false;
#endif
#if defined(CKMPM_HARNESS_SCENE_FIELD)
constexpr bool kField = true;
#else
constexpr bool kField = false;
#endif
constexpr uint32_t kRigidCount = 2048;
constexpr float kGravity = -9.8f;
constexpr float kFloorCells = 8.f;

// Host-only run parameters (read by Initialize / Simulate on the host).
inline uint32_t g_fps = 48;
inline uint32_t g_frames = 1;
inline float g_dt = 1e-4f;

typedef mpm::MPMDomainRange<kBlocks, kBlocks, kBlocks> DomainRange;
typedef mpm::MPMDomain<DomainRange, mpm::MPMDomainOffset<0, 0, 0>> Domain;
typedef mpm::MPMGridConfig<Domain> GridConfig;

class Config : public mpm::MPMConfigBase<Config> {
 public:
  friend class mpm::MPMConfigBase<Config>;
  constexpr Config() = default;

 protected:
  constexpr MPM_FORCE_INLINE MPM_HOST_DEV_FUNC auto GetDxImpl() const -> float { return kDx; }
  constexpr MPM_FORCE_INLINE MPM_HOST_DEV_FUNC auto GetBlockVolumeImpl() const -> uint32_t { return 64; }
  constexpr MPM_FORCE_INLINE MPM_HOST_DEV_FUNC auto GetBlockSizeImpl() const -> uint32_t { return 4; }
  constexpr MPM_FORCE_INLINE MPM_HOST_DEV_FUNC auto GetMaxParticleCountPerCellImpl() const -> uint32_t { return 64; }
  constexpr MPM_FORCE_INLINE MPM_HOST_DEV_FUNC auto GetMaxParticleCountPerBlockImpl() const -> uint32_t {
    return GetBlockVolumeImpl() * GetMaxParticleCountPerCellImpl();
  }
  constexpr MPM_FORCE_INLINE MPM_HOST_DEV_FUNC auto GetMaxParticleCountPerBucketImpl() const -> uint32_t { return 32; }
  constexpr MPM_FORCE_INLINE MPM_HOST_DEV_FUNC auto GetMaxActiveBlockCountImpl() const -> uint32_t { return kMaxBlocks; }
  MPM_FORCE_INLINE auto GetFpsImpl() const -> uint32_t { return g_fps; }
  MPM_FORCE_INLINE auto GetDtImpl() const -> float { return g_dt; }
  constexpr MPM_FORCE_INLINE MPM_HOST_DEV_FUNC auto GetCflImpl() const -> float { return 0.5f; }
  MPM_FORCE_INLINE auto GetTotalSimulatedFrameCountImpl() const -> uint32_t { return g_frames; }
  constexpr MPM_FORCE_INLINE MPM_HOST_DEV_FUNC auto GetGravityImpl() const -> float { return kGravity; }
  constexpr MPM_FORCE_INLINE MPM_HOST_DEV_FUNC auto GetMassClampImpl() const -> float { return 0.f; }
  constexpr MPM_FORCE_INLINE MPM_HOST_DEV_FUNC auto GetExistRigidParticleImpl() const -> bool { return kRigid; }
  constexpr MPM_FORCE_INLINE MPM_HOST_DEV_FUNC auto GetRigidParticleCountImpl() const -> uint32_t {
    return kRigid ? kRigidCount : 0u;
  }
  template <typename Scalar>
  constexpr MPM_FORCE_INLINE MPM_HOST_DEV_FUNC auto GetRigidParticleVelocityImpl(int frame) const
      -> mpm::Vector<Scalar, 3> {
    return mpm::Vector<Scalar, 3>{Scalar(2), Scalar(0.5) * Scalar(frame) - Scalar(1), Scalar(-1)};
  }
  constexpr MPM_FORCE_INLINE MPM_HOST_DEV_FUNC auto GetExistIrregularBoundaryImpl() const -> bool {
    return kSlipFloor || kField;
  }
  MPM_FORCE_INLINE MPM_HOST_DEV_FUNC auto ProcessGridCellVelocityImpl(const mpm::Vector<int, 3>& cell,
                                                                      mpm::Vector<float, 3>& velocity, int) const
      -> void {
    if (kField) {
      const bool fixed = cell[0] >= 24 && cell[0] < 32 && cell[1] < 14 && cell[2] >= 24 && cell[2] < 32;
      if (fixed) {
        velocity[0] = velocity[1] = velocity[2] = 0.f;
        return;
      }
      mpm::Vector<float, 3> n{0.f, 0.f, 0.f};
      bool wall = false;
      for (int a = 0; a < 3; ++a) {
        if (cell[a] < 8) {
          n[a] = 1.f;
          wall = true;
        } else if (cell[a] >= kBlocks * 4 - 8) {
          n[a] = -1.f;
          wall = true;
        }
      }
      if (wall) {
        n = n / n.Norm();
        const float d = n.Dot(velocity);
        velocity -= d * n;
      }
      return;
    }
    const int bx = cell[0] / 4, by = cell[1] / 4, bz = cell[2] / 4;
    const bool wall = bx < 2 || bx + 2 >= kBlocks || bz < 2 || bz + 2 >= kBlocks || by + 2 >= kBlocks;
    if (wall) {
      velocity[0] = velocity[1] = velocity[2] = 0.f;
    } else if (static_cast<float>(cell[1]) < kFloorCells) {
      velocity[1] = velocity[1] > 0.f ? velocity[1] : 0.f;
    }
  }
  // Simulate calls UpdateConfig once at the end of every substep (include/mpm_engine.cuh:866);
  // the state dump follows the particles from there.
  MPM_FORCE_INLINE MPM_HOST_DEV_FUNC auto UpdateConfigImpl(float, int) -> void {
#ifndef __CUDA_ARCH__
    on_substep();
#endif
  }
};

std::vector<mpm::Vector<float, 3>> read_xyz(const char* path) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) {
    std::fprintf(stderr, "cannot open %s\n", path);
    std::exit(2);
  }
  const size_t bytes = static_cast<size_t>(f.tellg());
  f.seekg(0);
  std::vector<mpm::Vector<float, 3>> v(bytes / 12);
  f.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(v.size() * 12));
  return v;
}

}  // namespace harness

// ---------------------------------------------------------------------------------------------
// State dump (mode 2).  The reference's particles carry no identity: a particle is an entry of
// its block's bucket list, and each substep's rebinning leaves, per entry of the next step's
// block list, an advection record (direction of the source block, index in it;
// include/mpm_particle.cuh:333-371).  The reference follows those records itself to export
// positions (RetrieveParticleBuffer, include/mpm_algorithm.cuh:1977-2020) and in G2P2G
// (:1496-1534).  The dump keeps one u32 id per particle entry of each of the two particle
// buffers, laid out like their buckets (entry i of the block in slot s sits at
// 32 * particleBinOffset_[s] + i), and carries it along the same records at the end of every
// substep, starting from the input indices that InitialSetup's binning stores in blockBucket_
// (BuildParticleCellBucket / ParticleCellBucketToBlock / CopyParticleArrayToParticleBuffer,
// :586-649, :974-1079).
namespace dump {

using namespace mpm;
using Engine = MPMEngine<harness::GridConfig>;
using Partition = Engine::Partition_;
constexpr uint32_t kBucket = 32;    // GetMaxParticleCountPerBucket
constexpr uint32_t kPerBlock = 4096;  // GetMaxParticleCountPerBlock (64 cells x 64)
static_assert(sizeof(MPMGridBlockCoordinate) == 3 * sizeof(int32_t), "block keys are read as int32 triples");

inline std::vector<uint64_t> g_ks;  // substep counts to dump at, ascending
inline size_t g_next = 0;
inline uint64_t g_substeps = 0;
inline std::string g_outdir;
inline bool g_active = false;
inline std::vector<std::array<uint32_t*, 2>> g_ids;  // per model, per particle buffer
inline uint32_t* g_counter = nullptr;
inline float* g_maxv = nullptr;
inline Engine::Grid_ g_grid;  // scratch copy of grid_[0] for the velocity read-back

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "dump: %s: %s\n", what, cudaGetErrorString(e));
    std::_Exit(3);
  }
}

// Ids of the particles InitialSetup wrote into `buf`: the input index of entry i of slot s.
template <typename Buffer>
__global__ void initial_ids_kernel(Buffer buf, uint32_t nblocks, uint32_t* ids) {
  const uint32_t s = blockIdx.x;
  if (s >= nblocks) return;
  const uint32_t n = buf.particleBucketSize_[s];
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
    ids[static_cast<size_t>(buf.particleBinOffset_[s]) * kBucket + i] = buf.blockBucket_[static_cast<size_t>(s) * kPerBlock + i];
}

// Walks the advection records of `rec` (one per entry of the blocks of `partition`) to the
// particle entries of `data` (blocks of `prev`), as RetrieveParticleBuffer does.  With id_dst
// it writes each source id at the entry the next G2P2G writes that particle to; with out_id it
// appends the particle (id, block key, every float attribute) to the output arrays.
template <typename Buffer>
__global__ void follow_kernel(Partition partition, Partition prev, Buffer data, Buffer rec, uint32_t nblocks,
                              const uint32_t* __restrict__ id_src, uint32_t* id_dst, uint32_t* counter,
                              uint32_t* out_id, int* out_key, float* out_attr, int nattr, uint32_t cap) {
  const uint32_t s = blockIdx.x;
  if (s >= nblocks) return;
  const uint32_t n = rec.particleBucketSize_[s];
  const auto key = partition.activeKeys_[s];
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const uint32_t r = rec.blockBucket_[static_cast<size_t>(s) * kPerBlock + i];
    const int dir = static_cast<int>(r / kPerBlock);
    const uint32_t src = r % kPerBlock;
    const MPMGridBlockCoordinate sk{key[0] + dir / 9 - 1, key[1] + (dir / 3) % 3 - 1, key[2] + dir % 3 - 1};
    const uint32_t ss = prev.Find(sk);
    const size_t lin = static_cast<size_t>(data.particleBinOffset_[ss]) * kBucket + src;
    const uint32_t id = id_src[lin];
    if (id_dst) id_dst[static_cast<size_t>(rec.particleBinOffset_[s]) * kBucket + i] = id;
    if (out_id) {
      const uint32_t o = atomicAdd(counter, 1u);
      if (o >= cap) continue;
      out_id[o] = id;
      out_key[3 * o] = key[0];
      out_key[3 * o + 1] = key[1];
      out_key[3 * o + 2] = key[2];
      const float* b = reinterpret_cast<const float*>(data.particleBuffer_) + (lin / kBucket) * kBucket * nattr;
      const size_t lane = lin % kBucket;
      for (int a = 0; a < nattr; ++a) out_attr[static_cast<size_t>(o) * nattr + a] = b[a * kBucket + lane];
    }
  }
}

// The velocity G2P gives a particle on the updated grid: 0.5 x the sum over both staggered grids
// of w_i v_i, with the reference's cell index, weights and summation order
// (CollectConservationMetric, include/mpm_algorithm.cuh:1270-1320), the node values read from
// the grid blocks instead of the shared tile they are copied into.  With rigid particles on, G2P
// reads attribute 3 of every particle as J and gives a particle with J == 0 (a rigid one) zero
// velocity (G2P2G, include/mpm_algorithm.cuh:1540-1543, 1609-1615); so does this read-back.
template <typename Grid>
__global__ void velocity_kernel(Partition partition, const Grid grid, uint32_t n, const float* attr, int nattr,
                                float* out_v) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  constexpr auto config = harness::Config{};
  const Vector<float, 3> pos{attr[static_cast<size_t>(p) * nattr], attr[static_cast<size_t>(p) * nattr + 1],
                             attr[static_cast<size_t>(p) * nattr + 2]};
  Vector<float, 3> vel = {};
  meta::ConstexprLoop<-1, 2, 2>([&](auto gw) -> void {
    constexpr int g = meta::ConstexprLoopIndex(gw);
    constexpr int gi = g == -1 ? 0 : 1;
    const auto cell = GetCellIndex<g>(config, pos);
    Vector<float, 3> local = pos * config.GetInvDx() - cell;
    Vector<float, 3> w;
    MPMKernel<SmoothLinear<float, g>>::OptimizedWeightComputation(local, w);
    meta::ConstexprLoop<0, 8>([&](auto mw) -> void {
      constexpr int m = meta::ConstexprLoopIndex(mw);
      constexpr int dx = (m & 4) >> 2, dy = (m & 2) >> 1, dz = m & 1;
      float weight = 1.f;
      weight *= dx == 0 ? w[0] : (1 - w[0]);
      weight *= dy == 0 ? w[1] : (1 - w[1]);
      weight *= dz == 0 ? w[2] : (1 - w[2]);
      const int cx = cell[0] + dx, cy = cell[1] + dy, cz = cell[2] + dz;
      const uint32_t slot = partition.Find(MPMGridBlockCoordinate{cx / 4, cy / 4, cz / 4});
      const auto* blk = grid.GetBlock(slot);
      const uint32_t idx = gi * 64 + (cx % 4) * 16 + (cy % 4) * 4 + (cz % 4);
      const Vector<float, 3> node{blk->template GetValue<1>(idx), blk->template GetValue<2>(idx),
                                  blk->template GetValue<3>(idx)};
      vel += weight * node;
    });
  });
  vel = 0.5f * vel;
  if (harness::kRigid && attr[static_cast<size_t>(p) * nattr + 3] == 0.f) vel = Vector<float, 3>{};
  out_v[3 * p] = vel[0];
  out_v[3 * p + 1] = vel[1];
  out_v[3 * p + 2] = vel[2];
}

template <typename T>
void write_raw(std::ofstream& f, const std::vector<T>& v) {
  f.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(sizeof(T) * v.size()));
}

// Carries every model's ids from the particle buffer the last substep wrote (roll index) to the
// entries the next substep writes (next roll index).
void step_ids(Engine* e) {
  cudaStream_t st = CudaUtil::GetCudaContext().GetComputeStream();
  const uint32_t r = e->GetRollIndex(), nx = e->GetNextRollIndex();
  const uint32_t na = e->activePartitionBlockCount_;
  for (size_t i = 0; i < g_ids.size(); ++i) {
    std::visit(
        [&](auto&& data) -> void {
          using B = std::decay_t<decltype(data)>;
          auto& rec = std::get<B>(e->particleBuffer_[nx][i]);
          if (na) follow_kernel<B><<<na, 128, 0, st>>>(e->partition_[r], e->partition_[nx], data, rec, na, g_ids[i][r],
                                                     g_ids[i][nx], nullptr, nullptr, nullptr, nullptr, 0, 0);
        },
        e->particleBuffer_[r][i]);
  }
  check(cudaGetLastError(), "follow (ids)");
  check(cudaStreamSynchronize(st), "ids sync");
}

// sets_k<K>.bin:    u32 K, NA, NN, NE, model count; i32 keys[NE][3] (slot order: particle
//                   blocks, neighbour additions, exterior additions); u32 counts[models][NA]
// state_m<i>_k<K>.bin: u32 n, attribute count A; u32 id[n]; i32 block key[n][3];
//                   f32 attributes[n][A] (the model's bucket attributes in order: x, y, z, then
//                   F / J / logJp as its particle type lays them out); f32 v[n][3]
void dump_at(Engine* e, uint64_t K, double next_dt) {
  auto& cu = CudaUtil::GetCudaContext();
  cudaStream_t st = cu.GetComputeStream();
  check(cudaStreamSynchronize(st), "dump sync");
  const uint32_t r = e->GetRollIndex(), nx = e->GetNextRollIndex();
  const uint32_t na = e->activePartitionBlockCount_, nn = e->activePartitionNeighborBlockCount_,
                 ne = e->activePartitionExteriorBlockCount_;
  constexpr auto config = harness::Config{};
  // Node velocities the next substep's G2P reads (UpdateGridVelocityAndQueryMax on a copy).
  g_grid.Copy(config, ne, e->grid_[0]);
  check(cudaMemsetAsync(g_maxv, 0, sizeof(float), st), "memset");
  cu.LaunchCompute({NextNearestMultipleOf<16>(nn) / 16, 512},
                   UpdateGridVelocityAndQueryMax<true, harness::Config, Engine::GridBlock_, Partition>, config, nn,
                   g_grid, e->partition_[r], next_dt, static_cast<int>(e->currentFrameIndex_), g_maxv);
  check(cudaStreamSynchronize(st), "grid update");

  std::vector<int32_t> keys(3 * static_cast<size_t>(ne));
  check(cudaMemcpy(keys.data(), e->partition_[r].activeKeys_, sizeof(int32_t) * keys.size(), cudaMemcpyDeviceToHost),
        "keys");
  std::vector<uint32_t> counts;
  const std::string tag = "_k" + std::to_string(K) + ".bin";
  for (size_t i = 0; i < g_ids.size(); ++i) {
    std::visit(
        [&](auto&& data) -> void {
          using B = std::decay_t<decltype(data)>;
          auto& rec = std::get<B>(e->particleBuffer_[nx][i]);
          const int nattr = static_cast<int>(B::Attribute::kSize_ / sizeof(float));
          std::vector<uint32_t> c(na);
          if (na)
            check(cudaMemcpy(c.data(), rec.particleBucketSize_, sizeof(uint32_t) * na, cudaMemcpyDeviceToHost), "counts");
          counts.insert(counts.end(), c.begin(), c.end());
          const uint32_t cap = static_cast<uint32_t>(e->particleCount_[i]);
          uint32_t *d_id = nullptr;
          int* d_key = nullptr;
          float *d_attr = nullptr, *d_v = nullptr;
          check(cudaMalloc(&d_id, sizeof(uint32_t) * cap), "alloc");
          check(cudaMalloc(&d_key, sizeof(int) * 3 * cap), "alloc");
          check(cudaMalloc(&d_attr, sizeof(float) * nattr * static_cast<size_t>(cap)), "alloc");
          check(cudaMalloc(&d_v, sizeof(float) * 3 * static_cast<size_t>(cap)), "alloc");
          check(cudaMemsetAsync(g_counter, 0, sizeof(uint32_t), st), "memset");
          if (na)
            follow_kernel<B><<<na, 128, 0, st>>>(e->partition_[r], e->partition_[nx], data, rec, na, g_ids[i][r],
                                                 nullptr, g_counter, d_id, d_key, d_attr, nattr, cap);
          check(cudaGetLastError(), "follow (dump)");
          uint32_t n = 0;
          check(cudaMemcpyAsync(&n, g_counter, sizeof(uint32_t), cudaMemcpyDeviceToHost, st), "count");
          check(cudaStreamSynchronize(st), "dump follow");
          if (n > cap) {
            std::fprintf(stderr, "dump: %u particles above the model's %u\n", n, cap);
            std::_Exit(3);
          }
          if (n) velocity_kernel<<<(n + 127) / 128, 128, 0, st>>>(e->partition_[r], g_grid, n, d_attr, nattr, d_v);
          check(cudaGetLastError(), "velocity");
          check(cudaStreamSynchronize(st), "velocity sync");
          std::vector<uint32_t> id(n);
          std::vector<int32_t> key(3 * static_cast<size_t>(n));
          std::vector<float> attr(static_cast<size_t>(nattr) * n), v(3 * static_cast<size_t>(n));
          check(cudaMemcpy(id.data(), d_id, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost), "d2h");
          check(cudaMemcpy(key.data(), d_key, sizeof(int32_t) * key.size(), cudaMemcpyDeviceToHost), "d2h");
          check(cudaMemcpy(attr.data(), d_attr, sizeof(float) * attr.size(), cudaMemcpyDeviceToHost), "d2h");
          check(cudaMemcpy(v.data(), d_v, sizeof(float) * v.size(), cudaMemcpyDeviceToHost), "d2h");
          cudaFree(d_id);
          cudaFree(d_key);
          cudaFree(d_attr);
          cudaFree(d_v);
          std::ofstream f(g_outdir + "/state_m" + std::to_string(i) + tag, std::ios::binary);
          const uint32_t hdr[2] = {n, static_cast<uint32_t>(nattr)};
          f.write(reinterpret_cast<const char*>(hdr), sizeof(hdr));
          write_raw(f, id);
          write_raw(f, key);
          write_raw(f, attr);
          write_raw(f, v);
        },
        e->particleBuffer_[r][i]);
  }
  std::ofstream f(g_outdir + "/sets" + tag, std::ios::binary);
  const uint32_t hdr[5] = {static_cast<uint32_t>(K), na, nn, ne, static_cast<uint32_t>(g_ids.size())};
  f.write(reinterpret_cast<const char*>(hdr), sizeof(hdr));
  write_raw(f, keys);
  write_raw(f, counts);
}

// After InitialSetup: ids of the initial particle entries, the K = 0 dump, and the ids of the
// entries the first substep writes.
void begin(Engine* e, const std::vector<uint64_t>& ks, const std::string& outdir) {
  g_ks = ks;
  g_outdir = outdir;
  g_active = true;
  cudaStream_t st = CudaUtil::GetCudaContext().GetComputeStream();
  check(cudaMalloc(&g_counter, sizeof(uint32_t)), "alloc");
  check(cudaMalloc(&g_maxv, sizeof(float)), "alloc");
  g_grid.Allocate(CudaDefaultAllocator{}, harness::kMaxBlocks);
  const uint32_t r = e->GetRollIndex();
  const uint32_t na = e->activePartitionBlockCount_;
  for (size_t i = 0; i < e->particleBuffer_[r].size(); ++i) {
    std::array<uint32_t*, 2> ids{};
    for (int b = 0; b < 2; ++b) {
      const size_t cap = std::visit([](auto&& buf) { return buf.particleBufferCapacity_; }, e->particleBuffer_[b][i]);
      check(cudaMalloc(&ids[b], sizeof(uint32_t) * cap), "alloc ids");
      check(cudaMemset(ids[b], 0xFF, sizeof(uint32_t) * cap), "memset ids");
    }
    g_ids.push_back(ids);
    std::visit(
        [&](auto&& buf) -> void {
          using B = std::decay_t<decltype(buf)>;
          if (na) initial_ids_kernel<B><<<na, 128, 0, st>>>(buf, na, g_ids[i][r]);
        },
        e->particleBuffer_[r][i]);
  }
  check(cudaGetLastError(), "initial ids");
  check(cudaStreamSynchronize(st), "initial ids sync");
  while (g_next < g_ks.size() && g_ks[g_next] == 0) {
    dump_at(e, 0, 0.0);  // the first substep advects with dt = 0 (include/mpm_engine.cuh:479-480)
    ++g_next;
  }
  if (g_next == g_ks.size()) std::_Exit(0);
  step_ids(e);
}

}  // namespace dump

namespace harness {

// Called by Simulate at the end of every substep, after its rebinning and roll.
void on_substep() {
  if (!dump::g_active) return;
  auto* e = dump::Engine::GetInstance();
  ++dump::g_substeps;
  if (dump::g_next < dump::g_ks.size() && dump::g_ks[dump::g_next] == dump::g_substeps) {
    dump::dump_at(e, dump::g_substeps, static_cast<double>(e->dt_));
    ++dump::g_next;
    if (dump::g_next == dump::g_ks.size()) {
      std::fflush(stdout);
      std::_Exit(0);
    }
  }
  dump::step_ids(e);
}

// Host time from before Initialize to the end of Simulate (which ends the process).
inline std::chrono::steady_clock::time_point g_e2e_start;
void print_e2e() {
  const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - g_e2e_start).count();
  std::printf("HARNESS e2e %.9f\n", s);
  std::fflush(stdout);
}

}  // namespace harness

int main(int argc, char** argv) {
  using namespace harness;
  if (argc != 7 && argc != 8) {
    std::fprintf(stderr, "usage: %s manifest fps frames dt outdir mode [K1,K2,...]\n", argv[0]);
    return 2;
  }
  g_fps = static_cast<uint32_t>(std::strtoul(argv[2], nullptr, 10));
  g_frames = static_cast<uint32_t>(std::strtoul(argv[3], nullptr, 10));
  g_dt = std::strtof(argv[4], nullptr);
  const std::string outdir = argv[5];
  const int mode = std::atoi(argv[6]);

  using namespace mpm;
  std::vector<MPMModelVariant> models;
  std::vector<std::vector<Vector<float, 3>>> xs, vs;  // kept alive: MPMModel copies them, spans must be valid
  std::ifstream manifest(argv[1]);
  std::string line;
  while (std::getline(manifest, line)) {
    if (line.empty()) continue;
    std::istringstream in(line);
    std::string mat, xf, vf;
    float p[8], mass, volume;
    in >> mat;
    for (float& q : p) in >> q;
    in >> mass >> volume >> xf >> vf;
    xs.push_back(read_xyz(xf.c_str()));
    vs.push_back(read_xyz(vf.c_str()));
    const auto xspan = std::span<const Vector<float, 3>>(xs.back());
    const auto vspan = std::span<const Vector<float, 3>>(vs.back());
    if (mat == "fc") {
      using M = MPMMaterial<MPMConstitutiveModel::kFixedCorotated>;
      models.emplace_back(MPMModel<M>{mass, volume, xspan, vspan, M{M::MaterialParameter_{p[0], p[1]}}});
    } else if (mat == "dp") {
      using M = MPMMaterial<MPMConstitutiveModel::kDruckerPragerStvkhencky>;
      models.emplace_back(MPMModel<M>{mass, volume, xspan, vspan, M{M::MaterialParameter_{p[0], p[1]}}});
    } else if (mat == "linear") {
      using M = MPMMaterial<MPMConstitutiveModel::kLinear>;
      models.emplace_back(MPMModel<M>{mass, volume, xspan, vspan, M{M::MaterialParameter_{p[0], p[1]}}});
    } else if (mat == "vm") {
      using M = MPMMaterial<MPMConstitutiveModel::kVonMises>;
      models.emplace_back(MPMModel<M>{mass, volume, xspan, vspan, M{M::MaterialParameter_{p[0], p[1], p[2]}}});
    } else if (mat == "nacc") {
      using M = MPMMaterial<MPMConstitutiveModel::kNonAssociatedCamClay>;
      models.emplace_back(
          MPMModel<M>{mass, volume, xspan, vspan, M{M::MaterialParameter_{p[0], p[1], p[2], p[3], p[4], p[5], p[6] != 0.f}}});
    } else {
      using M = MPMMaterial<MPMConstitutiveModel::kFluid>;
      models.emplace_back(MPMModel<M>{mass, volume, xspan, vspan, M{M::MaterialParameter_{p[0], p[1], p[2], p[3]}}});
    }
  }
  if (models.empty()) {
    std::fprintf(stderr, "empty manifest\n");
    return 2;
  }
  std::vector<uint64_t> ks;
  if (mode == 2) {
    if (argc != 8) {
      std::fprintf(stderr, "mode 2 needs the substep counts to dump at\n");
      return 2;
    }
    std::istringstream in(argv[7]);
    std::string tok;
    while (std::getline(in, tok, ',')) ks.push_back(std::strtoull(tok.c_str(), nullptr, 10));
    std::sort(ks.begin(), ks.end());
    if (ks.empty()) return 2;
  }
  Config config;
  auto* engine = MPMEngine<GridConfig>::GetInstance();
  // The CUDA context exists before the end-to-end timer starts.
  CudaUtil::GetCudaContext().SetContext();
  cudaFree(nullptr);
  g_e2e_start = std::chrono::steady_clock::now();
  if (mode == 1) std::atexit(print_e2e);
  engine->Initialize(config);
  engine->InitializeParticle(config, models);
  engine->InitialSetup(config);
  if (mode == 2) dump::begin(engine, ks, outdir);
  // Simulate ends the process itself (include/mpm_engine.cuh:908).
  engine->Simulate(config, outdir, false, mode == 0, mode == 1 || mode == 2);
  return 0;
}
