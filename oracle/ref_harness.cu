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
// Usage: ref_<scene> <manifest> <fps> <frames> <dt> <outdir> <mode>
//   manifest: one model per line: <material> <p0> ... <p7> <mass> <volume> <x.bin> <v.bin>
//   material and parameters, in the field order of each MaterialParameter_
//   (include/mpm_material.cuh:24-257): fc | dp | linear: lambda mu; fluid: bulk
//   gamma viscosity J0; vm: mu lambda yield; nacc: mu lambda alpha0 beta
//   hardeningFactor M hardeningOn
//   x.bin / v.bin: float32 xyz triples (v.bin holds 1 or n velocities)
//   mode 0: export raw positions every frame (outdir/model_0_particle_frame_<k>.txt)
//   mode 1: profile mode, no export; the reference prints its MPMBenchmark statistics
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <span>
#include <string>
#include <vector>

#include "mpm_engine.cuh"

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
  MPM_FORCE_INLINE MPM_HOST_DEV_FUNC auto UpdateConfigImpl(float, int) -> void {}
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

int main(int argc, char** argv) {
  using namespace harness;
  if (argc != 7) {
    std::fprintf(stderr, "usage: %s manifest fps frames dt outdir mode\n", argv[0]);
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
  Config config;
  auto* engine = MPMEngine<GridConfig>::GetInstance();
  engine->Initialize(config);
  engine->InitializeParticle(config, models);
  engine->InitialSetup(config);
  // Simulate ends the process itself (include/mpm_engine.cuh:908).
  engine->Simulate(config, outdir, false, mode == 0, mode == 1);
  return 0;
}
