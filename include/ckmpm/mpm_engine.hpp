// ckmpm/mpm_engine.hpp -- header-only C++ shim over the C ABI (ckmpm.h) that
// keeps the reference's engine/material/model/config names and call order, so
// existing scene code of AppledoreM/CKMPM changes little to run on this engine:
//
//   reference (include/mpm_engine.cuh, include/mpm_model.h, ...)      this shim
//   MPMEngine<GridConfig>::GetInstance()                      ->    ckmpm::MPMEngine (an ordinary object)
//   Initialize(config)            (:171)                      ->    Initialize(config)
//   InitializeParticle(config, models) (:92)                  ->    InitializeParticle(config, models)
//   InitialSetup(config)          (:216)                      ->    InitialSetup(config)
//   Simulate(config, dir, conservation, binary, profile) (:457) ->  the same call, or Simulate(config, export_fn);
//                                                                  both return instead of exiting
//   MPMModel<MPMMaterial<k>>(mass, volume, x, v, material)    ->    ckmpm::MPMModel(mass, volume, x, v, material)
//   MPMConfigBase<Derived> getters (include/mpm_config.h)     ->    ckmpm::MPMConfig (run-time fields, same getters)
//
// Differences are at the boundary only: scene constants are run-time values,
// errors throw ckmpm::Error (the reference calls exit()/abort()), and Simulate
// returns instead of ending the process.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "../ckmpm.h"

namespace ckmpm {

struct Error : std::runtime_error {
  ckmpm_status code;
  Error(ckmpm_status c, const std::string& what) : std::runtime_error(what), code(c) {}
};

inline void check(ckmpm_status s, const ckmpm_scene* h, const char* where) {
  if (s != CKMPM_OK) throw Error(s, std::string(where) + ": " + ckmpm_last_error(h));
}

using Vector3 = std::array<float, 3>;

// ComputeLameParameters (include/mpm_material.cuh:277-283).
inline std::array<float, 2> ComputeLameParameters(float E, float nu) {
  return {E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))};
}

// MPMConstitutiveModel (include/mpm_material.cuh:10-18).
enum class MPMConstitutiveModel : int32_t {
  kFixedCorotated = CKMPM_FIXED_COROTATED,
  kLinear = CKMPM_LINEAR,
  kDruckerPragerStvkhencky = CKMPM_DRUCKER_PRAGER,
  kFluid = CKMPM_FLUID,
  kVonMises = CKMPM_VON_MISES,
  kNonAssociatedCamClay = CKMPM_NACC,
};

// MPMMaterial<k>::MaterialParameter_ collapsed into one run-time value type;
// p holds each model's parameters in its field order (include/mpm_material.cuh:24-257).
struct MPMMaterial {
  MPMConstitutiveModel kind = MPMConstitutiveModel::kFixedCorotated;
  float p[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  static MPMMaterial FixedCorotated(float lambda, float mu) {
    return {MPMConstitutiveModel::kFixedCorotated, {lambda, mu}};
  }
  static MPMMaterial Linear(float lambda, float mu) { return {MPMConstitutiveModel::kLinear, {lambda, mu}}; }
  static MPMMaterial DruckerPrager(float lambda, float mu) {
    return {MPMConstitutiveModel::kDruckerPragerStvkhencky, {lambda, mu}};
  }
  static MPMMaterial Fluid(float bulk, float gamma, float viscosity, float J0 = 1.0f) {
    return {MPMConstitutiveModel::kFluid, {bulk, gamma, viscosity, J0}};
  }
  static MPMMaterial VonMises(float mu, float lambda, float yieldStress) {
    return {MPMConstitutiveModel::kVonMises, {mu, lambda, yieldStress}};
  }
  static MPMMaterial NonAssociatedCamClay(float mu, float lambda, float alpha0, float beta, float hardeningFactor,
                                          float m, bool hardeningOn) {
    return {MPMConstitutiveModel::kNonAssociatedCamClay,
            {mu, lambda, alpha0, beta, hardeningFactor, m, hardeningOn ? 1.f : 0.f}};
  }
  ckmpm_material c() const {
    ckmpm_material m{};
    m.kind = static_cast<int32_t>(kind);
    for (int i = 0; i < 8; ++i) m.p[i] = p[i];
    return m;
  }
};

// MPMModel (include/mpm_model.h:11-59).
class MPMModel {
 public:
  MPMModel(float particleMass, float particleVolume, std::vector<Vector3> particlePosition,
           std::vector<Vector3> particleVelocity, MPMMaterial material, double freezeTime = 0.0)
      : mass_(particleMass), volume_(particleVolume), x_(std::move(particlePosition)),
        v_(std::move(particleVelocity)), material_(material), freeze_(freezeTime) {
    if (v_.size() != 1 && v_.size() != x_.size())
      throw Error(CKMPM_ERR_INVALID, "particle velocity must hold 1 or n entries");
  }
  float GetParticleMass() const { return mass_; }
  float GetParticleVolume() const { return volume_; }
  uint32_t GetParticleCount() const { return static_cast<uint32_t>(x_.size()); }
  const MPMMaterial& GetParticleMaterial() const { return material_; }
  const std::vector<Vector3>& GetParticlePosition() const { return x_; }
  const std::vector<Vector3>& GetParticleVelocity() const { return v_; }
  bool IsFreezed(double elapsedSeconds) const { return elapsedSeconds < freeze_; }

 private:
  float mass_, volume_;
  std::vector<Vector3> x_, v_;
  MPMMaterial material_;
  double freeze_;
};

// MPMConfigBase getters as run-time fields (include/mpm_config.h:17-123).
struct MPMConfig {
  float dx = 1.f / 64.f;
  std::array<int32_t, 3> domainBlocks = {16, 16, 16};  // MPMDomainRange<Bx, By, Bz>
  float gravity = -9.8f;
  float massClamp = 0.f;
  float dt = 1e-4f;
  float cfl = 0.5f;
  uint32_t fps = 48;
  uint32_t totalFrames = 1;
  ckmpm_boundary_kind boundary = CKMPM_BOUNDARY_STICKY_BLOCKS;
  float floorCells = 8.f;
  uint32_t maxParticleCountPerBlock = 4096;
  bool trackIds = true;
  int32_t device = 0;
  // Rigid particles (GetExistRigidParticle / GetRigidParticleCount /
  // GetRigidParticleVelocity(frame), include/mpm_config.h:92-106).
  bool existRigidParticle = false;
  uint32_t rigidParticleCount = 0;
  std::function<Vector3(int)> rigidParticleVelocity = [](int) { return Vector3{0.f, 0.f, 0.f}; };
  // boundary == CKMPM_BOUNDARY_FIELD: the irregular-boundary hook (GetExistIrregularBoundary /
  // ProcessGridCellVelocity, include/mpm_config.h:108-117) as one ckmpm_cell_rule per cell
  // (x-major over 4 * domainBlocks cells per axis) and 3 floats per cell.
  std::vector<uint8_t> boundaryRule;
  std::vector<float> boundaryParam;

  float GetDx() const { return dx; }
  float GetInvDx() const { return 1.f / dx; }
  uint32_t GetBlockSize() const { return 4; }
  uint32_t GetBlockVolume() const { return 64; }
  uint32_t GetMaxParticleCountPerBlock() const { return maxParticleCountPerBlock; }
  uint32_t GetFps() const { return fps; }
  float GetDt() const { return dt; }
  float GetCfl() const { return cfl; }
  uint32_t GetTotalSimulatedFrameCount() const { return totalFrames; }
  float GetGravity() const { return gravity; }
  float GetMassClamp() const { return massClamp; }
  bool GetExistRigidParticle() const { return existRigidParticle; }
  uint32_t GetRigidParticleCount() const { return rigidParticleCount; }
  Vector3 GetRigidParticleVelocity(int frame) const { return rigidParticleVelocity(frame); }

  ckmpm_scene_desc c() const {
    ckmpm_scene_desc d{};
    d.dx = dx;
    for (int i = 0; i < 3; ++i) d.domain_blocks[i] = domainBlocks[i];
    d.gravity = gravity;
    d.mass_clamp = massClamp;
    d.boundary = boundary;
    d.floor_cells = floorCells;
    d.max_particles_per_block = maxParticleCountPerBlock;
    d.device = device;
    d.flags = trackIds ? CKMPM_FLAG_TRACK_IDS : 0u;
    return d;
  }
};

// MPMEngine (include/mpm_engine.cuh:29-974) with the same call order.
class MPMEngine {
 public:
  MPMEngine() = default;
  MPMEngine(const MPMEngine&) = delete;
  MPMEngine& operator=(const MPMEngine&) = delete;
  ~MPMEngine() {
    if (scene_) ckmpm_destroy(scene_);
  }

  // Initialize: dt = min(config dt, 1 / fps) (include/mpm_engine.cuh:178).
  void Initialize(const MPMConfig& config) {
    const ckmpm_scene_desc d = config.c();
    check(ckmpm_create(&d, &scene_), nullptr, "ckmpm_create");
    dt_ = std::min(config.GetDt(), 1.0f / static_cast<float>(config.GetFps()));
    if (config.GetExistRigidParticle()) {
      const Vector3 v = config.GetRigidParticleVelocity(0);
      check(ckmpm_set_rigid(scene_, config.GetRigidParticleCount(), v.data()), scene_, "ckmpm_set_rigid");
    }
    if (config.boundary == CKMPM_BOUNDARY_FIELD && !config.boundaryRule.empty())
      check(ckmpm_set_boundary_field(scene_, config.boundaryRule.data(),
                                     config.boundaryParam.empty() ? nullptr : config.boundaryParam.data()),
            scene_, "ckmpm_set_boundary_field");
  }

  // InitializeParticle: one engine model per MPMModel; dt shrinks by the CFL
  // bound of the initial velocities (include/mpm_engine.cuh:109-117).
  void InitializeParticle(const MPMConfig& config, const std::vector<MPMModel>& models) {
    for (const auto& m : models) {
      float vmax = 0.f;
      for (const auto& v : m.GetParticleVelocity()) vmax = std::max(vmax, std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
      if (vmax > 0.f) dt_ = std::min(dt_, config.GetDx() * config.GetCfl() / vmax);
      const ckmpm_material mat = m.GetParticleMaterial().c();
      int32_t idx = 0;
      check(ckmpm_add_model(scene_, &mat, m.GetParticleCount(), m.GetParticlePosition()[0].data(),
                            m.GetParticleVelocity()[0].data(), static_cast<uint32_t>(m.GetParticleVelocity().size()),
                            m.GetParticleMass(), m.GetParticleVolume(), &idx),
            scene_, "ckmpm_add_model");
      counts_.push_back(m.GetParticleCount());
    }
  }

  void InitialSetup(const MPMConfig&) { check(ckmpm_setup(scene_), scene_, "ckmpm_setup"); }

  // Simulate: GetTotalSimulatedFrameCount() frames; every substep takes
  // nextDt = min(dt_, time left in the frame, dx cfl / max|v|) on the device
  // (include/mpm_engine.cuh:514-557); export(frame, engine) runs after every
  // frame (the ExportParticleToModel point, :880-883).  Returns the simulated
  // time instead of ending the process.
  double Simulate(const MPMConfig& config, const std::function<void(uint32_t, MPMEngine&)>& exportFrame = {}) {
    double total = 0.0;
    for (uint32_t f = 0; f < config.GetTotalSimulatedFrameCount(); ++f) {
      if (config.GetExistRigidParticle()) {  // the hook is evaluated per frame (include/mpm_algorithm.cuh:1614)
        const Vector3 v = config.GetRigidParticleVelocity(static_cast<int>(f));
        check(ckmpm_set_rigid_velocity(scene_, v.data()), scene_, "ckmpm_set_rigid_velocity");
      }
      double elapsed = 0.0;
      check(ckmpm_step_adaptive(scene_, 1u << 30, dt_, config.GetCfl(), 1.0 / config.GetFps(), &elapsed), scene_,
            "ckmpm_step_adaptive");
      total += elapsed;
      if (exportFrame) exportFrame(f, *this);
    }
    return total;
  }

  // The reference's own signature, Simulate(config, exportRootPath,
  // collectConservationMetric, exportParticlePositionAsBinary, profileMode)
  // (include/mpm_engine.cuh:457-909), so scene code calls it unchanged:
  //  * exportParticlePositionAsBinary: after every frame, each model's positions as
  //    raw float32 xyz in <root>/model_<i>_particle_frame_<frame>.txt (:433-444);
  //    without it the reference writes Partio .bgeo files, which are not written here;
  //  * collectConservationMetric: before every substep, one record of 13 float32
  //    (time, Eulerian linear and angular momentum (zero), Lagrangian sum(v) and
  //    sum(x cross v)) per model in <root>/conservationMetric_model_<i>.bin (:494-603),
  //    stepping one substep at a time;
  //  * profileMode: no export.
  // Returns the simulated time (the reference ends the process).
  double Simulate(const MPMConfig& config, const std::string& exportRootPath, bool collectConservationMetric,
                  bool exportParticlePositionAsBinary, bool profileMode) {
    const bool metric = collectConservationMetric && !profileMode;
    const bool binary = exportParticlePositionAsBinary && !profileMode;
    const size_t nmodels = counts_.size();
    std::vector<FILE*> metricFiles;
    if (metric)
      for (size_t i = 0; i < nmodels; ++i) {
        const std::string path = exportRootPath + "/conservationMetric_model_" + std::to_string(i) + ".bin";
        FILE* f = std::fopen(path.c_str(), "wb");
        if (!f) {
          for (FILE* g : metricFiles) std::fclose(g);
          throw Error(CKMPM_ERR_INVALID, "cannot open " + path);
        }
        metricFiles.push_back(f);
      }
    auto record = [&]() {
      const double t = GetTime()[0];
      for (size_t i = 0; i < nmodels; ++i) {
        const std::array<Vector3, 4> m = GetConservationMetric(static_cast<int32_t>(i));
        float row[13] = {static_cast<float>(t)};
        for (int r = 0; r < 4; ++r)
          for (int k = 0; k < 3; ++k) row[1 + 3 * r + k] = m[r][k];
        std::fwrite(row, sizeof(float), 13, metricFiles[i]);
      }
    };
    double total = 0.0;
    try {
      for (uint32_t f = 0; f < config.GetTotalSimulatedFrameCount(); ++f) {
        if (config.GetExistRigidParticle()) {
          const Vector3 v = config.GetRigidParticleVelocity(static_cast<int>(f));
          check(ckmpm_set_rigid_velocity(scene_, v.data()), scene_, "ckmpm_set_rigid_velocity");
        }
        double frameTime = 1.0 / config.GetFps();
        for (;;) {
          if (metric) record();
          double elapsed = 0.0;
          check(ckmpm_step_adaptive(scene_, metric ? 1u : (1u << 30), dt_, config.GetCfl(), frameTime, &elapsed),
                scene_, "ckmpm_step_adaptive");
          total += elapsed;
          frameTime = 0.0;  // later calls continue this frame
          const std::array<double, 2> t = GetTime();
          if (!metric || !(t[1] - t[0] > 0.0)) break;
        }
        if (binary)
          for (size_t i = 0; i < nmodels; ++i) {
            const std::vector<Vector3> x = GetParticlePosition(static_cast<int32_t>(i));
            const std::string path = exportRootPath + "/model_" + std::to_string(i) + "_particle_frame_" +
                                     std::to_string(f) + ".txt";
            FILE* out = std::fopen(path.c_str(), "wb");
            if (!out) throw Error(CKMPM_ERR_INVALID, "cannot open " + path);
            std::fwrite(x.data(), sizeof(float), 3 * x.size(), out);
            std::fclose(out);
          }
      }
    } catch (...) {
      for (FILE* g : metricFiles) std::fclose(g);
      throw;
    }
    for (FILE* g : metricFiles) std::fclose(g);
    return total;
  }

  // Positions of a model (input order when ids are tracked), the export path's
  // RetrieveParticleBuffer + copy (include/mpm_engine.cuh:386-454).
  std::vector<Vector3> GetParticlePosition(int32_t model) {
    uint32_t n = 0;
    check(ckmpm_get_count(scene_, model, &n), scene_, "ckmpm_get_count");
    std::vector<Vector3> x(n);
    uint32_t out = 0;
    check(ckmpm_get_state(scene_, model, n ? x[0].data() : nullptr, nullptr, nullptr, nullptr, nullptr, n, &out),
          scene_, "ckmpm_get_state");
    return x;
  }

  // Full per-particle state of a model in input order when ids are tracked:
  // x, v (the velocity the next G2P interpolates), F (row-major 3x3) and aux
  // (J, logJp or the rigid flag), as ckmpm_get_state returns them.
  struct ParticleState {
    std::vector<Vector3> x, v;
    std::vector<std::array<float, 9>> F;
    std::vector<float> aux;
  };
  ParticleState GetParticleState(int32_t model) {
    uint32_t n = 0;
    check(ckmpm_get_count(scene_, model, &n), scene_, "ckmpm_get_count");
    ParticleState st;
    st.x.resize(n);
    st.v.resize(n);
    st.F.resize(n);
    st.aux.resize(n);
    uint32_t out = 0;
    if (n)
      check(ckmpm_get_state(scene_, model, st.x[0].data(), st.v[0].data(), st.F[0].data(), st.aux.data(), nullptr, n,
                            &out),
            scene_, "ckmpm_get_state");
    return st;
  }

  // The reference's conservation metric of one model (CollectConservationMetric,
  // include/mpm_algorithm.cuh:1082-1361): rows Eulerian linear and angular
  // momentum (zero, as the reference leaves them), Lagrangian sum(v) and
  // sum(x cross v), per unit particle mass, summed in double.
  std::array<Vector3, 4> GetConservationMetric(int32_t model) {
    const ParticleState st = GetParticleState(model);
    double l[3] = {0, 0, 0}, a[3] = {0, 0, 0};
    for (size_t i = 0; i < st.x.size(); ++i) {
      const auto& x = st.x[i];
      const auto& v = st.v[i];
      for (int k = 0; k < 3; ++k) l[k] += v[k];
      a[0] += static_cast<double>(x[1]) * v[2] - static_cast<double>(x[2]) * v[1];
      a[1] += static_cast<double>(x[2]) * v[0] - static_cast<double>(x[0]) * v[2];
      a[2] += static_cast<double>(x[0]) * v[1] - static_cast<double>(x[1]) * v[0];
    }
    std::array<Vector3, 4> m{};
    for (int k = 0; k < 3; ++k) {
      m[2][k] = static_cast<float>(l[k]);
      m[3][k] = static_cast<float>(a[k]);
    }
    return m;
  }

  // Simulated time (double) and the end of the current adaptive frame.
  std::array<double, 2> GetTime() {
    std::array<double, 2> t{};
    check(ckmpm_get_time(scene_, t.data()), scene_, "ckmpm_get_time");
    return t;
  }

  float GetDt() const { return dt_; }
  ckmpm_scene* Handle() { return scene_; }

 private:
  ckmpm_scene* scene_ = nullptr;
  float dt_ = 0.f;
  std::vector<uint32_t> counts_;
};

}  // namespace ckmpm
