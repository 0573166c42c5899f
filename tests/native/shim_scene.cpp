// A scene written the way the reference's scene executables are
// (tests/fluid_dam_break/test_fluid_dam_break.cu:5-18: Initialize ->
// InitializeParticle -> InitialSetup -> Simulate), against the C++ shim
// include/ckmpm/mpm_engine.hpp and the engine library, with a plain host
// compiler.  Used by tests/test_gpu_cpp_shim.py.
//
// usage: shim_scene <x.bin> <out.bin> <mass> <volume> <lambda> <mu> <frames> [rigid_count [export_dir]]
//   x.bin: float32 xyz triples; the cube falls with v0 = (0, -1, 0) on the
//   1/64 grid (16^3 blocks, sticky walls), dt = 2^-14, 1024 frames per second.
//   With rigid_count > 0 the model is von Mises (mu, lambda, yield 100) and its
//   first rigid_count particles are rigid with velocity (1, 0.5 frame, 0).
//   out.bin: positions after the last frame (input order).  With export_dir the
//   scene calls the reference's own Simulate signature, writing per-frame raw
//   positions and the per-substep conservation metric there.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <vector>

#include "ckmpm/mpm_engine.hpp"

int main(int argc, char** argv) {
  if (argc < 8) {
    std::fprintf(stderr, "usage: %s x.bin out.bin mass volume lambda mu frames [rigid_count]\n", argv[0]);
    return 2;
  }
  std::ifstream in(argv[1], std::ios::binary | std::ios::ate);
  const size_t bytes = static_cast<size_t>(in.tellg());
  in.seekg(0);
  std::vector<ckmpm::Vector3> x(bytes / 12);
  in.read(reinterpret_cast<char*>(x.data()), static_cast<std::streamsize>(x.size() * 12));
  const float mass = std::strtof(argv[3], nullptr), volume = std::strtof(argv[4], nullptr);
  const float lambda = std::strtof(argv[5], nullptr), mu = std::strtof(argv[6], nullptr);
  const uint32_t frames = static_cast<uint32_t>(std::strtoul(argv[7], nullptr, 10));
  const uint32_t rigid = argc > 8 ? static_cast<uint32_t>(std::strtoul(argv[8], nullptr, 10)) : 0u;
  const char* exportDir = argc > 9 ? argv[9] : nullptr;

  ckmpm::MPMConfig config;
  config.dx = 1.f / 64.f;
  config.domainBlocks = {16, 16, 16};
  config.dt = 1.f / 16384.f;
  config.fps = 1024;
  config.totalFrames = frames;
  ckmpm::MPMMaterial material = ckmpm::MPMMaterial::FixedCorotated(lambda, mu);
  if (rigid > 0) {
    material = ckmpm::MPMMaterial::VonMises(mu, lambda, 100.f);
    config.existRigidParticle = true;
    config.rigidParticleCount = rigid;
    config.rigidParticleVelocity = [](int frame) { return ckmpm::Vector3{1.f, 0.5f * static_cast<float>(frame), 0.f}; };
  }
  std::vector<ckmpm::MPMModel> models;
  models.emplace_back(mass, volume, x, std::vector<ckmpm::Vector3>{{0.f, -1.f, 0.f}}, material);

  try {
    ckmpm::MPMEngine simulator;
    simulator.Initialize(config);
    simulator.InitializeParticle(config, models);
    simulator.InitialSetup(config);
    if (exportDir) {  // the reference's call, as in its scene executables
      simulator.Simulate(config, exportDir, true, true, false);
      return 0;
    }
    std::vector<ckmpm::Vector3> last;
    std::array<ckmpm::Vector3, 4> metric{};
    simulator.Simulate(config, [&](uint32_t frame, ckmpm::MPMEngine& e) {
      if (frame + 1 == frames) {
        last = e.GetParticlePosition(0);
        metric = e.GetConservationMetric(0);
      }
    });
    // The Lagrangian momentum of the last frame on stderr, for the test to compare.
    std::fprintf(stderr, "metric %.9g %.9g %.9g %.9g %.9g %.9g\n", metric[2][0], metric[2][1], metric[2][2],
                 metric[3][0], metric[3][1], metric[3][2]);
    std::ofstream out(argv[2], std::ios::binary);
    out.write(reinterpret_cast<const char*>(last.data()), static_cast<std::streamsize>(last.size() * 12));
  } catch (const ckmpm::Error& err) {
    std::fprintf(stderr, "ckmpm error %d: %s\n", static_cast<int>(err.code), err.what());
    return 1;
  }
  return 0;
}
