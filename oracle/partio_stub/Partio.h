// TEST INFRASTRUCTURE ONLY.  A do-nothing stand-in for the Partio particle-IO
// library, which the reference includes only for its .bgeo frame exporter
// (include/mpm_io.h:15-16,67-157) and whose submodule is empty.  It provides the
// handful of names that exporter uses; nothing is ever written.  Positions are
// taken from the reference's raw binary export instead.
#pragma once

#include <cstddef>

namespace Partio {

enum ParticleAttributeType { NONE = 0, VECTOR = 1, FLOAT = 2, INT = 3 };

struct ParticleAttribute {
  int index = 0;
};

class ParticlesDataMutable {
 public:
  ParticleAttribute addAttribute(const char*, ParticleAttributeType, int) { return ParticleAttribute{}; }
  int addParticles(std::size_t) { return 0; }
  template <typename T>
  T* dataWrite(const ParticleAttribute&, int) {
    return reinterpret_cast<T*>(scratch_);
  }
  void release() { delete this; }

 private:
  double scratch_[8] = {};
};

inline ParticlesDataMutable* create() { return new ParticlesDataMutable(); }

inline void write(const char*, const ParticlesDataMutable&) {}

}  // namespace Partio
