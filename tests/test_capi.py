"""The C-ABI library builds, loads and exports every symbol include/ckmpm.h declares.

No compute calls: these run without a GPU.
"""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest
import torch

from ckmpm_b200 import _capi as capi
from ckmpm_b200 import scenes

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols() -> set[str]:
    text = (ROOT / "include" / "ckmpm.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(ckmpm_[a-z_0-9]+)\s*\(", text))


def test_header_declares_the_python_binding_surface():
    assert declared_symbols() == set(capi.EXPORTED)


def test_library_exports_every_declared_symbol(engine_lib):
    nm = subprocess.run(["nm", "-D", "--defined-only", str(capi.LIB_PATH)], capture_output=True, text=True,
                        check=True).stdout
    exported = set(re.findall(r"\bT (ckmpm_[a-z_0-9]+)$", nm, flags=re.M))
    missing = declared_symbols() - exported
    assert not missing, missing
    for name in declared_symbols():
        assert hasattr(engine_lib, name)


def test_version_string(engine_lib):
    assert engine_lib.ckmpm_version().decode().startswith("ckmpm-b200")


def test_null_arguments_are_rejected_without_a_device(engine_lib):
    h = C.c_void_p()
    assert engine_lib.ckmpm_create(None, C.byref(h)) == 1
    assert engine_lib.ckmpm_setup(None) == 1
    assert engine_lib.ckmpm_step(None, 1, C.c_float(1e-4)) == 1
    assert engine_lib.ckmpm_destroy(None) == 0


def test_scene_descriptor_is_checked_before_any_device_call(engine_lib):
    """ckmpm_create / ckmpm_create_batch refuse a malformed descriptor with CKMPM_ERR_INVALID and a
    message, before they look for a device; with no device a valid descriptor fails with
    CKMPM_ERR_CUDA (there is no CPU path to fall back to)."""
    def desc(**kw):
        d = scenes.jelly_cube()[0].to_c()
        for k, v in kw.items():
            if k == "domain_blocks":
                for a in range(3):
                    d.domain_blocks[a] = v[a]
            else:
                setattr(d, k, v)
        return d

    bad = [(dict(dx=0.0), "dx"), (dict(dx=-1.0), "dx"), (dict(domain_blocks=(0, 16, 16)), "domain_blocks"),
           (dict(domain_blocks=(4097, 16, 16)), "domain_blocks"),
           (dict(domain_blocks=(4096, 4096, 32)), "too large"), (dict(boundary=9), "boundary"),
           (dict(max_particles_per_block=4097), "4096")]
    for kw, word in bad:
        h = C.c_void_p()
        d = desc(**kw)
        assert engine_lib.ckmpm_create(C.byref(d), C.byref(h)) == capi.CKMPM_ERR_INVALID, kw
        assert not h
        assert word in engine_lib.ckmpm_last_error(None).decode(), (kw, engine_lib.ckmpm_last_error(None))
    h = C.c_void_p()
    d = desc()
    assert engine_lib.ckmpm_create_batch(C.byref(d), 0, C.byref(h)) == capi.CKMPM_ERR_INVALID
    if not torch.cuda.is_available():
        assert engine_lib.ckmpm_create(C.byref(d), C.byref(h)) == 2  # CKMPM_ERR_CUDA
        assert not h and "no CUDA device" in engine_lib.ckmpm_last_error(None).decode()
    else:
        pytest.skip("a device is present: the no-device answer is not testable here")


def test_header_compiles_as_c():
    src = '#include "ckmpm.h"\nint main(void){ ckmpm_scene_desc d; (void)d; return (int)CKMPM_OK; }\n'
    out = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", str(ROOT / "include"), "-x", "c", "-",
                          "-fsyntax-only"], input=src, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr


def test_cpp_shim_compiles_with_every_material():
    """include/ckmpm/mpm_engine.hpp (the reference-shaped C++ API) builds with a
    plain host compiler, maps each MPMMaterial factory onto ckmpm_material and
    carries the rigid-particle and boundary hooks."""
    src = """#include "ckmpm/mpm_engine.hpp"
int main() {
  using ckmpm::MPMMaterial;
  const MPMMaterial all[] = {MPMMaterial::FixedCorotated(1, 2), MPMMaterial::Linear(1, 2),
                             MPMMaterial::DruckerPrager(1, 2), MPMMaterial::Fluid(1, 7.15f, 0.1f),
                             MPMMaterial::VonMises(2, 1, 3), MPMMaterial::NonAssociatedCamClay(2, 1, -0.01f, 0.5f, 0.8f, 2.36f, true)};
  const int kinds[] = {CKMPM_FIXED_COROTATED, CKMPM_LINEAR, CKMPM_DRUCKER_PRAGER, CKMPM_FLUID, CKMPM_VON_MISES, CKMPM_NACC};
  for (int i = 0; i < 6; ++i) if (all[i].c().kind != kinds[i]) return 1;
  ckmpm::MPMConfig cfg;  // the rigid-particle hooks as run-time fields
  cfg.existRigidParticle = true;
  cfg.rigidParticleCount = 16;
  cfg.rigidParticleVelocity = [](int frame) { return ckmpm::Vector3{1.f, 0.f, static_cast<float>(frame)}; };
  if (!cfg.GetExistRigidParticle() || cfg.GetRigidParticleVelocity(2)[2] != 2.f) return 1;
  cfg.boundary = CKMPM_BOUNDARY_FIELD;  // the irregular-boundary hook as per-cell rules
  cfg.boundaryRule.assign(64 * 64 * 64, static_cast<uint8_t>(CKMPM_CELL_SLIP));
  cfg.boundaryParam.assign(3 * 64 * 64 * 64, 0.f);
  auto referenceCall = [](ckmpm::MPMEngine& e, const ckmpm::MPMConfig& c) {  // the reference's Simulate signature
    return e.Simulate(c, std::string("out"), true, true, false);
  };
  (void)referenceCall;
  return all[5].c().p[6] == 1.f ? 0 : 1;
}
"""
    out = subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", str(ROOT / "include"), "-x", "c++", "-",
                          "-fsyntax-only"], input=src, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
