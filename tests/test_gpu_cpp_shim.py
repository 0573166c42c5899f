"""A reference-style C++ scene through the header shim (include/ckmpm/mpm_engine.hpp).

tests/native/shim_scene.cpp is written the way the reference's scene
executables are (Initialize -> InitializeParticle -> InitialSetup -> Simulate
with a frame export), compiled here with g++ against include/ and linked to
the engine library.  Its positions after the last frame must equal, bit for
bit, those of the Python MPMEngine running the same configuration: both drive
the same C ABI with the same arguments.  A second run turns the rigid-particle
hooks on (the shim sets the velocity before every frame).
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from ckmpm_b200 import MPMEngine, scenes
from ckmpm_b200 import _capi as capi
from ckmpm_b200.engine import MPMMaterial, MPMModel, compute_lame_parameters

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
E, NU, FRAMES = 5e4, 0.3, 4


@pytest.fixture(scope="module")
def scene_binary(tmp_path_factory, engine_lib):
    out = tmp_path_factory.mktemp("shim") / "shim_scene"
    lib_dir = capi.LIB_PATH.parent
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", str(ROOT / "include"),
           str(ROOT / "tests" / "native" / "shim_scene.cpp"), "-L", str(lib_dir), "-lckmpm_b200",
           f"-Wl,-rpath,{lib_dir}", "-o", str(out)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return out


def python_run(model, rigid: int) -> np.ndarray:
    cfg, _ = scenes.jelly_cube(lo=(0.44, 0.44, 0.44), hi=(0.56, 0.56, 0.56))
    cfg.dt, cfg.fps, cfg.total_frames = 2.0 ** -14, 1024, FRAMES
    if rigid:
        cfg.exist_rigid_particle = True
        cfg.rigid_particle_count = rigid
        cfg.rigid_particle_velocity = lambda frame: (1.0, 0.5 * frame, 0.0)
    frames = {}
    eng = MPMEngine()
    eng.Initialize(cfg)
    eng.InitializeParticle(cfg, [model])
    eng.InitialSetup(cfg)
    eng.Simulate(cfg, export_callback=lambda f, scene: frames.__setitem__(f, scene.state(0).x.copy()))
    return frames[FRAMES - 1], eng.scene.conservation_metric(0)


@pytest.mark.parametrize("rigid", [0, 1500])
def test_cpp_scene_matches_python_engine(scene_binary, tmp_path, rigid):
    _, models = scenes.jelly_cube(lo=(0.44, 0.44, 0.44), hi=(0.56, 0.56, 0.56))
    m = models[0]
    lam, mu = compute_lame_parameters(E, NU)
    lam, mu = float(np.float32(lam)), float(np.float32(mu))
    mat = MPMMaterial.von_mises(mu, lam, 100.0) if rigid else MPMMaterial.fixed_corotated(lam, mu)
    model = MPMModel(m.particle_mass, m.particle_volume, m.particle_position,
                     np.asarray([[0.0, -1.0, 0.0]], np.float32), mat)
    xf, of = tmp_path / "x.bin", tmp_path / "out.bin"
    np.ascontiguousarray(m.particle_position, np.float32).tofile(xf)
    res = subprocess.run([str(scene_binary), str(xf), str(of), f"{m.particle_mass:.9g}", f"{m.particle_volume:.9g}",
                          f"{lam:.9g}", f"{mu:.9g}", str(FRAMES), str(rigid)], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    cpp = np.fromfile(of, np.float32).reshape(-1, 3)
    py, metric = python_run(model, rigid)
    assert cpp.shape == py.shape
    assert np.array_equal(cpp, py), np.abs(cpp - py).max()
    line = [ln for ln in res.stderr.splitlines() if ln.startswith("metric ")][0]
    cpp_metric = np.array([float(t) for t in line.split()[1:]]).reshape(2, 3)
    np.testing.assert_allclose(cpp_metric, metric[2:].astype(np.float32), rtol=1e-6, atol=1e-6)


def test_cpp_scene_reference_simulate_signature(scene_binary, tmp_path):
    """Simulate(config, exportRootPath, collectConservationMetric=true,
    exportParticlePositionAsBinary=true, profileMode=false), the reference's own
    call: per-frame raw position files and a per-substep conservation-metric file
    equal to the Python engine's."""
    from ckmpm_b200 import MPMEngine
    _, models = scenes.jelly_cube(lo=(0.44, 0.44, 0.44), hi=(0.56, 0.56, 0.56))
    m = models[0]
    lam, mu = compute_lame_parameters(E, NU)
    lam, mu = float(np.float32(lam)), float(np.float32(mu))
    xf = tmp_path / "x.bin"
    np.ascontiguousarray(m.particle_position, np.float32).tofile(xf)
    out = tmp_path / "ref_style"
    out.mkdir()
    res = subprocess.run([str(scene_binary), str(xf), str(tmp_path / "unused.bin"), f"{m.particle_mass:.9g}",
                          f"{m.particle_volume:.9g}", f"{lam:.9g}", f"{mu:.9g}", str(FRAMES), "0", str(out)],
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    cfg, _ = scenes.jelly_cube(lo=(0.44, 0.44, 0.44), hi=(0.56, 0.56, 0.56))
    cfg.dt, cfg.fps, cfg.total_frames = 2.0 ** -14, 1024, FRAMES
    model = MPMModel(m.particle_mass, m.particle_volume, m.particle_position,
                     np.asarray([[0.0, -1.0, 0.0]], np.float32), MPMMaterial.fixed_corotated(lam, mu))
    py_root = tmp_path / "py"
    eng = MPMEngine()
    eng.Initialize(cfg)
    eng.InitializeParticle(cfg, [model])
    eng.InitialSetup(cfg)
    eng.Simulate(cfg, export_root=py_root, collect_conservation_metric=True)
    for f in range(FRAMES):
        a = np.fromfile(out / f"model_0_particle_frame_{f}.txt", np.float32)
        b = np.fromfile(py_root / f"model_0_particle_frame_{f}.txt", np.float32)
        assert np.array_equal(a, b), f
    ma = np.fromfile(out / "conservationMetric_model_0.bin", np.float32).reshape(-1, 13)
    mb = np.fromfile(py_root / "conservationMetric_model_0.bin", np.float32).reshape(-1, 13)
    assert ma.shape == mb.shape and ma.shape[0] >= 16 * FRAMES
    np.testing.assert_allclose(ma, mb, rtol=1e-6, atol=1e-6)
