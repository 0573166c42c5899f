"""ckmpm_simulate_noalloc: the allocation-free entry point, checked against the allocating path.

Callers that cannot allocate device memory -- code running inside another
framework's CUDA-graph capture, plugins whose host owns the memory budget,
real-time loops that cannot take the synchronisation of a cudaMalloc -- use
ckmpm_simulate_noalloc, which keeps all its scratch in one fixed device array.
These tests call it through the C ABI twice in a row on the same inputs and
compare each result with ckmpm_create / ckmpm_add_model / ckmpm_setup /
ckmpm_step / ckmpm_get_state, within the parity tolerances of
tests/test_gpu_engine.py (positions 2e-6, F 5e-5, velocities 1e-4 x max|v|).
This file runs last so that, if it fails, every other test has already run.
"""
import ctypes as C

import numpy as np
import pytest

from ckmpm_b200 import Scene, scenes
from ckmpm_b200 import _capi as capi

pytestmark = pytest.mark.gpu

X_TOL = 2e-6
F_TOL = 5e-5
V_REL = 1e-4


def _noalloc(lib, cfg, model, nsteps, dt, torch):
    dev = torch.device("cuda", cfg.device)
    x = torch.from_numpy(np.ascontiguousarray(model.particle_position)).to(dev)
    v = torch.from_numpy(np.ascontiguousarray(model.particle_velocity)).to(dev)
    n = x.shape[0]
    xo = torch.zeros((n, 3), dtype=torch.float32, device=dev)
    vo = torch.zeros((n, 3), dtype=torch.float32, device=dev)
    Fo = torch.zeros((n, 3, 3), dtype=torch.float32, device=dev)
    ao = torch.zeros((n,), dtype=torch.float32, device=dev)
    desc = cfg.to_c()
    mat = model.material.to_c()
    nlive = C.c_uint32()
    msg = C.c_char_p()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(dev)[0]
    code = lib.ckmpm_simulate_noalloc(C.byref(desc), C.byref(mat), n, C.c_void_p(x.data_ptr()),
                                      C.c_void_p(v.data_ptr()), v.shape[0], model.particle_mass,
                                      model.particle_volume, nsteps, dt, None, C.c_void_p(xo.data_ptr()),
                                      C.c_void_p(vo.data_ptr()), C.c_void_p(Fo.data_ptr()), C.c_void_p(ao.data_ptr()),
                                      C.byref(nlive), C.byref(msg))
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info(dev)[0]
    return (code, (msg.value or b"").decode(), nlive.value, xo.cpu().numpy(), vo.cpu().numpy(), Fo.cpu().numpy(),
            free_before - free_after)


def test_noalloc_matches_allocating_path_twice(engine_lib):
    torch = pytest.importorskip("torch")
    cfg, models = scenes.jelly_cube(lo=(0.44, 0.44, 0.44), hi=(0.56, 0.56, 0.56), v0=(0.3, -1.0, 0.2))
    nsteps, dt = 24, 1e-4
    s = Scene(cfg)
    s.add_model(models[0])
    s.setup()
    s.step(nsteps, dt)
    ref = s.state(0)
    s.close()
    vtol = V_REL * float(np.abs(ref.v).max()) + 1e-6
    for call in range(2):
        code, msg, nlive, xo, vo, Fo, used = _noalloc(engine_lib, cfg, models[0], nsteps, dt, torch)
        assert code == capi.CKMPM_OK, msg
        assert nlive == len(ref.id)
        assert np.abs(xo[ref.id] - ref.x).max() <= X_TOL
        assert np.abs(Fo[ref.id] - ref.F).max() <= F_TOL
        assert np.abs(vo[ref.id] - ref.v).max() <= vtol
        if call == 1:
            # Inputs and outputs were allocated by the test before the call; the
            # call itself takes no device memory.
            assert used < (1 << 20), used


@pytest.mark.parametrize("kind", ["von_mises", "nacc"])
def test_noalloc_other_materials(engine_lib, kind):
    """The von Mises and NACC cubes through the allocation-free entry point, against the
    allocating path (NACC compared through F F^T, its F being fixed only up to a rotation)."""
    torch = pytest.importorskip("torch")
    cfg, models = scenes.material_cube(kind)
    nsteps, dt = 24, 1e-4
    s = Scene(cfg)
    s.add_model(models[0])
    s.setup()
    s.step(nsteps, dt)
    ref = s.state(0)
    s.close()
    code, msg, nlive, xo, vo, Fo, used = _noalloc(engine_lib, cfg, models[0], nsteps, dt, torch)
    assert code == capi.CKMPM_OK, msg
    assert nlive == len(ref.id)
    assert np.abs(xo[ref.id] - ref.x).max() <= X_TOL
    Fa, Fb = Fo[ref.id].astype(np.float64), ref.F.astype(np.float64)
    if kind == "nacc":
        Fa, Fb = Fa @ Fa.transpose(0, 2, 1), Fb @ Fb.transpose(0, 2, 1)
    assert np.abs(Fa - Fb).max() <= F_TOL
    assert np.abs(vo[ref.id] - ref.v).max() <= V_REL * float(np.abs(ref.v).max()) + 1e-6


def test_noalloc_rejects_sizes_beyond_its_limits(engine_lib):
    torch = pytest.importorskip("torch")
    cfg, models = scenes.jelly_cube(lo=(0.44, 0.44, 0.44), hi=(0.56, 0.56, 0.56))
    big = np.zeros((65537, 3), np.float32) + 0.5
    m = models[0]
    m_big = type(m)(m.particle_mass, m.particle_volume, big, m.particle_velocity, m.material)
    code, msg = _noalloc(engine_lib, cfg, m_big, 1, 1e-4, torch)[:2]
    assert code == 3 and "65536" in msg  # CKMPM_ERR_CAPACITY
    cfg_big, _ = scenes.jelly_cube(dx=1 / 128, lo=(0.44, 0.44, 0.44), hi=(0.56, 0.56, 0.56))  # 32^3 blocks
    code, msg = _noalloc(engine_lib, cfg_big, m, 1, 1e-4, torch)[:2]
    assert code == 3 and "4096" in msg
