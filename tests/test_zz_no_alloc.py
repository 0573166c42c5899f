"""ckmpm_simulate_noalloc: the allocation-free entry point, checked against the allocating path.

Callers that cannot allocate device memory -- plugins whose host runtime owns
the device memory budget through its own pool, loops that cannot take the
synchronisation of a cudaMalloc -- use ckmpm_simulate_noalloc, which keeps all
its scratch in one fixed device array.  These tests call it through the C ABI
twice in a row on the same inputs and compare each result with ckmpm_create /
ckmpm_add_model / ckmpm_setup / ckmpm_step / ckmpm_get_state, within the parity
tolerances of tests/test_gpu_engine.py (positions 2e-6, F 5e-5, velocities
1e-4 x max|v|), on the legacy default stream and on a caller's stream, for a
sticky-wall solid, a fluid on the slip floor and per-particle velocities.  The
call synchronises its stream, so on a capturing stream it must refuse with
CKMPM_ERR_INVALID.  This file runs last so that, if it fails, every other test
has already run.
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


def _noalloc(lib, cfg, model, nsteps, dt, torch, stream=None):
    """One call; stream: a torch.cuda.Stream to run on (None: the legacy default stream)."""
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
                                      model.particle_volume, nsteps, dt,
                                      C.c_void_p(stream.cuda_stream) if stream is not None else None,
                                      C.c_void_p(xo.data_ptr()),
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


def _allocating(cfg, model, nsteps, dt):
    s = Scene(cfg)
    s.add_model(model)
    s.setup()
    s.step(nsteps, dt)
    ref = s.state(0)
    s.close()
    return ref


def _check(res, ref, check_F=True):
    code, msg, nlive, xo, vo, Fo, used = res
    assert code == capi.CKMPM_OK, msg
    assert nlive == len(ref.id)
    assert np.abs(xo[ref.id] - ref.x).max() <= X_TOL
    if check_F:
        assert np.abs(Fo[ref.id] - ref.F).max() <= F_TOL
    assert np.abs(vo[ref.id] - ref.v).max() <= V_REL * float(np.abs(ref.v).max()) + 1e-6


def test_noalloc_fluid_on_slip_floor_on_a_caller_stream(engine_lib):
    """A J-fluid box thrown onto the slip floor (no F kept: identity written out), run on a
    torch stream the caller owns."""
    import dataclasses
    torch = pytest.importorskip("torch")
    cfg, models = scenes.fluid_box(lo=(0.3, 0.13, 0.3), hi=(0.45, 0.3, 0.45), v0=(0.5, -2.0, -0.25))
    cfg = dataclasses.replace(cfg, boundary="slip_floor", floor_cells=8.0)
    nsteps, dt = 40, 1e-4
    ref = _allocating(cfg, models[0], nsteps, dt)
    assert np.array_equal(ref.F, np.broadcast_to(np.eye(3, dtype=np.float32), ref.F.shape))
    stream = torch.cuda.Stream()
    res = _noalloc(engine_lib, cfg, models[0], nsteps, dt, torch, stream)
    _check(res, ref)


def test_noalloc_per_particle_velocities(engine_lib):
    """nv = n: every particle its own initial velocity."""
    torch = pytest.importorskip("torch")
    cfg, models = scenes.jelly_cube(lo=(0.44, 0.44, 0.44), hi=(0.56, 0.56, 0.56))
    m = models[0]
    rng = np.random.default_rng(3)
    v = rng.uniform(-1.5, 1.5, (m.GetParticleCount(), 3)).astype(np.float32)
    m = type(m)(m.particle_mass, m.particle_volume, m.particle_position, v, m.material)
    nsteps, dt = 24, 1e-4
    ref = _allocating(cfg, m, nsteps, dt)
    _check(_noalloc(engine_lib, cfg, m, nsteps, dt, torch), ref)


def test_noalloc_refuses_a_capturing_stream(engine_lib):
    """The call synchronises its stream, which a CUDA-graph capture cannot record: on a stream
    that is capturing it returns CKMPM_ERR_INVALID before enqueuing anything, and the capture
    stays valid."""
    torch = pytest.importorskip("torch")
    cfg, models = scenes.jelly_cube(lo=(0.44, 0.44, 0.44), hi=(0.56, 0.56, 0.56))
    stream = torch.cuda.Stream()
    assert _noalloc(engine_lib, cfg, models[0], 2, 1e-4, torch, stream)[0] == capi.CKMPM_OK  # set-up done
    dev = torch.device("cuda", cfg.device)
    m = models[0]
    x = torch.from_numpy(np.ascontiguousarray(m.particle_position)).to(dev)
    v = torch.from_numpy(np.ascontiguousarray(m.particle_velocity)).to(dev)
    desc, mat = cfg.to_c(), m.material.to_c()
    msg = C.c_char_p()
    nlive = C.c_uint32()
    y = torch.zeros(4, device=dev)
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=stream, capture_error_mode="thread_local"):
        y += 1.0  # the caller's own captured work
        code = engine_lib.ckmpm_simulate_noalloc(C.byref(desc), C.byref(mat), x.shape[0], C.c_void_p(x.data_ptr()),
                                                 C.c_void_p(v.data_ptr()), v.shape[0], m.particle_mass,
                                                 m.particle_volume, 2, 1e-4, C.c_void_p(stream.cuda_stream), None,
                                                 None, None, None, C.byref(nlive), C.byref(msg))
    assert code == capi.CKMPM_ERR_INVALID
    assert b"capturing" in (msg.value or b"")
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(y.cpu(), torch.ones(4))  # the capture stayed valid


def test_noalloc_first_call_in_a_fresh_process_takes_no_memory(engine_lib):
    """In a new process, the first call on the device (which does the per-device set-up) takes
    no device memory: the scratch array is placed with the library's device code, not by the
    call."""
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    code = f"""
import ctypes as C, sys
sys.path.insert(0, {str(root)!r})
import numpy as np, torch
from ckmpm_b200 import Scene, scenes
from ckmpm_b200 import _capi as capi
lib = capi.lib()
cfg, models = scenes.jelly_cube(lo=(0.44, 0.44, 0.44), hi=(0.56, 0.56, 0.56))
s = Scene(cfg)  # loads the library's device code on this device, then frees what it allocated
s.close()
m = models[0]
dev = torch.device('cuda', 0)
x = torch.from_numpy(np.ascontiguousarray(m.particle_position)).to(dev)
v = torch.from_numpy(np.ascontiguousarray(m.particle_velocity)).to(dev)
xo = torch.zeros_like(x)
desc, mat = cfg.to_c(), m.material.to_c()
nlive, msg = C.c_uint32(), C.c_char_p()
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info(dev)[0]
rc = lib.ckmpm_simulate_noalloc(C.byref(desc), C.byref(mat), x.shape[0], C.c_void_p(x.data_ptr()),
                                C.c_void_p(v.data_ptr()), v.shape[0], m.particle_mass, m.particle_volume, 8, 1e-4,
                                None, C.c_void_p(xo.data_ptr()), None, None, None, C.byref(nlive), C.byref(msg))
torch.cuda.synchronize()
free1 = torch.cuda.mem_get_info(dev)[0]
print(rc, free0 - free1)
"""
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    rc, used = (int(t) for t in out.stdout.split()[-2:])
    assert rc == capi.CKMPM_OK
    assert used < (1 << 20), used
