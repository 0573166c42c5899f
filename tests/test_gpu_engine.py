"""Parity of the CUDA engine (through the C ABI) against the FP64 oracle.

Tolerances (FP32 engine vs FP64 oracle on the same seeded inputs):
  * one constitutive update: |d tau| <= 8 ulp(1) * K + 2e-5 |tau| with K the
    material's stiffness (2 mu + 3 lambda; bulk * gamma for the fluid), since tau
    is K-Lipschitz in F; F within 2e-5 relative;
  * after N substeps: positions within 2e-6 (absolute, domain [0,1]),
    deformation gradients within 5e-5, velocities within 1e-4 x max|v| + 1e-6,
    J / logJp within 5e-5;
  * Drucker-Prager: at the ~1e-5 strains of a column settling under gravity,
    FP32 rounding of singular values near 1 is a visible part of the Hencky
    strain, which the zero-pressure branch and the logJp volume correction of
    the return map (include/mpm_material.cuh:400-445) carry into the stress, so
    velocities differ by up to ~0.6 % of max|v| between any two implementations
    (this engine, the FP64 oracle, the reference build: the oracle and the
    reference differ from each other by as much on the full column).  Compared
    as: every velocity within 1 % of max|v|, x within the tolerance above, F and
    logJp within twice theirs;
  * integer outputs (block sets, per-block counts, live counts): exact.
"""
import numpy as np
import pytest

from ckmpm_b200 import Scene, scenes
from ckmpm_b200 import _capi as capi
from ckmpm_b200.engine import MPMConfig, MPMMaterial, MPMModel

pytestmark = pytest.mark.gpu

X_TOL = 2e-6
F_TOL = 5e-5
V_REL = 1e-4
AUX_TOL = 5e-5


def run_engine(cfg, models, nsteps, dt):
    s = Scene(cfg)
    for m in models:
        s.add_model(m)
    s.setup()
    if nsteps:
        s.step(nsteps, dt)
    return s


def run_oracle(oracle_mod, cfg, models, nsteps, dt):
    o = oracle_mod.OracleScene(cfg, models)
    o.setup()
    if nsteps:
        o.step(nsteps, dt)
    return o


def compare(s, o, model=0, x_tol=X_TOL, f_tol=F_TOL, v_rel=V_REL, aux_tol=AUX_TOL, check_aux=False,
            branchy=False, f_left=False):
    """f_left: compare F F^T instead of F (NACC stores F = U S V, fixed only up to
    a rotation on the right; everything the model computes depends on F F^T)."""
    g = s.state(model)
    r = o.state(model)
    alive = np.nonzero(r["alive"])[0]
    assert len(g.id) == len(alive), "live particle counts differ"
    assert np.array_equal(g.id, alive.astype(np.uint32))
    ex = np.abs(g.x - r["x"][alive]).max(axis=1)
    Fg, Fo = g.F.astype(np.float64), r["F"][alive].reshape(-1, 3, 3)
    if f_left:
        Fg, Fo = Fg @ Fg.transpose(0, 2, 1), Fo @ Fo.transpose(0, 2, 1)
    eF = np.abs(Fg - Fo).max(axis=(1, 2))
    ev = np.abs(g.v - r["v"][alive]).max(axis=1)
    vmax = np.abs(r["v"][alive]).max()
    ea = np.abs(g.aux - r["aux"][alive]) if check_aux else np.zeros(1)
    w = int(np.argmax(ev))
    print(f"max |dx|={ex.max():.3e} |dF|={eF.max():.3e} |dv|={ev.max():.3e} (p99 {np.percentile(ev, 99):.3e}, "
          f"vmax {vmax:.3e}, worst at x={r['x'][alive][w]}) |daux|={ea.max():.3e}")
    vtol = v_rel * vmax + 1e-6
    if branchy:
        assert ev.max() <= 1e-2 * vmax + 1e-6
        assert ex.max() <= x_tol
        assert eF.max() <= 2 * f_tol and ea.max() <= 2 * aux_tol
    else:
        assert ex.max() <= x_tol
        assert eF.max() <= f_tol
        assert ev.max() <= vtol
        assert ea.max() <= aux_tol
    return ex.max(), eF.max(), ev.max()


def test_constitutive_matches_oracle(engine_lib, oracle_mod):
    rng = np.random.default_rng(7)
    n = 512
    for kind, params in [(0, [2.9e4, 1.9e4, 0, 0]), (2, [2.0e5, 1.35e5, 0, 0]), (3, [1e5, 7.15, 0.1, 1.0]),
                         (4, [2.0e4, 3.0e4, 300.0, 0]), (5, [1.0e4, 2.0e4, -0.04, 0.5, 10.0, 1.0, 1.0, 0])]:
        Cm = (0.5 * rng.normal(size=(n, 3, 3))).astype(np.float32)
        F = (np.eye(3)[None] + 0.15 * rng.normal(size=(n, 3, 3))).astype(np.float32)
        if kind == 2:
            F[: n // 4] = np.eye(3) * 1.02  # expansion branch of the return map
        if kind == 5:
            F[: n // 4] = np.eye(3) * 0.7  # pressure beyond p0: the clamped branch
        aux = (np.full(n, 1.0) if kind == 3 else np.full(n, params[2] if kind == 5 else 0.0)).astype(np.float32)
        dt = 1e-3
        cm = capi.Material()
        cm.kind = kind
        for i, p in enumerate(params):
            cm.p[i] = p
        Fg, ag, tg = F.copy(), aux.copy(), np.zeros_like(F)
        S = np.zeros((n, 3), np.float32)
        capi.check(engine_lib.ckmpm_debug_constitutive(cm, n, capi.fptr(Cm), dt, capi.fptr(Fg), capi.fptr(ag),
                                                       capi.fptr(tg), None, capi.fptr(S), None), "debug")
        for i in range(n):
            Fo, ao, to = oracle_mod.constitutive(kind, params, Cm[i].astype(np.float64), dt,
                                                 F[i].astype(np.float64), float(aux[i]))
            K = params[0] * params[1] if kind == 3 else 5 * max(params[0], params[1])
            assert np.abs(tg[i] - to).max() <= 8 * 2.0 ** -23 * K + 2e-5 * np.abs(to).max(), (kind, i)
            if kind != 3:
                # NACC stores F = U S V (fixed up to a right rotation): compare F F^T
                a, b = (Fg[i] @ Fg[i].T, Fo @ Fo.T) if kind == 5 else (Fg[i], Fo)
                assert np.abs(a - b).max() <= 2e-5 * max(1.0, np.abs(b).max()), (kind, i)
            assert abs(ag[i] - ao) <= 2e-5 * max(1.0, abs(ao)), (kind, i)
        if kind != 3:
            # singular values of the trial F (before the return map) match the oracle's SVD
            for i in range(0, n, 17):
                Ft = (np.eye(3) + dt * Cm[i].astype(np.float64)) @ F[i].astype(np.float64)
                _, So, _ = oracle_mod.svd3(Ft)
                assert np.abs(S[i] - So).max() <= 3e-6 * max(1.0, So[0])


def test_near_identity_deformation_stays_unrotated(engine_lib):
    """A deformation gradient within rounding of the identity (a free-falling or rigidly moving
    body: F = I + dt C with dt C ~ 1e-11) leaves the SVD's pairs unrotated, as the reference's SVD
    does: V is exactly the identity, fixed-corotated stress is exactly zero, and the Drucker-Prager
    tension branch's re-projected F = U V^T stays within 1e-10 of the identity instead of picking
    up the ~1e-7 rounding of 45-degree rotations every substep."""
    rng = np.random.default_rng(9)
    n = 256
    F0 = (np.eye(3) + rng.normal(scale=1e-11, size=(n, 3, 3))).astype(np.float32)
    Cm = np.zeros((n, 3, 3), np.float32)
    lam, mu = 1.0e5, 1.35e5
    for kind in (capi.FIXED_COROTATED, capi.DRUCKER_PRAGER):
        cm = capi.Material()
        cm.kind = kind
        cm.p[0], cm.p[1] = lam, mu
        F, aux, tau = F0.copy(), np.zeros(n, np.float32), np.zeros((n, 3, 3), np.float32)
        U, S, V = np.zeros_like(F), np.zeros((n, 3), np.float32), np.zeros_like(F)
        capi.check(engine_lib.ckmpm_debug_constitutive(cm, n, capi.fptr(Cm), 1e-4, capi.fptr(F), capi.fptr(aux),
                                                       capi.fptr(tau), capi.fptr(U), capi.fptr(S), capi.fptr(V)),
                   "debug")
        assert np.array_equal(V, np.broadcast_to(np.eye(3, dtype=np.float32), V.shape)), kind
        assert np.abs(S - 1.0).max() == 0.0, kind
        if kind == capi.FIXED_COROTATED:
            assert not tau.any()
        else:
            assert np.abs(F.astype(np.float64) - np.eye(3)).max() <= 1e-10
            assert np.abs(tau).max() <= 1e-3  # Pa: at most rounding of a zero strain


def test_setup_binning_exact(engine_lib, oracle_mod):
    cfg, models = scenes.jelly_cube()
    s = run_engine(cfg, models, 0, 0.0)
    o = oracle_mod.OracleScene(cfg, models)
    for which in (0, 1, 2):
        kg, cg = s.blocks(0, which)
        ko, co = o.blocks(0, which)
        assert np.array_equal(kg, ko)
        assert np.array_equal(cg, co)
    assert s.count(0) == len(models[0].particle_position)


def test_jelly_parity(engine_lib, oracle_mod):
    cfg, models = scenes.jelly_cube(lo=(0.42, 0.42, 0.42), hi=(0.58, 0.58, 0.58))
    s = run_engine(cfg, models, 40, 1e-4)
    o = run_oracle(oracle_mod, cfg, models, 40, 1e-4)
    compare(s, o)
    assert s.counters()["lost"] == 0


def test_jelly_rebinning_tracks_positions(engine_lib, oracle_mod):
    # Blocks after many substeps equal the blocks recomputed from the engine's own positions.
    cfg, models = scenes.jelly_cube(lo=(0.40, 0.45, 0.40), hi=(0.56, 0.6, 0.52), v0=(1.5, -2.0, 0.7))
    s = run_engine(cfg, models, 200, 1e-4)
    st = s.state(0)
    K = (np.floor(st.x.astype(np.float32) / np.float32(cfg.dx) + np.float32(0.25)).astype(int) - 2) // 4
    uniq, cnt = np.unique(K, axis=0, return_counts=True)
    kg, cg = s.blocks(0, 0)
    assert np.array_equal(kg, uniq.astype(np.int32))
    assert np.array_equal(cg, cnt.astype(np.uint32))
    o = run_oracle(oracle_mod, cfg, models, 200, 1e-4)
    compare(s, o, x_tol=1e-5, f_tol=2e-4, v_rel=5e-4)


def test_sand_parity(engine_lib, oracle_mod):
    cfg, models = scenes.small_sand()
    s = run_engine(cfg, models, 30, 5e-5)
    o = run_oracle(oracle_mod, cfg, models, 30, 5e-5)
    compare(s, o, check_aux=True, branchy=True)


def test_fluid_parity(engine_lib, oracle_mod):
    cfg, models = scenes.fluid_box()
    s = run_engine(cfg, models, 30, 5e-5)
    o = run_oracle(oracle_mod, cfg, models, 30, 5e-5)
    compare(s, o, check_aux=True)


def test_two_models_share_the_grid(engine_lib, oracle_mod):
    cfg, m1 = scenes.jelly_cube(lo=(0.3, 0.3, 0.3), hi=(0.42, 0.42, 0.42), v0=(1.0, 0.0, 0.0))
    _, m2 = scenes.fluid_box(lo=(0.44, 0.3, 0.3), hi=(0.55, 0.4, 0.42), v0=(-1.0, 0.0, 0.0))
    models = m1 + m2
    s = run_engine(cfg, models, 60, 1e-4)
    o = run_oracle(oracle_mod, cfg, models, 60, 1e-4)
    compare(s, o, model=0)
    compare(s, o, model=1, check_aux=True)
    ku, cu = s.blocks(-1, 0)
    ko, co = o.blocks(-1, 0)
    assert np.array_equal(ku, ko) and np.array_equal(cu, co)


def test_deterministic_bitwise(engine_lib):
    """Two runs, and runs at every launch shape, give the same bits (exact integer
    P2G and grid sums: the order in which blocks deposit does not matter)."""
    cfg, models = scenes.jelly_cube(v0=(0.7, -1.3, 0.4))
    a = run_engine(cfg, models, 50, 1e-4).state(0)
    runs = [run_engine(cfg, models, 50, 1e-4).state(0)]
    for shape in ((1024, 1, 8), (128, 3, 32), (192, 5, 8)):
        s = Scene(cfg)
        s.set_tuning(*shape)
        for m in models:
            s.add_model(m)
        s.setup()
        s.step(50, 1e-4)
        runs.append(s.state(0))
    for b in runs:
        assert np.array_equal(a.x.view(np.uint32), b.x.view(np.uint32))
        assert np.array_equal(a.F.view(np.uint32), b.F.view(np.uint32))
        assert np.array_equal(a.v.view(np.uint32), b.v.view(np.uint32))


@pytest.mark.parametrize("scene", ["jelly", "sand"])
def test_setup_lays_particles_out_across_cells(engine_lib, scene):
    """Setup's particle layout: within every block the particles are stored by (rank within
    their cell, cell), the cells numbered x-major over the block, so 32 consecutive particles
    lie in 32 different cells of a half block wherever the counts allow.  Read back in storage
    order (a scene without ids exports in block order), each block's sequence of keys
    (occurrences of its cell so far, cell) must increase strictly, and two setups of the same
    scene store the particles in the same order."""
    cfg, models = scenes.jelly_cube(track_ids=False) if scene == "jelly" else scenes.small_sand(track_ids=False)
    xs = []
    for _ in range(2):
        s = run_engine(cfg, models, 0, 1e-4)
        xs.append(s.state(0).x)
        s.close()
    x = xs[0]
    assert np.array_equal(xs[0], xs[1]), "the storage order differs between two setups of the same scene"
    c = (x.astype(np.float32) * np.float32(1.0 / cfg.dx) + np.float32(0.25)).astype(np.int64)
    block = (c - 2) // 4  # all positions are well inside the domain: floor equals truncation
    cell = ((c - 2) % 4) @ np.array([16, 4, 1])
    starts = np.flatnonzero(np.any(block[1:] != block[:-1], axis=1)) + 1
    runs = np.split(np.arange(len(x)), starts)
    assert len({tuple(block[r[0]]) for r in runs}) == len(runs), "a block's particles are not contiguous"
    full_warps = 0
    for r in runs:
        seen = {}
        keys = []
        for ci in cell[r]:
            keys.append(seen.get(ci, 0) * 64 + ci)
            seen[ci] = seen.get(ci, 0) + 1
        assert all(a < b for a, b in zip(keys, keys[1:])), "block not in (rank, cell) order"
        full_warps += sum(len(set(cell[r][i:i + 32])) == 32 for i in range(0, len(r) - 31, 32))
    assert full_warps > 0


def _relayout_cases():
    from ckmpm_b200.engine import compute_lame_parameters
    cfg_j, jelly = scenes.jelly_cube(lo=(0.4, 0.42, 0.38), hi=(0.6, 0.58, 0.55), v0=(1.0, -1.0, 0.3))
    cfg_s, sand = scenes.small_sand()
    cfg_m, m1 = scenes.jelly_cube(lo=(0.3, 0.3, 0.3), hi=(0.42, 0.42, 0.42), v0=(1.0, 0.0, 0.0))
    _, m2 = scenes.fluid_box(lo=(0.44, 0.3, 0.3), hi=(0.55, 0.4, 0.42), v0=(-1.0, 0.0, 0.0))
    lam, mu = compute_lame_parameters(5e4, 0.3)
    lin = MPMModel(m1[0].particle_mass, m1[0].particle_volume, m1[0].particle_position,
                   np.asarray([[0.6, -0.8, 0.2]], np.float32), MPMMaterial.linear(lam, mu))
    return {"jelly_fc": (cfg_j, jelly, 1e-4), "sand_dp": (cfg_s, sand, 5e-5), "two_models": (cfg_m, m1 + m2, 1e-4),
            "linear": (cfg_m, [lin], 1e-4)}


@pytest.mark.parametrize("case", ["jelly_fc", "sand_dp", "two_models", "linear"])
def test_relayout_changes_no_result(engine_lib, case):
    """ckmpm_set_reorder_interval: re-laying out every block's particles every 10
    substeps (before graph chunks, between single substeps, and in the adaptive
    loop) leaves every particle's x, v, F, aux and the counters bit for bit as
    never re-laying out does; only where the particles are stored changes."""
    cfg, models, dt = _relayout_cases()[case]
    runs = []
    for every in (0, 10):
        s = Scene(cfg)
        s.set_reorder_interval(every)
        for m in models:
            s.add_model(m)
        s.setup()
        s.step(47, dt)
        s.step_async(23, dt)
        s.status_check()
        s.step_adaptive(25, dt, 0.4, 25 * dt)
        runs.append(([s.state(i) for i in range(len(models))], s.counters()))
        s.close()
    (a, ca), (b, cb) = runs
    assert ca == cb
    for sa, sb in zip(a, b):
        assert np.array_equal(sa.id, sb.id)
        for name in ("x", "v", "F", "aux"):
            assert np.array_equal(getattr(sa, name).view(np.uint32), getattr(sb, name).view(np.uint32)), (case, name)


def test_first_substep_has_zero_advection(engine_lib):
    cfg, models = scenes.jelly_cube()
    s = run_engine(cfg, models, 1, 1e-4)
    st = s.state(0)
    assert np.array_equal(st.x, models[0].particle_position[st.id])
    assert s.dt_pair() == (np.float32(1e-4), np.float32(1e-4))


def test_particles_leaving_domain_are_counted(engine_lib, oracle_mod):
    # Start outside the sticky layer moving out fast, with no walls in the way:
    # a particle spawned in the last block leaves the domain.
    cfg = MPMConfig(dx=1 / 64, domain_blocks=(16, 16, 16), gravity=0.0)
    x = np.array([[0.5, 0.5, 0.5], [0.5, 0.5, 0.51], [1.2, 0.5, 0.5]], np.float32)
    m = MPMModel(1e-4, 1e-7, x, np.zeros((1, 3), np.float32), MPMMaterial.fixed_corotated(1e2, 1e2))
    s = run_engine(cfg, [m], 3, 1e-4)
    assert s.count(0) == 2
    assert s.counters()["lost"] == 1


def test_full_block_next_to_lone_particles(engine_lib, oracle_mod):
    """Ragged extremes of the per-block work: one block holding the maximum of
    4096 particles (64 per cell over its 64 cells, the reference's bucket
    capacity) and three blocks holding one particle each.  Ten substeps match
    the FP64 oracle, and no capacity or consistency flag is raised."""
    from ckmpm_b200.engine import compute_lame_parameters
    dx, b = 1 / 64, 7
    # Block b along an axis takes int(x / dx + 0.25) in [4b + 2, 4b + 5], so
    # x / dx in [4b + 1.75, 4b + 5.75): a 16^3 lattice over [4b + 1.85, 4b + 5.65].
    g = (4 * b + 1.85 + (np.arange(16) + 0.5) / 16 * 3.8) * dx
    full = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    lone = np.array([[0.2, 0.2, 0.2], [0.8, 0.3, 0.7], [0.3, 0.75, 0.25]])
    x = np.concatenate([full, lone]).astype(np.float32)
    v = np.random.default_rng(3).uniform(-0.2, 0.2, x.shape).astype(np.float32)
    lam, mu = compute_lame_parameters(5e4, 0.3)
    vol = dx ** 3 / 64
    m = MPMModel(1000.0 * vol, vol, x, v, MPMMaterial.fixed_corotated(lam, mu))
    cfg = MPMConfig(dx=dx, domain_blocks=(16, 16, 16), gravity=-9.8)
    s = run_engine(cfg, [m], 0, 1e-4)
    keys, counts = s.blocks()  # right after setup: also the +dx/4 grid's blocks, with no particles
    assert sorted(counts[counts > 0].tolist()) == [1, 1, 1, 4096]
    assert [b, b, b] in keys[counts > 0].tolist()
    s.step(10, 1e-4)
    o = run_oracle(oracle_mod, cfg, [m], 10, 1e-4)
    assert s.count(0) == len(x)
    compare(s, o)


def test_async_position_export(engine_lib):
    """ckmpm_export_positions_async: each model's buffer receives the positions
    as of the export, not those of substeps enqueued after it, bit for bit
    what state() returns; export_wait gives the live count; ckmpm_get_state
    after an export waits for its copy; a short buffer is refused."""
    import torch
    cfg, m1 = scenes.jelly_cube(lo=(0.3, 0.3, 0.3), hi=(0.42, 0.42, 0.42), v0=(1.0, 0.0, 0.0))
    _, m2 = scenes.fluid_box(lo=(0.44, 0.3, 0.3), hi=(0.55, 0.4, 0.42), v0=(-1.0, 0.0, 0.0))
    models = [m1[0], m2[0]]
    s = run_engine(cfg, models, 6, 1e-4)
    ref = [s.state(i).x for i in range(2)]
    bufs = [torch.zeros((len(m.particle_position), 3), dtype=torch.float32).pin_memory().numpy() for m in models]
    for i in range(2):
        s.export_positions_async(i, bufs[i])
    s.step_async(25, 1e-4)
    n = s.export_wait()
    assert n == len(ref[1])
    for i in range(2):
        assert np.array_equal(bufs[i][:len(ref[i])], ref[i]), i
    later = s.state(0).x
    assert not np.array_equal(later, ref[0])
    s.export_positions_async(0, bufs[0])
    again = s.state(0).x  # reuses the staging buffer after the copy
    assert s.export_wait() == len(again)
    assert np.array_equal(bufs[0][:len(again)], again) and np.array_equal(again, later)
    pageable = np.zeros_like(bufs[1])
    s.export_positions_async(1, pageable)
    s.export_wait()
    assert np.array_equal(pageable[:len(ref[1])], s.state(1).x)
    with pytest.raises(capi.CkmpmError):
        s.export_positions_async(0, np.zeros((3, 3), np.float32))
    s.close()


def test_capacity_overflow_is_reported(engine_lib):
    cfg, models = scenes.jelly_cube()
    cfg.max_particles_per_block = 64  # a full block holds 512 particles at 8 ppc
    s = Scene(cfg)
    s.add_model(models[0])
    s.setup()
    with pytest.raises(capi.CkmpmError) as ei:
        s.step(1, 1e-4)
    assert ei.value.code == 3


def test_invalid_arguments(engine_lib):
    cfg, models = scenes.jelly_cube()
    with pytest.raises(capi.CkmpmError):
        Scene(MPMConfig(dx=-1.0, domain_blocks=(4, 4, 4)))
    s = Scene(cfg)
    with pytest.raises(capi.CkmpmError):
        s.setup()  # no models
    with pytest.raises(capi.CkmpmError):
        s.step(1, 1e-4)  # before setup
    s.add_model(models[0])
    s.setup()
    with pytest.raises(capi.CkmpmError):
        s.add_model(models[0])  # after setup
    with pytest.raises(capi.CkmpmError):
        s.step(1, -1.0)


@pytest.mark.parametrize("kind", ["von_mises", "nacc", "linear"])
def test_other_materials_parity(engine_lib, oracle_mod, kind):
    """The reference's von Mises, non-associated Cam-clay and linear models
    (mpm_algorithm.cuh:107-520, mpm_material.cuh:480-669) against the FP64
    oracle after 40 substeps of a cube loaded by its initial velocity field."""
    cfg, models = scenes.material_cube(kind)
    s = run_engine(cfg, models, 40, 1e-4)
    o = run_oracle(oracle_mod, cfg, models, 40, 1e-4)
    compare(s, o, check_aux=(kind == "nacc"), f_left=(kind == "nacc"))


def test_rigid_particles_parity(engine_lib, oracle_mod):
    """Rigid particles (include/mpm_algorithm.cuh:1063-1069, 1540-1543,
    1609-1624): the first 2048 particles of the von Mises cube are rigid and
    their velocity changes every 10 substeps; engine and oracle agree on every
    particle (rigid ones: x exactly advected, F = I, v = 0, aux = 0)."""
    cfg, models = scenes.material_cube("von_mises")
    R = 2048
    vel = [(2.0, -1.0, 0.5), (0.0, 1.5, -1.0), (-1.0, 0.0, 0.0), (0.5, 0.5, 0.5)]
    s = Scene(cfg)
    s.set_rigid(R, vel[0])
    s.add_model(models[0])
    s.setup()
    o = oracle_mod.OracleScene(cfg, models)
    o.set_rigid(R, vel[0])
    o.setup()
    for v in vel:
        s.set_rigid_velocity(v)
        o.set_rigid_velocity(v)
        s.step(10, 1e-4)
        o.step(10, 1e-4)
    compare(s, o, check_aux=True)
    g = s.state(0)
    rigid = g.id < R
    assert rigid.sum() == R and np.all(g.aux[rigid] == 0.0) and np.all(g.aux[~rigid] == 1.0)
    assert np.abs(g.v[rigid]).max() == 0.0
    assert np.abs(g.F[rigid] - np.eye(3, dtype=np.float32)).max() == 0.0


def test_rigid_particles_api(engine_lib):
    cfg, models = scenes.material_cube("von_mises")
    s = Scene(cfg)
    with pytest.raises(capi.CkmpmError, match="rigid particles are off"):
        s.set_rigid_velocity((1.0, 0.0, 0.0))
    with pytest.raises(capi.CkmpmError, match="finite"):
        s.set_rigid(4, (float("nan"), 0.0, 0.0))
    s.add_model(models[0])
    s.setup()
    with pytest.raises(capi.CkmpmError, match="before ckmpm_setup"):
        s.set_rigid(4, (1.0, 0.0, 0.0))
    # Rigid particles off: the von Mises flag stays 1 and no particle is rigid.
    s.step(4, 1e-4)
    assert np.all(s.state(0).aux == 1.0)


def test_model_entirely_outside_the_domain(engine_lib):
    """A model whose particles all lie outside the domain is dropped at setup
    (counted as lost, zero live particles, empty state) and leaves the other
    model's simulation bitwise unchanged."""
    cfg, models = scenes.jelly_cube(lo=(0.44, 0.44, 0.44), hi=(0.56, 0.56, 0.56))
    m = models[0]
    out = MPMModel(m.particle_mass, m.particle_volume, (m.particle_position + 2.0).astype(np.float32),
                   m.particle_velocity, m.material)
    s = run_engine(cfg, [m, out], 12, 1e-4)
    alone = run_engine(cfg, [m], 12, 1e-4)
    assert s.count(1) == 0 and s.counters()["lost"] == len(out.particle_position)
    empty = s.state(1)
    assert empty.x.shape == (0, 3) and empty.id.shape == (0,)
    a, b = s.state(0), alone.state(0)
    for name in ("id", "x", "v", "F"):
        assert np.array_equal(getattr(a, name), getattr(b, name)), name


def test_conservation_metric(engine_lib, oracle_mod, tmp_path):
    """The reference's conservation metric (Lagrangian sum(v) and sum(x cross v)
    before every substep, include/mpm_engine.cuh:573-603): written as 13 float32
    per substep; collecting it steps one substep at a time without changing a
    bit of the simulation; its x and z momentum of a free-flying cube stay at
    N v0 (APIC transfers conserve momentum; gravity acts on y only); and it
    matches the FP64 oracle's sums at the end."""
    from ckmpm_b200 import MPMEngine
    cfg, models = scenes.jelly_cube(lo=(0.44, 0.44, 0.44), hi=(0.56, 0.56, 0.56), v0=(0.3, -1.0, 0.2))
    cfg.dt, cfg.fps, cfg.total_frames = 2.0 ** -14, 1024, 4
    n = len(models[0].particle_position)
    finals = {}
    for mode in ("fixed", "adaptive"):
        for collect in (False, True):
            eng = MPMEngine()
            eng.Initialize(cfg)
            eng.InitializeParticle(cfg, models)
            eng.InitialSetup(cfg)
            root = tmp_path / f"{mode}_{collect}"
            eng.Simulate(cfg, fixed_substeps_per_frame=16 if mode == "fixed" else None,
                         export_root=root if collect else None, collect_conservation_metric=collect)
            finals[(mode, collect)] = eng.scene.state(0).x.copy()
            if collect:
                rec = np.fromfile(root / "conservationMetric_model_0.bin", np.float32).reshape(-1, 13)
                assert rec.shape[0] == 64 and np.all(np.diff(rec[:, 0]) >= 0)
                assert np.all(rec[:, 1:7] == 0.0)  # the Eulerian rows stay zero, as in the reference
                np.testing.assert_allclose(rec[:, 7], n * 0.3, rtol=1e-5)
                np.testing.assert_allclose(rec[:, 9], n * 0.2, rtol=1e-5)
                last = eng.scene.conservation_metric(0)
        assert np.array_equal(finals[(mode, False)], finals[(mode, True)]), mode
    o = run_oracle(oracle_mod, cfg, models, 64, cfg.dt)
    r = o.state(0)
    ref = np.array([r["v"].sum(axis=0), np.cross(r["x"], r["v"]).sum(axis=0)])
    s = run_engine(cfg, models, 64, cfg.dt)
    got = s.conservation_metric(0)[2:]
    assert np.abs(got - ref).max() <= 5e-5 * np.abs(ref).max(), (got, ref)


def test_momentum_conserved_on_the_full_sand_column(engine_lib):
    """Size-independent property at the benchmark's full size (1.69M particles):
    the column starts at rest and nothing acts on it along x or z but its own
    stress (the slip floor only limits v_y, the walls are far), so the
    Lagrangian x and z momentum stay at zero up to FP32 noise."""
    cfg, models = scenes.sand_column(track_ids=False)
    s = run_engine(cfg, models, 200, cfg.dt)
    st = s.state(0)
    n, vmax = len(st.v), float(np.abs(st.v).max())
    m = s.conservation_metric(0)[2]
    assert vmax > 1e-3
    assert abs(m[0]) <= 1e-4 * n * vmax and abs(m[2]) <= 1e-4 * n * vmax, (m, n, vmax)
    assert s.counters()["lost"] == 0


def field_scene():
    """A fluid box in a boundary field with every rule: slip walls, a fixed box,
    a driven (velocity) box, a rotating box and a one-sided floor."""
    from ckmpm_b200.boundary import BoundaryField
    cfg, models = scenes.fluid_box(lo=(0.13, 0.13, 0.3), hi=(0.45, 0.3, 0.55), v0=(-2.0, -3.0, 1.0))
    cfg.boundary = "field"
    bf = BoundaryField(cfg).slip_walls(8).separate_below(10).fixed_box((24, 0, 24), (32, 14, 32))
    bf.velocity_box((10, 16, 30), (14, 20, 34), (0.5, 0.25, -0.5))
    bf.rotating_box((16, 12, 20), (22, 18, 26), center=(0.3, 0.23, 0.36), axis=(0, 0, -1), factor=2.0)
    cfg.boundary_field = bf.arrays()
    return cfg, models, bf


def test_boundary_field_parity(engine_lib, oracle_mod):
    """Per-cell boundary rules (the irregular-boundary hook as data,
    include/mpm_algorithm.cuh:795-799) against the FP64 oracle with the same
    field; a VELOCITY cell with mass reports its prescribed velocity."""
    cfg, models, bf = field_scene()
    s = run_engine(cfg, models, 40, 1e-4)
    o = run_oracle(oracle_mod, cfg, models, 40, 1e-4)
    compare(s, o, check_aux=True)
    # Changing the field after setup applies to the substeps after the call.
    bf.fixed_box((0, 0, 0), tuple(bf.shape))
    s.set_boundary_field(*bf.arrays())
    o.set_boundary_field(*bf.arrays())
    s.step(4, 1e-4)
    o.step(4, 1e-4)
    g = s.state(0)
    assert np.abs(g.v).max() == 0.0  # every node is fixed now
    compare(s, o, check_aux=True)


def test_boundary_field_api(engine_lib):
    cfg, models, bf = field_scene()
    rule, param = bf.arrays()
    plain, _ = scenes.fluid_box()
    s = Scene(plain)
    with pytest.raises(capi.CkmpmError, match="not CKMPM_BOUNDARY_FIELD"):
        s.set_boundary_field(rule, param)
    cfg.boundary_field = None
    s = Scene(cfg)
    bad = rule.copy()
    bad[0, 0, 0] = 9
    with pytest.raises(capi.CkmpmError, match="unknown cell rule"):
        s.set_boundary_field(bad, param)
    with pytest.raises(capi.CkmpmError, match="need param"):
        s.set_boundary_field(rule, None)
    nanp = param.copy()
    nanp[0, 0, 0, 0] = np.nan
    with pytest.raises(capi.CkmpmError, match="finite"):
        s.set_boundary_field(rule, nanp)
    # Without a field every cell is free: the box falls through the wall bands.
    s.add_model(models[0])
    s.setup()
    s.step(4, 1e-4)
    assert s.counters()["status"] == 0


def test_non_finite_inputs(engine_lib):
    """A non-finite or out-of-range initial velocity is an error status from
    ckmpm_setup (the reference stops when the grid velocity turns infinite,
    include/mpm_engine.cuh:545-549); a non-finite position drops the particle
    at binning and counts it as lost."""
    cfg, models = scenes.jelly_cube(lo=(0.44, 0.44, 0.44), hi=(0.56, 0.56, 0.56))
    m = models[0]
    for bad in (np.nan, np.inf, 1e6):
        v = np.repeat(np.asarray([[0.0, -1.0, 0.0]], np.float32), len(m.particle_position), 0)
        v[17, 1] = bad
        s = Scene(cfg)
        s.add_model(MPMModel(m.particle_mass, m.particle_volume, m.particle_position, v, m.material))
        with pytest.raises(capi.CkmpmError, match="NUMERIC"):
            s.setup()
    x = m.particle_position.copy()
    x[5, 0] = np.nan
    s = Scene(cfg)
    s.add_model(MPMModel(m.particle_mass, m.particle_volume, x, m.particle_velocity, m.material))
    s.setup()
    s.step(4, 1e-4)
    assert s.counters()["lost"] == 1 and s.count(0) == len(x) - 1


def test_full_sand_column_relayout_is_bitwise_neutral(engine_lib):
    """Size-independent property at the benchmark's full size and length: the 1.69M-particle column
    over 2000 substeps with the default re-layout (every 128 substeps, 15 re-layouts) and with none
    gives every particle the same bits, loses none and raises no status."""
    cfg, models = scenes.sand_column(track_ids=True)
    states = []
    for every in (128, 0):
        s = Scene(cfg)
        s.set_reorder_interval(every)
        s.add_model(models[0])
        s.setup()
        s.step(2000, cfg.dt)
        c = s.counters()
        assert c["lost"] == 0 and c["status"] == 0 and c["window_skips"] == 0, c
        states.append(s.state(0))
        s.close()
    a, b = states
    for name in ("id", "x", "v", "F", "aux"):
        assert np.array_equal(getattr(a, name).view(np.uint32), getattr(b, name).view(np.uint32)), name


def test_full_sand_column_is_bitwise_reproducible(engine_lib):
    """Size-independent property at the benchmark's full size: two runs of the
    1.69M-particle column (200 substeps) give the same bits, and the same block
    sets and per-block counts."""
    cfg, models = scenes.sand_column(track_ids=True)
    a = run_engine(cfg, models, 200, cfg.dt)
    b = run_engine(cfg, models, 200, cfg.dt)
    sa, sb = a.state(0), b.state(0)
    for name in ("id", "x", "v", "F", "aux"):
        assert np.array_equal(getattr(sa, name).view(np.uint32), getattr(sb, name).view(np.uint32)), name
    for which in (0, 1, 2):
        ka, ca = a.blocks(-1, which)
        kb, cb = b.blocks(-1, which)
        assert np.array_equal(ka, kb) and np.array_equal(ca, cb), which
