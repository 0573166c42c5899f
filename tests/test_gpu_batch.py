"""Batched scenes (ckmpm_create_batch / ckmpm_add_batch) through the C ABI.

A batch advances every scene in the same launches.  Each scene must come out
bit for bit as it does in a batch of its own: the P2G tile and the grid hold
exact integer sums, so neither the other scenes nor the order in which blocks
deposit changes a bit (x, v, F, aux, ids).  Launch shape (ckmpm_set_tuning,
ckmpm_autotune) and checkpoint save/restore must not change any bit either.
Against the same scene run alone through the single-scene kernel, which is
compiled per material, a scene agrees to the last bits of x, v and F (the two
instantiations may fuse a multiply-add differently), with identical ids and
block sets.  Three scenes are also checked against the FP64 oracle with the
tolerances of the plain-path parity tests.
"""
import numpy as np
import pytest

from ckmpm_b200 import CkmpmError, Scene, scenes
from ckmpm_b200.batch import SceneBatch

pytestmark = pytest.mark.gpu

DT = 1e-4
# Plain-path parity tolerances (the same values as the single-scene tests).
X_TOL, F_TOL, V_REL, AUX_TOL = 2e-6, 5e-5, 1e-4, 5e-5


def small_batch(n=9, seed=3, n_min=500, n_max=6000):
    return scenes.batched_scenes(n_scenes=n, seed=seed, n_min=n_min, n_max=n_max)


def run_batch(cfg, models, nsteps, tuning=None):
    b = SceneBatch(cfg, models)
    b.setup()
    if tuning is not None:
        b.set_tuning(*tuning)
    if nsteps:
        b.step(nsteps, DT)
    return b


def run_alone(cfg, model, nsteps):
    s = Scene(cfg)
    s.add_model(model)
    s.setup()
    if nsteps:
        s.step(nsteps, DT)
    return s


def assert_same_state(a, b, what):
    for name in ("id", "x", "v", "F", "aux"):
        pa, pb = getattr(a, name), getattr(b, name)
        assert pa.shape == pb.shape, (what, name, pa.shape, pb.shape)
        if not np.array_equal(pa, pb):
            d = np.abs(pa.astype(np.float64) - pb.astype(np.float64)).max()
            raise AssertionError(f"{what}: {name} differs (max |diff| {d:.3e})")


# Batch against the single-scene kernel: last-bit differences from multiply-add
# fusion, grown over a few dozen substeps.
ALONE_X, ALONE_F, ALONE_V = 1e-6, 1e-5, 1e-5


def assert_close_to_alone(a, b, what):
    assert np.array_equal(a.id, b.id), f"{what}: ids differ"
    dx = np.abs(a.x.astype(np.float64) - b.x).max(initial=0.0)
    dF = np.abs(a.F.astype(np.float64) - b.F).max(initial=0.0)
    dv = np.abs(a.v.astype(np.float64) - b.v).max(initial=0.0)
    da = np.abs(a.aux.astype(np.float64) - b.aux).max(initial=0.0)
    vmax = np.abs(b.v).max(initial=0.0)
    ndiff = int(np.any(a.x != b.x, axis=1).sum())
    print(f"{what}: {ndiff} of {len(a.id)} positions differ; |dx| {dx:.1e} |dF| {dF:.1e} |dv| {dv:.1e} |daux| {da:.1e}")
    assert dx <= ALONE_X and dF <= ALONE_F and da <= ALONE_F and dv <= ALONE_V * (1.0 + vmax), what


def check_against_alone_and_own_batch(cfg, models, b, nsteps):
    """Each scene of batch b: bit for bit as in a batch of its own, close to
    the scene run alone, with the same block sets."""
    st = b.state()
    for i, m in enumerate(models):
        got = b.scene_state(i, st)
        own = run_batch(cfg, [m], nsteps)
        assert_same_state(got, own.state(), f"scene {i} ({m.material.kind}, {len(m.particle_position)} particles)")
        own.close()
        alone = run_alone(cfg, m, nsteps)
        assert_close_to_alone(got, alone.state(0), f"scene {i} ({m.material.kind})")
        for which in (0, 2):
            kb, cb = b.blocks_in(i, which)
            ka, ca = alone.blocks(-1, which)
            assert np.array_equal(kb, ka) and np.array_equal(cb, ca), (i, which)
        alone.close()


def test_batch_scenes_equal_each_scene_on_its_own(engine_lib):
    cfg, models = small_batch()
    b = run_batch(cfg, models, 24)
    check_against_alone_and_own_batch(cfg, models, b, 24)
    assert {m.material.kind for m in models} == {"fixed_corotated", "fluid", "drucker_prager"}
    c = b.counters()
    assert c["steps"] == 24 and c["status"] == 0 and c["timeouts"] == 0


def test_batch_scenes_match_oracle(engine_lib, oracle_mod):
    cfg, models = small_batch(n=12, seed=5, n_min=800, n_max=3000)
    picked = {}
    for i, m in enumerate(models):
        picked.setdefault(m.material.kind, i)
    idx = sorted(picked.values())
    sub = [models[i] for i in idx]
    b = run_batch(cfg, sub, 16)
    st = b.state()
    for j, m in enumerate(sub):
        o = oracle_mod.OracleScene(cfg, [m])
        o.setup()
        o.step(16, DT)
        r = o.state(0)
        g = b.scene_state(j, st)
        alive = np.nonzero(r["alive"])[0]
        assert np.array_equal(g.id, alive.astype(np.uint32))
        ex = np.abs(g.x - r["x"][alive]).max(axis=1)
        eF = np.abs(g.F - r["F"][alive]).max(axis=(1, 2))
        ev = np.abs(g.v - r["v"][alive]).max(axis=1)
        ea = np.abs(g.aux - r["aux"][alive])
        vmax = np.abs(r["v"][alive]).max()
        print(f"{m.material.kind}: n={len(alive)} |dx|={ex.max():.2e} |dF|={eF.max():.2e} |dv|={ev.max():.2e} "
              f"(vmax {vmax:.2e}) |daux|={ea.max():.2e}")
        if m.material.kind == "drucker_prager":
            assert np.percentile(ev, 99) <= 0.03 * vmax + 1e-6 and ev.max() <= 0.05 * vmax + 1e-6
            assert np.percentile(ex, 99) <= X_TOL and ex.max() <= 10 * X_TOL
            assert np.percentile(eF, 99) <= F_TOL and np.percentile(ea, 99) <= AUX_TOL
        else:
            assert ex.max() <= X_TOL and eF.max() <= F_TOL and ea.max() <= AUX_TOL
            assert ev.max() <= V_REL * vmax + 1e-6


def test_launch_shape_does_not_change_results(engine_lib):
    cfg, models = small_batch(n=6, seed=7)
    ref = run_batch(cfg, models, 16).state()
    for tuning in ((128, 1, 2), (128, 5, 32), (192, 5, 8), (256, 2, 8), (256, 4, 64), (1024, 1, 8)):
        got = run_batch(cfg, models, 16, tuning).state()
        assert_same_state(got, ref, f"tuning {tuning}")


def test_autotune_leaves_state_unchanged(engine_lib):
    cfg, models = small_batch(n=6, seed=11)
    ref = run_batch(cfg, models, 10).state()
    b = SceneBatch(cfg, models)
    b.setup()
    b.step(4, DT)
    best, tried = b.autotune(4, DT)
    assert len(tried) >= 4 and all(t["probe_ms"] > 0 for t in tried)
    assert best["probe_ms"] == min(t["probe_ms"] for t in tried)
    assert b.tuning()["threads"] == best["threads"]
    assert b.counters()["steps"] == 4
    b.step(6, DT)
    assert_same_state(b.state(), ref, "after autotune")


def test_checkpoint_roundtrip(engine_lib):
    import torch
    cfg, models = small_batch(n=5, seed=13)
    b = run_batch(cfg, models, 8)
    buf = torch.empty(b.checkpoint_bytes(), dtype=torch.uint8, device="cuda")
    b.checkpoint_save(buf.data_ptr())
    b.step(7, DT)
    first = b.state()
    b.checkpoint_restore(buf.data_ptr())
    assert b.counters()["steps"] == 8
    b.step(7, DT)
    assert_same_state(b.state(), first, "after restore")


def test_batch_argument_errors(engine_lib):
    cfg, models = small_batch(n=3, seed=1)
    bad = scenes.MPMModel(models[0].particle_mass, models[0].particle_volume, models[0].particle_position,
                          models[0].particle_velocity, scenes.MPMMaterial.fixed_corotated(1e4, 0.0))
    with pytest.raises(CkmpmError):
        SceneBatch(cfg, [models[0], bad])
    b = SceneBatch(cfg, models)
    with pytest.raises(CkmpmError):
        b.set_tuning(64, 1, 8)
    with pytest.raises(CkmpmError):
        b.set_tuning(256, 1, 7)
    with pytest.raises(CkmpmError):
        b.step(1, DT)  # before setup
    b.setup()
    with pytest.raises(CkmpmError):
        b.blocks_in(3)


def test_batch_with_every_material_equals_scenes_on_their_own(engine_lib):
    """von Mises, NACC and linear scenes (the kinds the batched workload does not
    draw) next to fixed-corotated, fluid and Drucker-Prager scenes in one batch:
    every scene bit for bit as in a batch of its own, and close to the scene
    run alone."""
    cfg, models = small_batch(n=6, seed=5)
    for kind in ("von_mises", "nacc", "linear"):
        c2, m2 = scenes.material_cube(kind)
        assert c2.dx == cfg.dx and tuple(c2.domain_blocks) == tuple(cfg.domain_blocks)
        models.append(m2[0])
    b = run_batch(cfg, models, 24)
    check_against_alone_and_own_batch(cfg, models, b, 24)
    assert {"von_mises", "nacc", "linear"} <= {m.material.kind for m in models}
    assert b.counters()["status"] == 0


def test_batch_with_ragged_scenes(engine_lib):
    """A one-particle scene and a scene whose particles fill one block to the
    4096-particle maximum, batched with ordinary scenes: each bit for bit as in
    a batch of its own, and close to the scene run alone."""
    from ckmpm_b200.engine import MPMMaterial, MPMModel, compute_lame_parameters
    cfg, models = small_batch(n=3, seed=21)
    dx = cfg.dx
    lam, mu = compute_lame_parameters(5e4, 0.3)
    vol = dx ** 3 / 64
    g = (4 * 9 + 1.85 + (np.arange(16) + 0.5) / 16 * 3.8) * dx  # one block along each axis
    full = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3).astype(np.float32)
    rng = np.random.default_rng(4)
    models.append(MPMModel(1000.0 * vol, vol, full, rng.uniform(-0.3, 0.3, full.shape).astype(np.float32),
                           MPMMaterial.fixed_corotated(lam, mu)))
    models.insert(1, MPMModel(1000.0 * vol, vol, np.array([[0.41, 0.52, 0.47]], np.float32),
                              np.array([[0.5, -0.2, 0.1]], np.float32), MPMMaterial.fixed_corotated(lam, mu)))
    b = run_batch(cfg, models, 0)
    # Right after setup the set also holds the blocks of the +dx/4 grid's cells, with no particles.
    keys, counts = b.blocks_in(len(models) - 1, 0)
    assert keys[counts > 0].tolist() == [[9, 9, 9]] and counts[counts > 0].tolist() == [4096]
    c1 = b.blocks_in(1, 0)[1]
    assert c1[c1 > 0].tolist() == [1]
    b.step(24, DT)
    check_against_alone_and_own_batch(cfg, models, b, 24)
    assert b.counters()["status"] == 0


def test_batch_shares_a_boundary_field(engine_lib):
    """A batch of boundary="field" scenes shares one per-cell field (slip walls
    and a fixed box); each scene comes out bit for bit as in a batch of its own
    with the field, and close to the scene run alone with it."""
    from ckmpm_b200.boundary import BoundaryField
    cfg, models = small_batch(n=4, seed=13)
    cfg.boundary = "field"
    cfg.boundary_field = BoundaryField(cfg).slip_walls(8).fixed_box((20, 0, 20), (44, 12, 44)).arrays()
    b = run_batch(cfg, models, 16)
    check_against_alone_and_own_batch(cfg, models, b, 16)


def test_batch_relayout_changes_no_result(engine_lib):
    """A batch re-laid out every 10 substeps (ckmpm_set_reorder_interval; every scene's blocks
    gather their particles into the setup order) gives the same particles bit for bit as one
    never re-laid out."""
    cfg, models = small_batch()
    runs = []
    for every in (0, 10):
        b = SceneBatch(cfg, models)
        b.set_reorder_interval(every)
        b.setup()
        b.step(37, DT)
        runs.append(b.state())
        b.close()
    assert_same_state(runs[0], runs[1], "batch with and without re-layout")


def test_batch_from_concatenated_inputs(engine_lib):
    """SceneBatch given the scenes' inputs already concatenated (x, v of every particle, here in
    pinned host memory) equals the batch that concatenates them itself, bit for bit; malformed
    arrays are refused."""
    import torch
    cfg, models = small_batch()
    ref = run_batch(cfg, models, 12).state()
    x = np.concatenate([m.particle_position for m in models]).astype(np.float32)
    v = np.concatenate([np.broadcast_to(m.particle_velocity, m.particle_position.shape) for m in models])
    xp = torch.from_numpy(np.ascontiguousarray(x)).pin_memory()
    vp = torch.from_numpy(np.ascontiguousarray(v, np.float32)).pin_memory()
    b = SceneBatch(cfg, models, x=xp.numpy(), v=vp.numpy())
    b.setup()
    b.step(12, DT)
    st = b.state()
    b.close()
    for q in ("x", "v", "F", "aux", "id"):
        assert np.array_equal(getattr(st, q), getattr(ref, q)), q
    with pytest.raises(ValueError):
        SceneBatch(cfg, models, x=x[:-1], v=v[:-1])
    with pytest.raises(ValueError):
        SceneBatch(cfg, models, x=x)

