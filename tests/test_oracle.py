"""Self-checks of the FP64 oracle: the identities the reference's algorithm satisfies.

The oracle (oracle/ckmpm_oracle.cpp) is the checker for the CUDA path; these
tests pin its arithmetic independently of any GPU: SVD conventions, the CK
weights, conservation of mass and momentum by P2G, exact transport of a
uniform velocity field, the first-step dt = 0 rule and the block sets.
"""
import math

import numpy as np
import pytest

from ckmpm_b200 import scenes
from ckmpm_b200.engine import MPMConfig, MPMMaterial, MPMModel


def test_svd_conventions(oracle_mod):
    rng = np.random.default_rng(0)
    mats = [rng.normal(size=(3, 3)) for _ in range(50)]
    mats += [np.eye(3), np.diag([2.0, 2.0, 2.0]), np.diag([1.0, 1.0, -1.0]), np.diag([3.0, 1e-7, 1e-7])]
    mats += [np.diag([1.5, 1.5, 0.5]) @ np.linalg.qr(rng.normal(size=(3, 3)))[0]]
    for A in mats:
        U, S, V = oracle_mod.svd3(A)
        assert np.allclose(U @ np.diag(S) @ V.T, A, atol=1e-12 * max(1.0, np.abs(A).max()))
        assert np.allclose(U @ U.T, np.eye(3), atol=1e-12)
        assert np.allclose(V @ V.T, np.eye(3), atol=1e-12)
        assert np.linalg.det(U) > 0 and np.linalg.det(V) > 0
        assert S[0] >= S[1] - 1e-12 >= abs(S[2]) - 2e-12
        assert S[0] >= 0 and S[1] >= 0
        if abs(np.linalg.det(A)) > 1e-9:
            assert np.sign(S[2]) == np.sign(np.linalg.det(A))


def test_ck_weight_partition_and_bounds(oracle_mod):
    for o in np.linspace(0, 1, 101)[:-1]:
        w0 = oracle_mod.ck_w0(o)
        assert 0.0 <= w0 <= 1.0
        assert math.isclose(w0, 1 - o + math.sin(2 * math.pi * o) / (2 * math.pi), abs_tol=1e-15)
    # The two staggered grids' first moments cancel: sum_g (w1 - o_g) = 0
    # for offsets half a cell apart (mpm_kernel.cuh:91-114 construction).
    for s in np.linspace(0.3, 7.7, 37):
        tot = 0.0
        for g in (-1, 1):
            base = int(s - 0.25 * g)
            o = s - base - 0.25 * g
            tot += (1 - oracle_mod.ck_w0(o)) - o
        assert abs(tot) < 1e-12


def _rigid_scene(v0, gravity=0.0):
    cfg, models = scenes.jelly_cube(lo=(0.45, 0.45, 0.45), hi=(0.55, 0.55, 0.55), v0=v0, gravity=gravity)
    # A "material" with negligible stiffness so the test isolates transport.
    models[0].material = MPMMaterial.fixed_corotated(1e-6, 1e-6)
    return cfg, models


def test_uniform_translation_is_exact(oracle_mod):
    v0 = (0.3, -0.2, 0.1)
    cfg, models = _rigid_scene(v0)
    o = oracle_mod.OracleScene(cfg, models)
    o.setup()
    dt = 1e-3
    o.step(1, dt)  # first substep advects with dt = 0 (mpm_engine.cuh:479-480)
    st = o.state(0)
    assert np.allclose(st["x"], models[0].particle_position, atol=1e-12)
    o.step(10, dt)
    st = o.state(0)
    expect = models[0].particle_position.astype(np.float64) + np.asarray(v0) * 10 * dt
    assert np.allclose(st["x"], expect, atol=1e-10)
    assert np.allclose(st["v"], np.asarray(v0)[None, :], atol=1e-10)
    assert np.allclose(st["F"], np.eye(3)[None], atol=1e-9)


def test_p2g_conserves_mass_and_momentum(oracle_mod):
    cfg, models = scenes.jelly_cube(lo=(0.42, 0.44, 0.46), hi=(0.58, 0.57, 0.55), v0=(0.5, -1.0, 0.25),
                                    gravity=0.0)
    o = oracle_mod.OracleScene(cfg, models)
    o.setup()
    m = models[0]
    _, g = o.grid()
    # Each staggered grid carries the full mass (partition of unity per grid).
    assert np.isclose(g[:, 0].sum(), 2 * m.particle_mass * m.GetParticleCount(), rtol=1e-12)
    p0 = g[:, 1:4].sum(axis=(0, 2, 3))
    o.step(3, 2e-4)
    _, g = o.grid()
    assert np.isclose(g[:, 0].sum(), 2 * m.particle_mass * m.GetParticleCount(), rtol=1e-12)
    p1 = g[:, 1:4].sum(axis=(0, 2, 3))
    assert np.allclose(p0, p1, rtol=1e-9, atol=1e-12)


def test_block_sets(oracle_mod):
    cfg, models = scenes.jelly_cube()
    o = oracle_mod.OracleScene(cfg, models)
    keys, counts = o.blocks(0, 0)
    x = models[0].particle_position.astype(np.float64)
    K = ((np.floor(x / cfg.dx + 0.25).astype(int) - 2) // 4)
    uniq, cnt = np.unique(K, axis=0, return_counts=True)
    # Right after setup the reference's partition also holds the blocks of the +dx/4 grid's
    # cells (ActivateBlocksWithParticles, include/mpm_algorithm.cuh:713-736), with no particles.
    K2 = ((np.floor(x / cfg.dx - 0.25).astype(int) - 2) // 4)
    allk = np.unique(np.concatenate([uniq, K2]), axis=0)
    c = dict(zip(map(tuple, uniq), cnt))
    assert len(allk) > len(uniq)
    assert np.array_equal(keys, allk.astype(np.int32))
    assert np.array_equal(counts, np.array([c.get(tuple(k), 0) for k in allk], np.uint32))
    kn, _ = o.blocks(0, 1)
    ke, _ = o.blocks(0, 2)
    sa, sn, se = {tuple(k) for k in keys}, {tuple(k) for k in kn}, {tuple(k) for k in ke}
    assert sa <= sn <= se
    for (a, b, c) in sa:
        for d in np.ndindex(2, 2, 2):
            assert (a + d[0], b + d[1], c + d[2]) in sn
        for d in np.ndindex(3, 3, 3):
            assert (a + d[0] - 1, b + d[1] - 1, c + d[2] - 1) in se


def test_sticky_walls_stop_particles(oracle_mod):
    # Particles driven into the wall stop at the two-block sticky layer.
    cfg, models = scenes.jelly_cube(lo=(0.2, 0.2, 0.45), hi=(0.3, 0.3, 0.55), v0=(-2.0, 0.0, 0.0), gravity=0.0)
    o = oracle_mod.OracleScene(cfg, models)
    o.setup()
    o.step(400, 2e-4)
    st = o.state(0)
    assert st["alive"].all()
    assert st["x"][:, 0].min() > 6 * cfg.dx


def test_drucker_prager_return_map_projects(oracle_mod):
    lam, mu = 1e4, 1e4
    rng = np.random.default_rng(3)
    for _ in range(20):
        F = np.eye(3) + 0.2 * rng.normal(size=(3, 3))
        if np.linalg.det(F) <= 0.1:
            continue
        Fn, logjp, tau = oracle_mod.constitutive(2, [lam, mu, 0, 0], np.zeros((3, 3)), 0.0, F, 0.0)
        U, S, V = np.linalg.svd(Fn)
        eps = np.log(np.maximum(np.abs(S), 1e-4))
        tr = eps.sum()
        dev = eps - tr / 3
        ys = 0.816496580927726 * 2 * 0.5 / 2.5
        # After projection: either expanded (tr >= 0, F -> rotation) or inside the cone.
        if tr < -1e-12:
            assert np.linalg.norm(dev) + (3 * lam + 2 * mu) / (2 * mu) * tr * ys <= 1e-6
        assert np.allclose(tau, tau.T, atol=1e-8 * max(1, np.abs(tau).max()))


def test_fluid_pressure(oracle_mod):
    prm = [1e4, 7.0, 0.0, 1.0]
    Cm = np.diag([0.1, 0.1, 0.1])
    F, J, tau = oracle_mod.constitutive(3, prm, Cm, 1e-2, np.eye(3), 1.0)
    J_expect = 1.0 + 0.3 * 1e-2
    p = 1e4 * (J_expect ** -7.0 - 1.0)
    assert math.isclose(J, J_expect, rel_tol=1e-12)
    assert np.allclose(tau, -p * J_expect * np.eye(3), rtol=1e-12)


def test_out_of_domain_particles_are_dropped(oracle_mod):
    cfg = MPMConfig(dx=1 / 64, domain_blocks=(16, 16, 16), gravity=0.0)
    x = np.array([[0.5, 0.5, 0.5], [1.5, 0.5, 0.5], [-0.2, 0.5, 0.5]], np.float32)
    m = MPMModel(1e-3, 1e-6, x, np.zeros((1, 3), np.float32), MPMMaterial.fixed_corotated(1e3, 1e3))
    o = oracle_mod.OracleScene(cfg, [m])
    st = o.state(0)
    assert st["alive"].tolist() == [True, False, False]


def test_von_mises_projects_onto_the_yield_surface(oracle_mod):
    """Von Mises (mpm_algorithm.cuh:404-490): a trial strain outside the surface
    ends with |dev log S| = yield / (2 mu), volume (tr log S) unchanged; inside,
    F is untouched and tau is the StVK-Hencky stress of F."""
    mu, lam, ys = 2.0e4, 3.0e4, 200.0
    C = np.zeros((3, 3))
    F = np.diag([1.2, 0.9, 1.0])
    Fo, _, tau = oracle_mod.constitutive(4, [mu, lam, ys], C, 0.0, F, 0.0)
    S = np.linalg.svd(Fo, compute_uv=False)
    eps = np.log(S)
    dev = eps - eps.mean()
    assert abs(np.linalg.norm(dev) - ys / (2 * mu)) < 1e-12
    assert abs(eps.sum() - np.log(np.linalg.svd(F, compute_uv=False)).sum()) < 1e-12
    F2 = np.diag([1.001, 0.9995, 1.0])
    Fo2, _, tau2 = oracle_mod.constitutive(4, [mu, 1e4 * lam, 1e6], C, 0.0, F2, 0.0)
    assert np.allclose(Fo2, F2, atol=1e-15)
    ls = np.log(np.diag(F2))
    expect = np.diag((2 * mu * ls + 1e4 * lam * ls.sum()))  # tau = P F^T = diag(phi_i s_i)
    assert np.allclose(tau2, expect, rtol=1e-10, atol=1e-8)


def test_nacc_rest_state_and_hardening(oracle_mod):
    """NACC (mpm_material.cuh:520-669): F = I carries no stress and no plastic
    flow; a strong compression leaves [pMin, p0], projects to J = Je_new with
    the clamped pressure K (1 - J^2) / 2 = p0, and hardens:
    logJp += log(Je_trial / Je_new) < 0 raises p0."""
    prm = [1.0e4, 2.0e4, -0.04, 0.5, 10.0, 1.0, 1.0]
    C = np.zeros((3, 3))
    F, a, tau = oracle_mod.constitutive(5, prm, C, 0.0, np.eye(3), -0.04)
    assert np.allclose(tau, 0, atol=1e-9) and np.allclose(F, np.eye(3)) and a == -0.04
    Fc = np.eye(3) * 0.7  # p_trial = K (1 - Je^2) / 2 = 0.44 K > p0 = 0.41 K
    Fn, a2, tau2 = oracle_mod.constitutive(5, prm, C, 0.0, Fc, -0.04)
    p0 = (2 * prm[0] / 3 + prm[1]) * (1e-5 + np.sinh(prm[4] * 0.04))
    assert abs(-np.trace(tau2) / 3 - p0) < 1e-9 * p0  # isotropic projection: tau = -p0 I
    assert np.allclose(tau2, -p0 * np.eye(3), atol=1e-9 * p0)
    je = 0.7 ** 3
    jn = np.linalg.det(Fn)
    assert a2 < -0.04 and abs(a2 - (-0.04 + np.log(je / jn))) < 1e-12  # p0 grows with -logJp


def test_linear_stored_stress(oracle_mod):
    """The linear model's update (mpm_algorithm.cuh:107-191): Q <- (Q + 50 (C +
    C^T - I) dt) det F, rows 1 and 2 zeroed, on a fresh particle (Q = 0)."""
    cfg, _ = __import__("ckmpm_b200").scenes.jelly_cube()
    from ckmpm_b200.engine import MPMMaterial, MPMModel
    x = np.array([[0.5, 0.5, 0.5]], np.float32)
    m = MPMModel(1.0, 1.0 / 8 / 64 ** 3, x, np.array([[0.1, 0.0, 0.0]], np.float32), MPMMaterial.linear(1.0, 1.0))
    o = oracle_mod.OracleScene(cfg, [m])
    o.setup()
    o.step(1, 1e-4)
    st = o.state(0)
    assert np.isfinite(st["x"]).all() and np.allclose(st["F"][0], np.eye(3))


def test_rigid_particles(oracle_mod):
    """Rigid particles (include/mpm_algorithm.cuh:1063-1069, 1609-1624): the first
    R particles of a von Mises model move by dt * velocity (the first substep
    advects with dt = 0), keep F = I and report v = 0; they deposit mass with
    zero momentum, so the deformable rest of the cube moves differently from a
    run without them.  The rigid flag is aux (1 deformable, 0 rigid)."""
    cfg, models = scenes.material_cube("von_mises")
    R, dt, n = 2048, 1e-4, 12
    vr = np.array([2.0, -1.0, 0.5])
    o = oracle_mod.OracleScene(cfg, models)
    o.set_rigid(R, vr)
    o.setup()
    x0 = o.state(0)["x"].copy()
    o.step(n, dt)
    st = o.state(0)
    assert np.array_equal(st["aux"][:R], np.zeros(R)) and np.all(st["aux"][R:] == 1.0)
    np.testing.assert_allclose(st["x"][:R] - x0[:R], np.tile((n - 1) * dt * vr, (R, 1)), rtol=0, atol=1e-12)
    assert np.abs(st["F"][:R] - np.eye(3)).max() == 0.0
    assert np.abs(st["v"][:R]).max() == 0.0
    free = oracle_mod.OracleScene(cfg, models)
    free.setup()
    free.step(n, dt)
    ref = free.state(0)
    assert np.all(ref["aux"] == 1.0)
    # The deformable particles next to the rigid slab feel its zero-momentum mass.
    assert np.abs(st["x"][R:] - ref["x"][R:]).max() > 1e-7
    # A velocity change applies to the following substeps only.
    o.set_rigid_velocity(-vr)
    o.step(3, dt)
    np.testing.assert_allclose(o.state(0)["x"][:R] - st["x"][:R], np.tile(-3 * dt * vr, (R, 1)), rtol=0, atol=1e-12)


def _field_cube(rule_kind, param=None, v0=(1.0, -0.5, 0.25)):
    """Cube in a boundary field whose every cell carries one rule (oracle)."""
    from ckmpm_b200.boundary import BoundaryField
    cfg, models = scenes.jelly_cube(lo=(0.45, 0.45, 0.45), hi=(0.55, 0.55, 0.55), v0=v0, gravity=0.0)
    cfg.boundary = "field"
    bf = BoundaryField(cfg)
    bf.rule[...] = rule_kind
    if param is not None:
        bf.param[...] = np.asarray(param, np.float32)
    cfg.boundary_field = bf.arrays()
    return cfg, models


def test_boundary_field_rules(oracle_mod):
    """The per-cell rules of a boundary field (the reference's irregular-boundary
    hook as data, mpm_algorithm.cuh:795-799), one rule over the whole domain:
    the velocity the next G2P reads is the rule applied to the free velocity."""
    v0 = np.array([1.0, -0.5, 0.25])
    n = np.array([0.0, 0.6, 0.8])  # a unit normal
    u = np.array([0.3, 0.2, -0.1])
    expect = {
        0: v0,                            # free
        1: np.zeros(3),                   # fixed
        2: v0 - (n @ v0) * n,             # slip
        3: u,                             # prescribed velocity
        4: v0 if n @ v0 >= 0 else v0 - (n @ v0) * n,  # separate: n . v = -0.1 < 0, so projected
    }
    for kind, want in expect.items():
        param = u if kind == 3 else n
        cfg, models = _field_cube(kind, param)
        o = oracle_mod.OracleScene(cfg, models)
        o.setup()
        v = o.state(0)["v"]
        np.testing.assert_allclose(v, np.tile(want, (len(v), 1)), atol=1e-9, err_msg=f"rule {kind}")


def test_boundary_field_helpers():
    """BoundaryField builds the reference scenes' hook rules: slip walls with the
    normalised sum of face normals, fixed and rotating boxes, a one-sided floor."""
    from ckmpm_b200.boundary import FIXED, SEPARATE, SLIP, VELOCITY, BoundaryField
    cfg, _ = scenes.jelly_cube()
    bf = BoundaryField(cfg).slip_walls(8)
    assert bf.shape == (64, 64, 64)
    assert bf.rule[30, 30, 30] == 0 and bf.rule[3, 30, 30] == SLIP and bf.rule[60, 3, 30] == SLIP
    np.testing.assert_allclose(bf.param[3, 30, 30], [1, 0, 0])
    np.testing.assert_allclose(bf.param[60, 3, 30], np.array([-1, 1, 0]) / np.sqrt(2), rtol=1e-7)
    np.testing.assert_allclose(bf.param[0, 63, 0], np.array([1, -1, 1]) / np.sqrt(3), rtol=1e-7)
    bf.fixed_box((20, 0, 20), (24, 4, 24)).separate_below(2)
    assert bf.rule[21, 3, 21] == FIXED and bf.rule[40, 1, 40] == SEPARATE
    bf.rotating_box((10, 10, 10), (20, 20, 12), center=(0.25, 0.25, 0.0), axis=(0, 0, -1), factor=2.0)
    c = (15, 10, 11)
    r = np.array([c[0] / 64 - 0.25, c[1] / 64 - 0.25, 0.0])
    v = bf.param[c]
    assert bf.rule[c] == VELOCITY
    np.testing.assert_allclose(np.linalg.norm(v), 2.0 * np.linalg.norm(r), rtol=1e-6)
    assert abs(v @ r) < 1e-7  # tangential
