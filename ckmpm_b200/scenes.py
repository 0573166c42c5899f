"""Seeded synthetic scenes with the shapes, sizes and materials of the benchmark configurations.

Particles are seeded on a sub-cell lattice of spacing dx / ppc^(1/3) with a
uniform jitter of one lattice spacing per particle (numpy PCG64, seed 0 unless
given), kept when inside the shape.  Particle volume is dx^3 / ppc and mass
rho * volume, as the reference's scenes do
(tests/fluid_dam_break/test_fluid_dam_break.cuh:39-42).
"""
from __future__ import annotations

import math

import numpy as np

from .engine import MPMConfig, MPMMaterial, MPMModel, compute_lame_parameters


def lattice(lo, hi, spacing: float, rng: np.random.Generator) -> np.ndarray:
    """Jittered lattice points inside the box [lo, hi)."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    n = np.maximum(np.ceil((hi - lo) / spacing).astype(int), 0)
    if n.min() <= 0:
        return np.zeros((0, 3), np.float32)
    idx = np.stack(np.meshgrid(*[np.arange(k) for k in n], indexing="ij"), -1).reshape(-1, 3).astype(np.float64)
    pts = lo + (idx + rng.random(idx.shape)) * spacing
    keep = np.all(pts < hi, axis=1)
    return pts[keep]


def box_particles(lo, hi, dx: float, ppc: int, rng) -> np.ndarray:
    return lattice(lo, hi, dx / round(ppc ** (1 / 3)), rng).astype(np.float32)


def sphere_particles(center, r: float, dx: float, ppc: int, rng) -> np.ndarray:
    c = np.asarray(center, np.float64)
    pts = lattice(c - r, c + r, dx / round(ppc ** (1 / 3)), rng)
    keep = np.sum((pts - c) ** 2, axis=1) < r * r
    return pts[keep].astype(np.float32)


def cylinder_y_particles(center_xz, y0: float, r: float, h: float, dx: float, ppc: int, rng) -> np.ndarray:
    cx, cz = center_xz
    pts = lattice((cx - r, y0, cz - r), (cx + r, y0 + h, cz + r), dx / round(ppc ** (1 / 3)), rng)
    keep = (pts[:, 0] - cx) ** 2 + (pts[:, 2] - cz) ** 2 < r * r
    return pts[keep].astype(np.float32)


def jelly_cube(seed: int = 0, dx: float = 1 / 64, lo=(0.4, 0.4, 0.4), hi=(0.6, 0.6, 0.6), ppc: int = 8,
               E: float = 5e4, nu: float = 0.3, rho: float = 1000.0, v0=(0.0, -1.0, 0.0), gravity: float = -9.8,
               dt: float = 1e-4, track_ids: bool = True) -> tuple[MPMConfig, list[MPMModel]]:
    """Jelly cube, fixed-corotated: dx=1/64, cube [0.4,0.6]^3 at 8 ppc (~16.8k particles),
    E=5e4, nu=0.3, rho=1000, v0=(0,-1,0), g=-9.8, dt=1e-4, sticky walls."""
    rng = np.random.default_rng(seed)
    x = box_particles(lo, hi, dx, ppc, rng)
    n_cells = round(1.0 / dx)
    cfg = MPMConfig(dx=dx, domain_blocks=(n_cells // 4,) * 3, gravity=gravity, dt=dt, track_ids=track_ids)
    lam, mu = compute_lame_parameters(E, nu)
    vol = dx ** 3 / ppc
    return cfg, [MPMModel(rho * vol, vol, x, np.asarray([v0], np.float32), MPMMaterial.fixed_corotated(lam, mu))]


def sand_column(seed: int = 0, dx: float = 1 / 256, r: float = 0.1, h: float = 0.4, ppc: int = 8,
                E: float = 3.5e5, nu: float = 0.3, rho: float = 1600.0, gravity: float = -9.8,
                dt: float = 5e-5, track_ids: bool = True) -> tuple[MPMConfig, list[MPMModel]]:
    """Sand column collapse, Drucker-Prager (friction angle 30 deg): dx=1/256, cylinder r=0.1,
    h=0.4 standing on y0 = 8 dx at (0.5, 0.5), 8 ppc (~1.69M particles), E=3.5e5, nu=0.3,
    rho=1600, dt=5e-5, slip floor at 8 cells."""
    rng = np.random.default_rng(seed)
    y0 = 8 * dx
    x = cylinder_y_particles((0.5, 0.5), y0, r, h, dx, ppc, rng)
    n_cells = round(1.0 / dx)
    cfg = MPMConfig(dx=dx, domain_blocks=(n_cells // 4,) * 3, gravity=gravity, dt=dt, boundary="slip_floor",
                    floor_cells=8.0, track_ids=track_ids)
    lam, mu = compute_lame_parameters(E, nu)
    vol = dx ** 3 / ppc
    return cfg, [MPMModel(rho * vol, vol, x, np.zeros((1, 3), np.float32), MPMMaterial.drucker_prager(lam, mu))]


def dam_break_mixed(seed: int = 0, dx: float = 1 / 512, ppc: int = 8, n_spheres: int = 64, r: float = 0.03,
                    fluid_hi=(0.4, 0.6, 1.0), bulk: float = 1e5, gamma: float = 7.15, viscosity: float = 0.1,
                    E: float = 1e5, nu: float = 0.3, rho: float = 1000.0, dt: float = 2e-5,
                    gravity: float = -9.8, track_ids: bool = False) -> tuple[MPMConfig, list[MPMModel]]:
    """Mixed large scene: J-fluid dam-break block [0,0.4]x[0,0.6]x[0,1] clipped to the
    two-block sticky margin (bulk 1e5, gamma 7.15 and viscosity 0.1 as the reference's
    dam-break scene) plus 64 fixed-corotated spheres r=0.03 (E=1e5, nu=0.3) at seeded
    positions with v0 ~ U(-2,2)^3; 8 ppc; dt=2e-5."""
    rng = np.random.default_rng(seed)
    margin = 8 * dx
    lo = np.array([margin] * 3)
    hi = np.minimum(np.asarray(fluid_hi), 1.0 - margin)
    xf = box_particles(lo, hi, dx, ppc, rng)
    spheres, vels = [], []
    for _ in range(n_spheres):
        c = rng.uniform(margin + r + 4 * dx, 1.0 - margin - r - 4 * dx, 3)
        c[0] = rng.uniform(hi[0] + r + 4 * dx, 1.0 - margin - r - 4 * dx)
        p = sphere_particles(c, r, dx, ppc, rng)
        spheres.append(p)
        vels.append(np.repeat(rng.uniform(-2, 2, (1, 3)).astype(np.float32), len(p), 0))
    xs = np.concatenate(spheres) if spheres else np.zeros((0, 3), np.float32)
    vs = np.concatenate(vels) if vels else np.zeros((1, 3), np.float32)
    n_cells = round(1.0 / dx)
    cfg = MPMConfig(dx=dx, domain_blocks=(n_cells // 4,) * 3, gravity=gravity, dt=dt, track_ids=track_ids)
    vol = dx ** 3 / ppc
    lam, mu = compute_lame_parameters(E, nu)
    models = [MPMModel(rho * vol, vol, xf, np.zeros((1, 3), np.float32), MPMMaterial.fluid(bulk, gamma, viscosity))]
    if len(xs):
        models.append(MPMModel(rho * vol, vol, xs, vs, MPMMaterial.fixed_corotated(lam, mu)))
    return cfg, models


def fluid_box(seed: int = 0, dx: float = 1 / 64, lo=(0.3, 0.3, 0.3), hi=(0.5, 0.6, 0.5), ppc: int = 8,
              bulk: float = 1e4, gamma: float = 7.15, viscosity: float = 0.1, rho: float = 1000.0,
              gravity: float = -9.8, v0=(0.5, 0.0, -0.25), track_ids: bool = True) -> tuple[MPMConfig, list[MPMModel]]:
    """Small J-fluid box for parity tests."""
    rng = np.random.default_rng(seed)
    x = box_particles(lo, hi, dx, ppc, rng)
    n_cells = round(1.0 / dx)
    cfg = MPMConfig(dx=dx, domain_blocks=(n_cells // 4,) * 3, gravity=gravity, track_ids=track_ids)
    vol = dx ** 3 / ppc
    return cfg, [MPMModel(rho * vol, vol, x, np.asarray([v0], np.float32), MPMMaterial.fluid(bulk, gamma, viscosity))]


def small_sand(seed: int = 0, dx: float = 1 / 64, r: float = 0.1, h: float = 0.25, ppc: int = 8,
               E: float = 3.5e5, nu: float = 0.3, rho: float = 1600.0, gravity: float = -9.8,
               track_ids: bool = True) -> tuple[MPMConfig, list[MPMModel]]:
    """Small Drucker-Prager column on the slip floor, for parity tests."""
    rng = np.random.default_rng(seed)
    y0 = 8 * dx
    x = cylinder_y_particles((0.5, 0.5), y0, r, h, dx, ppc, rng)
    n_cells = round(1.0 / dx)
    cfg = MPMConfig(dx=dx, domain_blocks=(n_cells // 4,) * 3, gravity=gravity, boundary="slip_floor",
                    floor_cells=8.0, track_ids=track_ids)
    lam, mu = compute_lame_parameters(E, nu)
    vol = dx ** 3 / ppc
    return cfg, [MPMModel(rho * vol, vol, x, np.zeros((1, 3), np.float32), MPMMaterial.drucker_prager(lam, mu))]


def material_cube(kind: str, seed: int = 0, dx: float = 1 / 64, lo=(0.42, 0.42, 0.42), hi=(0.58, 0.58, 0.58),
                  ppc: int = 8, rho: float = 1000.0, gravity: float = -9.8,
                  track_ids: bool = True) -> tuple[MPMConfig, list[MPMModel]]:
    """Small cube of one of the reference's other materials, with an initial
    velocity field that loads it at once (parity tests):
    * 'von_mises': E 2e4, nu 0.3, yield stress 100 Pa, shear v = (20 (y - 0.5), 0, 0);
    * 'nacc': E 2e4, nu 0.4 (mu, lambda in the model's field order), alpha0 -0.01,
      beta 0.5, hardening factor 0.8, M 2.36, hardening on (the reference's oreo
      scene, tests/oreo/test_oreo.cuh), converging v = -10 (x - centre);
    * 'linear': E 5e4, nu 0.3, v0 = (0, -1, 0)."""
    rng = np.random.default_rng(seed)
    x = box_particles(lo, hi, dx, ppc, rng)
    c = (np.asarray(lo) + np.asarray(hi)) / 2
    if kind == "von_mises":
        lam, mu = compute_lame_parameters(2e4, 0.3)
        mat = MPMMaterial.von_mises(mu, lam, 100.0)
        v = np.zeros_like(x)
        v[:, 0] = 20.0 * (x[:, 1] - c[1])
    elif kind == "nacc":
        lam, mu = compute_lame_parameters(2e4, 0.4)
        mat = MPMMaterial.nacc(mu, lam, -0.01, 0.5, 0.8, 2.36, True)
        v = (-10.0 * (x - c)).astype(np.float32)
    elif kind == "linear":
        lam, mu = compute_lame_parameters(5e4, 0.3)
        mat = MPMMaterial.linear(lam, mu)
        v = np.asarray([[0.0, -1.0, 0.0]], np.float32)
    else:
        raise ValueError(kind)
    n_cells = round(1.0 / dx)
    cfg = MPMConfig(dx=dx, domain_blocks=(n_cells // 4,) * 3, gravity=gravity, track_ids=track_ids)
    vol = dx ** 3 / ppc
    return cfg, [MPMModel(rho * vol, vol, x, np.asarray(v, np.float32), mat)]


def batched_scenes(n_scenes: int = 256, seed: int = 0, dx: float = 1 / 64, ppc: int = 8, n_min: int = 2000,
                   n_max: int = 200000, dt: float = 1e-4, gravity: float = -9.8) -> tuple[MPMConfig, list[MPMModel]]:
    """Batched form: n_scenes independent scenes on a 64^3 domain (dx = 1/64,
    sticky walls), one model each.  Per scene: target particle count
    log-uniform in [n_min, n_max] at 8 ppc; shape box (aspect ratios
    U(0.7, 1.4)) or sphere with equal odds; material uniform over
    {fixed-corotated, J-fluid, Drucker-Prager}; E ~ logU[1e4, 1e6],
    nu ~ U[0.2, 0.4]; rho 1000 (1600 for sand); v0 ~ U(-1, 1)^3 per scene; centre
    uniform where the shape keeps one block of room inside the two-block
    sticky margin.  The fluid's bulk modulus is E / gamma (gamma 7.15,
    viscosity 0.1), so its acoustic stiffness bulk * gamma is the drawn E.
    Actual counts follow the jittered lattice, not the target exactly."""
    rng = np.random.default_rng(seed)
    n_cells = round(1.0 / dx)
    cfg = MPMConfig(dx=dx, domain_blocks=(n_cells // 4,) * 3, gravity=gravity, dt=dt, track_ids=True)
    lo_free, hi_free = 12 * dx, 1.0 - 12 * dx
    vol = dx ** 3 / ppc
    models = []
    for _ in range(n_scenes):
        target = math.exp(rng.uniform(math.log(n_min), math.log(n_max)))
        volume = target / ppc * dx ** 3
        kind = int(rng.integers(0, 3))
        E = math.exp(rng.uniform(math.log(1e4), math.log(1e6)))
        nu = float(rng.uniform(0.2, 0.4))
        v0 = rng.uniform(-1.0, 1.0, 3).astype(np.float32)
        if rng.random() < 0.5:
            a = rng.uniform(0.7, 1.4, 3)
            ext = a * (volume / np.prod(a)) ** (1 / 3)
            ext = np.minimum(ext, hi_free - lo_free - 2 * dx)
            c = rng.uniform(lo_free + ext / 2, hi_free - ext / 2)
            x = box_particles(c - ext / 2, c + ext / 2, dx, ppc, rng)
        else:
            r = min((3 * volume / (4 * math.pi)) ** (1 / 3), (hi_free - lo_free) / 2 - dx)
            c = rng.uniform(lo_free + r, hi_free - r, 3)
            x = sphere_particles(c, r, dx, ppc, rng)
        if kind == 0:
            lam, mu = compute_lame_parameters(E, nu)
            mat, rho = MPMMaterial.fixed_corotated(lam, mu), 1000.0
        elif kind == 1:
            mat, rho = MPMMaterial.fluid(E / 7.15, 7.15, 0.1), 1000.0
        else:
            lam, mu = compute_lame_parameters(E, nu)
            mat, rho = MPMMaterial.drucker_prager(lam, mu), 1600.0
        models.append(MPMModel(rho * vol, vol, x, np.repeat(v0[None], len(x), 0), mat))
    return cfg, models


def diff_cube(seed: int = 0, dx: float = 1 / 64, half: float = 0.1445, ppc: int = 8, E: float = 5e4,
              log_e_sigma: float = 0.2, nu: float = 0.3, rho: float = 1000.0, nsteps: int = 200, dt: float = 1e-4,
              checkpoint_every: int = 1, gravity: float = -9.8) -> dict:
    """Differentiable form: fixed-corotated cube of ~50k particles (8 ppc, side
    2 * half centred at 0.5) on a 64^3 grid with sticky walls; per-particle
    log E ~ N(log E, log_e_sigma), nu = 0.3; v0 ~ U(-0.5, 0.5)^3 shared by all
    particles (learnable per particle); 200 substeps of dt = 1e-4, every
    substep kept as a checkpoint (x, F and the node velocities: ~2.2 GB of HBM,
    so the backward recomputes nothing); target = initial centre of mass +
    U(-0.05, 0.05)^3."""
    rng = np.random.default_rng(seed)
    x = box_particles((0.5 - half,) * 3, (0.5 + half,) * 3, dx, ppc, rng)
    n = len(x)
    logE = (math.log(E) + log_e_sigma * rng.standard_normal(n)).astype(np.float32)
    v0 = np.repeat(rng.uniform(-0.5, 0.5, (1, 3)), n, 0).astype(np.float32)
    target = (x.astype(np.float64).mean(0) + rng.uniform(-0.05, 0.05, 3)).astype(np.float32)
    n_cells = round(1.0 / dx)
    cfg = MPMConfig(dx=dx, domain_blocks=(n_cells // 4,) * 3, gravity=gravity, dt=dt, track_ids=True)
    vol = dx ** 3 / ppc
    return {"config": cfg, "x0": x, "v0": v0, "logE": logE, "target": target, "mass": rho * vol, "volume": vol,
            "nu": nu, "nsteps": nsteps, "dt": dt, "checkpoint_every": checkpoint_every}


WORKLOADS = {
    "jelly_cube": jelly_cube,
    "sand_column": sand_column,
    "dam_break_mixed": dam_break_mixed,
    "batched_256": batched_scenes,
}
