"""The timed CPU baseline (oracle/pic_baseline.cpp, the python-src PIC demo restated in C++/OpenMP)
against a float64 NumPy restatement of the demo's substep, on a small grid.

The demo (python-src/python_demo.py:101-215) is a Taichi program that cannot run here; its substep is
restated below, vectorised over particles, in the demo's own order: clear the grid; P2G on the two
staggered grids with the compact kernel's stencil (compact_kernel_stencil :60-67), mass w m and
momentum w m v + dt PF grad_w (compact_kernel_gradient :69-74, compute_fixed_corotated :84-91); grid
update v = mv / m above 1e-8 m_p, gravity on y, zero within `wall` cells of the edge (:146-164); G2P
v = 1/2 sum w v_i, x += dt v, F <- (I + dt/2 sum v_i grad_w^T) F (:167-192).  The C++ baseline runs
in float32 on one thread here, so the two agree to float32 rounding.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest


def pic_numpy(x, v0, n_grid, E, nu, rho, gravity, wall, dt, nsteps):
    """float64 restatement of the demo's substep; returns (x, v, F, grid mass per staggered grid)."""
    x = np.array(x, np.float64)
    n = len(x)
    v = np.broadcast_to(np.asarray(v0, np.float64), (n, 3)).copy()
    F = np.broadcast_to(np.eye(3), (n, 3, 3)).copy()
    dx = 1.0 / n_grid
    vol = dx ** 3 / 8
    mass = rho * vol
    mu, lam = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
    two_pi = 2 * np.pi
    offsets = np.array([(i, j, k) for i in range(2) for j in range(2) for k in range(2)])
    masses = []

    def stencil(sign):
        base = np.trunc(x * n_grid - sign * 0.25).astype(np.int64)
        off = x * n_grid - (base + 0.25 * sign)
        st0 = 1 - off + np.sin(two_pi * off) / two_pi
        return base, off, np.stack([st0, 1 - st0], axis=-1)  # (n, 3, 2)

    def node_terms(off, st, I):
        kx, ky, kz = st[:, 0, I[0]], st[:, 1, I[1]], st[:, 2, I[2]]
        dw = off - I
        grad = np.sign(dw) * (np.cos(two_pi * np.abs(dw)) - 1)
        return kx * ky * kz, n_grid * np.stack([ky * kz, kx * kz, kx * ky], axis=-1) * grad

    for _ in range(nsteps):
        gm = np.zeros((n_grid, n_grid, n_grid, 2))
        gmv = np.zeros((n_grid, n_grid, n_grid, 2, 3))
        U, S, Vt = np.linalg.svd(F)
        R = U @ Vt
        J = S.prod(axis=1)
        PF = -vol * (2 * mu * (F - R) @ F.transpose(0, 2, 1) + (lam * (J - 1) * J)[:, None, None] * np.eye(3))
        for w, sign in enumerate((-1, 1)):
            base, off, st = stencil(sign)
            for I in offsets:
                wgt, gr = node_terms(off, st, I)
                c = base + I
                idx = (c[:, 0], c[:, 1], c[:, 2], np.full(n, w))
                np.add.at(gm, idx, wgt * mass)
                np.add.at(gmv, idx, (wgt * mass)[:, None] * v + dt * np.einsum("pij,pj->pi", PF, gr))
        masses.append(gm.sum(axis=(0, 1, 2)))
        gv = np.where((gm > mass * 1e-8)[..., None], gmv / np.where(gm > 0, gm, 1)[..., None], 0.0)
        gv[..., 1] += dt * gravity
        i = np.arange(n_grid)
        edge = (i < wall) | (i >= n_grid - wall)
        out = edge[:, None, None] | edge[None, :, None] | edge[None, None, :]
        gv[out] = 0.0
        vel = np.zeros((n, 3))
        Cv = np.zeros((n, 3, 3))
        for w, sign in enumerate((-1, 1)):
            base, off, st = stencil(sign)
            for I in offsets:
                wgt, gr = node_terms(off, st, I)
                c = base + I
                gvel = gv[c[:, 0], c[:, 1], c[:, 2], w]
                vel += wgt[:, None] * gvel
                Cv += gvel[:, :, None] * gr[:, None, :]
        vel *= 0.5
        x = x + dt * vel
        v = vel
        F = (np.eye(3) + 0.5 * dt * Cv) @ F
    return x, v, F, np.array(masses)


@pytest.fixture(scope="module")
def pic_lib():
    from oracle import oracle as O
    O.build()
    L = C.CDLL(str(O.PIC_LIB))
    f = C.POINTER(C.c_float)
    L.pic_run.restype = C.c_double
    L.pic_run.argtypes = [C.c_int, f, f, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                          C.c_double, C.c_int, C.c_int, C.POINTER(C.c_int)]
    return L


def run_cpp(L, x, v0, n_grid, E, nu, rho, gravity, wall, dt, nsteps, threads=1):
    x = np.ascontiguousarray(x, np.float32).copy()
    v = np.ascontiguousarray(v0, np.float32)
    f = C.POINTER(C.c_float)
    th = C.c_int()
    L.pic_run(len(x), x.ctypes.data_as(f), v.ctypes.data_as(f), len(v), n_grid, E, nu, rho, gravity, wall, dt,
              nsteps, threads, C.byref(th))
    return x, th.value


def cube(n_grid, lo, hi, seed=0):
    from ckmpm_b200 import scenes
    return scenes.box_particles(lo, hi, 1.0 / n_grid, 8, np.random.default_rng(seed))


def test_pic_baseline_matches_the_demo_restated(pic_lib):
    """A spinning, falling jelly cube on a 32^3 grid: 12 substeps, every particle's position within
    float32 rounding of the float64 restatement (displacements here reach ~4e-3)."""
    n_grid = 32
    x0 = cube(n_grid, (0.35, 0.4, 0.35), (0.6, 0.65, 0.6))
    c = x0.mean(axis=0)
    v0 = np.cross(np.array([0.0, 0.0, 6.0]), x0 - c) + np.array([0.2, -1.0, 0.1])
    args = dict(n_grid=n_grid, E=5e4, nu=0.3, rho=1000.0, gravity=-9.8, wall=3, dt=2e-4, nsteps=12)
    xr, vr, Fr, masses = pic_numpy(x0, v0, **args)
    xc, threads = run_cpp(pic_lib, x0, v0.astype(np.float32), **args)
    assert threads == 1
    moved = np.abs(xr - x0).max()
    assert moved > 1e-3
    err = np.abs(xc.astype(np.float64) - xr).max()
    print(f"max |x_cpp - x_numpy| = {err:.2e} (largest displacement {moved:.2e})")
    assert err <= 2e-6, err
    # the restatement deposits every particle's full mass on each staggered grid
    m = 1000.0 * (1.0 / n_grid) ** 3 / 8
    assert np.allclose(masses, len(x0) * m, rtol=1e-12)


def test_pic_baseline_threads_agree(pic_lib):
    """All host threads (the timed configuration) against one thread: the same positions up to the
    order of the OpenMP atomic sums."""
    n_grid = 32
    x0 = cube(n_grid, (0.4, 0.4, 0.4), (0.6, 0.6, 0.6), seed=1)
    v0 = np.array([[0.0, -1.0, 0.0]], np.float32)
    args = dict(n_grid=n_grid, E=5e4, nu=0.3, rho=1000.0, gravity=-9.8, wall=3, dt=2e-4, nsteps=10)
    x1, _ = run_cpp(pic_lib, x0, v0, threads=1, **args)
    xn, _ = run_cpp(pic_lib, x0, v0, threads=0, **args)
    assert np.abs(x1.astype(np.float64) - xn).max() <= 1e-6
