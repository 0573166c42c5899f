"""The hand-written adjoint of the differentiable substep, on CPU in double.

tests/native/diff_check.cpp drives the generic forward and adjoint of
ckmpm_b200/csrc/diff_math.cuh (the code the GPU kernels instantiate with
float) in double precision on a small dense grid; the gradients of a linear
functional of (xT, FT) with respect to x0, v0 and log E must match central
finite differences of that forward to 1e-6 relative (the derivation is exact;
what remains is the O(eps^2) truncation of the differences).
"""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

SRC = Path(__file__).resolve().parent / "native" / "diff_check.cpp"


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    out = tmp_path_factory.mktemp("diffcheck") / "diff_check.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", str(out), str(SRC)], check=True)
    L = C.CDLL(str(out))
    d = C.POINTER(C.c_double)
    L.diff_rollout.argtypes = [C.c_int, d, d, d, C.c_double, C.c_double, C.c_double, C.c_int, C.c_double, C.c_int,
                               C.c_double, d, d, d, d, d, d, d]
    return L


def _p(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


@pytest.mark.parametrize("nsteps", [2, 12, 30])
def test_adjoint_matches_central_differences(harness, nsteps):
    rng = np.random.default_rng(nsteps)
    nc, dx = 32, 1 / 32
    g = np.stack(np.meshgrid(*[np.arange(0.40, 0.50, dx / 2)] * 3, indexing="ij"), -1).reshape(-1, 3)
    x0 = g + rng.random(g.shape) * dx / 2
    n = len(x0)
    v0 = np.tile([0.3, -0.5, 0.2], (n, 1)) + 0.1 * rng.standard_normal((n, 3))
    logE = np.log(1e4) + 0.2 * rng.standard_normal(n)
    nu, vol = 0.3, dx ** 3 / 8
    mass = 1000 * vol
    gxT = rng.standard_normal((n, 3))
    gFT = 0.1 * rng.standard_normal((n, 9))

    def run(x0, v0, logE, grad=False):
        xT, FT = np.zeros((n, 3)), np.zeros((n, 9))
        gx, gv, gE = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n)
        bad = harness.diff_rollout(n, _p(x0), _p(v0), _p(logE), nu, mass, vol, nsteps, 1e-3, nc, -9.8, _p(xT),
                                   _p(FT), _p(gxT) if grad else None, _p(gFT) if grad else None, _p(gx), _p(gv),
                                   _p(gE))
        assert bad == 0
        return (gxT * xT).sum() + (gFT * FT).sum(), gx, gv, gE

    _, gx, gv, gE = run(x0, v0, logE, True)
    args = {"x0": x0, "v0": v0, "logE": logE}
    for name, grad, eps in (("v0", gv, 1e-5), ("logE", gE, 1e-5), ("x0", gx, 1e-7)):
        d = rng.standard_normal(args[name].shape)
        a = dict(args)
        a[name] = args[name] + eps * d
        lp = run(**a)[0]
        a[name] = args[name] - eps * d
        lm = run(**a)[0]
        fd = (lp - lm) / (2 * eps)
        ad = float((grad * d).sum())
        print(f"{nsteps} substeps, {name}: fd {fd:.10e} adjoint {ad:.10e}")
        assert abs(fd - ad) <= 1e-6 * abs(fd) + 1e-9, (name, fd, ad)


def test_checkpoint_interval_by_memory():
    """The rollout keeps every substep when its checkpoints fit the budget and
    picks the smallest interval that fits otherwise (host logic, no GPU)."""
    from ckmpm_b200.diff import auto_checkpoint_interval, rollout_bytes
    from ckmpm_b200.engine import MPMConfig
    cfg = MPMConfig(dx=1 / 64, domain_blocks=(16, 16, 16))
    n, nsteps = 50_626, 200
    full = rollout_bytes(cfg, n, nsteps, 1)
    # 200 checkpoints of x, F (48 B per particle) and 2 x 64^3 node velocities (16 B)
    assert full == 200 * (48 * n + 16 * 2 * 64 ** 3) + 48 * n + 16 * 2 * 64 ** 3
    assert auto_checkpoint_interval(cfg, n, nsteps, full) == 1
    k = auto_checkpoint_interval(cfg, n, nsteps, full // 4)
    assert k > 1 and rollout_bytes(cfg, n, nsteps, k) <= full // 4 < rollout_bytes(cfg, n, nsteps, k - 1)
    # nothing fits: the interval of least memory (the checkpoints fall with it, the tape grows)
    least = auto_checkpoint_interval(cfg, n, nsteps, 0)
    assert all(rollout_bytes(cfg, n, nsteps, least) <= rollout_bytes(cfg, n, nsteps, e) for e in range(1, nsteps + 1))
    assert 1 < least < nsteps
