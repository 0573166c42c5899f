"""Differentiable rollout (ckmpm_diff_*, ckmpm_b200.diff) on the GPU.

  * its FP32 forward against the plain engine (uniform E) and against the FP64
    oracle with per-particle E: positions within 2e-6, F within 5e-5 after 40
    substeps (the plain-path parity tolerances);
  * gradients through torch.autograd against FP64 central finite differences
    of the oracle (per-particle Lame parameters, double inputs): within 1e-3
    relative, for directions in v0, log E and x0 and a linear functional of
    (xT, FT) that depends on all of them;
  * checkpointing: every-10, every-7, every-1 (the whole tape kept, no
    recomputation) and one-segment runs give the same xT and the same
    gradients, bit for bit (the forward's node sums and the adjoint's
    node-velocity sums are both exact integers), and so does a repeated run;
  * at the config-5 scale (50.6k particles, 200 substeps, a checkpoint at every
    substep):
    per-particle d loss / d log E and d loss / d v0 on a seeded sample of
    particles against FP64 central differences of the oracle.
"""
import numpy as np
import pytest

from ckmpm_b200 import Scene, scenes
from ckmpm_b200.engine import MPMMaterial, MPMModel

pytestmark = pytest.mark.gpu


def small_case(nsteps=40, every=10, half=0.06, seed=4):
    d = scenes.diff_cube(seed=seed, half=half, nsteps=nsteps, checkpoint_every=every)
    rng = np.random.default_rng(seed)
    d["v0"] = (d["v0"] + 0.1 * rng.standard_normal(d["v0"].shape)).astype(np.float32)
    return d


def lame(logE, nu):
    E = np.exp(np.asarray(logE, np.float64))
    return E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))


def make_sim(d):
    from ckmpm_b200.diff import DiffRollout
    return DiffRollout(d["config"], len(d["x0"]), d["mass"], d["volume"], d["nu"], d["nsteps"], d["dt"],
                       d["checkpoint_every"])


def tensors(d):
    import torch
    return (torch.tensor(d["x0"], device="cuda"), torch.tensor(d["v0"], device="cuda"),
            torch.tensor(d["logE"], device="cuda"))


def oracle_state(oracle_mod, d, x0, v0, logE):
    lam, mu = lame(logE, d["nu"])
    m = MPMModel(d["mass"], d["volume"], np.asarray(x0, np.float32), np.asarray(v0, np.float32),
                 MPMMaterial.fixed_corotated(float(lam[0]), float(mu[0])))
    o = oracle_mod.OracleScene(d["config"], [m])
    o.set_state(0, x=np.asarray(x0, np.float64))
    o.set_initial_velocity(0, np.asarray(v0, np.float64))
    o.set_lame(0, lam, mu)
    o.setup()
    o.step(d["nsteps"], d["dt"])
    st = o.state(0)
    assert st["alive"].all()
    o.close()
    return st["x"], st["F"].reshape(-1, 9)


def test_forward_matches_plain_engine(engine_lib):
    from ckmpm_b200.diff import rollout
    d = small_case()
    d["logE"][:] = np.log(5e4)
    sim = make_sim(d)
    xT, FT = rollout(sim, *tensors(d))
    lam, mu = lame(d["logE"][:1], d["nu"])
    s = Scene(d["config"])
    s.add_model(MPMModel(d["mass"], d["volume"], d["x0"], d["v0"], MPMMaterial.fixed_corotated(float(lam[0]),
                                                                                               float(mu[0]))))
    s.setup()
    s.step(d["nsteps"], d["dt"])
    st = s.state(0)
    ex = np.abs(xT.cpu().numpy() - st.x).max()
    eF = np.abs(FT.cpu().numpy() - st.F).max()
    print(f"diff forward vs plain engine: |dx| {ex:.3e} |dF| {eF:.3e}")
    assert ex <= 2e-6 and eF <= 5e-5


def test_forward_matches_oracle_per_particle_E(engine_lib, oracle_mod):
    from ckmpm_b200.diff import rollout
    d = small_case()
    sim = make_sim(d)
    xT, FT = rollout(sim, *tensors(d))
    xo, Fo = oracle_state(oracle_mod, d, d["x0"], d["v0"], d["logE"])
    ex = np.abs(xT.cpu().numpy() - xo).max()
    eF = np.abs(FT.cpu().numpy().reshape(-1, 9) - Fo).max()
    print(f"diff forward vs FP64 oracle: |dx| {ex:.3e} |dF| {eF:.3e}")
    assert ex <= 2e-6 and eF <= 5e-5


def test_gradients_match_fp64_finite_differences(engine_lib, oracle_mod):
    import torch
    from ckmpm_b200.diff import rollout
    d = small_case()
    n = len(d["x0"])
    rng = np.random.default_rng(11)
    c = rng.standard_normal((n, 3)) / n
    e = rng.standard_normal((n, 9)) / n
    sim = make_sim(d)
    x0, v0, lE = (t.requires_grad_() for t in tensors(d))
    xT, FT = rollout(sim, x0, v0, lE)
    loss = (torch.tensor(c, device="cuda", dtype=torch.float32) * xT).sum() + \
           (torch.tensor(e, device="cuda", dtype=torch.float32) * FT.reshape(n, 9)).sum()
    loss.backward()
    grads = {"x0": x0.grad.cpu().numpy().astype(np.float64), "v0": v0.grad.cpu().numpy().astype(np.float64),
             "logE": lE.grad.cpu().numpy().astype(np.float64)}
    base = {"x0": d["x0"].astype(np.float64), "v0": d["v0"].astype(np.float64), "logE": d["logE"].astype(np.float64)}

    def L(args):
        x, F = oracle_state(oracle_mod, d, args["x0"], args["v0"], args["logE"])
        return float((c * x).sum() + (e * F).sum())

    dirs = []
    for a in range(3):
        u = np.zeros((n, 3))
        u[:, a] = 1.0
        dirs.append(("v0", u, 1e-4))
    dirs.append(("logE", rng.standard_normal(n), 1e-4))
    dirs.append(("x0", rng.standard_normal((n, 3)), 1e-6))
    results = []
    for name, u, eps in dirs:
        a = dict(base)
        a[name] = base[name] + eps * u
        lp = L(a)
        a[name] = base[name] - eps * u
        lm = L(a)
        fd = (lp - lm) / (2 * eps)
        ad = float((grads[name] * u).sum())
        results.append((name, fd, ad))
        print(f"{name}: fd {fd:.8e} adjoint {ad:.8e} rel {abs(fd - ad) / max(abs(fd), 1e-30):.2e}")
    scale = max(abs(fd) for _, fd, _ in results)
    for name, fd, ad in results:
        assert abs(fd - ad) <= 1e-3 * abs(fd) + 1e-5 * scale, (name, fd, ad)


def test_checkpointing_gives_the_same_rollout_and_gradients(engine_lib):
    import torch
    from ckmpm_b200.diff import rollout
    out = []
    for every in (10, 40, 7, 1):
        d = small_case(every=every)
        sim = make_sim(d)
        x0, v0, lE = (t.requires_grad_() for t in tensors(d))
        xT, FT = rollout(sim, x0, v0, lE)
        target = torch.tensor(d["target"], device="cuda")
        loss = ((xT.mean(0) - target) ** 2).sum() + 1e-3 * (FT ** 2).sum()
        loss.backward()
        out.append((xT.detach().cpu().numpy(), x0.grad.cpu().numpy(), v0.grad.cpu().numpy(), lE.grad.cpu().numpy()))
        sim.close()
    for other in out[1:]:
        assert np.array_equal(other[0], out[0][0])
        for a, b in zip(other[1:], out[0][1:]):
            assert np.array_equal(a, b)


def test_gradients_are_bitwise_reproducible(engine_lib):
    import torch
    from ckmpm_b200.diff import rollout
    d = small_case()
    sim = make_sim(d)
    res = []
    for _ in range(2):
        x0, v0, lE = (t.requires_grad_() for t in tensors(d))
        xT, FT = rollout(sim, x0, v0, lE)
        ((xT.mean(0) - torch.tensor(d["target"], device="cuda")) ** 2).sum().backward()
        res.append((x0.grad.cpu().numpy(), v0.grad.cpu().numpy(), lE.grad.cpu().numpy()))
    for a, b in zip(*res):
        assert np.array_equal(a, b)
    sim.close()


def _oracle_loss(args):
    """FP64 loss sum_p c_p . xT_p of one oracle rollout (a spawn-pool worker)."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    from oracle import oracle as O
    d, v0, logE = args
    lam, mu = lame(logE, d["nu"])
    m = MPMModel(d["mass"], d["volume"], d["x0"], np.asarray(v0, np.float32), MPMMaterial.fixed_corotated(1.0, 1.0))
    o = O.OracleScene(d["config"], [m])
    o.set_state(0, x=d["x0"].astype(np.float64))
    o.set_initial_velocity(0, np.asarray(v0, np.float64))
    o.set_lame(0, lam, mu)
    o.setup()
    o.step(d["nsteps"], d["dt"])
    x = o.state(0)["x"]
    o.close()
    return float((d["c"] * x).sum())


def test_config5_per_particle_gradients_against_fp64_differences(engine_lib, oracle_mod):
    """The config-5 rollout (50.6k particles, 200 substeps, every substep kept): d loss / d log E_p
    and d loss / d v0_p (along a random unit direction) for 6 seeded particles p, against FP64
    central differences of the oracle's rollout with per-particle Lame parameters (24 rollouts of
    50.6k particles x 200 substeps, run in a spawn pool on the host cores).  The config-5 loss
    |com(xT) - target|^2 does not depend on any particle's stiffness (internal forces conserve
    momentum, and the cube touches nothing in its 20 ms), so the loss here is a seeded linear
    functional of the final positions, sum_p c_p . xT_p, and every particle's v0 carries a seeded
    0.2 m/s perturbation so that the cube deforms.  Bound: 2e-3 of the difference plus 1e-3 of the
    largest sampled derivative of the same kind."""
    import multiprocessing as mp
    import os
    import torch
    from ckmpm_b200.diff import rollout
    d = scenes.diff_cube()
    n = len(d["x0"])
    rng = np.random.default_rng(23)
    d["v0"] = (d["v0"] + 0.2 * rng.standard_normal((n, 3))).astype(np.float32)
    d["c"] = rng.standard_normal((n, 3))
    sim = make_sim(d)
    x0, v0, lE = (t.requires_grad_() for t in tensors(d))
    xT, _ = rollout(sim, x0, v0, lE)
    (torch.tensor(d["c"], device="cuda", dtype=torch.float32) * xT).sum().backward()
    gv, ge = v0.grad.cpu().numpy().astype(np.float64), lE.grad.cpu().numpy().astype(np.float64)
    sim.close()
    picks = rng.choice(n, 6, replace=False)
    dirs = rng.standard_normal((6, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    v0b, lEb = d["v0"].astype(np.float64), d["logE"].astype(np.float64)
    jobs, meta = [], []
    for k, p in enumerate(picks):
        for kind, eps in (("logE", 1e-2), ("v0", 1e-3)):
            for sgn in (1, -1):
                v, e = v0b.copy(), lEb.copy()
                if kind == "logE":
                    e[p] += sgn * eps
                else:
                    v[p] += sgn * eps * dirs[k]
                jobs.append((d, v, e))
            meta.append((kind, k, p, eps))
    with mp.get_context("spawn").Pool(min(len(jobs), max(1, os.cpu_count() or 1))) as pool:
        losses = pool.map(_oracle_loss, jobs)
    rows = []
    for j, (kind, k, p, eps) in enumerate(meta):
        fd = (losses[2 * j] - losses[2 * j + 1]) / (2 * eps)
        ad = float(ge[p]) if kind == "logE" else float(gv[p] @ dirs[k])
        rows.append((kind, p, fd, ad))
        print(f"{kind} particle {p}: fd {fd:.6e} adjoint {ad:.6e} rel {abs(fd - ad) / max(abs(fd), 1e-30):.2e}")
    for kind in ("logE", "v0"):
        scale = max(abs(fd) for kd, _, fd, _ in rows if kd == kind)
        assert scale > 0
        for kd, p, fd, ad in rows:
            if kd == kind:
                assert abs(fd - ad) <= 2e-3 * abs(fd) + 1e-3 * scale, (kind, p, fd, ad)
