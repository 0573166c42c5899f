"""Differentiable rollout (ckmpm_diff_*, ckmpm_b200.diff) on the GPU.

  * its FP32 forward against the plain engine (uniform E) and against the FP64
    oracle with per-particle E: positions within 2e-6, F within 5e-5 after 40
    substeps (the plain-path parity tolerances);
  * gradients through torch.autograd against FP64 central finite differences
    of the oracle (per-particle Lame parameters, double inputs): within 1e-3
    relative, for directions in v0, log E and x0 and a linear functional of
    (xT, FT) that depends on all of them;
  * checkpointing: every-10 and one-segment runs give the same xT and the same
    gradients (to float-atomic reordering, 1e-4 relative).
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
    for every in (10, 40, 7):
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
            assert np.allclose(a, b, rtol=1e-4, atol=1e-4 * np.abs(b).max())


def test_backward_needs_its_own_forward(engine_lib):
    import torch
    from ckmpm_b200 import CkmpmError
    from ckmpm_b200.diff import rollout
    d = small_case(nsteps=6, every=3)
    sim = make_sim(d)
    with pytest.raises(CkmpmError):
        sim.backward(None, None, torch.device("cuda"))
    x0, v0, lE = (t.requires_grad_() for t in tensors(d))
    xT, _ = rollout(sim, x0, v0, lE)
    rollout(sim, *tensors(d))  # a second forward replaces the checkpoints
    with pytest.raises(RuntimeError):
        xT.sum().backward()
