"""The FP64 oracle against the reference CUDA build's own outputs (golden fixtures).

tests/golden/*.npz hold the positions that the reference's stock
MPMEngine::Simulate exported on a B200 for seeded scenes
(tests/golden/make_golden.py, oracle/ref_harness.cu): a fixed-corotated cube,
a J-fluid box, a Drucker-Prager column on the slip floor, von Mises,
non-associated Cam-clay and linear cubes loaded by shear, converging and
uniform initial velocity fields, a fluid box against slip walls and a fixed box,
and the column and the fluid box with the material constants of the
reference's sand_armadillo and fluid_dam_break scenes, 128 substeps of
dt = 2^-14.  The reference exports unordered positions, so particles are
matched by nearest neighbour (spacing dx/2 = 7.8e-3 is far above the errors).

Tolerance on positions after N substeps: 1e-6 + N * 2^-24.  The reference
updates x += dt v in FP32; with a constant
increment round-to-nearest drifts by up to half an ulp of x (<= 2^-24 on
[0.5, 1)) per substep in the same direction for every particle, which the FP64
oracle does not do (measured: 1.19e-8 per substep on the cube, exactly that
rounding).  The reference's run-to-run spread, stored with each fixture, is
below this.
"""
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def load_meta():
    return json.loads((GOLDEN / "golden.json").read_text())


def golden_cases():
    import sys
    sys.path.insert(0, str(GOLDEN))
    import make_golden
    return list(make_golden.golden_scenes()), make_golden


def tolerance(name: str, nsub: int) -> float:
    return 1e-6 + nsub * 2.0 ** -24


def nn_error(x: np.ndarray, ref: np.ndarray) -> float:
    from oracle import ref_runner
    i, d = ref_runner.match_nn(x, ref)
    assert len(set(i.tolist())) == len(ref), (
        f"nearest-neighbour matching is not one-to-one (max distance {d.max():.3e}, "
        f"mean offset {(ref[i] - x).mean(axis=0)})")
    return float(d.max())


def test_fixtures_match_the_seeded_inputs():
    cases, mg = golden_cases()
    meta = load_meta()
    for name, family, cfg, model in cases:
        m = meta[name]
        assert m["input_sha"] == mg.checksum(model.particle_position), name
        assert m["n"] == len(model.particle_position)
        spread = max(m["reference_run_to_run_spread"])
        assert spread <= tolerance(name, 128), (name, spread)


def adaptive_dt(cfg, model) -> float:
    """dt_ of the reference's Initialize + InitializeParticle (include/mpm_engine.cuh:109-117,178)."""
    dt = np.float32(min(np.float32(cfg.dt), np.float32(1.0) / np.float32(cfg.fps)))
    vmax = float(np.max(np.linalg.norm(model.particle_velocity.astype(np.float64), axis=1)))
    if vmax > 0:
        dt = min(dt, np.float32(cfg.dx * cfg.cfl / vmax))
    return float(dt)


def test_oracle_matches_reference_adaptive(oracle_mod):
    _, mg = golden_cases()
    meta = load_meta()["jelly_adaptive"]
    cfg, model = mg.adaptive_scene()
    assert meta["input_sha"] == mg.checksum(model.particle_position)
    fx = np.load(GOLDEN / "jelly_adaptive.npz")
    o = oracle_mod.OracleScene(cfg, [model])
    o.setup()
    dt = adaptive_dt(cfg, model)
    total = 0
    for k in meta["kept_frames"]:
        total += o.step_frame(dt, cfg.cfl, 1.0 / cfg.fps)
        x = o.state(0)["x"]
        err = nn_error(x, fx[f"frame{k}"])
        print(f"jelly_adaptive frame {k} ({total} substeps): oracle vs reference {err:.3e}")
        assert err <= tolerance("jelly_adaptive", total), (k, err)


def test_oracle_matches_reference_build(oracle_mod):
    cases, _ = golden_cases()
    meta = load_meta()
    for name, family, cfg, model in cases:
        m = meta[name]
        fx = np.load(GOLDEN / f"{name}.npz")
        o = oracle_mod.OracleScene(cfg, [model])
        o.setup()
        done = 0
        for k in m["kept_frames"]:
            target = (k + 1) * m["substeps_per_frame"]
            o.step(target - done, m["dt"])
            done = target
            st = o.state(0)
            x = st["x"][st["alive"]]
            ref = fx[f"frame{k}"]
            assert len(x) == len(ref) == m["counts"][k]
            err = nn_error(x, ref)
            print(f"{name} frame {k} ({target} substeps): oracle vs reference {err:.3e}")
            assert err <= tolerance(name, target), (name, k, err)


def test_oracle_matches_reference_rigid(oracle_mod):
    """Rigid particles: the reference with its rigid-particle hooks on (harness
    family RIGID: the von Mises cube's first 2048 particles move with a velocity
    that changes every frame) against the oracle driven frame by frame."""
    _, mg = golden_cases()
    meta = load_meta()["vm_rigid"]
    cfg, model = mg.rigid_scene()
    assert meta["input_sha"] == mg.checksum(model.particle_position)
    assert max(meta["reference_run_to_run_spread"]) <= tolerance("vm_rigid", 128)
    fx = np.load(GOLDEN / "vm_rigid.npz")
    o = oracle_mod.OracleScene(cfg, [model])
    o.set_rigid(cfg.GetRigidParticleCount(), cfg.GetRigidParticleVelocity(0))
    o.setup()
    for k in range(meta["frames"]):
        o.set_rigid_velocity(cfg.GetRigidParticleVelocity(k))
        o.step(meta["substeps_per_frame"], meta["dt"])
        if k not in meta["kept_frames"]:
            continue
        st = o.state(0)
        x = st["x"][st["alive"]]
        ref = fx[f"frame{k}"]
        assert len(x) == len(ref) == meta["counts"][k]
        err = nn_error(x, ref)
        print(f"vm_rigid frame {k}: oracle vs reference {err:.3e}")
        assert err <= tolerance("vm_rigid", (k + 1) * meta["substeps_per_frame"]), (k, err)
