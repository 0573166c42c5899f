"""The CUDA engine against the reference CUDA build's own outputs (golden fixtures).

Same fixtures and matching as tests/test_golden.py.  Both builds are FP32 and
round the position update the same way, so the tolerance is the oracle test's
(1e-6 + N * 2^-24 on positions, x 2 for Drucker-Prager), which bounds the
reference's run-to-run spread too.
"""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

from ckmpm_b200 import Scene

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def test_engine_matches_reference_build(engine_lib):
    import sys
    sys.path.insert(0, str(GOLDEN))
    import make_golden
    from test_golden import nn_error, tolerance
    meta = json.loads((GOLDEN / "golden.json").read_text())
    for name, family, cfg, model in make_golden.golden_scenes():
        m = meta[name]
        fx = np.load(GOLDEN / f"{name}.npz")
        s = Scene(cfg)
        s.add_model(model)
        s.setup()
        done = 0
        for k in m["kept_frames"]:
            target = (k + 1) * m["substeps_per_frame"]
            s.step(target - done, m["dt"])
            done = target
            x = s.state(0).x
            ref = fx[f"frame{k}"]
            assert len(x) == len(ref) == m["counts"][k]
            err = nn_error(x, ref)
            print(f"{name} frame {k} ({target} substeps): engine vs reference {err:.3e}")
            assert err <= tolerance(name, target), (name, k, err)
        s.close()


def test_engine_simulate_matches_reference_adaptive(engine_lib):
    """The reference-shaped MPMEngine.Simulate (adaptive CFL dt, frame clipping)
    against the reference's own Simulate on the same scene."""
    sys.path.insert(0, str(GOLDEN))
    import make_golden
    from test_golden import nn_error, tolerance
    from ckmpm_b200 import MPMEngine
    meta = json.loads((GOLDEN / "golden.json").read_text())["jelly_adaptive"]
    cfg, model = make_golden.adaptive_scene()
    fx = np.load(GOLDEN / "jelly_adaptive.npz")
    frames = {}
    eng = MPMEngine()
    eng.Initialize(cfg)
    eng.InitializeParticle(cfg, [model])
    eng.InitialSetup(cfg)
    n = eng.Simulate(cfg, export_callback=lambda f, scene: frames.__setitem__(f, scene.state(0).x.copy()))
    for k in meta["kept_frames"]:
        err = nn_error(frames[k], fx[f"frame{k}"])
        print(f"jelly_adaptive frame {k}: engine vs reference {err:.3e} ({n} substeps in total)")
        assert err <= tolerance("jelly_adaptive", n), (k, err)


def test_engine_rigid_matches_reference_build(engine_lib):
    """Rigid particles through the reference-shaped MPMEngine (the rigid hooks of
    MPMConfig, velocity set per frame by Simulate) against the reference with
    its own rigid hooks on."""
    sys.path.insert(0, str(GOLDEN))
    import make_golden
    from test_golden import nn_error, tolerance
    from ckmpm_b200 import MPMEngine
    meta = json.loads((GOLDEN / "golden.json").read_text())["vm_rigid"]
    cfg, model = make_golden.rigid_scene()
    fx = np.load(GOLDEN / "vm_rigid.npz")
    frames = {}
    eng = MPMEngine()
    eng.Initialize(cfg)
    eng.InitializeParticle(cfg, [model])
    eng.InitialSetup(cfg)
    eng.Simulate(cfg, export_callback=lambda f, scene: frames.__setitem__(f, scene.state(0).x.copy()),
                 fixed_substeps_per_frame=meta["substeps_per_frame"])
    for k in meta["kept_frames"]:
        err = nn_error(frames[k], fx[f"frame{k}"])
        print(f"vm_rigid frame {k}: engine vs reference {err:.3e}")
        assert err <= tolerance("vm_rigid", (k + 1) * meta["substeps_per_frame"]), (k, err)
