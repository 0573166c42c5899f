"""A JSON scene file (ckmpm_b200.engine.load_scene_json) run through the engine against the FP64 oracle.

The scene: a fixed-corotated cube read from a raw float32 .bin asset (the reference's asset
format, asset/*.bin) and a J-fluid box from a .npy file, materials given by E and nu (converted
by the reference's ComputeLameParameters) and by the fluid's own parameters, per-scene velocities,
and a per-cell boundary field built from the file's rules (slip walls and a fixed box).  Both the
engine and the oracle take the loaded configuration and models as they are; after 60 substeps
positions, deformation gradients and velocities agree within the parity tolerances of
tests/test_gpu_engine.py.
"""
import json

import numpy as np
import pytest

from ckmpm_b200 import Scene
from ckmpm_b200.engine import load_scene_json

pytestmark = pytest.mark.gpu


def test_json_scene_through_the_engine_matches_the_oracle(engine_lib, oracle_mod, tmp_path):
    from test_gpu_engine import compare
    rng = np.random.default_rng(3)
    dx = 1 / 64
    g = np.arange(0.40, 0.52, dx / 2) + dx / 4
    cube = np.stack(np.meshgrid(g, g + 0.05, g, indexing="ij"), -1).reshape(-1, 3)
    cube = (cube + rng.uniform(-dx / 8, dx / 8, cube.shape)).astype(np.float32)
    cube.tofile(tmp_path / "cube.bin")
    h = np.arange(0.22, 0.34, dx / 2) + dx / 4
    box = np.stack(np.meshgrid(h, h - 0.05, h + 0.3, indexing="ij"), -1).reshape(-1, 3).astype(np.float32)
    np.save(tmp_path / "fluid.npy", box)
    vol = dx ** 3 / 8
    spec = {
        "config": {"dx": dx, "domain_blocks": [16, 16, 16], "gravity": -9.8, "boundary": "field", "dt": 1e-4},
        "models": [
            {"material": {"kind": "fixed_corotated", "E": 5e4, "nu": 0.3}, "mass": 1000 * vol, "volume": vol,
             "positions": "cube.bin", "velocity": [[0.8, -1.5, 0.4]]},
            {"material": {"kind": "fluid", "bulk_": 1e4, "gamma_": 7.15, "viscosity_": 0.1}, "mass": 1000 * vol,
             "volume": vol, "positions": "fluid.npy", "velocity": [[-0.5, -1.0, 0.0]]},
        ],
        "boundary_rules": [{"slip_walls": 8}, {"fixed_box": [[28, 8, 28], [36, 14, 36]]}],
    }
    (tmp_path / "scene.json").write_text(json.dumps(spec))
    cfg, models = load_scene_json(tmp_path / "scene.json")
    nsteps, dt = 60, cfg.dt
    s = Scene(cfg)
    for m in models:
        s.add_model(m)
    s.setup()
    s.step(nsteps, dt)
    o = oracle_mod.OracleScene(cfg, models)
    o.setup()
    o.step(nsteps, dt)
    compare(s, o, model=0)
    compare(s, o, model=1, check_aux=True)
    assert s.counters()["lost"] == 0
    s.close()
    o.close()
