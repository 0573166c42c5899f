"""Scene and asset IO on the host: raw .bin particle files (the reference's
asset/*.bin format, float32 xyz triples) and JSON scene files with materials,
velocities and per-cell boundary rules.  No GPU needed."""
import json

import numpy as np
import pytest

from ckmpm_b200.boundary import FIXED, SLIP, VELOCITY
from ckmpm_b200.engine import load_raw_positions, load_scene_json


def test_raw_positions_roundtrip(tmp_path):
    x = np.random.default_rng(0).random((1000, 3)).astype(np.float32)
    f = tmp_path / "asset.bin"
    x.tofile(f)
    np.testing.assert_array_equal(load_raw_positions(f), x)
    (tmp_path / "bad.bin").write_bytes(b"\0" * 16)
    with pytest.raises(ValueError, match="xyz triples"):
        load_raw_positions(tmp_path / "bad.bin")


def test_scene_json_with_assets_and_boundary_rules(tmp_path):
    rng = np.random.default_rng(1)
    xa = (0.4 + 0.2 * rng.random((500, 3))).astype(np.float32)
    xa.tofile(tmp_path / "sand.bin")
    np.save(tmp_path / "jelly.npy", (0.3 + 0.1 * rng.random((200, 3))).astype(np.float32))
    spec = {
        "config": {"dx": 1 / 64, "domain_blocks": [16, 16, 16], "gravity": -2.0, "boundary": "field",
                   "dt": 5e-5, "fps": 48, "total_frames": 2},
        "models": [
            {"material": {"kind": "drucker_prager", "E": 1e4, "nu": 0.4}, "mass": 1e-4, "volume": 1e-7,
             "positions": "sand.bin"},
            {"material": {"kind": "fixed_corotated", "E": 5e4, "nu": 0.3}, "mass": 2e-4, "volume": 2e-7,
             "positions": "jelly.npy", "velocity": [[0.0, -1.0, 0.0]], "freeze_time": 0.5},
        ],
        "boundary_rules": [{"slip_walls": 8}, {"fixed_box": [[20, 0, 20], [30, 10, 30]]},
                           {"velocity_box": [[40, 20, 40], [42, 22, 42], [0.5, 0.0, 0.0]]}],
    }
    (tmp_path / "scene.json").write_text(json.dumps(spec))
    cfg, models = load_scene_json(tmp_path / "scene.json")
    assert cfg.domain_blocks == (16, 16, 16) and cfg.gravity == -2.0 and cfg.total_frames == 2
    assert [m.material.kind for m in models] == ["drucker_prager", "fixed_corotated"]
    np.testing.assert_array_equal(models[0].particle_position, xa)
    assert models[1].particle_position.shape == (200, 3) and models[1].freeze_time == 0.5
    np.testing.assert_array_equal(models[1].particle_velocity, [[0.0, -1.0, 0.0]])
    rule, param = cfg.boundary_field
    assert rule.shape == (64, 64, 64) and param.shape == (64, 64, 64, 3)
    assert rule[2, 30, 30] == SLIP and rule[25, 5, 25] == FIXED and rule[41, 21, 41] == VELOCITY
    np.testing.assert_array_equal(param[41, 21, 41], [0.5, 0.0, 0.0])
    assert rule[32, 32, 32] == 0

    spec["boundary_rules"] = [{"no_such_rule": 1}]
    (tmp_path / "bad.json").write_text(json.dumps(spec))
    with pytest.raises(ValueError, match="unknown boundary rule"):
        load_scene_json(tmp_path / "bad.json")
    spec["config"]["boundary"] = "sticky_blocks"
    spec["boundary_rules"] = [{"slip_walls": 8}]
    (tmp_path / "bad2.json").write_text(json.dumps(spec))
    with pytest.raises(ValueError, match='need config "boundary": "field"'):
        load_scene_json(tmp_path / "bad2.json")
