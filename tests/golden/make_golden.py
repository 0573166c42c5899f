"""Generate the golden fixtures: outputs of the reference CUDA build on seeded scenes.

Run on a machine with a GPU and the reference harness built (make -C oracle ref):

    python tests/golden/make_golden.py <outdir>

For each scene below it runs the reference's stock MPMEngine::Simulate
(oracle/_ref/ref_<family>, oracle/ref_harness.cu) twice and stores, per exported
frame, the reference's particle positions (unordered, as the reference exports
them), the largest nearest-neighbour distance between the two runs (the
reference's own run-to-run spread, from its float atomics), and the inputs'
checksum.  dt is a power of two and fps = 1 / (16 dt), so each frame is exactly
16 substeps and the reference's frame clipping never changes dt; the first
substep advects with dt = 0 as in the reference.  The fluid_walls fixture runs on
the harness's FIELD family, whose irregular-boundary hook (slip walls and a
fixed box of cells) the engine receives as a per-cell boundary field.  The rigid-particle fixture
runs on the harness's RIGID family, whose scene hooks make the first 2048
particles rigid with a per-frame velocity (rigid_velocity below).
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from ckmpm_b200 import scenes  # noqa: E402
from oracle import ref_runner  # noqa: E402

DT = 2.0 ** -14          # 6.103515625e-05, exact in float and double
SUBSTEPS_PER_FRAME = 16
FPS = 1024               # 1 / (16 * 2^-14)
FRAMES = 8               # 128 substeps
KEEP = (1, 7)            # frames stored: after 32 and 128 substeps


def golden_scenes():
    """(name, harness family, config, model) of every fixture."""
    cfg, m = scenes.jelly_cube(lo=(0.44, 0.44, 0.44), hi=(0.56, 0.56, 0.56), v0=(0.3, -1.0, 0.2))
    yield "jelly_fc", "jelly", cfg, m[0]
    cfg, m = scenes.fluid_box(lo=(0.32, 0.3, 0.34), hi=(0.44, 0.42, 0.46), v0=(0.5, 0.0, -0.25))
    yield "fluid", "jelly", cfg, m[0]
    cfg, m = scenes.small_sand(r=0.06, h=0.15)
    yield "sand_dp", "slip", cfg, m[0]
    for kind in ("von_mises", "nacc", "linear"):
        cfg, m = scenes.material_cube(kind)
        yield kind, "jelly", cfg, m[0]
    yield ("fluid_walls", "field") + wall_scene()
    # The reference scenes' own material constants: the sand of
    # tests/sand_armadillo (E 1e4, nu 0.4) and the fluid of tests/fluid_dam_break
    # (bulk 10, gamma 7.15, viscosity 0.1).
    cfg, m = scenes.small_sand(r=0.06, h=0.15, E=1e4, nu=0.4)
    yield "sand_scene_params", "slip", cfg, m[0]
    cfg, m = scenes.fluid_box(lo=(0.32, 0.3, 0.34), hi=(0.44, 0.42, 0.46), v0=(0.5, 0.0, -0.25), bulk=10.0)
    yield "fluid_scene_params", "jelly", cfg, m[0]


def wall_scene():
    """A J-fluid box thrown into the slip walls and over a fixed box of cells:
    the harness's FIELD family hook, and the same rules as a boundary field."""
    from ckmpm_b200.boundary import BoundaryField
    cfg, m = scenes.fluid_box(lo=(0.13, 0.13, 0.3), hi=(0.45, 0.3, 0.55), v0=(-2.0, -3.0, 1.0))
    cfg.boundary = "field"
    cfg.boundary_field = BoundaryField(cfg).slip_walls(8).fixed_box((24, 0, 24), (32, 14, 32)).arrays()
    return cfg, m[0]


# Adaptive-dt fixture: the reference's own Simulate picks every dt (CFL on the
# grid's max |v| binds, and each frame ends on a clipped substep).
ADAPTIVE = {"name": "jelly_adaptive", "family": "jelly", "dt": 2e-3, "fps": 48, "frames": 2}


def adaptive_scene():
    cfg, m = scenes.jelly_cube(lo=(0.44, 0.44, 0.44), hi=(0.56, 0.56, 0.56), v0=(6.0, 0.0, 0.0), E=2e4, gravity=-9.8)
    cfg.dt, cfg.fps, cfg.total_frames, cfg.cfl = ADAPTIVE["dt"], ADAPTIVE["fps"], ADAPTIVE["frames"], 0.5
    return cfg, m[0]


# Rigid-particle fixture: the von Mises cube on the harness's RIGID family
# (oracle/ref_harness.cu), where the reference's rigid-particle hooks are on:
# its first RIGID_COUNT particles move with rigid_velocity(frame).
RIGID = {"name": "vm_rigid", "family": "rigid"}
RIGID_COUNT = 2048


def rigid_velocity(frame: int) -> tuple[float, float, float]:
    return (2.0, 0.5 * frame - 1.0, -1.0)


def rigid_scene():
    cfg, m = scenes.material_cube("von_mises")
    cfg.exist_rigid_particle = True
    cfg.rigid_particle_count = RIGID_COUNT
    cfg.rigid_particle_velocity = rigid_velocity
    cfg.dt, cfg.fps, cfg.total_frames = DT, FPS, FRAMES
    return cfg, m[0]


def checksum(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, np.float32).tobytes()).hexdigest()[:16]


def main(outdir: str, only: list[str] | None = None) -> None:
    """Write the fixtures of every scene, or only of the named ones (merged into
    an existing golden.json)."""
    out = Path(outdir)
    out.mkdir(parents=True, exist_ok=True)
    meta_path = out / "golden.json"
    meta = json.loads(meta_path.read_text()) if (only and meta_path.exists()) else {}
    for name, family, cfg, model in golden_scenes():
        if only and name not in only:
            continue
        runs = []
        for _ in range(2):
            _, d = ref_runner.run(family, model, FPS, FRAMES, DT, 0)
            runs.append(ref_runner.frames_out(d, FRAMES))
        spread = []
        for k in range(FRAMES):
            _, dist = ref_runner.match_nn(runs[0][k], runs[1][k])
            spread.append(float(dist.max()))
        arrays = {f"frame{k}": runs[0][k] for k in KEEP}
        np.savez_compressed(out / f"{name}.npz", **arrays)
        meta[name] = {"family": family, "n": int(len(model.particle_position)),
                      "input_sha": checksum(model.particle_position), "dt": DT, "fps": FPS, "frames": FRAMES,
                      "substeps_per_frame": SUBSTEPS_PER_FRAME, "kept_frames": list(KEEP),
                      "reference_run_to_run_spread": spread,
                      "material": model.material.kind, "params": model.material.params(),
                      "mass": model.particle_mass, "volume": model.particle_volume,
                      "counts": [int(len(runs[0][k])) for k in range(FRAMES)]}
        print(name, meta[name]["n"], "spread", max(spread), flush=True)
    if not only or RIGID["name"] in only:
        cfg, model = rigid_scene()
        runs = []
        for _ in range(2):
            _, d = ref_runner.run(RIGID["family"], model, FPS, FRAMES, DT, 0)
            runs.append(ref_runner.frames_out(d, FRAMES))
        spread = [float(ref_runner.match_nn(runs[0][k], runs[1][k])[1].max()) for k in range(FRAMES)]
        np.savez_compressed(out / f"{RIGID['name']}.npz", **{f"frame{k}": runs[0][k] for k in KEEP})
        meta[RIGID["name"]] = {"family": RIGID["family"], "n": int(len(model.particle_position)),
                               "input_sha": checksum(model.particle_position), "dt": DT, "fps": FPS,
                               "frames": FRAMES, "substeps_per_frame": SUBSTEPS_PER_FRAME,
                               "kept_frames": list(KEEP), "rigid_count": RIGID_COUNT,
                               "rigid_velocity": [list(rigid_velocity(k)) for k in range(FRAMES)],
                               "reference_run_to_run_spread": spread,
                               "counts": [int(len(r)) for r in runs[0]]}
        print(RIGID["name"], meta[RIGID["name"]]["n"], "spread", max(spread), flush=True)
    if only and ADAPTIVE["name"] not in only:
        meta_path.write_text(json.dumps(meta, indent=1))
        return
    cfg, model = adaptive_scene()
    a = ADAPTIVE
    runs = []
    for _ in range(2):
        text, d = ref_runner.run(a["family"], model, a["fps"], a["frames"], a["dt"], 0)
        runs.append(ref_runner.frames_out(d, a["frames"]))
    spread = [float(ref_runner.match_nn(runs[0][k], runs[1][k])[1].max()) for k in range(a["frames"])]
    np.savez_compressed(out / f"{a['name']}.npz", **{f"frame{k}": runs[0][k] for k in range(a["frames"])})
    meta[a["name"]] = {"family": a["family"], "n": int(len(model.particle_position)),
                       "input_sha": checksum(model.particle_position), "dt": a["dt"], "fps": a["fps"],
                       "frames": a["frames"], "kept_frames": list(range(a["frames"])), "adaptive": True,
                       "reference_run_to_run_spread": spread, "counts": [int(len(r)) for r in runs[0]]}
    print(a["name"], meta[a["name"]]["n"], "spread", max(spread), flush=True)
    meta_path.write_text(json.dumps(meta, indent=1))


if __name__ == "__main__":
    # python tests/golden/make_golden.py [outdir] [scene names ...]
    main(sys.argv[1] if len(sys.argv) > 1 else str(Path(__file__).resolve().parent), sys.argv[2:] or None)
