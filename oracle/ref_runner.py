"""TEST INFRASTRUCTURE ONLY: runs the reference CUDA build (oracle/_ref/ref_*) through its own API.

The binaries are built from the reference's headers by oracle/Makefile (target
`ref`); see oracle/ref_harness.cu.  Used by tests/golden/make_golden.py (golden
fixtures) and by bench.py --impl reference (timing of the reference's
Simulate loop).  Never on the product path.
"""
from __future__ import annotations

import re
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"

KIND_NAMES = {0: "fc", 1: "linear", 2: "dp", 3: "fluid", 4: "vm", 5: "nacc"}


def binary(family: str) -> Path:
    return REF_DIR / f"ref_{family}"


def available(family: str) -> bool:
    return binary(family).exists()


def run(family: str, models, fps: int, frames: int, dt: float, mode: int, outdir: Path | None = None,
        timeout: float = 3600.0) -> tuple[str, Path]:
    """Run one reference simulation of one or more models; returns (stdout, outdir)."""
    if not isinstance(models, (list, tuple)):
        models = [models]
    outdir = Path(outdir or tempfile.mkdtemp(prefix="ckmpm_ref_"))
    outdir.mkdir(parents=True, exist_ok=True)
    lines = []
    for i, model in enumerate(models):
        x = np.ascontiguousarray(model.particle_position, np.float32)
        v = np.ascontiguousarray(model.particle_velocity, np.float32)
        xf, vf = outdir / f"x{i}.bin", outdir / f"v{i}.bin"
        x.tofile(xf)
        v.tofile(vf)
        p = " ".join(f"{float(t):.9g}" for t in model.material.params())
        lines.append(f"{KIND_NAMES[model.material.kind_code]} {p} {model.particle_mass:.9g} "
                     f"{model.particle_volume:.9g} {xf} {vf}")
    manifest = outdir / "models.txt"
    manifest.write_text("\n".join(lines) + "\n")
    cmd = [str(binary(family)), str(manifest), str(fps), str(frames), f"{dt:.9g}", str(outdir), str(mode)]
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if res.returncode != 0:
        raise RuntimeError(f"reference run failed ({res.returncode}): {res.stderr[-2000:]}")
    return res.stdout + res.stderr, outdir


def frames_out(outdir: Path, frames: int, model_index: int = 0) -> list[np.ndarray]:
    """Raw position exports of the reference (float32 xyz, unordered), one per frame."""
    out = []
    for k in range(frames):
        f = outdir / f"model_{model_index}_particle_frame_{k}.txt"
        out.append(np.fromfile(f, np.float32).reshape(-1, 3))
    return out


_BENCH = re.compile(r"MPMBenchmark task (.+?) \| Total duration: ([0-9.eE+-]+)s \| Epoch count: (\d+)")


def parse_benchmark(text: str) -> dict:
    """{task: (total_seconds, epochs)} from the reference's MPMBenchmark print (include/mpm_benchmark.h:37-40)."""
    return {m.group(1): (float(m.group(2)), int(m.group(3))) for m in _BENCH.finditer(text)}


def time_reference(family: str, cfg, models, steps: int, warmup: int) -> dict:
    """Particle-substeps/s of the reference's own Simulate loop (profile mode, no export).

    One frame of (warmup + steps) substeps at the scene's dt; the reference's
    host timer around its frame loop ("Total") and its substep count (epochs of
    "G2P2G (Cuda)") give the rate.  The loop includes the reference's per-substep
    host syncs and dt read-back, as in its stock Simulate.
    """
    dt = cfg.dt
    total = warmup + steps
    fps = max(1, int(round(1.0 / (total * dt))))
    text, _ = run(family, list(models), fps, 1, dt, 1)
    b = parse_benchmark(text)
    secs, _ = b["Total"]
    _, substeps = b["G2P2G (Cuda)"]
    n = sum(len(m.particle_position) for m in models)
    return {"value": n * substeps / secs, "substeps": substeps, "seconds": secs, "particles": n,
            "sample": f"reference CUDA build (oracle/_ref/ref_{family}) via MPMEngine::Simulate in profile mode: "
                      f"{substeps} substeps of the {n}-particle scene, host timer around its frame loop"}


def match_nn(a: np.ndarray, b: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Nearest-neighbour matching of two unordered particle sets: for each row of a,
    the index of its nearest row in b and the distance."""
    from scipy.spatial import cKDTree
    d, i = cKDTree(b.astype(np.float64)).query(a.astype(np.float64))
    return i, d
