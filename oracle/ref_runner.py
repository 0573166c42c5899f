"""TEST INFRASTRUCTURE ONLY: runs the reference CUDA build (oracle/_ref/ref_*) through its own API.

The binaries are built from the reference's headers by oracle/Makefile (target
`ref`); see oracle/ref_harness.cu.  Used by tests/golden/make_golden.py (golden
fixtures), by the live parity tests against the reference (state dumps after
K substeps, tests/test_gpu_ref_parity.py) and by bench.py --impl reference
(timing of the reference's Simulate loop).  Never on the product path.
"""
from __future__ import annotations

import os
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
        timeout: float = 3600.0, extra: list[str] | None = None, env: dict | None = None) -> tuple[str, Path]:
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
    cmd = [str(binary(family)), str(manifest), str(fps), str(frames), f"{dt:.9g}", str(outdir), str(mode),
           *(extra or [])]
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout,
                         env={**os.environ, **env} if env else None)
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


# Bucket attributes of each particle type (include/mpm_material.cuh:24-257, written by
# CopyParticleArrayToParticleBuffer, include/mpm_algorithm.cuh:974-1079): the columns of F, and
# of the aux scalar (logJp, J, alpha or the rigid flag), in a dumped attribute row.
ATTR_LAYOUT = {"fc": (3, None), "dp": (3, 12), "linear": (3, None), "fluid": (None, 3), "vm": (4, 3),
               "nacc": (4, 3)}


def dump(family: str, models, dt: float, ks, outdir: Path | None = None, timeout: float = 3600.0) -> dict:
    """State of the reference after each K in ks substeps at a fixed dt (mode 2 of the harness).

    Returns {K: {"na", "nn", "ne": ints, "keys": int32 (NE, 3) in the reference's slot order,
    "counts": uint32 (models, NA), "models": [per model: {"id", "block", "x", "F", "aux", "v"}
    sorted by id]}}.  Ids are input indices, carried through the reference's own advection
    records; a particle the reference dropped is absent.  F is (n, 3, 3) row-major (identity
    where the model keeps none), aux the model's scalar (0 where it keeps none), v the velocity
    the next substep's G2P gives the particle (zero for a rigid one, as G2P gives it)."""
    if not isinstance(models, (list, tuple)):
        models = [models]
    ks = sorted(set(int(k) for k in ks))
    # One frame of one second: no substep is clipped to a frame end, so every substep after the
    # first (dt = 0) advances by dt.
    if ks[-1] * dt >= 0.9:
        raise ValueError("the dump runs inside one one-second frame: K * dt must stay below 0.9 s")
    text, out = run(family, list(models), 1, 1, dt, 2, outdir, timeout, [",".join(map(str, ks))])
    res = {}
    for k in ks:
        f = out / f"sets_k{k}.bin"
        if not f.exists():
            raise RuntimeError(f"reference dump at substep {k} missing (the run ended early): {text[-2000:]}")
        raw = np.fromfile(f, np.uint32)
        kk, na, nn, ne, nm = (int(v) for v in raw[:5])
        keys = raw[5:5 + 3 * ne].view(np.int32).reshape(ne, 3)
        counts = raw[5 + 3 * ne:5 + 3 * ne + nm * na].reshape(nm, na)
        entry = {"na": na, "nn": nn, "ne": ne, "keys": keys, "counts": counts, "models": []}
        for i, model in enumerate(models):
            b = np.fromfile(out / f"state_m{i}_k{k}.bin", np.uint8)
            n, nattr = (int(v) for v in b[:8].view(np.uint32))
            o = 8
            ids = b[o:o + 4 * n].view(np.uint32); o += 4 * n
            blk = b[o:o + 12 * n].view(np.int32).reshape(n, 3); o += 12 * n
            attr = b[o:o + 4 * n * nattr].view(np.float32).reshape(n, nattr); o += 4 * n * nattr
            v = b[o:o + 12 * n].view(np.float32).reshape(n, 3)
            order = np.argsort(ids, kind="stable")
            kind = KIND_NAMES[model.material.kind_code]
            fcol, acol = ATTR_LAYOUT[kind]
            F = (attr[order, fcol:fcol + 9].reshape(n, 3, 3) if fcol is not None
                 else np.broadcast_to(np.eye(3, dtype=np.float32), (n, 3, 3)).copy())
            aux = attr[order, acol].copy() if acol is not None else np.zeros(n, np.float32)
            entry["models"].append({"id": ids[order].copy(), "block": blk[order].copy(),
                                    "x": attr[order, :3].copy(), "F": F, "aux": aux, "v": v[order].copy()})
        res[k] = entry
    return res


def time_reference_e2e(family: str, cfg, models, steps: int, warmup: int) -> dict:
    """Like time_reference, plus the harness's host timer from before Initialize to the end of
    the frame loop (setup included).  The CUDA context and, with eager module loading, every
    kernel of the binary are loaded before that timer starts, as they are for the engine's
    end-to-end run, which follows its device-resident one in the same process."""
    dt = cfg.dt
    total = warmup + steps
    fps = max(1, int(round(1.0 / (total * dt))))
    text, _ = run(family, list(models), fps, 1, dt, 1, env={"CUDA_MODULE_LOADING": "EAGER"})
    b = parse_benchmark(text)
    secs, _ = b["Total"]
    _, substeps = b["G2P2G (Cuda)"]
    m = re.search(r"HARNESS e2e ([0-9.eE+-]+)", text)
    e2e = float(m.group(1)) if m else None
    n = sum(len(m_.particle_position) for m_ in models)
    return {"value": n * substeps / secs, "substeps": substeps, "seconds": secs, "particles": n,
            "e2e_seconds": e2e, "e2e_value": (n * substeps / e2e) if e2e else None}
