"""Generate the state-dump fixture: the reference CUDA build's full particle state after K substeps.

Run on a machine with a GPU and the reference harness built (make -C oracle ref):

    python tests/golden/make_dumps.py <outdir>

For each scene below it runs the reference's own MPMEngine twice through the harness's state
dump (oracle/ref_runner.dump, mode 2 of oracle/ref_harness.cu) and stores, for every 8th
particle by id of the first run, its position, the velocity the next G2P gives it, F and the
model's scalar after 100 and 500 substeps (for NACC, whose F is fixed only up to a rotation on the
right, F F^T in place of F), and per quantity the largest difference between the
two runs over those particles (the reference's own run-to-run spread from its float atomics; v
relative to the first run's max |v|).  The golden position fixtures hold positions only; these
pin the FP64 oracle's v, F and scalar too (tests/test_oracle_dumps.py).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from ckmpm_b200 import scenes  # noqa: E402
from oracle import ref_runner  # noqa: E402

KS = (100, 500)
EVERY = 8
QUANTITIES = ("x", "v", "F", "aux")


def dump_scenes():
    """(name, harness family, config, models) of every dumped scene."""
    cfg, m = scenes.jelly_cube(lo=(0.44, 0.44, 0.44), hi=(0.56, 0.56, 0.56), v0=(0.3, -1.0, 0.2), track_ids=True)
    yield "jelly_fc", "jelly", cfg, m
    cfg, m = scenes.fluid_box(lo=(0.32, 0.3, 0.34), hi=(0.44, 0.42, 0.46), v0=(0.5, 0.0, -0.25), track_ids=True)
    yield "fluid", "jelly", cfg, m
    cfg, m = scenes.small_sand(r=0.06, h=0.15, track_ids=True)
    yield "sand_dp", "slip", cfg, m
    for kind in ("von_mises", "nacc", "linear"):
        cfg, m = scenes.material_cube(kind, track_ids=True)
        yield kind, "jelly", cfg, m


def main(outdir: Path) -> None:
    out = {}
    for name, family, cfg, models in dump_scenes():
        runs = [ref_runner.dump(family, models, cfg.dt, KS) for _ in range(2)]
        for k in KS:
            a, b = (r[k]["models"][0] for r in runs)
            if not np.array_equal(a["id"], b["id"]):
                raise RuntimeError(f"{name}: the two reference runs kept different particles at {k}")
            keep = a["id"] % EVERY == 0
            out[f"{name}_{k}_id"] = a["id"][keep].astype(np.uint32)
            scale_v = max(float(np.abs(a["v"]).max()), 1e-6)
            for q in QUANTITIES:
                qa = np.asarray(a[q], np.float64)[keep]
                qb = np.asarray(b[q], np.float64)[keep]
                if q == "F" and name == "nacc":  # NACC's F is fixed only up to a rotation on the right
                    qa, qb = qa @ qa.transpose(0, 2, 1), qb @ qb.transpose(0, 2, 1)
                qa = qa.reshape(int(keep.sum()), -1)
                qb = qb.reshape(int(keep.sum()), -1)
                out[f"{name}_{k}_{q}"] = qa.astype(np.float32)
                spread = float(np.abs(qa - qb).max()) if qa.size else 0.0
                out[f"{name}_{k}_{q}_spread"] = np.float64(spread / scale_v if q == "v" else spread)
    outdir.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(outdir / "ref_dumps.npz", **out)
    print(f"wrote {outdir / 'ref_dumps.npz'}")


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent)
