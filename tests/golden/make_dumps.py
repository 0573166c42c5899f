"""Generate the state-dump fixture: the reference CUDA build's full particle state after K substeps.

Run on a machine with a GPU and the reference harness built (make -C oracle ref):

    python tests/golden/make_dumps.py <outdir>

For the von Mises cube in shear and the linear cube falling (scenes.material_cube on the
jelly grid, dt = 1e-4) it runs the reference's own MPMEngine once through the harness's state
dump (oracle/ref_runner.dump, mode 2 of oracle/ref_harness.cu) and stores, for every 8th
particle by id, its position, the velocity the next G2P gives it, F and the model's scalar
after 100 and 500 substeps.  The golden position fixtures hold positions only; these pin the
FP64 oracle's v and F too (tests/test_oracle_dumps.py).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from ckmpm_b200 import scenes  # noqa: E402
from oracle import ref_runner  # noqa: E402

KINDS = ("von_mises", "linear")
KS = (100, 500)
EVERY = 8


def main(outdir: Path) -> None:
    out = {}
    for kind in KINDS:
        cfg, models = scenes.material_cube(kind, track_ids=True)
        d = ref_runner.dump("jelly", models, cfg.dt, KS)
        for k in KS:
            m = d[k]["models"][0]
            keep = m["id"] % EVERY == 0
            out[f"{kind}_{k}_id"] = m["id"][keep].astype(np.uint32)
            for q in ("x", "v", "F", "aux"):
                out[f"{kind}_{k}_{q}"] = np.asarray(m[q])[keep].astype(np.float32)
    outdir.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(outdir / "ref_dumps.npz", **out)
    print(f"wrote {outdir / 'ref_dumps.npz'}")


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent)
