"""The FP64 oracle against the reference CUDA build's full particle state (CPU; fixture made by
tests/golden/make_dumps.py through the reference harness's state dump, two reference runs).

The golden position fixtures pin the oracle's positions; these pin its velocities, F and scalar as
well: a fixed-corotated cube thrown sideways, a J-fluid box, a Drucker-Prager column on the slip
floor, the von Mises cube in shear, the NACC cube squeezed (F F^T for F, as NACC fixes F only up to a
rotation on the right) and the linear cube falling (3,547 to 8,626 particles, dt = 1e-4), every 8th
particle by id, after 100 and 500 substeps.

Bound, per quantity, as in the live engine-vs-reference test: max(8 x the reference's run-to-run
difference, a floor).  Floors: x 1e-6 + K 2^-24 (the reference rounds x += dt v to FP32 once per
substep, the oracle keeps FP64: on the FC cube after 500 substeps this alone is 1.4e-5), v 1e-4 of
max |v|, F and the scalar 1e-4; on the von Mises cube v 2.5e-4, since in plastic shear the
reference's own rounding shows more than its run-to-run spread (the oracle measured 8.9e-5 there,
the reference's two runs 8.7e-6).  The von Mises scalar is not compared: without rigid particles
the reference writes its unread J register (0) into the flag's slot (include/mpm_algorithm.cuh:
1540-1543, 1643-1644, 512-516) while the oracle keeps the flag (1).
"""
import sys
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
import make_dumps  # noqa: E402  (the fixture's own scene definitions)

FIXTURE = GOLDEN / "ref_dumps.npz"
KS = make_dumps.KS
SPREAD_FACTOR = 8.0
FLOOR = {"v": 1e-4, "F": 1e-4, "aux": 1e-4}
FLOOR_SCENE = {"von_mises": {"v": 2.5e-4}}
NO_SCALAR = ("von_mises",)

SCENES = {name: (cfg, models) for name, _, cfg, models in make_dumps.dump_scenes()}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_oracle_state_matches_reference_dump(oracle_mod, name):
    d = np.load(FIXTURE)
    cfg, models = SCENES[name]
    o = oracle_mod.OracleScene(cfg, models)
    o.setup()
    done = 0
    for k in KS:
        o.step(k - done, cfg.dt)
        done = k
        st = o.state(0)
        ids = d[f"{name}_{k}_id"].astype(np.int64)
        scale_v = max(float(np.abs(d[f"{name}_{k}_v"]).max()), 1e-6)
        for q in ("x", "v", "F", "aux"):
            if q == "aux" and name in NO_SCALAR:
                continue
            ours = np.asarray(st[q], np.float64)[ids]
            if q == "F" and name == "nacc":  # the fixture holds F F^T for NACC
                ours = ours.reshape(-1, 3, 3)
                ours = ours @ ours.transpose(0, 2, 1)
            ours = ours.reshape(len(ids), -1)
            ref = d[f"{name}_{k}_{q}"].astype(np.float64).reshape(len(ids), -1)
            err = float(np.abs(ours - ref).max())
            if q == "v":
                err /= scale_v
            floor = 1e-6 + k * 2.0 ** -24 if q == "x" else FLOOR_SCENE.get(name, {}).get(q, FLOOR[q])
            bound = max(SPREAD_FACTOR * float(d[f"{name}_{k}_{q}_spread"]), floor)
            assert err <= bound, (name, k, q, err, bound)
