"""One scene decomposed over ranks (ckmpm_b200/decomp.py) against the same scene on one engine.

Every rank of a 2- and 3-way decomposition runs in this process on the one GPU: each rank is its
own engine scene holding the particles of its slab, and the exchange after setup and after every
substep sums the blocks more than one rank deposited into (ckmpm_dd_mark / ckmpm_dd_pack /
ckmpm_dd_unpack, the reduction a sum over the local buffers instead of an NCCL all-reduce).  No
kernel waits on another: the host runs the ranks' substeps one after another.  Because the grid
holds exact integer sums, every particle must come out bit for bit as in the undecomposed scene:
positions, velocities, deformation gradients and logJp / J, after tens of substeps, for a
fixed-corotated cube, a Drucker-Prager column on the slip floor and a two-model scene.
"""
from __future__ import annotations

import numpy as np
import pytest

from ckmpm_b200 import Scene, scenes
from ckmpm_b200.decomp import local_decomposition

pytestmark = pytest.mark.gpu


def _cases():
    cfg_j, jelly = scenes.jelly_cube(lo=(0.4, 0.42, 0.38), hi=(0.6, 0.58, 0.55), v0=(1.0, -1.0, 0.3))
    cfg_s, sand = scenes.small_sand()
    cfg_m, m1 = scenes.jelly_cube(lo=(0.3, 0.3, 0.3), hi=(0.42, 0.42, 0.42), v0=(1.0, 0.0, 0.0))
    _, m2 = scenes.fluid_box(lo=(0.44, 0.3, 0.3), hi=(0.55, 0.4, 0.42), v0=(-1.0, 0.0, 0.0))
    return {"jelly_fc": (cfg_j, jelly, 1e-4), "sand_dp": (cfg_s, sand, 5e-5), "two_models": (cfg_m, m1 + m2, 1e-4)}


@pytest.mark.parametrize("case", ["jelly_fc", "sand_dp", "two_models"])
@pytest.mark.parametrize("world", [2, 3])
def test_decomposed_scene_equals_the_scene_bit_for_bit(engine_lib, case, world):
    cfg, models, dt = _cases()[case]
    nsteps = 60
    ref = Scene(cfg)
    for m in models:
        ref.add_model(m)
    ref.setup()
    ref.step(nsteps, dt)
    d = local_decomposition(cfg, models, world)
    d.setup()
    d.step(nsteps, dt)
    assert d.shared_blocks_last > 0  # the slabs do share grid blocks
    for i in range(len(models)):
        a, b = ref.state(i), d.state(i)
        assert np.array_equal(a.id, b.id), (case, i)
        for name in ("x", "v", "F", "aux"):
            assert np.array_equal(getattr(a, name), getattr(b, name)), (case, world, i, name)
    d.close()
    ref.close()
