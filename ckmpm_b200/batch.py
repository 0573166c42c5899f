"""Batched scenes: many independent scenes advanced together in the same launches.

No counterpart in the reference, whose MPMEngine is a per-GridConfig singleton
(include/mpm_engine.cuh:80-90): there, one process runs one scene.  Here a
SceneBatch holds up to 65536 scenes that share dx, the domain extent, gravity
and the boundary rule, each with one model of its own material; every substep
of every scene runs in one persistent fused launch plus the rebinning, replayed
from CUDA graphs.  A scene's result does not depend, by a single bit, on the
other scenes of the batch or on the launch shape; against the same scene run
alone (a kernel compiled per material) it agrees to the last bits of x, v and
F, as the two compilations may fuse a multiply-add differently.

Across GPUs the scenes shard with no data exchange: shard_scenes() assigns
scenes to ranks by a greedy longest-first bin-pack on their particle counts.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _capi as capi
from .engine import MPMConfig, MPMModel, ParticleState, Scene


def shard_scenes(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest-processing-time-first bin-pack of scene costs onto `world` ranks.

    Scenes in decreasing cost order go to the rank with the least load so far
    (lowest rank on ties); each rank's list is returned in ascending scene
    order.  Deterministic, so every rank computes the same assignment.
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0.0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        shards[r].append(i)
        load[r] += float(costs[i])
    return [sorted(s) for s in shards]


def reduce_over_ranks(ms: float, live: float, device="cuda") -> tuple[float, float]:
    """The only cross-rank step of a sharded batch: the slowest rank's time
    (max) and the live particles of all ranks (sum).  Identity without an
    initialised process group of more than one rank."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1):
        return ms, live
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    n = torch.tensor([live], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(n, op=dist.ReduceOp.SUM)
    return float(t.item()), float(n.item())


class SceneBatch(Scene):
    """A ckmpm_scene handle holding a batch (ckmpm_create_batch + ckmpm_add_batch).

    The Scene methods (setup, step, step_async, status_check, counters,
    tuning, autotune, checkpoints) apply to the whole batch; state() returns
    every live particle in input order with its scene index.
    """

    def __init__(self, config: MPMConfig, scenes: Sequence[MPMModel], x: np.ndarray | None = None,
                 v: np.ndarray | None = None):
        """x, v (optional): every scene's positions and per-particle velocities already concatenated in
        scene order, float32 C-contiguous arrays of shape (total particles, 3), the layout
        ckmpm_add_batch takes; in pinned host memory the upload is a DMA.  Without them they are
        concatenated from the scenes (a scene with one velocity row gives it to all its particles)."""
        if not scenes:
            raise ValueError("empty batch")
        if len(scenes) > capi.MAX_BATCH_SCENES:
            raise ValueError(f"at most {capi.MAX_BATCH_SCENES} scenes per batch")
        self.config = config
        self._h = C.c_void_p()
        self._exports_in_flight: list[np.ndarray] = []
        self.models = list(scenes)
        self.counts = np.array([len(m.particle_position) for m in scenes], np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.counts)])
        total = int(self.counts.sum())
        if (x is None) != (v is None):
            raise ValueError("give both x and v, or neither")
        if x is None:
            x = np.ascontiguousarray(np.concatenate([m.particle_position for m in scenes]), np.float32)
            v = np.ascontiguousarray(np.concatenate([
                m.particle_velocity if len(m.particle_velocity) == len(m.particle_position)
                else np.repeat(m.particle_velocity, len(m.particle_position), 0) for m in scenes]), np.float32)
        for name, a in (("x", x), ("v", v)):
            if a.dtype != np.float32 or not a.flags.c_contiguous or a.shape != (total, 3):
                raise ValueError(f"{name} must be a C-contiguous float32 array of shape ({total}, 3)")
        L = capi.lib()
        desc = config.to_c()
        capi.check(L.ckmpm_create_batch(C.byref(desc), len(scenes), C.byref(self._h)), "ckmpm_create_batch", None)
        arr = (capi.BatchScene * len(scenes))()
        for i, m in enumerate(scenes):
            arr[i].material = m.material.to_c()
            arr[i].mass = m.particle_mass
            arr[i].volume = m.particle_volume
            arr[i].n = len(m.particle_position)
        capi.check(L.ckmpm_add_batch(self._h, len(scenes), arr, capi.fptr(x), capi.fptr(v)), "ckmpm_add_batch",
                   self._h)
        if config.boundary == "field" and config.boundary_field is not None:
            self.set_boundary_field(*config.boundary_field)  # one field, shared by every scene of the batch

    @property
    def n_scenes(self) -> int:
        return len(self.models)

    def add_model(self, model: MPMModel) -> int:
        raise TypeError("a SceneBatch takes its scenes at construction")

    def state(self, model: int = 0) -> ParticleState:
        """All live particles, ordered by input index (the concatenation of the scenes)."""
        return super().state(0)

    def scene_of(self, ids: np.ndarray) -> np.ndarray:
        """Scene index of each particle id."""
        return np.searchsorted(self.offsets, np.asarray(ids, np.int64), side="right") - 1

    def scene_state(self, scene: int, st: ParticleState | None = None) -> ParticleState:
        """The live particles of one scene (ids local to the scene)."""
        st = st if st is not None else self.state()
        sel = self.scene_of(st.id) == scene
        return ParticleState(st.x[sel], st.v[sel], st.F[sel], st.aux[sel],
                             (st.id[sel].astype(np.int64) - self.offsets[scene]).astype(np.uint32))

    def blocks_in(self, scene: int, which: int = 0) -> tuple[np.ndarray, np.ndarray]:
        n = C.c_uint32()
        L = capi.lib()
        code = L.ckmpm_get_blocks_in(self._h, scene, -1, which, None, None, 0, C.byref(n))
        if code not in (capi.CKMPM_OK, 6):
            capi.check(code, "ckmpm_get_blocks_in", self._h)
        keys = np.zeros((n.value, 3), np.int32)
        counts = np.zeros(n.value, np.uint32)
        capi.check(L.ckmpm_get_blocks_in(self._h, scene, -1, which, capi.iptr(keys), capi.uptr(counts), n.value,
                                         C.byref(n)), "ckmpm_get_blocks_in", self._h)
        return keys, counts
