"""One scene decomposed over several GPUs (row f3; no counterpart in the reference, whose engine
runs on one GPU, src/cuda_util.cu:5-17).

Ownership, not space, is what is split: the particles are divided once, at setup, into slabs of
block columns along x (contiguous ranges of the initial block's x index, balanced by particle
count), and every rank simulates only its own particles, for the whole run.  Each rank keeps the
whole dense grid (180 GB of HBM holds 2 x 1 GB for a 64^3-block domain, 2 x 8 GB for 128^3) and
deposits only its own particles into it.  Before each substep reads the grid, the ranks exchange
the blocks that more than one of them deposited into -- at first the one layer of block columns
where two slabs meet, later wherever the slabs have interpenetrated -- and sum them.  The grid
holds exact 64-bit integer sums (ckmpm_b200/csrc/kernels.cuh, flush_tile), so the sum over ranks
is independent of their number and order: every rank reads, bit for bit, the grid of the
undecomposed scene, and every particle evolves exactly as it would there.  Particles never
migrate, so no particle state crosses NVLink; only the shared grid blocks do (4 KB each).

Exchange after ckmpm_setup and after every substep (include/ckmpm.h, ckmpm_dd_*; exchange()):
  1. ckmpm_dd_mark: a per-block int32 mask of this rank's deposit blocks;
  2. all-reduce (sum) of the masks; the blocks with a count of 2 or more, in block order;
  3. ckmpm_dd_pack into a buffer of 512 int64 per block; all-reduce (sum, int64);
  4. ckmpm_dd_unpack.
Across GPUs the all-reduces run over torch.distributed (NCCL); with every rank in one process
(the single-GPU test), as a sum over the local scenes.  exchange() takes any grid with mark /
pack / unpack, so the host-side protocol also runs over gloo on CPU grids
(tests/test_decomp_host.py).  Fixed dt only (the adaptive dt's grid maximum would need one more
all-reduce per substep).
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Sequence

import numpy as np

from . import _capi as capi
from .engine import MPMConfig, MPMModel, ParticleState, Scene


def slab_owners(models: Sequence[MPMModel], dx: float, world: int) -> list[np.ndarray]:
    """Owner rank of every particle of every model: rank r owns the particles whose initial
    block x index falls in its slab, slabs being contiguous ranges of block columns cut so that
    the particle counts are as even as whole columns allow.  Deterministic, so every rank
    computes the same split."""
    if world < 1:
        raise ValueError("world must be >= 1")
    inv = np.float32(1.0 / dx)
    bx = [((np.asarray(m.particle_position, np.float32)[:, 0] * inv + np.float32(0.25)).astype(np.int64) - 2) // 4
          for m in models]
    allbx = np.concatenate(bx) if bx else np.zeros(0, np.int64)
    if allbx.size == 0:
        return [np.zeros(0, np.int32) for _ in models]
    lo, hi = int(allbx.min()), int(allbx.max())
    cols = np.bincount(allbx - lo, minlength=hi - lo + 1)
    cum = np.cumsum(cols)
    total = int(cum[-1])
    # slab r starts at the column boundary whose running count is nearest r / world of the particles
    cuts = []
    for r in range(1, world):
        target = total * r / world
        i = int(np.searchsorted(cum, target, side="left"))  # first column whose running count reaches it
        after = i + 1 if i < len(cum) and (i == 0 or abs(cum[i] - target) < abs(cum[i - 1] - target)) else i
        cuts.append(lo + max(after, (cuts[-1] - lo + 1) if cuts else 1))
    return [np.searchsorted(np.asarray(cuts, np.int64), b, side="right").astype(np.int32) for b in bx]


class EngineGrid:
    """The grid of one engine scene, as the exchange sees it (ckmpm_dd_*, include/ckmpm.h)."""

    def __init__(self, scene: Scene):
        import torch
        self.scene = scene
        self.torch = torch
        n = C.c_uint32()
        capi.check(capi.lib().ckmpm_dd_blocks(scene._h, C.byref(n)), "ckmpm_dd_blocks", scene._h)
        self.n_blocks = n.value

    def mark(self, mask) -> None:
        capi.check(capi.lib().ckmpm_dd_mark(self.scene._h, C.c_void_p(mask.data_ptr())), "ckmpm_dd_mark",
                   self.scene._h)

    def pack(self, blocks, buf) -> None:
        capi.check(capi.lib().ckmpm_dd_pack(self.scene._h, C.c_void_p(blocks.data_ptr()), blocks.numel(),
                                            C.c_void_p(buf.data_ptr())), "ckmpm_dd_pack", self.scene._h)

    def unpack(self, blocks, buf) -> None:
        capi.check(capi.lib().ckmpm_dd_unpack(self.scene._h, C.c_void_p(blocks.data_ptr()), blocks.numel(),
                                              C.c_void_p(buf.data_ptr())), "ckmpm_dd_unpack", self.scene._h)

    def sync(self) -> None:
        # the engine runs on the scene's stream; the reductions on torch's current stream
        self.torch.cuda.synchronize()


def exchange(grids: Sequence, reduce: Callable, device) -> int:
    """One grid exchange over the grids this process holds (one per rank it drives).

    reduce(list of tensors) returns the tensor summed over every rank of the decomposition.
    Returns the number of blocks summed (those more than one rank deposited into)."""
    import torch
    masks = [torch.zeros(g.n_blocks, dtype=torch.int32, device=device) for g in grids]
    for g, m in zip(grids, masks):
        g.mark(m)
    for g in grids:
        g.sync()
    count = reduce(masks)
    shared = torch.nonzero(count >= 2).flatten().to(torch.int32)
    if shared.numel() == 0:
        return 0
    bufs = [torch.empty((shared.numel(), 512), dtype=torch.int64, device=device) for _ in grids]
    for g, b in zip(grids, bufs):
        g.pack(shared, b)
    for g in grids:
        g.sync()
    total = reduce(bufs)
    for g in grids:
        g.unpack(shared, total)
    for g in grids:
        g.sync()
    return int(shared.numel())


def local_reduce(tensors):
    """Every rank in this process: the sum of their tensors."""
    total = tensors[0].clone()
    for t in tensors[1:]:
        total += t
    return total


def distributed_reduce(group=None):
    """This process's one rank: an all-reduce (sum) over torch.distributed -- NCCL across GPUs,
    gloo on the host."""
    def reduce(tensors):
        import torch.distributed as dist
        (t,) = tensors
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        return t
    return reduce


class DecomposedScene:
    """This process's share of one decomposed scene: the ranks given by `ranks` (all of them
    when one process drives every rank on one GPU, else this process's rank alone)."""

    def __init__(self, config: MPMConfig, models: Sequence[MPMModel], world: int, ranks: Sequence[int],
                 reduce: Callable, device):
        self.config = config
        self.world = world
        self.ranks = list(ranks)
        self.owners = slab_owners(models, config.dx, world)
        self.global_ids: list[list[np.ndarray]] = []  # [local rank][model] -> global ids
        self.scenes: list[Scene] = []
        for r in self.ranks:
            s = Scene(config)
            gids = []
            for m, own in zip(models, self.owners):
                sel = np.nonzero(own == r)[0]
                gids.append(sel.astype(np.uint32))
                x = np.ascontiguousarray(m.particle_position[sel], np.float32)
                v = m.particle_velocity
                v = np.ascontiguousarray(v if len(v) == 1 else v[sel], np.float32)
                if len(sel) == 0:  # a rank with no particle of this model keeps one far outside the domain
                    x = np.full((1, 3), -1.0, np.float32)
                    v = np.zeros((1, 3), np.float32)
                s.add_model(MPMModel(m.particle_mass, m.particle_volume, x, v, m.material, m.freeze_time))
            self.scenes.append(s)
            self.global_ids.append(gids)
        self.reduce = reduce
        self.device = device
        self.grids: list[EngineGrid] = []
        self.shared_blocks_last = 0

    def set_stream(self, stream_handle: int | None) -> None:
        for s in self.scenes:
            s.set_stream(stream_handle)

    def exchange(self) -> int:
        self.shared_blocks_last = exchange(self.grids, self.reduce, self.device)
        return self.shared_blocks_last

    def setup(self) -> None:
        for s in self.scenes:
            s.setup()
        self.grids = [EngineGrid(s) for s in self.scenes]
        self.exchange()

    def step(self, nsteps: int, dt: float) -> None:
        for _ in range(nsteps):
            for s in self.scenes:
                s.step_async(1, dt)
            self.exchange()
        for s in self.scenes:
            s.status_check()

    def state(self, model: int = 0) -> ParticleState:
        """This process's particles of `model` with global ids (input order of the whole model),
        sorted by id."""
        parts = []
        for s, gids in zip(self.scenes, self.global_ids):
            st = s.state(model)
            g = gids[model]
            keep = st.id < len(g)
            parts.append((st, g[st.id[keep]], keep))
        ids = np.concatenate([p[1] for p in parts])
        order = np.argsort(ids, kind="stable")

        def cat(name):
            return np.concatenate([getattr(p[0], name)[p[2]] for p in parts])[order]
        return ParticleState(cat("x"), cat("v"), cat("F"), cat("aux"), ids[order])

    def close(self) -> None:
        for s in self.scenes:
            s.close()


def local_decomposition(config: MPMConfig, models: Sequence[MPMModel], world: int, device=None) -> DecomposedScene:
    """Every rank of a `world`-way decomposition in this process, on one GPU: the exchange sums
    the ranks' buffers directly.  Bit for bit the same particles as the undecomposed scene."""
    import torch
    dev = device if device is not None else torch.device("cuda", config.device)
    return DecomposedScene(config, models, world, range(world), local_reduce, dev)


def distributed_decomposition(config: MPMConfig, models: Sequence[MPMModel], group=None) -> DecomposedScene:
    """This rank's share, the exchange an all-reduce over torch.distributed (NCCL across GPUs)."""
    import torch
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    dev = torch.device("cuda", config.device)
    return DecomposedScene(config, models, world, [rank], distributed_reduce(group), dev)
