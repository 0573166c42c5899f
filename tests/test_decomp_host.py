"""The host side of one scene decomposed over ranks (ckmpm_b200/decomp.py), over gloo on CPU.

Two or three ranks each deposit only the particles they own -- the slabs slab_owners() cuts --
into a dense grid of exact 64-bit fixed-point sums, with the CK dual-grid weights of the substep's
P2G (two grids at -dx/4 and +dx/4, w0 = 1 - o + sin(2 pi o) / (2 pi) per axis), then run the
engine's exchange protocol (decomp.exchange: per-block masks summed over ranks, the blocks two or
more ranks deposited into packed, summed over ranks, unpacked).  Every block a rank deposited
into must then hold, bit for bit, the sums of the undecomposed scene.  The GPU side (the same
protocol over the engine's ckmpm_dd_* kernels) is tests/test_gpu_decomp.py.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from ckmpm_b200 import scenes
from ckmpm_b200.decomp import distributed_reduce, exchange, local_reduce, slab_owners

SCALE = float(2 ** 36)  # the engine's fixed-point unit: 2^-36 of a particle mass


class CpuGrid:
    """A dense grid of int64 sums per block ([m, mvx, mvy, mvz] x 2 grids x 64 cells = 512), with
    the mark / pack / unpack of the engine's ckmpm_dd_* on torch CPU tensors."""

    def __init__(self, dims):
        self.dims = dims
        self.n_blocks = int(np.prod(dims))
        self.g = torch.zeros((self.n_blocks, 512), dtype=torch.int64)
        self.touched = torch.zeros(self.n_blocks, dtype=torch.bool)

    def deposit(self, x, v, dx):
        """CK-weighted mass and momentum of particles (per unit particle mass) as exact sums."""
        xs = x.astype(np.float64) / dx
        for gi, g in enumerate((-1, 1)):
            base = np.floor(xs - 0.25 * g).astype(np.int64)
            o = xs - base - 0.25 * g
            w0 = 1 - o + np.sin(2 * np.pi * o) / (2 * np.pi)
            for n in range(8):
                d = np.array([(n >> 2) & 1, (n >> 1) & 1, n & 1])
                w = np.prod(np.where(d == 0, w0, 1 - w0), axis=1)
                c = base + d
                blk = ((c[:, 0] // 4) * self.dims[1] + c[:, 1] // 4) * self.dims[2] + c[:, 2] // 4
                cell = (c[:, 0] % 4) * 16 + (c[:, 1] % 4) * 4 + (c[:, 2] % 4)
                vals = [w, w * v[:, 0], w * v[:, 1], w * v[:, 2]]
                for ch, val in enumerate(vals):
                    q = np.rint(val * SCALE).astype(np.int64)
                    col = ch * 128 + gi * 64 + cell
                    self.g.index_put_((torch.from_numpy(blk), torch.from_numpy(col)), torch.from_numpy(q),
                                      accumulate=True)
                self.touched[torch.from_numpy(np.unique(blk))] = True

    def mark(self, mask):
        mask.copy_(self.touched.to(torch.int32))

    def pack(self, blocks, buf):
        b = blocks.long()
        buf.copy_(torch.where(self.touched[b][:, None], self.g[b], torch.zeros_like(self.g[b])))

    def unpack(self, blocks, buf):
        self.g[blocks.long()] = buf

    def sync(self):
        pass


def _scene(seed=0):
    # two models (a jelly cube and a sand column) whose slabs interleave along x
    cfg, jelly = scenes.jelly_cube(seed=seed, lo=(0.3, 0.3, 0.35), hi=(0.55, 0.5, 0.6), v0=(0.5, -1.0, 0.2))
    _, sand = scenes.small_sand(seed=seed)
    rng = np.random.default_rng(seed)
    v_sand = rng.uniform(-1, 1, (len(sand[0].particle_position), 3)).astype(np.float32)
    return cfg, [(jelly[0].particle_position, np.broadcast_to(jelly[0].particle_velocity, jelly[0].particle_position.shape)),
                 (sand[0].particle_position, v_sand)], jelly + sand


def _undecomposed(cfg, parts):
    g = CpuGrid(cfg.domain_blocks)
    for x, v in parts:
        g.deposit(x, v, cfg.dx)
    return g


def test_slab_owners_are_contiguous_balanced_and_deterministic():
    cfg, parts, models = _scene()
    for world in (1, 2, 3, 5):
        owners = slab_owners(models, cfg.dx, world)
        assert [len(o) for o in owners] == [len(m.particle_position) for m in models]
        allx = np.concatenate([m.particle_position[:, 0] for m in models])
        allo = np.concatenate(owners)
        counts = np.bincount(allo, minlength=world)
        assert counts.sum() == len(allx) and (counts > 0).all()
        # slabs are contiguous in x: every particle of rank r lies left of every particle of rank r + 1
        for r in range(world - 1):
            assert allx[allo == r].max() < allx[allo == r + 1].min() + cfg.dx * 4
        # every cut within one block column's particles of its share r / world
        col = np.bincount(((allx / cfg.dx + 0.25).astype(int) - 2) // 4)
        below = np.cumsum(counts)[:-1]
        assert all(abs(below[r - 1] - len(allx) * r / world) <= col.max() for r in range(1, world))
        assert all(np.array_equal(a, b) for a, b in zip(owners, slab_owners(models, cfg.dx, world)))


def test_local_exchange_equals_the_undecomposed_grid():
    cfg, parts, models = _scene(1)
    ref = _undecomposed(cfg, parts)
    for world in (2, 3):
        owners = slab_owners(models, cfg.dx, world)
        grids = [CpuGrid(cfg.domain_blocks) for _ in range(world)]
        for r, g in enumerate(grids):
            for (x, v), own in zip(parts, owners):
                g.deposit(x[own == r], v[own == r], cfg.dx)
        n = exchange(grids, local_reduce, "cpu")
        assert n > 0
        for g in grids:
            t = g.touched
            assert torch.equal(g.g[t], ref.g[t])  # bit for bit on every block this rank reads


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cfg, parts, models = _scene(2)
        owners = slab_owners(models, cfg.dx, world)
        g = CpuGrid(cfg.domain_blocks)
        for (x, v), own in zip(parts, owners):
            g.deposit(x[own == rank], v[own == rank], cfg.dx)
        n = exchange([g], distributed_reduce(), "cpu")
        ref = _undecomposed(cfg, parts)
        t = g.touched
        out[rank] = (n, int(t.sum()), bool(torch.equal(g.g[t], ref.g[t])))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_over_gloo_equals_the_undecomposed_grid(world):
    """world ranks as processes over gloo: after one exchange every rank's grid equals the
    undecomposed scene's on every block it deposited into, bit for bit."""
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == list(range(world))
    shared = {res[r][0] for r in range(world)}
    assert len(shared) == 1 and shared.pop() > 0  # every rank summed the same blocks
    assert all(res[r][2] for r in range(world))
