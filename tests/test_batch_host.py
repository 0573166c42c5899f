"""Host logic of the batched form, on CPU: the scene generator, the shard
assignment across ranks, and the sharded run's cross-rank reduction over a
world_size-2 gloo process group (the GPU side of a sharded batch has no
collective; each rank runs its own SceneBatch)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ckmpm_b200 import scenes
from ckmpm_b200.batch import reduce_over_ranks, shard_scenes


def test_scene_batch_checks_concatenated_inputs_before_any_device_call():
    """SceneBatch(cfg, scenes, x=, v=) refuses inputs that are not the scenes' concatenation
    (float32, C-contiguous, shape (total, 3), both or neither) before it creates anything."""
    from ckmpm_b200.batch import SceneBatch
    cfg, models = scenes.batched_scenes(n_scenes=3, seed=2, n_min=500, n_max=900)
    total = sum(len(m.particle_position) for m in models)
    good = np.zeros((total, 3), np.float32)
    for x, v in ((good[:-1], good[:-1]), (good.astype(np.float64), good), (good, good[:, :2]),
                 (np.asfortranarray(good), good), (good, None), (None, good)):
        with pytest.raises(ValueError):
            SceneBatch(cfg, models, x=x, v=v)


def test_batched_scenes_follow_the_configuration():
    cfg, models = scenes.batched_scenes(n_scenes=48, seed=0)
    assert len(models) == 48 and cfg.domain_blocks == (16, 16, 16) and abs(cfg.dx - 1 / 64) < 1e-12
    counts = np.array([len(m.particle_position) for m in models])
    assert counts.min() >= 1000 and counts.max() <= 230000
    kinds = {m.material.kind for m in models}
    assert kinds == {"fixed_corotated", "fluid", "drucker_prager"}
    for m in models:
        x = m.particle_position
        # inside the sticky margin (2 blocks) with one block of room
        assert x.min() >= 12 / 64 - 1e-6 and x.max() <= 1 - 12 / 64 + 1e-6
        assert len(m.particle_velocity) == len(x) and np.all(np.abs(m.particle_velocity) <= 1.0)
        assert np.allclose(m.particle_velocity, m.particle_velocity[0])
        assert m.particle_volume == pytest.approx((1 / 64) ** 3 / 8)
    cfg2, again = scenes.batched_scenes(n_scenes=48, seed=0)
    assert all(np.array_equal(a.particle_position, b.particle_position) for a, b in zip(models, again))


def test_shard_scenes_is_a_balanced_partition():
    rng = np.random.default_rng(1)
    costs = np.exp(rng.uniform(np.log(2e3), np.log(2e5), 256))
    for world in (1, 2, 3, 4, 8):
        shards = shard_scenes(costs, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(256))
        loads = [costs[s].sum() for s in shards]
        # longest-first greedy: every rank within one largest scene of the lightest
        assert max(loads) - min(loads) <= costs.max() + 1e-9
        assert shards == shard_scenes(costs, world)
    assert shard_scenes([5.0, 1.0, 1.0, 1.0], 2) == [[0], [1, 2, 3]]
    with pytest.raises(ValueError):
        shard_scenes([1.0], 0)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, counts, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard_scenes(counts, world)[rank]
        shards = [None] * world
        dist.all_gather_object(shards, mine)
        live = float(sum(counts[i] for i in mine))
        fake_ms = 10.0 + rank  # the slowest rank must win
        ms, total = reduce_over_ranks(fake_ms, live, device="cpu")
        out[rank] = (shards, ms, total)
    finally:
        dist.destroy_process_group()


def test_sharded_batch_over_gloo_world_size_2():
    _, models = scenes.batched_scenes(n_scenes=24, seed=2, n_max=20000)
    counts = [len(m.particle_position) for m in models]
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), counts, out), nprocs=world, join=True)
        res = dict(out)
    shards0, ms0, total0 = res[0]
    shards1, ms1, total1 = res[1]
    assert shards0 == shards1 == shard_scenes(counts, world)
    assert sorted(shards0[0] + shards0[1]) == list(range(24))
    assert ms0 == ms1 == 11.0
    assert total0 == total1 == float(sum(counts))


def test_reduce_over_ranks_without_a_process_group():
    assert reduce_over_ranks(3.0, 7.0, device="cpu") == (3.0, 7.0)


def _oracle_scene_state(cfg, model, nsteps):
    from oracle import oracle as O
    o = O.OracleScene(cfg, [model])
    o.setup()
    o.step(nsteps, cfg.dt)
    st = o.state(0)
    o.close()
    return st["x"].copy(), st["F"].copy()


def _shard_rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cfg, models = scenes.batched_scenes(n_scenes=8, seed=5, n_min=300, n_max=1200)
        mine = shard_scenes([len(m.particle_position) for m in models], world)[rank]
        res = {i: _oracle_scene_state(cfg, models[i], 6) for i in mine}
        gathered = [None] * world
        dist.all_gather_object(gathered, res)
        if rank == 0:
            union = {}
            for g in gathered:
                union.update(g)
            out["union"] = union
    finally:
        dist.destroy_process_group()


def test_sharded_scenes_through_the_oracle_equal_the_unsharded_run():
    """Each of two gloo ranks runs its shard of a small batch through the FP64 oracle; the union
    of their results, gathered over the process group, is the unsharded run scene for scene."""
    from oracle import oracle as O
    O.build()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_shard_rank_main, args=(2, _free_port(), out), nprocs=2, join=True)
        union = dict(out)["union"]
    cfg, models = scenes.batched_scenes(n_scenes=8, seed=5, n_min=300, n_max=1200)
    assert sorted(union) == list(range(8))
    for i, m in enumerate(models):
        x, F = _oracle_scene_state(cfg, m, 6)
        assert np.array_equal(union[i][0], x) and np.array_equal(union[i][1], F), i
