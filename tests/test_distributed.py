"""Pass sharding and the film reduction, on CPU ranks with the gloo backend."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from helpers import sb  # noqa: F401  (registers the package)
from spectral_b200 import distributed as sd


def test_block_range_partitions():
    for total in (0, 1, 7, 11, 275 // 25):
        for world in (1, 2, 3, 8):
            spans = [sd.block_range(total, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == total
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            assert max(b - a for a, b in spans) - min(b - a for a, b in spans) <= 1
    p = sd.pass_indices(4, 25, 1, 2)
    assert p[0] == (50, 0) and p[-1] == (99, 24) and len(p) == 50
    with pytest.raises(ValueError):
        sd.block_range(4, 2, 2)


def test_scene_shard_partitions_and_balances():
    rng = np.random.default_rng(3)
    costs = rng.uniform(1, 100, size=37)
    for world in (1, 2, 3, 8):
        shards = [sd.scene_shard(costs, r, world) for r in range(world)]
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(costs)))  # a partition
        loads = [costs[s].sum() for s in shards]
        # greedy LPT: no rank exceeds the mean load by more than the largest scene
        assert max(loads) <= costs.sum() / world + costs.max() + 1e-9
        assert shards == [sd.scene_shard(list(costs), r, world) for r in range(world)]  # deterministic
    # more ranks than scenes: some ranks get none
    assert [sd.scene_shard([5, 1], r, 3) for r in range(3)] == [[0], [1], []]
    with pytest.raises(ValueError):
        sd.scene_shard([1, -1], 0, 1)
    with pytest.raises(ValueError):
        sd.scene_shard([1], 1, 1)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rng = np.random.default_rng(rank)
    nb = 2 + rank  # uneven block counts
    blocks = rng.uniform(size=(nb, 3, 4, 5))
    mean = torch.from_numpy(blocks.mean(0).copy())
    m2 = torch.from_numpy((blocks ** 2).sum(0))
    mean, m2, total = sd.reduce_film(mean, m2, nb)
    q.put((rank, mean.numpy(), m2.numpy(), total))
    dist.destroy_process_group()


def test_reduce_film_gloo_world2():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    allb = np.concatenate([np.random.default_rng(r).uniform(size=(2 + r, 3, 4, 5)) for r in range(world)])
    for rank, mean, m2, total in res:
        assert total == allb.shape[0]
        assert np.allclose(mean, allb.mean(0), rtol=1e-13)
        assert np.allclose(m2, (allb ** 2).sum(0), rtol=1e-13)


def _grad_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    first, last = sd.adjoint_range(7, rank, world)
    # each rank's partial gradient: a stand-in sum over its own passes
    g = torch.zeros(79, dtype=torch.float64)
    for p in range(first, last):
        g += torch.from_numpy(np.random.default_rng(p).normal(size=79))
    sd.reduce_gradient(g)
    q.put((rank, g.numpy()))
    dist.destroy_process_group()


def test_reduce_gradient_gloo_world2():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_grad_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = sum(np.random.default_rng(p).normal(size=79) for p in range(7))
    for _, g in res:
        assert np.allclose(g, want, rtol=1e-13, atol=1e-13)
    with pytest.raises(TypeError):
        sd.reduce_gradient(torch.zeros(3, dtype=torch.float32))


def _shard_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    costs = [9, 1, 4, 4, 7, 2]
    idx = sd.scene_shard(costs, rank, world)
    blocks = [10 * i + 1 for i in idx]  # a rank's own per-scene results
    q.put((rank, idx, sd.gather_scene_blocks(blocks, idx, len(costs)).tolist()))
    dist.destroy_process_group()


def test_scene_shard_gather_gloo_world2():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(res[0][1] + res[1][1]) == list(range(6))
    # LPT: 9 -> r0, 7 -> r1, 4 -> r1 (7 < 9), 4 -> r0 (9 < 11), 2 -> r1 (11 < 13), 1 -> r0 (13 = 13, lower rank)
    assert res[0][1] == [0, 1, 3] and res[1][1] == [2, 4, 5]
    for _, _, gathered in res:
        assert gathered == [10 * i + 1 for i in range(6)]
