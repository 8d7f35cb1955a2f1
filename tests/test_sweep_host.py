"""Scene sharding of the batched sweep on the host: the partition, and the
gather of every scene's result over two gloo ranks (CPU; the per-rank scene
runner is replaced by a host function, no GPU)."""
import multiprocessing as mp
import os
import socket

import numpy as np

from mpmwarpydw_b200.sweep import SceneResult, partition, run_sharded


def test_partition_covers_every_scene_once_and_balances():
    rng = np.random.default_rng(4)
    counts = rng.integers(20_000, 500_001, 64).tolist()
    for world in (1, 2, 3, 8):
        parts = partition(counts, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [sum(counts[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(counts)
        assert parts == partition(counts, world)  # deterministic


class _Scene:
    def __init__(self, n):
        self.n = n


def _fake_runner(scenes, steps, chunk, device):
    return [SceneResult(i, s.n, s.n, 0.001 * s.n, (float(s.n), 0.0, -float(steps)), 1.0) for i, s in enumerate(scenes)]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        scenes = [_Scene(n) for n in (30_000, 480_000, 75_000, 210_000, 20_000, 333_000, 90_000)]
        res = run_sharded(scenes, steps=7, runner=_fake_runner)
        if rank == 0:
            q.put([(r.index, r.particles, r.momentum[2]) for r in res])
        else:
            q.put(res)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_run_sharded_gathers_every_scene_once_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res0 = [g for g in got if g is not None]
    assert len(res0) == 1 and got.count(None) == 1
    res = res0[0]
    assert [r[0] for r in res] == list(range(7))
    assert [r[1] for r in res] == [30_000, 480_000, 75_000, 210_000, 20_000, 333_000, 90_000]
    assert all(r[2] == -7.0 for r in res)
