"""Batched parameter sweeps: many independent scenes of uneven size.

Each scene keeps its own state objects and grid.  ``SceneBatch`` advances all
of them together: every scene's ``mpmw_run_substeps`` call goes to its own
CUDA stream, and the whole batch step is captured once into a CUDA graph
(fork/join across the scene streams) that is replayed, so one graph launch
runs every scene's substeps concurrently on the GPU.

Across GPUs the scenes shard with no data-path exchange: :func:`partition`
assigns scenes to ranks by particle count (longest first, each to the least
loaded rank), each rank runs its scenes, and the per-scene results are
gathered on rank 0 at the end (:func:`run_sharded`), the only collective.
"""
from __future__ import annotations

import heapq
from dataclasses import dataclass

import torch


def partition(counts, world: int):
    """Scene indices per rank: longest-processing-time-first bin packing of the
    scenes' particle counts over ``world`` ranks (deterministic; ties by index)."""
    heap = [(0, r) for r in range(world)]
    heapq.heapify(heap)
    out = [[] for _ in range(world)]
    for i in sorted(range(len(counts)), key=lambda i: (-int(counts[i]), i)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(counts[i]), r))
    return [sorted(v) for v in out]


@dataclass
class SceneResult:
    index: int
    particles: int
    active: int
    mean_damage: float
    momentum: tuple
    max_abs_velocity: float


class SceneBatch:
    """Independent scenes stepped together (one CUDA graph over per-scene streams)."""

    def __init__(self, scenes, device="cuda:0", sort=True):
        from . import domains
        from .bind import workspace
        from .engine import sort_particles
        self.device = torch.device(device)
        self.states = []
        for d in scenes:
            sim, mpm, xpbd = domains.build(d, device=self.device)
            if sort:
                sort_particles(sim, mpm, xpbd)
            workspace(mpm, sim.nPoints, self.device)
            self.states.append((sim, mpm, xpbd))
        self.streams = [torch.cuda.Stream(device=self.device) for _ in self.states]
        self.graph = None
        self.graph_steps = 0
        torch.cuda.synchronize(self.device)

    @property
    def particles(self):
        return sum(s[0].nPoints for s in self.states)

    def _launch(self, k):
        from .utils.simulationRoutines import run_mpm_substeps
        cur = torch.cuda.current_stream(self.device)
        for (sim, mpm, xpbd), s in zip(self.states, self.streams):
            s.wait_stream(cur)
            with torch.cuda.stream(s):
                run_mpm_substeps(sim, mpm, xpbd, k)
        for s in self.streams:
            cur.wait_stream(s)

    def step(self, k: int):
        """k substeps of every scene (eager: per-scene streams, no graph)."""
        self._launch(k)

    def capture(self, k: int):
        """Capture one batch step of k substeps per scene into a CUDA graph.
        The eager warm-up needed before capture advances every scene by k."""
        self._launch(k)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream(device=self.device)
        cap.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.graph(g, stream=cap):
            self._launch(k)
        self.graph, self.graph_steps = g, k
        return g

    def replay(self):
        self.graph.replay()

    def results(self):
        out = []
        for i, (sim, mpm, xpbd) in enumerate(self.states):
            act = (sim.activeLabel == 1)
            v = sim.particle_v
            m = sim.particle_mass
            mom = (m[:, None] * v).sum(0).double().cpu().tolist()
            out.append(SceneResult(i, sim.nPoints, int(act.sum().item()),
                                   float(mpm.particle_damage[act].double().mean().item()) if act.any() else 0.0,
                                   tuple(mom), float(v.abs().max().item())))
        return out


def run_sharded(scenes, steps: int, chunk: int = 50, device=None, group=None, runner=None):
    """Run ``scenes`` for ``steps`` substeps sharded over the ranks of the
    default process group (or ``group``); rank 0 returns every scene's
    SceneResult in scene order, other ranks return None.

    ``runner(my_scenes, steps, chunk, device) -> list[SceneResult]`` runs one
    rank's share (default: a SceneBatch replaying a captured graph of ``chunk``
    substeps); the result indices are the positions within ``my_scenes``."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    counts = [s.n for s in scenes]
    mine = partition(counts, world)[rank]
    run = runner or _run_batch
    local = run([scenes[i] for i in mine], steps, chunk, device)
    local = [SceneResult(mine[r.index], r.particles, r.active, r.mean_damage, r.momentum, r.max_abs_velocity)
             for r in local]
    if world == 1:
        return sorted(local, key=lambda r: r.index)
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(local, gathered, dst=0, group=group)
    if rank != 0:
        return None
    allr = [r for part in gathered for r in part]
    return sorted(allr, key=lambda r: r.index)


def _run_batch(scenes, steps, chunk, device):
    if not scenes:
        return []
    dev = device or torch.device("cuda", torch.cuda.current_device())
    b = SceneBatch(scenes, device=dev)
    done = 0
    if steps >= 2 * chunk:
        b.capture(chunk)
        done = chunk
        while done + chunk <= steps:
            b.replay()
            done += chunk
    if steps > done:
        b.step(steps - done)
    torch.cuda.synchronize(dev)
    return b.results()
