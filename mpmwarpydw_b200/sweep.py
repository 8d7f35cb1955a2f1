"""Batched parameter sweeps: many independent scenes of uneven size.

Two ways to step a batch:

- ``ConcatBatch`` concatenates the scenes' particles (each scene padded with
  inactive particles to a multiple of 256) into one set of SoA arrays, keeps
  each scene's grid, and steps every scene with one launch per kernel
  (``mpmw_batch_run_substeps``): a CTA finds its scene in a table passed as a
  kernel parameter.  The batch step can be captured as a CUDA graph.
- ``SceneBatch`` keeps each scene's own state objects and gives every
  scene's ``mpmw_run_substeps`` call its own CUDA stream; the whole batch step
  is captured once into a CUDA graph (fork/join across the scene streams).

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

    def check(self, where: str = "batch", log=print) -> int:
        """Read and clear the device status word after the batch ran (raises on
        a non-finite position; logs out-of-grid stencils, bad scene-table
        entries and bounded-wait timeouts)."""
        from .bind import check_status
        return check_status(self.device, where, log)

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


_CHUNK = 256  # scene offsets are multiples of this (the batch entry points require it)
_TUNED = {}   # (scenes, log2 particles) -> (group count, kernel options) chosen by ConcatBatch.tune


def scene_groups(counts, groups: int):
    """Split scenes 0..len(counts)-1 into ``groups`` contiguous ranges of
    roughly equal particle count: a list of (first, last) pairs."""
    n = len(counts)
    groups = max(1, min(int(groups), n))
    total = float(sum(counts))
    out, first, acc = [], 0, 0
    for i, c in enumerate(counts):
        acc += c
        left_scenes, left_groups = n - i - 1, groups - len(out) - 1
        if left_groups > 0 and (acc >= total * (len(out) + 1) / groups or left_scenes == left_groups):
            out.append((first, i + 1))
            first = i + 1
    out.append((first, n))
    return out


class ConcatBatch:
    """Independent scenes stepped by one launch per kernel over concatenated
    particle arrays (``mpmw_batch_run_substeps``).

    ``fields[name]`` holds every scene's particles of that mpmw_particles_t
    field; scene i owns columns ``offsets[i]:offsets[i] + counts[i]`` (the
    rest of its 256-aligned range is inactive padding).  The per-scene state
    objects built from the domains keep their grids, which the batch steps in
    place; :meth:`sync_scenes` copies the particle results back into them."""

    def __init__(self, scenes, device="cuda:0", sort=True):
        import ctypes

        from . import _lib, domains
        from .bind import grid_from_state, params_from_states, particle_storage, particles_struct, status_word
        from .engine import sort_particles
        if not scenes:
            raise ValueError("a batch needs at least one scene")
        self.device = torch.device(device)
        self.states = []
        for d in scenes:
            sim, mpm, xpbd = domains.build(d, device=self.device)
            if sort:
                sort_particles(sim, mpm, xpbd)
            self.states.append((sim, mpm, xpbd))
        self.counts = [s[0].nPoints for s in self.states]
        offs = [0]
        for c in self.counts:
            offs.append(offs[-1] + -(-c // _CHUNK) * _CHUNK)
        self.offsets = offs
        self.total = offs[-1]
        per = [particle_storage(*st) for st in self.states]
        self.fields = {}
        self._aos = {}  # field -> values per particle of a flat per-particle (AoS) array, e.g. cov (6)
        for name in per[0]:
            parts = [p[name] for p in per]
            if all(t is None for t in parts):
                self.fields[name] = None
                continue
            if any(t is None for t in parts):
                raise ValueError(f"field {name} is present in some scenes only")
            t0, c0 = parts[0], self.counts[0]
            k = t0.numel() // c0 if t0.dim() == 1 and t0.numel() != c0 else 0
            self._aos[name] = k
            cols = []
            for t, c, o0, o1 in zip(parts, self.counts, offs[:-1], offs[1:]):
                if k:  # AoS: k values per particle, padding appended row by row
                    t = t.view(c, k)
                cols.append(t)
                if o1 - o0 > c:  # inactive padding (active label 0)
                    shape = (o1 - o0 - c, k) if k else (*t.shape[:-1], o1 - o0 - c)
                    cols.append(torch.zeros(*shape, dtype=t.dtype, device=t.device))
            cat = torch.cat(cols, dim=0 if k else -1)
            self.fields[name] = (cat.reshape(-1) if k else cat).contiguous()
        self.P = particles_struct(self.total, **self.fields)
        n = len(self.states)
        self.grids = (_lib.Grid * n)(*[grid_from_state(mpm) for _, mpm, _ in self.states])
        self.prms = (_lib.Params * n)(*[params_from_states(sim, mpm) for sim, mpm, _ in self.states])
        self.offs = (ctypes.c_int64 * (n + 1))(*offs)
        L = _lib.lib()
        self.ws = torch.empty(int(L.mpmw_batch_workspace_bytes(self.grids, n, self.total)), dtype=torch.uint8,
                              device=self.device)
        self.status = status_word(self.device)
        self.graph = None
        self.graph_steps = 0
        self.groups = 1
        self.options = (True, True)
        self.tuning = {}
        self._streams = []
        self.prepare()
        torch.cuda.synchronize(self.device)

    def prepare(self):
        """(Re)write the scene table (grids, parameters, tensor maps) into the
        workspace; needed again after a scene's parameters change."""
        import ctypes

        from . import _lib
        from .bind import stream_handle
        _lib.check(_lib.lib().mpmw_batch_prepare(ctypes.byref(self.P), self.grids, self.prms, self.offs,
                                                 len(self.states), self.ws.data_ptr(), self.ws.numel(),
                                                 stream_handle(torch.cuda.current_stream(self.device))),
                   "batch_prepare")

    @property
    def particles(self):
        return sum(self.counts)

    def step(self, k: int, groups=None):
        """k substeps of every scene.  The scenes run as ``groups`` contiguous
        ranges (default: ``self.groups``), each range one launch per kernel
        on its own stream; 1 group is a single launch per kernel; 0 runs the
        fused substeps of all scenes in one persistent launch
        (mpmw_batch_run_persistent)."""
        import ctypes

        from . import _lib
        from .bind import stream_handle
        L = _lib.lib()
        groups = self.groups if groups is None else groups
        cur = torch.cuda.current_stream(self.device)
        if groups == 0:
            _lib.check(L.mpmw_batch_run_persistent(ctypes.byref(self.P), int(k), self.status.data_ptr(),
                                                   self.ws.data_ptr(), self.ws.numel(), stream_handle(cur)),
                       "batch_run_persistent")
            return
        ranges = scene_groups(self.counts, groups)
        if len(ranges) == 1:
            _lib.check(L.mpmw_batch_run_substeps(ctypes.byref(self.P), int(k), self.status.data_ptr(),
                                                 self.ws.data_ptr(), self.ws.numel(), stream_handle(cur)),
                       "batch_run_substeps")
            return
        while len(self._streams) < len(ranges):
            self._streams.append(torch.cuda.Stream(device=self.device))
        for (a, b), st in zip(ranges, self._streams):
            st.wait_stream(cur)
            _lib.check(L.mpmw_batch_run_range(ctypes.byref(self.P), a, b, int(k), self.status.data_ptr(),
                                              self.ws.data_ptr(), self.ws.numel(), stream_handle(st)),
                       "batch_run_range")
        for st in self._streams[:len(ranges)]:
            cur.wait_stream(st)

    def set_options(self, gather_tile: bool = True, read_ahead: bool = True):
        """Launch options of the batch's kernels (mpmw_batch_set_options): the
        G2P grid tile by TMA or gathers through L1, particle fields read ahead
        by bulk copies or loaded plainly.  Same results either way."""
        from . import _lib
        _lib.check(_lib.lib().mpmw_batch_set_options(self.ws.data_ptr(), int(bool(gather_tile)),
                                                     int(bool(read_ahead))), "batch_set_options")
        self.options = (bool(gather_tile), bool(read_ahead))

    def _rate(self, k, groups):
        self.step(k, groups)
        torch.cuda.synchronize(self.device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        self.step(k, groups)
        e1.record()
        torch.cuda.synchronize(self.device)
        return self.particles * k / (e0.elapsed_time(e1) * 1e-3)

    def tune(self, k: int = 5, candidates=None, reuse: bool = True):
        """Pick the launch configuration that steps this batch fastest: first
        the kernels' options (grid tile by TMA or L1 gathers, bulk read-ahead
        or plain loads) with one group, then the number of scene groups
        (streams) with the best options, and the one persistent launch for
        all scenes (groups = 0).  Each candidate runs k substeps to
        warm up and k timed, so the tuning advances every scene by 2 k
        substeps per candidate.  The choice is kept in ``self.groups`` /
        ``self.options`` and, per batch shape, for later batches."""
        import math
        key = (len(self.counts), int(round(math.log2(max(1, self.particles)))))
        if reuse and key in _TUNED:
            g, opts = _TUNED[key]
            self.set_options(*opts)
            self.groups = g
            return self.groups
        n = len(self.counts)
        self.tuning = {}
        for opts in ((True, True), (True, False), (False, True), (False, False)):
            self.set_options(*opts)
            self.tuning[(1, opts)] = self._rate(k, 1)
        best_opts = max(((o, r) for (g, o), r in self.tuning.items()), key=lambda t: t[1])[0]
        self.set_options(*best_opts)
        cands = sorted({c for c in (candidates or (0, 1, 2, 4, 8, 16, 32, n)) if c == 0 or 1 < c <= n})
        for g in cands:
            self.tuning[(g, best_opts)] = self._rate(k, g)
        (self.groups, opts) = max(self.tuning, key=self.tuning.get)
        self.set_options(*opts)
        _TUNED[key] = (self.groups, opts)
        return self.groups

    def capture(self, k: int):
        """Capture one batch step of k substeps into a CUDA graph.  The eager
        warm-up needed before capture advances every scene by k."""
        self.step(k)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream(device=self.device)
        cap.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.graph(g, stream=cap):
            self.step(k)
        self.graph, self.graph_steps = g, k
        return g

    def replay(self):
        self.graph.replay()

    def scene_field(self, i: int, name: str):
        """Scene i's part of a concatenated field (a view): columns of a SoA
        field, rows (particle, k) of an AoS one."""
        t = self.fields[name]
        o, c = self.offsets[i], self.counts[i]
        k = self._aos[name]
        return t.view(-1, k)[o:o + c] if k else t[..., o:o + c]

    def sync_scenes(self):
        """Copy every scene's particle state back into its state objects."""
        from .bind import particle_storage
        for i, st in enumerate(self.states):
            for name, dst in particle_storage(*st).items():
                if dst is not None:
                    src = self.scene_field(i, name)
                    dst.copy_(src.reshape(dst.shape) if self._aos[name] else src)

    def check(self, where: str = "batch", log=print) -> int:
        """Read and clear the device status word after the batch ran (raises on
        a non-finite position; logs out-of-grid stencils, bad scene-table
        entries and bounded-wait timeouts)."""
        from .bind import check_status
        return check_status(self.device, where, log)

    def results(self):
        out = []
        for i, c in enumerate(self.counts):
            act = self.scene_field(i, "active") == 1
            v = self.scene_field(i, "v")            # (3, n)
            m = self.scene_field(i, "mass")
            d = self.scene_field(i, "damage")
            mom = (m[None, :] * v).sum(1).double().cpu().tolist()
            out.append(SceneResult(i, c, int(act.sum().item()),
                                   float(d[act].double().mean().item()) if act.any() else 0.0,
                                   tuple(mom), float(v.abs().max().item())))
        return out


def run_sharded(scenes, steps: int, chunk: int = 50, device=None, group=None, runner=None):
    """Run ``scenes`` for ``steps`` substeps sharded over the ranks of the
    default process group (or ``group``); rank 0 returns every scene's
    SceneResult in scene order, other ranks return None.

    ``runner(my_scenes, steps, chunk, device) -> list[SceneResult]`` runs one
    rank's share (default: a tuned ConcatBatch replaying a captured graph of
    ``chunk`` substeps); the result indices are the positions within
    ``my_scenes``."""
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


def _run_batch(scenes, steps, chunk, device, tune_k: int = 5):
    if not scenes:
        return []
    dev = device or torch.device("cuda", torch.cuda.current_device())
    b = ConcatBatch(scenes, device=dev)
    done = 0
    n_cands = 4 + len({c for c in (2, 4, 8, 16, 32, len(scenes)) if 1 < c <= len(scenes)})
    if steps >= 2 * tune_k * n_cands + 2 * chunk:
        b.tune(tune_k, reuse=False)
        done = 2 * tune_k * len(b.tuning)
    if steps - done >= 2 * chunk:
        b.capture(chunk)
        done += chunk
        while done + chunk <= steps:
            b.replay()
            done += chunk
    if steps > done:
        b.step(steps - done)
    torch.cuda.synchronize(dev)
    b.check(f"sweep of {len(scenes)} scenes")
    return b.results()
