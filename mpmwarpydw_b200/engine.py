"""Multi-step execution: spatial particle ordering and CUDA-graph replay.

``sort_particles`` reorders every per-particle array of the three state
objects into 4x4x4-cell block order (a one-time set-up step; the reference's
results do not depend on particle order).  Consecutive particles then share
grid cells, which is what the scatter's per-CTA counting sort (long segments of
one base cell) and the G2P kernels' grid tiles (one TMA copy per CTA) rely on.  ``sim.particle_order`` keeps, for each
stored particle, its index in the original input so results can be written
back in input order (:func:`original_order`).

``SubstepGraph`` captures ``k`` MPM substeps (one library call) into a CUDA
graph and replays it; host work per replay is one launch.
``SubstepGraphCache`` keeps such graphs per call (k and every captured
address and parameter), which is how the driver steps between its checks.
"""
from __future__ import annotations

import torch

from . import _lib
from .bind import grid_from_state, params_from_states, particles_from_states, status_word, stream_handle, workspace
from .state import Mat33Field, ScalarField, Sym33Field, Vec3Field


def block_sort_key(x_n3: torch.Tensor, minBounds, inv_dx: float, dims, block: int = 4) -> torch.Tensor:
    """int64 key: (block index in C order) * block^3 + (cell index inside the block).

    The cell is the particle's stencil base, int((x - minBounds) * inv_dx - 0.5)
    in FP32 with truncation (utils/mpmRoutines.py:514-517), so particles sharing
    a key scatter to the same 27 nodes."""
    mb = torch.as_tensor(minBounds, dtype=torch.float32, device=x_n3.device)
    inv = torch.tensor(inv_dx, dtype=torch.float32, device=x_n3.device)
    gp = (x_n3.to(torch.float32) - mb) * inv
    cell = (gp - 0.5).to(torch.int64)  # truncation toward zero, as the kernels
    d = torch.as_tensor(dims, dtype=torch.int64, device=x_n3.device)
    cell = torch.minimum(torch.clamp(cell, min=0), d - 1)
    nb = (d + block - 1) // block
    b = cell // block
    r = cell % block
    bidx = (b[:, 0] * nb[1] + b[:, 1]) * nb[2] + b[:, 2]
    ridx = (r[:, 0] * block + r[:, 1]) * block + r[:, 2]
    return bidx * (block ** 3) + ridx


def _permute_state(obj, perm: torch.Tensor, n: int):
    for cls in type(obj).__mro__:
        for name, desc in list(vars(cls).items()):
            if not isinstance(desc, (ScalarField, Vec3Field, Mat33Field, Sym33Field)):
                continue
            s = desc.storage(obj)
            if s is None:
                continue
            if isinstance(desc, ScalarField):
                if s.numel() == n:
                    s.copy_(s[perm])
                elif s.numel() % n == 0:
                    k = s.numel() // n
                    v = s.view(n, k)
                    v.copy_(v[perm])
            else:
                s.copy_(s[:, perm])


def block_order(sim, mpm, block: int = 4) -> torch.Tensor:
    """The stable order of the particles by :func:`block_sort_key`, computed on
    the device by the library (``mpmw_block_sort``: key kernel + stable LSD
    radix sort); an int64 permutation (position i holds particle perm[i])."""
    import ctypes
    n = sim.nPoints
    dev = sim.device
    perm = torch.empty(n, dtype=torch.int32, device=dev)
    if n == 0:
        return perm.long()
    L = _lib.lib()
    need = int(L.mpmw_block_sort_workspace_bytes(n))
    ws = getattr(mpm, "_mpmw_sort_ws", None)
    if ws is None or ws.numel() < need:
        ws = torch.empty(max(need, 256), dtype=torch.uint8, device=dev)
        mpm._mpmw_sort_ws = ws
    prm = params_from_states(sim, mpm)
    dims = (ctypes.c_int32 * 3)(*[int(d) for d in mpm.gridDims])
    _lib.check(L.mpmw_block_sort(sim._s_particle_x.data_ptr(), n, ctypes.byref(prm), dims, int(block),
                                 perm.data_ptr(), ws.data_ptr(), ws.numel(), stream_handle()), "block_sort")
    return perm.long()


def sort_particles(sim, mpm, xpbd=None, block: int = 4):
    """Reorder all per-particle state into block order (returns the permutation).

    The order comes from the library's device sort (:func:`block_order`); the
    fields are gathered through it in place.  Used at set-up and, by the
    driver, every ``resort_interval`` substeps, as particles drift out of the
    cells their CTA covers."""
    n = sim.nPoints
    perm = block_order(sim, mpm, block)
    for obj in (sim, mpm, xpbd):
        if obj is not None:
            _permute_state(obj, perm, n)
    prev = getattr(sim, "particle_order", None)
    sim.particle_order = perm if prev is None else prev[perm]
    return perm


def original_order(sim, t: torch.Tensor) -> torch.Tensor:
    """Return a per-particle tensor (first dim N) in the original input order."""
    order = getattr(sim, "particle_order", None)
    if order is None:
        return t
    out = torch.empty_like(t)
    out[order] = t
    return out


class SubstepGraph:
    """CUDA graph of ``k`` consecutive MPM substeps on fixed state buffers."""

    def __init__(self, sim, mpm, xpbd, k: int, warmup: bool = True):
        """With ``warmup`` the k substeps run once eagerly before capture (so
        every kernel is loaded); that run advances the simulation."""
        self.k = int(k)
        self.P = particles_from_states(sim, mpm, xpbd)
        self.G = grid_from_state(mpm)
        self.prm = params_from_states(sim, mpm)
        self.status = status_word(sim.device)
        self.ws = workspace(mpm, sim.nPoints, sim.device)
        self.graph = torch.cuda.CUDAGraph()
        self.stream = torch.cuda.Stream(device=sim.device)
        self.stream.wait_stream(torch.cuda.current_stream())
        if warmup:
            with torch.cuda.stream(self.stream):
                self._call()
        torch.cuda.current_stream().wait_stream(self.stream)
        torch.cuda.synchronize(sim.device)
        with torch.cuda.graph(self.graph, stream=self.stream):
            self._call()

    def _call(self):
        _lib.check(_lib.lib().mpmw_run_substeps(self.P, self.G, self.prm, self.k, self.status.data_ptr(),
                                                 self.ws.data_ptr(), self.ws.numel(), stream_handle()),
                   "run_substeps")

    def replay(self):
        self.graph.replay()


class SubstepGraphCache:
    """Runs ``k`` MPM substeps through a replayed CUDA graph when the same call
    was captured before, else directly (and captures it for next time).

    A graph holds the device addresses and parameters of its capture, so the
    key is everything it bakes in: k, the particle, grid and parameter structs
    byte for byte (pointers, counts, dt, gravity, flags), the workspace and the
    status word.  A changed parameter (the gravity pulse, a new dt) is a new
    key; nothing captured is ever replayed on other buffers or values.  On
    small scenes a replay saves the per-launch host work (a 64,000-particle
    block: 24.5 instead of 29.6 us per substep)."""

    def __init__(self, max_graphs: int = 8):
        self.max_graphs = int(max_graphs)
        self._graphs = {}

    def _key(self, sim, mpm, xpbd, k):
        return (int(k), bytes(particles_from_states(sim, mpm, xpbd)), bytes(grid_from_state(mpm)),
                bytes(params_from_states(sim, mpm)), workspace(mpm, sim.nPoints, sim.device).data_ptr(),
                status_word(sim.device).data_ptr())

    def run(self, sim, mpm, xpbd, k: int):
        key = self._key(sim, mpm, xpbd, k)
        g = self._graphs.get(key)
        if g is not None:
            g.replay()
            return
        if len(self._graphs) >= self.max_graphs:
            self._graphs.pop(next(iter(self._graphs)))  # oldest first
        # the capture's warm-up run is this call's k substeps
        self._graphs[key] = SubstepGraph(sim, mpm, xpbd, k, warmup=True)


class DeviceLoop:
    """Phase-1 substeps with the driver's stop test on the device
    (runMPMYDW.py:656-727; ``mpmw_loop_*``).

    One CUDA graph whose while node runs ``chunk`` fused substeps, the
    statistics and the driver's check (residual, damage stall) until the phase
    ends or the segment's substep budget runs out, with no host round trip in
    between.  The graph bakes in the particle, grid and parameter structs: make
    a new loop when a parameter (dt, gravity) changes."""

    def __init__(self, sim, mpm, xpbd, chunk, n_steps, residual_threshold, stall_threshold, stall_steps, min_steps):
        import ctypes
        self.chunk = int(chunk)
        self.P = particles_from_states(sim, mpm, xpbd)
        self.G = grid_from_state(mpm)
        self.prm = params_from_states(sim, mpm)
        self.key = bytes(self.prm)
        self.status = status_word(sim.device)
        self.ws = workspace(mpm, sim.nPoints, sim.device)
        self.state = torch.zeros(ctypes.sizeof(_lib.LoopState) // 8, dtype=torch.float64, device=sim.device)
        self.lp = _lib.LoopParams(self.chunk, int(n_steps), int(min_steps), int(stall_steps),
                                  float(residual_threshold), float(stall_threshold))
        self.stream = torch.cuda.Stream(device=sim.device)
        self.handle = ctypes.c_void_p()
        _lib.check(_lib.lib().mpmw_loop_create(ctypes.byref(self.P), ctypes.byref(self.G), ctypes.byref(self.prm),
                                               ctypes.byref(self.lp), self.state.data_ptr(), self.status.data_ptr(),
                                               self.ws.data_ptr(), self.ws.numel(), ctypes.byref(self.handle),
                                               stream_handle(self.stream)), "loop_create")

    def _write(self, st):
        self.state.copy_(torch.frombuffer(bytearray(bytes(st)), dtype=torch.float64))

    def read(self):
        """The loop state (an ``_lib.LoopState``) after the last launch."""
        raw = self.state.cpu().numpy().tobytes()
        return _lib.LoopState.from_buffer_copy(raw)

    def run(self, counter, stall, residual, prev_damage, segment):
        """Run chunks from the given monitor state for at most ``segment``
        substeps (at least one chunk; segment is rounded down to whole
        chunks); returns the state after the last chunk."""
        segment = (int(segment) // self.chunk) * self.chunk
        if segment < self.chunk:
            raise ValueError("a device segment runs at least one chunk")
        st = _lib.LoopState()
        st.counter, st.stall, st.stopped_early, st.segment_left = int(counter), int(stall), 0, segment
        st.residual, st.prev_damage = float(residual), float(prev_damage)
        cur = torch.cuda.current_stream(self.state.device)
        self._write(st)
        self.stream.wait_stream(cur)
        _lib.check(_lib.lib().mpmw_loop_launch(self.handle, stream_handle(self.stream)), "loop_launch")
        cur.wait_stream(self.stream)
        return self.read()

    def close(self):
        if self.handle:
            _lib.lib().mpmw_loop_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PhaseLoop(DeviceLoop):
    """Phase 1 of a big step with its XPBD steps and gravity pulse inside one
    CUDA graph (``mpmw_phase_loop_create``; runMPMYDW.py:646-727): each
    iteration of the graph's while node runs ``chunk`` fused substeps with the
    pulse gravity or the plain one (an IF node per case, the chunk the pulse
    ends in split at that substep), the XPBD step when the chunk's last
    substep index is a positive multiple of ``xpbd_ratio``, the statistics and
    the driver's check.  Chunks start at counters = ``phase`` (mod chunk); with
    XPBD steps that is 1 mod chunk and chunk must divide xpbd_ratio, so that
    every XPBD substep ends a chunk.  The graph bakes in the structs: make a
    new loop when dt or the base gravity changes."""

    def __init__(self, sim, mpm, xpbd, chunk, n_steps, residual_threshold, stall_threshold, stall_steps, min_steps,
                 xpbd_ratio=0, pulse_steps=0, pulse_gravity=None, gravity=None):
        """``gravity``: the plain gravity (default sim.gravity); ``pulse_gravity``:
        the gravity of the first ``pulse_steps`` substeps."""
        import ctypes

        from .bind import params_struct
        from .utils.xpbdRoutines import xpbd_structs
        self.chunk = int(chunk)
        self.xpbd_ratio, self.pulse_steps = int(xpbd_ratio), int(pulse_steps)
        self.phase = (1 % self.chunk) if self.xpbd_ratio > 0 else 0
        self.P = particles_from_states(sim, mpm, xpbd)
        self.G = grid_from_state(mpm)
        self.prm = params_from_states(sim, mpm)
        self.prm_pulse = params_from_states(sim, mpm)
        base = tuple(float(g) for g in (gravity if gravity is not None else sim.gravity))
        for i in range(3):
            self.prm.gravity[i] = base[i]
        pg = tuple(float(g) for g in (pulse_gravity if pulse_gravity is not None else base))
        for i in range(3):
            self.prm_pulse.gravity[i] = pg[i]
        self.key = (bytes(self.prm), bytes(self.prm_pulse), self.chunk, self.xpbd_ratio, self.pulse_steps)
        self.status = status_word(sim.device)
        self.ws = workspace(mpm, sim.nPoints, sim.device)
        self.state = torch.zeros(ctypes.sizeof(_lib.LoopState) // 8, dtype=torch.float64, device=sim.device)
        self.lp = _lib.PhaseParams(_lib.LoopParams(self.chunk, int(n_steps), int(min_steps), int(stall_steps),
                                                   float(residual_threshold), float(stall_threshold)),
                                   self.xpbd_ratio, self.pulse_steps, self.phase)
        self._keep = []
        X = H = Q = QP = None
        xws, xws_n = None, 0
        if self.xpbd_ratio > 0:
            _, X, Q = xpbd_structs(sim, mpm, xpbd)
            _, _, QP = xpbd_structs(sim, mpm, xpbd)
            for i in range(3):
                Q.gravity[i] = base[i]
                QP.gravity[i] = pg[i]
            hg = xpbd.particle_grid
            hg.cell_width = float(sim.dx)
            hg._ensure(sim.nPoints)
            hg.n = sim.nPoints
            H = hg.struct()
            xw = hg.workspace()
            xws, xws_n = xw.data_ptr(), xw.numel()
            self._keep += [X, Q, QP, H, xw]
        self.stream = torch.cuda.Stream(device=sim.device)
        self.handle = ctypes.c_void_p()
        ref = lambda o: ctypes.byref(o) if o is not None else None  # noqa: E731
        _lib.check(_lib.lib().mpmw_phase_loop_create(
            ctypes.byref(self.P), ctypes.byref(self.G), ctypes.byref(self.prm), ctypes.byref(self.prm_pulse),
            ref(X), ref(H), ref(Q), ref(QP), ctypes.byref(self.lp), self.state.data_ptr(), self.status.data_ptr(),
            self.ws.data_ptr(), self.ws.numel(), xws, xws_n, ctypes.byref(self.handle), stream_handle(self.stream)),
            "phase_loop_create")

    def run(self, counter, stall, residual, prev_damage, segment):
        """As DeviceLoop.run; ``counter`` must be = phase (mod chunk)."""
        if int(counter) % self.chunk != self.phase:
            raise ValueError(f"phase loop: chunks start at counters = {self.phase} mod {self.chunk}, not {counter}")
        return super().run(counter, stall, residual, prev_damage, segment)


class XPBDLoop(DeviceLoop):
    """Phase 2 of a big step (runMPMYDW.py:780-844) in one CUDA graph
    (``mpmw_xpbd_loop_create``): XPBD-only steps until ``max_steps`` ran or the
    sleeping fraction of the XPBD particles reaches ``sleep_ratio``."""

    def __init__(self, sim, mpm, xpbd, max_steps, sleep_ratio):
        import ctypes

        from .utils.xpbdRoutines import xpbd_structs
        self.chunk = 1
        P, X, Q = xpbd_structs(sim, mpm, xpbd, xpbd_only=True)
        hg = xpbd.particle_grid
        hg.cell_width = float(sim.dx)
        hg._ensure(sim.nPoints)
        hg.n = sim.nPoints
        H = hg.struct()
        xw = hg.workspace()
        self._keep = [P, X, Q, H, xw]
        self.state = torch.zeros(ctypes.sizeof(_lib.LoopState) // 8, dtype=torch.float64, device=sim.device)
        self.stream = torch.cuda.Stream(device=sim.device)
        self.handle = ctypes.c_void_p()
        _lib.check(_lib.lib().mpmw_xpbd_loop_create(ctypes.byref(P), ctypes.byref(X), ctypes.byref(H),
                                                    ctypes.byref(Q), int(max_steps), float(sleep_ratio),
                                                    self.state.data_ptr(), status_word(sim.device).data_ptr(),
                                                    xw.data_ptr(), xw.numel(), ctypes.byref(self.handle),
                                                    stream_handle(self.stream)),
                   "xpbd_loop_create")

    def run_steps(self, done, budget):
        """Run from ``done`` steps for at most ``budget`` more (at least one);
        returns the loop state (counter = steps done, stopped_early = 1 on the
        sleep-ratio stop, stats[0:2] = XPBD total / sleeping)."""
        st = _lib.LoopState()
        st.counter, st.stall, st.stopped_early, st.segment_left = int(done), 0, 0, int(budget)
        cur = torch.cuda.current_stream(self.state.device)
        self._write(st)
        self.stream.wait_stream(cur)
        _lib.check(_lib.lib().mpmw_loop_launch(self.handle, stream_handle(self.stream)), "loop_launch")
        cur.wait_stream(self.stream)
        return self.read()
