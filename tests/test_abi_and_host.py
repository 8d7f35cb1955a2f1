"""CPU tests of the C-ABI library (loads, exports every declared symbol, rejects
bad arguments without touching a GPU) and of the host-side logic."""
import ctypes
import json

import numpy as np
import pytest


def test_library_exports_every_declared_symbol():
    from mpmwarpydw_b200 import _lib
    L = _lib.lib()
    names = _lib.exported_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.mpmw_version() >= 1


def test_argument_errors_are_reported_not_raised():
    from mpmwarpydw_b200 import _lib
    L = _lib.lib()
    prm = _lib.Params()
    rc = L.mpmw_stress(None, ctypes.byref(prm), None, None)
    assert rc == 1 and b"NULL" in L.mpmw_last_error()
    G = _lib.Grid()
    rc = L.mpmw_grid_update(ctypes.byref(G), ctypes.byref(prm), None)
    assert rc == 1 and b"dims" in L.mpmw_last_error()
    P = _lib.Particles(); P.n = -1
    rc = L.mpmw_stats(ctypes.byref(P), None, None)
    assert rc == 1
    prm.boundary_condition = 42
    G.dims[0] = G.dims[1] = G.dims[2] = 4
    rc = L.mpmw_grid_op(ctypes.byref(G), ctypes.byref(prm), 0, None)
    assert rc == 1  # null grid buffers are rejected before the enum


def test_particle_counts_beyond_32_bits_are_rejected():
    """Particle indices, worklists and hash ids are 32-bit: a count above
    2^31 - 1 is an argument error, reported before any device work."""
    from mpmwarpydw_b200 import _lib
    L = _lib.lib()
    big = 2 ** 31
    P = _lib.Particles(); P.n = big
    G = _lib.Grid(); G.dims[0] = G.dims[1] = G.dims[2] = 4
    prm = _lib.Params()
    rc = L.mpmw_substep(ctypes.byref(P), ctypes.byref(G), ctypes.byref(prm), None, None)
    assert rc == 1 and b"2147483647" in L.mpmw_last_error()
    out = (ctypes.c_double * 7)()  # never written: the count is rejected first
    rc = L.mpmw_stats(ctypes.byref(P), out, None)
    assert rc == 1 and b"2147483647" in L.mpmw_last_error()
    X, q, H = _lib.XPBD(), _lib.XPBDParams(), _lib.Hash()
    for i in range(3):
        H.dims[i] = 8
    H.cell_width = 1.0
    rc = L.mpmw_xpbd_step(ctypes.byref(P), ctypes.byref(X), ctypes.byref(H), ctypes.byref(q), None, None, 0, None)
    assert rc == 1 and b"2147483647" in L.mpmw_last_error()
    rc = L.mpmw_hash_build(None, big, ctypes.byref(H), None, 0, None)
    assert rc == 1 and b"2147483647" in L.mpmw_last_error()
    f = (ctypes.c_float * 1)()  # never read: the count is rejected first
    rc = L.mpmw_mu_lam_bulk(big, f, f, f, f, f, None)
    assert rc == 1 and b"2147483647" in L.mpmw_last_error()


def test_getargs_merge_rules(tmp_path):
    from mpmwarpydw_b200.utils.getArgs import get_args
    cfg = tmp_path / "c.json"
    cfg.write_text(json.dumps({"dt": 2e-4, "E": 5e9, "boundaryCondition": "plane_strain_y_global",
                               "not_a_flag": 3, "_comment": "x"}))
    a = get_args(["--config", str(cfg), "--E", "7e9"], verbose=False)
    assert a.dt == 2e-4                 # JSON over default
    assert a.E == 7e9                   # CLI over JSON
    assert a.boundaryCondition == "plane_strain_y_global"  # JSON bypasses the CLI choices
    assert not hasattr(a, "not_a_flag")
    assert a.volumetric_locking_correction == 1 and a.rpic_damping == 0.2 and a.eff == 0.05  # reference defaults


def test_reference_configs_load():
    """Every benchmark JSON of the reference loads through get_args: known keys
    are applied, unknown keys ignored (utils/getArgs.py:145-148).  Reads the
    reference checkout named by MPMW_REFERENCE_ROOT; skipped without it."""
    import glob
    import os
    from mpmwarpydw_b200.utils.getArgs import get_args
    root = os.environ.get("MPMW_REFERENCE_ROOT", "")
    files = sorted(glob.glob(os.path.join(root, "benchmarks", "*", "config_*.json"))) if root else []
    if not files:
        pytest.skip("no reference checkout (set MPMW_REFERENCE_ROOT)")
    for f in files:
        cfg = json.load(open(f))
        a = get_args(["--config", f], verbose=False)
        for k, v in cfg.items():
            if hasattr(a, k) and not k.startswith("_"):
                assert getattr(a, k) == v, (os.path.basename(f), k)


def test_domain_sizes():
    from mpmwarpydw_b200 import domains
    d = domains.tunnel()
    assert d.n == 3_873_600 and d.gridDims == (120, 70, 120)
    b = domains.block_collapse()
    assert b.n == 64_000 and b.gridDims == (40, 40, 40)
    assert abs(b.overrides["alpha"] - 0.23094) < 1e-5
    assert abs(domains.friction_angle_to_alpha(35.0) - 0.27296) < 1e-5


def test_grid_geometry_mask():
    from mpmwarpydw_b200.scene import grid_geometry
    from mpmwarpydw_b200.utils.getArgs import defaults
    a = defaults()
    a.boundary_padding_mask = "000001"
    a.grid_padding = 10.0
    x = np.array([[0, 0, 0], [10, 10, 10]], np.float32)
    dx, mn, mx, dims = grid_geometry(a, x, np.full(2, 0.125), dx=1.0)
    assert np.allclose(mn, [-2, -2, -2]) and np.allclose(mx, [12, 12, 20]) and dims == (14, 14, 22)
    with pytest.raises(ValueError):
        a.boundary_padding_mask = "0101"
        grid_geometry(a, x, np.full(2, 0.125), dx=1.0)


def test_block_sort_key_groups_blocks():
    import torch
    from mpmwarpydw_b200.engine import block_sort_key
    x = torch.tensor([[0.5, 0.5, 0.5], [4.5, 0.5, 0.5], [1.5, 0.5, 0.5], [0.5, 0.5, 4.5]])
    k = block_sort_key(x, (0, 0, 0), 1.0, (8, 8, 8))
    # particles 0 and 2 share block (0,0,0); particle 3 is in block (0,0,1); particle 1 in block (1,0,0)
    assert k[0] // 64 == k[2] // 64 and k[0] < k[2] < k[3] < k[1]


def test_batch_arguments_are_checked_before_any_device_work():
    """mpmw_batch_prepare rejects a bad scene table with MPMW_E_ARG (and a short
    workspace with MPMW_E_WORKSPACE) before it touches a device, and
    mpmw_batch_run_substeps refuses a workspace that was never prepared: the
    pointers below are host addresses that no kernel ever sees."""
    from mpmwarpydw_b200 import _lib
    L = _lib.lib()
    buf = (ctypes.c_float * 128)()
    addr = ctypes.addressof(buf) + (-ctypes.addressof(buf)) % 256  # 256-byte aligned host address
    P = _lib.Particles(); P.n = 512
    for f in ("x", "v", "C", "F", "F_trial", "stress", "vol", "mass", "density", "mu", "lam", "ys", "alpha",
              "hardening", "softening", "strain_criteria", "eta_shear", "eta_bulk", "acc_strain", "damage",
              "active", "material", "x_pc", "v_pc"):
        setattr(P, f, addr)
    grids = (_lib.Grid * 2)()
    prms = (_lib.Params * 2)()
    for g in grids:
        g.dims[0] = g.dims[1] = g.dims[2] = 4
        g.mv = g.v = addr
    for p in prms:
        p.boundary_condition = -1

    def prepare(offsets, nscenes=2, ws=None, ws_bytes=0):
        offs = (ctypes.c_int64 * len(offsets))(*offsets)
        return L.mpmw_batch_prepare(ctypes.byref(P), grids, prms, offs, nscenes, ws, ws_bytes, None)

    need = L.mpmw_batch_workspace_bytes(grids, 2, 512)
    assert need > L.mpmw_workspace_bytes(512)  # worklist plus the scene table
    assert prepare([0, 100, 512]) == 1 and b"multiples of 256" in L.mpmw_last_error()
    assert prepare([0, 256, 500]) == 1 and b"particle count" in L.mpmw_last_error()
    assert prepare([0, 512, 512]) == 1 and b"increase" in L.mpmw_last_error()
    assert prepare([0], nscenes=0) == 1 and b"scenes" in L.mpmw_last_error()
    prms[1].vlc = 1
    assert prepare([0, 256, 512]) == 1 and b"locking" in L.mpmw_last_error()
    prms[1].vlc = 0
    assert prepare([0, 256, 512]) == 4 and b"workspace" in L.mpmw_last_error()
    assert prepare([0, 256, 512], ws=addr + 4, ws_bytes=need) == 1 and b"aligned" in L.mpmw_last_error()
    assert prepare([0, 256, 512], ws=addr, ws_bytes=need - 256) == 4 and b"workspace" in L.mpmw_last_error()
    grids[1].dims[2] = 0
    assert prepare([0, 256, 512]) == 1 and b"dims" in L.mpmw_last_error()
    assert L.mpmw_batch_workspace_bytes(grids, 2, 512) == 0
    rc = L.mpmw_batch_run_substeps(ctypes.byref(P), 3, None, addr, need, None)
    assert rc == 1 and b"not prepared" in L.mpmw_last_error()


def test_scene_groups_are_contiguous_balanced_and_never_empty():
    """The batch's scene ranges (one stream each) cover every scene once, in
    order, with min(groups, scenes) non-empty ranges of similar particle count."""
    import random

    from mpmwarpydw_b200.sweep import scene_groups
    rng = random.Random(5)
    for _ in range(200):
        counts = [rng.randint(1, 1000) for _ in range(rng.randint(1, 40))]
        g = rng.randint(1, 50)
        r = scene_groups(counts, g)
        assert len(r) == min(g, len(counts))
        assert r[0][0] == 0 and r[-1][1] == len(counts)
        assert all(a < b for a, b in r) and all(r[i][1] == r[i + 1][0] for i in range(len(r) - 1))
    # equal scenes split evenly
    assert scene_groups([10] * 8, 4) == [(0, 2), (2, 4), (4, 6), (6, 8)]


def test_device_segments_stop_before_host_events():
    """The device loop runs whole chunks only: each ends within nSteps and by
    the end of a gravity pulse, and none holds an XPBD substep (a positive
    multiple of the XPBD ratio), which the host runs with its chunk."""
    import random

    from mpmwarpydw_b200.runMPMYDW import device_segment
    rng = random.Random(3)
    for _ in range(500):
        c, k, ratio = rng.randint(0, 300), rng.randint(1, 12), rng.randint(1, 60)
        n_steps, pulse = rng.randint(c, 400), rng.choice([0, rng.randint(1, 300)])
        seg = device_segment(c, k, ratio, n_steps, pulse)
        assert seg % k == 0 and c + seg <= n_steps
        for a in range(c, c + seg, k):
            assert not any(m % ratio == 0 for m in range(max(a, 1), a + k))
            assert not (pulse and a < pulse < a + k)
        # the next chunk is one the host must run (or there is none)
        a = c + seg
        nxt_ok = (a + k <= n_steps and not (pulse and a < pulse < a + k)
                  and not any(m % ratio == 0 for m in range(max(a, 1), a + k)))
        assert not nxt_ok


def test_xpbd_step_workspace_covers_the_persistent_form():
    """mpmw_xpbd_step runs as one persistent launch only with a workspace of
    mpmw_xpbd_step_workspace_bytes(n, dims): a 16 KB header (barrier
    arrivals, XPBD count, tile tickets, scan chunk sums), one bit per hash
    cell, then an area that holds the radix sort's buffers and, after the
    build, 32 B of contact records per point.  Host-side size query only."""
    import ctypes

    from mpmwarpydw_b200 import _lib
    L = _lib.lib()
    for n, d in ((1, (1, 1, 1)), (1000, (128, 128, 128)), (3_873_600, (120, 70, 120))):
        dims = (ctypes.c_int32 * 3)(*d)
        need = int(L.mpmw_xpbd_step_workspace_bytes(n, dims))
        ncell = d[0] * d[1] * d[2]
        bits = (ncell + 31) // 32 * 4
        assert need >= 16384 + bits + 32 * n
        assert need >= int(L.mpmw_hash_workspace_bytes(n))
