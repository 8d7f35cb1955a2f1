"""mpmw_hash_build_noalloc (static scratch, no allocation) against mpmw_hash_build
(caller workspace), through the C ABI.  The hash is integer work: bit-exact.

Kept in a file of its own that pytest collects last, so it runs both alone in a
fresh process and after every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HASH_DIMS = (128, 128, 128)


def _points(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-3, 40, (n, 3)).astype(np.float32)
    if n > 10:
        x[: n // 10] = x[0]  # a crowded cell
    return x


def _hash_arrays(torch, n, dev):
    ncell = int(np.prod(HASH_DIMS))
    return dict(point_ids=torch.empty(max(n, 1), dtype=torch.int32, device=dev),
                cell_starts=torch.full((ncell,), -7, dtype=torch.int32, device=dev),
                cell_ends=torch.full((ncell,), -7, dtype=torch.int32, device=dev),
                point_cells=torch.empty(max(n, 1), dtype=torch.int32, device=dev))


def _struct(a, w):
    from mpmwarpydw_b200 import _lib
    h = _lib.Hash()
    for i in range(3):
        h.dims[i] = HASH_DIMS[i]
    h.cell_width = w
    for k in ("point_ids", "cell_starts", "cell_ends", "point_cells"):
        setattr(h, k, a[k].data_ptr())
    return h


def test_noalloc_hash_matches_workspace_hash_twice():
    import torch

    from mpmwarpydw_b200 import _lib
    L = _lib.lib()
    dev = "cuda:0"
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    for n, w, seed in ((70_000, 1.0, 11), (5_000, 0.25, 12)):   # two calls in a row, different sizes
        x = torch.as_tensor(_points(n, seed).T.copy(), device=dev)  # SoA [3][n]
        ref = _hash_arrays(torch, n, dev)
        ws = torch.empty(int(L.mpmw_hash_workspace_bytes(n)), dtype=torch.uint8, device=dev)
        _lib.check(L.mpmw_hash_build(x.data_ptr(), n, ctypes.byref(_struct(ref, w)), ws.data_ptr(), ws.numel(),
                                     stream), "hash_build")
        got = _hash_arrays(torch, n, dev)
        _lib.check(L.mpmw_hash_build_noalloc(x.data_ptr(), n, ctypes.byref(_struct(got, w)), stream),
                   "hash_build_noalloc")
        torch.cuda.synchronize()
        for k in ("point_ids", "point_cells"):
            assert torch.equal(got[k][:n], ref[k][:n]), k
        for k in ("cell_starts", "cell_ends"):
            assert torch.equal(got[k], ref[k]), k


def test_noalloc_hash_rejects_too_many_points():
    import torch

    from mpmwarpydw_b200 import _lib
    L = _lib.lib()
    a = _hash_arrays(torch, 1, "cuda:0")
    n = 1048576 + 1
    rc = L.mpmw_hash_build_noalloc(None, n, ctypes.byref(_struct(a, 1.0)), None)
    assert rc == 1  # MPMW_E_ARG, before any device work
    assert b"1048576" in L.mpmw_last_error()
