"""The bounded mbarrier wait every TMA and bulk-copy consumer uses
(mpmwarpydw_b200/csrc/mpmw_tma.cuh): a wait on a barrier that completes
returns at once; a wait on a barrier that nothing completes gives up after
its wall-time bound (200 ms) with a false result, and the CUDA context stays
usable.  The probe kernel is test code (tests/csrc/wait_probe.cu), built with
nvcc against the library's own header."""
import ctypes
import os
import subprocess
import tempfile

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "wait_probe.cu")
BOUND_NS = 200_000_000


def _build(outdir):
    from mpmwarpydw_b200 import build as B
    so = os.path.join(outdir, "wait_probe.so")
    cmd = [B.nvcc(), *B.ARCH, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-o", so, SRC]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return so


def test_probe_builds():
    with tempfile.TemporaryDirectory() as d:
        assert os.path.getsize(_build(d)) > 0


@pytest.mark.gpu
def test_bounded_wait_returns_and_times_out():
    import torch
    torch.cuda.init()
    with tempfile.TemporaryDirectory() as d:
        lib = ctypes.CDLL(_build(d))
        lib.wait_probe.restype = ctypes.c_int
        lib.wait_probe.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_uint), ctypes.POINTER(ctypes.c_ulonglong)]
        ok, ns = ctypes.c_uint(7), ctypes.c_ulonglong(0)
        assert lib.wait_probe(1, ctypes.byref(ok), ctypes.byref(ns)) == 0
        assert ok.value == 1 and ns.value < 1_000_000          # completed phase: returns within 1 ms
        ok, ns = ctypes.c_uint(7), ctypes.c_ulonglong(0)
        assert lib.wait_probe(0, ctypes.byref(ok), ctypes.byref(ns)) == 0
        assert ok.value == 0                                     # never completed: gives up
        assert BOUND_NS <= ns.value < 10 * BOUND_NS              # after its bound, not much later
        ok = ctypes.c_uint(7)
        assert lib.wait_probe(1, ctypes.byref(ok), ctypes.byref(ns)) == 0 and ok.value == 1  # context usable
    x = torch.arange(4, device="cuda:0")
    assert int(x.sum().item()) == 6
