"""The reference's XPBD kernel surface (utils/xpbdRoutines.py), backed by libmpmw."""
from __future__ import annotations

import torch


class HashGrid:
    """Spatial hash with the interface of ``wp.HashGrid(dim_x, dim_y, dim_z)``.

    ``build(points, radius)`` hashes (N, 3) CUDA points into cells of width
    ``radius``; the sorted point order and per-cell ranges stay on the device."""

    def __init__(self, dim_x, dim_y, dim_z, device="cuda:0"):
        self.dims = (int(dim_x), int(dim_y), int(dim_z))
        self.device = torch.device(device)
        self.cell_width = None
        self.point_ids = None
        self.cell_starts = None
        self.cell_ends = None
        self.point_cells = None
        self.id = self  # the reference passes grid.id into kernels

    def build(self, points, radius):
        raise NotImplementedError("HashGrid.build: XPBD kernels are not built yet")


def xpbd_step(sim, mpm, xpbd, xpbd_only=False):
    raise NotImplementedError("xpbdSimulationStep: XPBD kernels are not built yet")
