"""Host results of the reference's sample programs (test infrastructure).

grid-points (halloc samples/grid-points/grid-points.cu:82-99): the cell of
each point, and per cell the number of points and the sum of mix32(point
index), the digest the device's ha_grid_check_c computes.  The cell index
follows the sample's float32 arithmetic: floor(p * ncells), clamped.
"""
from __future__ import annotations

import numpy as np

from oracle.phase import mix32


def grid_cells(pts: np.ndarray, ncells: int) -> np.ndarray:
    c = np.floor(pts.astype(np.float32) * np.float32(ncells)).astype(np.int64)
    c = np.clip(c, 0, ncells - 1)
    return c[:, 0] + ncells * (c[:, 1] + ncells * c[:, 2])


def grid_expect(pts: np.ndarray, ncells: int):
    """(count, hsum) per cell, ncells^3 entries each."""
    cell = grid_cells(pts, ncells)
    n3 = ncells ** 3
    count = np.bincount(cell, minlength=n3).astype(np.uint32)
    h = mix32(np.arange(len(pts), dtype=np.uint32)).astype(np.uint64)
    hsum = np.zeros(n3, np.uint64)
    np.add.at(hsum, cell, h)
    return count, hsum
