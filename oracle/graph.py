"""CPU CSR of the device random-graph build (test infrastructure).

Same hashes as ha_graph_build_c: degree of u = number of thresholds <=
mix32(u ^ seed); k-th neighbour = mix32(mix32(u ^ seed ^ 0xABCDEF01) +
k * 0x9E3779B9) mod n.  Returns (offsets, cols) with offsets[0] = 0.
"""
from __future__ import annotations

import numpy as np

from .phase import mix32


def graph_csr(n: int, seed: int, thresholds: np.ndarray):
    u = np.arange(n, dtype=np.uint32)
    deg = np.searchsorted(np.asarray(thresholds, np.uint32), mix32(u ^ np.uint32(seed)),
                          side="right").astype(np.int64)
    offsets = np.zeros(n + 1, np.int64)
    np.cumsum(deg, out=offsets[1:])
    src = np.repeat(u, deg)
    k = (np.arange(offsets[-1], dtype=np.int64) - np.repeat(offsets[:-1], deg)).astype(np.uint32)
    base = mix32(src ^ np.uint32(seed) ^ np.uint32(0xABCDEF01))
    cols = mix32(base + k * np.uint32(0x9E3779B9)) % np.uint32(n)
    return offsets, cols.astype(np.uint32)
