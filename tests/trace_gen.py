"""Seeded serial trace generator shared by the golden-fixture script and the
tests.  A trace is a list of ops: op >= 0 is hamalloc(op); op < 0 frees the
block returned by op index -(op + 1)."""
from __future__ import annotations

import numpy as np


def make_trace(n: int, sizes, pfree: float, seed: int, live_cap: int | None = None,
               drain: float = 0.0, tail: int = 0) -> list:
    """n random ops (malloc of a size drawn from `sizes`, or, with probability
    pfree, free of a random live block); then frees `drain` of the remaining
    live blocks; then `tail` more mallocs."""
    rng = np.random.default_rng(seed)
    ops: list = []
    live: list = []
    sizes = list(sizes)
    for _ in range(n):
        if live and (rng.random() < pfree or (live_cap and len(live) >= live_cap)):
            j = live.pop(int(rng.integers(len(live))))
            ops.append(-(j + 1))
        else:
            ops.append(int(sizes[int(rng.integers(len(sizes)))]))
            live.append(len(ops) - 1)
    if drain:
        rng.shuffle(live)
        k = int(drain * len(live))
        ops.extend(-(j + 1) for j in live[:k])
        live = live[k:]
    for _ in range(tail):
        ops.append(int(sizes[int(rng.integers(len(sizes)))]))
    return ops
