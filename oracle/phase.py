"""Host replay of the mixed-size phase workload (test infrastructure).

The device workload (ha_phase_round_c / ha_phase_run_c) takes every
decision from a hash of (seed, thread, slot, round): whether an empty slot is
filled, the block size, the payload base, whether a live block is freed.
Replaying the same hashes here gives, for any device scheduling, the exact
number of allocations and frees, the slots filled after every round and the
sums of all payload words written and read back -- provided no allocation
failed, which the device reports separately.
"""
from __future__ import annotations

import numpy as np

MASK32 = 0xFFFFFFFF


def mix32(x) -> np.ndarray:
    """The "lowbias32" integer finaliser, as in the device kernels."""
    x = np.array(x, dtype=np.uint32, copy=True)
    x ^= x >> np.uint32(16)
    x *= np.uint32(0x7FEB352D)
    x ^= x >> np.uint32(15)
    x *= np.uint32(0x846CA68B)
    x ^= x >> np.uint32(16)
    return x


def slot_hash(seed: int, i: np.ndarray, s: int, rnd: int) -> np.ndarray:
    key = ((i.astype(np.uint32) << np.uint32(2)) | np.uint32(s))
    return mix32(key ^ np.uint32((rnd * 0x9E3779B9) & MASK32) ^ np.uint32(seed))


def words_sum(base: np.ndarray, nbytes: np.ndarray) -> int:
    """Sum over blocks of the 32-bit words base, base+1, ... (mod 2^32 each)
    filling nbytes // 4 words."""
    m = (nbytes.astype(np.int64) // 8) * 2
    b = base.astype(np.int64)
    wrapped = np.maximum(0, b + m - (1 << 32))
    return int((m * b + m * (m - 1) // 2 - (wrapped << 32)).sum())


class PhaseReplay:
    def __init__(self, nthreads: int, nslots: int, seed: int, size_set):
        self.n, self.nslots, self.seed = nthreads, nslots, seed
        self.size_set = np.asarray(size_set, np.uint32)
        self.i = np.arange(nthreads, dtype=np.uint32)
        self.filled = np.zeros((nslots, nthreads), bool)
        self.size = np.zeros((nslots, nthreads), np.uint32)
        self.base = np.zeros((nslots, nthreads), np.uint32)
        self.wsum = self.rsum = self.mallocs = self.frees = 0

    def alloc_round(self, rnd: int, thr: int) -> int:
        for s in range(self.nslots):
            h = slot_hash(self.seed, self.i, s, rnd)
            take = ~self.filled[s] & (h < np.uint32(thr))
            sz = self.size_set[mix32(h ^ np.uint32(0xA5A5A5A5)) % np.uint32(len(self.size_set))]
            base = mix32(h ^ np.uint32(0x5EED5EED))
            self.size[s, take] = sz[take]
            self.base[s, take] = base[take]
            self.filled[s] |= take
            self.wsum += words_sum(base[take], sz[take])
            self.mallocs += int(take.sum())
        return int(self.filled.sum())

    def free_round(self, rnd: int, thr: int) -> int:
        for s in range(self.nslots):
            live = self.filled[s]
            if thr == MASK32:
                take = live
            else:
                take = live & (slot_hash(self.seed, self.i, s, rnd) < np.uint32(thr))
            self.rsum += words_sum(self.base[s, take], self.size[s, take])
            self.frees += int(take.sum())
            self.filled[s] &= ~take
        return int(self.filled.sum())

    def run(self, periods: int, thr_alloc: int, thr_free: int, target_filled: int,
            max_rounds: int) -> dict:
        """The schedule of ha_phase_run_c."""
        rnd = 0
        alloc_rounds = free_rounds = 0
        for _ in range(periods):
            for _ in range(max_rounds):
                filled = self.alloc_round(rnd, thr_alloc)
                rnd += 1
                alloc_rounds += 1
                if filled >= target_filled:
                    break
            self.free_round(rnd, thr_free)
            rnd += 1
            free_rounds += 1
        filled = self.free_round(rnd, MASK32)
        free_rounds += 1
        return {"alloc_rounds": alloc_rounds, "free_rounds": free_rounds, "filled": filled,
                "wsum": self.wsum, "rsum": self.rsum, "mallocs": self.mallocs,
                "frees": self.frees}


# ---- the reference's own form of the phase workload ---------------------------
#
# halloc tst/perf/phase-throughput/phase-throughput.cu:17-48 (one launch per
# try) and tst/common/common.h:80-117, 209-235 (per-thread generator, draws,
# next_action, next_alloc_sz with the uniform distribution).


def wang_next(st: np.ndarray) -> np.ndarray:
    """Thomas Wang's 32-bit integer hash, the reference's drandom() step
    (tst/common/common.h:86-91); returns the new states."""
    x = np.array(st, dtype=np.uint32, copy=True)
    x = (x ^ np.uint32(61)) ^ (x >> np.uint32(16))
    x *= np.uint32(9)
    x ^= x >> np.uint32(4)
    x *= np.uint32(0x27D4EB2D)
    x ^= x >> np.uint32(15)
    return x


def wang_next_scalar(x: int) -> int:
    """The same step on a Python int (for known-answer checks)."""
    x = ((x ^ 61) ^ (x >> 16)) & MASK32
    x = (x * 9) & MASK32
    x ^= x >> 4
    x = (x * 0x27D4EB2D) & MASK32
    x ^= x >> 15
    return x


class PhaseRefReplay:
    """Replays the reference-form phase workload thread by thread: the
    decisions, block sizes, generator states and per-thread block counts are
    exactly the device's, whatever the scheduling, as long as no allocation
    failed.  sizes[k, i] is the size of thread i's k-th live block (0 when
    the thread holds nothing)."""

    def __init__(self, states: np.ndarray, nallocs: int, probs, smin: int, smax: int,
                 niters: int = 1):
        self.st = np.array(states, dtype=np.uint32, copy=True)
        self.n = len(self.st)
        self.nallocs, self.niters = nallocs, niters
        self.p = np.asarray(probs, np.float32).reshape(2, 2)
        self.smin, self.smax = smin, smax
        self.ctr = np.zeros(self.n, np.uint32)
        self.sizes = np.zeros((nallocs, self.n), np.uint32)
        self.mallocs = self.frees = self.bytes = 0

    def _draw_in(self, mask: np.ndarray, a: int, b: int) -> np.ndarray:
        nxt = wang_next(self.st)
        self.st = np.where(mask, nxt, self.st)
        return np.uint32(a) + (nxt & np.uint32(0x00FFFFFF)) % np.uint32(b - a + 1)

    def _draw_bool(self, mask: np.ndarray, p: np.ndarray) -> np.ndarray:
        inner = (p > 0) & (p < 1)
        k = self._draw_in(mask & inner, 0, (1 << 20) - 1)
        frac = np.float32(1.0 / (1 << 20)) * k.astype(np.float32)
        return np.where(inner, frac <= p, p >= 1)

    def step(self, itry: int) -> None:
        every = np.ones(self.n, bool)
        for it in range(self.niters):
            phase = (itry * self.niters + it) % 2
            holding = self.ctr > 0
            p = np.where(holding, self.p[phase, 1], self.p[phase, 0]).astype(np.float32)
            act = self._draw_bool(every, p)
            alloc = act & ~holding
            free = act & holding
            for k in range(self.nallocs):
                if self.smin == self.smax:
                    sz = np.full(self.n, self.smin, np.uint32)
                else:
                    sz = self._draw_in(alloc, self.smin, self.smax)
                self.sizes[k] = np.where(alloc, sz, np.where(free, 0, self.sizes[k]))
                self.bytes += int(sz[alloc].sum(dtype=np.uint64))
            self.mallocs += int(alloc.sum()) * self.nallocs
            self.frees += int(free.sum()) * self.nallocs
            self.ctr = np.where(alloc, self.nallocs, np.where(free, 0, self.ctr)).astype(
                np.uint32)

    def rest(self) -> None:
        self.frees += int(self.ctr.sum())
        self.ctr[:] = 0
        self.sizes[:] = 0
