"""Workload drivers built on the C ABI: the batched request stream, the
degree table of the random-graph build, the generator seeds of the
reference-form phase workload and the inputs of the sample programs.

The batched stream (64 batches of log-uniform size between 1,024 and
1,048,576 requests; block sizes geometric over the 16 size classes with
p = 0.3 per class step; 1 % large requests uniform in 4..64 KiB that take the
CUDA-heap path; lifetimes uniform over 1..8 batches) is generated on the host
from a seed and served either by per-batch kernel launches (plain form) or by
one persistent kernel, optionally replayed from a CUDA graph.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import HallocError, _addr, _check, _stream, load

CLASS_BYTES = [16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768, 1024, 1536, 2048, 3072]


@dataclass
class BatchedPlan:
    req_size: np.ndarray     # uint32, nreq
    batch_start: np.ndarray  # uint32, nbatch + 1
    free_start: np.ndarray   # uint32, nbatch + 2
    free_ids: np.ndarray     # uint32, nreq
    nbatch: int

    @property
    def nreq(self) -> int:
        return int(self.req_size.shape[0])


def batched_plan(seed: int = 1, nbatch: int = 64, min_batch: int = 1024,
                 max_batch: int = 1 << 20, p_class: float = 0.3, large_frac: float = 0.01,
                 large_lo: int = 4096, large_hi: int = 65536, max_life: int = 8) -> BatchedPlan:
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(min_batch), np.log(max_batch), nbatch))
    counts = np.maximum(1, np.rint(sizes)).astype(np.int64)
    nreq = int(counts.sum())
    w = p_class * (1 - p_class) ** np.arange(16)
    cls = rng.choice(16, size=nreq, p=w / w.sum())
    req_size = np.asarray(CLASS_BYTES, np.uint32)[cls]
    large = rng.random(nreq) < large_frac
    req_size[large] = rng.integers(large_lo, large_hi + 1, int(large.sum()), dtype=np.uint32)
    batch_start = np.zeros(nbatch + 1, np.uint32)
    batch_start[1:] = np.cumsum(counts)
    batch_of = np.repeat(np.arange(nbatch), counts)
    step = np.minimum(batch_of + rng.integers(1, max_life + 1, nreq), nbatch)
    free_ids = np.argsort(step, kind="stable").astype(np.uint32)
    free_start = np.zeros(nbatch + 2, np.uint32)
    free_start[1:] = np.cumsum(np.bincount(step, minlength=nbatch + 1))
    return BatchedPlan(req_size, batch_start, free_start, free_ids, nbatch)


class _CPlan(ctypes.Structure):
    _fields_ = [("nbatch", ctypes.c_uint32), ("nreq", ctypes.c_uint32),
                ("req_size", ctypes.c_void_p), ("req_ptr", ctypes.c_void_p),
                ("free_ids", ctypes.c_void_p), ("h_batch_start", ctypes.c_void_p),
                ("h_free_start", ctypes.c_void_p), ("acc", ctypes.c_void_p)]


ACC = ("failed", "mismatches", "id_sum", "mallocs", "frees", "late")


class BatchedRunner:
    """Device copies of a plan (torch tensors) and the two ways of serving
    it: per-batch launches and the persistent kernel."""

    def __init__(self, plan: BatchedPlan, torch):
        lib = load()
        for name, res, args in (
                ("ha_batched_plain_c", ctypes.c_int, [ctypes.POINTER(_CPlan), ctypes.c_uint32,
                                                      ctypes.c_void_p]),
                ("ha_batched_prepare_c", ctypes.c_int,
                 [ctypes.POINTER(_CPlan), ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                  ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
                ("ha_batched_launch_c", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
                ("ha_batched_run_noalloc_c", ctypes.c_int,
                 [ctypes.POINTER(_CPlan), ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                  ctypes.c_void_p]),
                ("ha_batched_release_c", ctypes.c_int, [ctypes.c_void_p])):
            f = getattr(lib, name)
            f.restype, f.argtypes = res, args
        self.lib, self.plan, self.torch = lib, plan, torch
        dev = "cuda"
        self.d_size = torch.from_numpy(plan.req_size.view(np.int32)).to(dev)
        self.d_ptr = torch.zeros(plan.nreq, dtype=torch.int64, device=dev)
        self.d_free = torch.from_numpy(plan.free_ids.view(np.int32)).to(dev)
        self.d_acc = torch.zeros(8, dtype=torch.int64, device=dev)
        self.h_batch = np.ascontiguousarray(plan.batch_start)
        self.h_free = np.ascontiguousarray(plan.free_start)
        self.c = _CPlan(plan.nbatch, plan.nreq, _addr(self.d_size), _addr(self.d_ptr),
                        _addr(self.d_free), self.h_batch.ctypes.data, self.h_free.ctypes.data,
                        _addr(self.d_acc))
        self.handles = []

    def plain(self, block: int = 256, stream=None) -> None:
        _check(self.lib.ha_batched_plain_c(ctypes.byref(self.c), block, _stream(stream)),
               "ha_batched_plain_c")

    def prepare(self, block: int = 1024, ctas_per_sm: int = 0, task_items: int = 8192,
                graph: bool = True):
        h = ctypes.c_void_p()
        _check(self.lib.ha_batched_prepare_c(ctypes.byref(self.c), block, ctas_per_sm,
                                             task_items, 1 if graph else 0, ctypes.byref(h)),
               "ha_batched_prepare_c")
        self.handles.append(h)
        return h

    def run_noalloc(self, block: int = 256, ctas_per_sm: int = 0, task_items: int = 2048,
                    stream=None) -> int:
        """The persistent form through ha_batched_run_noalloc_c, which
        allocates nothing (for callers that cannot call cudaMalloc).  Returns
        the C return code (HA_ERANGE for a plan beyond its fixed limits)."""
        return self.lib.ha_batched_run_noalloc_c(ctypes.byref(self.c), block, ctas_per_sm,
                                                 task_items, _stream(stream))

    def launch(self, handle, stream=None) -> None:
        _check(self.lib.ha_batched_launch_c(handle, _stream(stream)), "ha_batched_launch_c")

    def release(self) -> None:
        for h in self.handles:
            self.lib.ha_batched_release_c(h)
        self.handles = []

    def acc(self) -> dict:
        return dict(zip(ACC, self.d_acc.cpu().tolist()))

    def verify(self, acc: dict | None = None) -> dict:
        a = acc or self.acc()
        n = self.plan.nreq
        ok = (a["failed"] == 0 and a["mismatches"] == 0 and a["late"] == 0 and
              a["mallocs"] == n and a["frees"] == n and a["id_sum"] == n * (n - 1) // 2)
        if not ok:
            raise HallocError(f"batched run failed verification: {a}")
        return a


def poisson_thresholds(lam: float = 16.0) -> np.ndarray:
    """32-bit thresholds of the Poisson(lam) CDF for ha_graph_build_c: a
    vertex whose hash is h gets degree #{k : t[k] <= h}."""
    p = np.exp(-lam)
    cdf, out, k = p, [], 0
    while True:
        t = min(int(cdf * 2**32), 2**32 - 1)
        out.append(t)
        if t >= 2**32 - 1 or k > 10 * lam + 100:
            break
        k += 1
        p *= lam / k
        cdf += p
    out[-1] = 2**32 - 1
    return np.asarray(out, np.uint32)


def group_seeds(nthreads: int, group: int, seed: int) -> np.ndarray:
    """Initial generator states for the reference-form phase workload
    (ha_phase_ref_step_c): one seed per group of `group` consecutive
    threads, as halloc's drandom_init (tst/common/common.cu:358-383, period
    1) seeds them, drawn from a seeded numpy generator instead of random()."""
    rng = np.random.default_rng(seed)
    per_group = rng.integers(0, 1 << 31, (nthreads + group - 1) // group, dtype=np.uint32)
    return np.repeat(per_group, group)[:nthreads].astype(np.uint32)


def sample_points(n: int, seed: int) -> np.ndarray:
    """n points in [0, 1)^3 on the 1/65536 lattice of halloc's grid-points
    sample (samples/grid-points/grid-points.cu:45-54), float32 (n, 3),
    seeded."""
    rng = np.random.default_rng(seed)
    return (rng.integers(0, 65536, (n, 3)) / 65536.0).astype(np.float32)


def sample_lengths(n: int, period: int, lo: int, hi: int, seed: int) -> np.ndarray:
    """String lengths in [lo, hi], equal within groups of `period`
    consecutive strings, as halloc's add-strings sample draws them
    (samples/add-strings/add-strings.cu:44-53), seeded."""
    rng = np.random.default_rng(seed)
    per = rng.integers(lo, hi + 1, (n + period - 1) // period)
    return np.repeat(per, period)[:n].astype(np.int32)
