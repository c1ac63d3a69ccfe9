"""halloc-b200: host side of the B200 device allocator.

The allocator lives in device code (``hamalloc`` / ``hafree``,
include/halloc.h).  This module binds the C ABI of ``libhalloc_b200.so``
(include/halloc_c.h) with ctypes, mirroring the reference's host interface
(``ha_init(halloc_opts_t)``, ``ha_shutdown``, ``ha_extfrag``) and its test
harness wrappers (batch malloc / free, the private-throughput loop).

Device buffers are passed as integers (device addresses, e.g.
``tensor.data_ptr()``) or as objects with a ``data_ptr()`` method; streams
as integers (``torch.cuda.current_stream().cuda_stream``) or None for the
default stream.  There is no CPU fallback: every call needs the native
library and a CUDA device, and raises HallocError otherwise.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

__all__ = [
    "HallocError", "HallocOpts", "init", "shutdown", "extfrag", "stats", "status",
    "clear_status", "set_wait_limit", "dump_state", "l2_persist", "malloc_batch",
    "free_batch", "phase_round", "phase_run", "phase_ref_step", "phase_ref_run", "phase_ref_latency", "grid_insert",
    "grid_check", "grid_free", "strings_alloc", "strings_concat", "strings_free",
    "strings_check", "graph_build", "graph_gather", "serve_run",
    "throughput", "throughput_host", "cuda_throughput", "trace",
    "atomic_peak", "debug_set_head_lock", "set_hash_scale", "set_heads", "set_surge",
    "close_surges", "set_growth", "grow",
    "trim", "ST_GROW", "library_path", "load", "ST_TIMEOUT", "ST_BAD_FREE", "ST_LIVELOCK",
]

PKG = os.path.dirname(os.path.abspath(__file__))
SO_PATH = os.path.join(PKG, "libhalloc_b200.so")

HA_OK, HA_EINVAL, HA_ECUDA, HA_ESTATE, HA_ERANGE = 0, -1, -2, -3, -4
ST_TIMEOUT, ST_BAD_FREE, ST_LIVELOCK, ST_GROW = 0x1, 0x2, 0x4, 0x8
NSIZES = 16
NSETS = 37
NONE = 0xFFFFFFFF

_ERR = {HA_EINVAL: "invalid argument", HA_ECUDA: "CUDA error",
        HA_ESTATE: "wrong allocator state (not / already initialised)",
        HA_ERANGE: "size beyond a documented limit"}


class HallocError(RuntimeError):
    pass


@dataclass
class HallocOpts:
    """Mirror of ``halloc_opts_t`` (include/halloc.h; defaults of halloc
    src/halloc.h:30-33)."""

    memory: int = 512 << 20
    halloc_fraction: float = 0.75
    busy_fraction: float = 0.835
    roomy_fraction: float = 0.6
    sparse_fraction: float = 0.012
    sb_sz_sh: int = 22


class _COpts(ctypes.Structure):
    _fields_ = [("memory", ctypes.c_uint64), ("halloc_fraction", ctypes.c_double),
                ("busy_fraction", ctypes.c_double), ("roomy_fraction", ctypes.c_double),
                ("sparse_fraction", ctypes.c_double), ("sb_sz_sh", ctypes.c_int32)]


class _CStats(ctypes.Structure):
    _fields_ = [("pool_base", ctypes.c_uint64), ("pool_bytes", ctypes.c_uint64),
                ("cuda_heap_bytes", ctypes.c_uint64), ("used_chunks", ctypes.c_uint64),
                ("used_bytes", ctypes.c_uint64), ("nsbs", ctypes.c_uint32),
                ("sb_sz", ctypes.c_uint32), ("free_slabs", ctypes.c_uint32),
                ("head_slabs", ctypes.c_uint32), ("status", ctypes.c_uint32),
                ("n_head_changes", ctypes.c_uint32), ("n_null", ctypes.c_uint32),
                ("heap_limit_ok", ctypes.c_uint32), ("head", ctypes.c_uint32 * 16),
                ("cached", ctypes.c_uint32 * 16), ("growth", ctypes.c_uint32),
                ("committed_slabs", ctypes.c_uint32), ("unit_bytes", ctypes.c_uint64),
                ("surge_level", ctypes.c_uint32 * 16), ("n_surge_changes", ctypes.c_uint32),
                ("free_count", ctypes.c_uint32)]


class _CPhaseResult(ctypes.Structure):
    _fields_ = [("alloc_rounds", ctypes.c_uint32), ("free_rounds", ctypes.c_uint32),
                ("kernel_ms", ctypes.c_double), ("filled", ctypes.c_uint64),
                ("acc", ctypes.c_uint64 * 6)]


SERVE_HIST = 1024


class _CServeCfg(ctypes.Structure):
    _fields_ = [("njobs", ctypes.c_uint32), ("seed", ctypes.c_uint32),
                ("lam", ctypes.c_double), ("occupancy_limit", ctypes.c_double),
                ("mean_life", ctypes.c_double), ("block_bytes", ctypes.c_uint32),
                ("min_len", ctypes.c_uint32), ("max_len", ctypes.c_uint32),
                ("grow_min", ctypes.c_uint32), ("grow_max", ctypes.c_uint32),
                ("cta_threads", ctypes.c_uint32), ("ctas_per_sm", ctypes.c_uint32),
                ("job_ids", ctypes.c_void_p), ("njob_ids", ctypes.c_uint32),
                ("results", ctypes.c_void_p), ("grow_bytes", ctypes.c_uint64),
                ("prereleased", ctypes.c_uint32)]


class _CServeResult(ctypes.Structure):
    _fields_ = [("seconds", ctypes.c_double), ("cycles_per_ns", ctypes.c_double),
                ("jobs_done", ctypes.c_uint64), ("allocs", ctypes.c_uint64),
                ("alloc_failures", ctypes.c_uint64), ("refusals", ctypes.c_uint64),
                ("peak_live_blocks", ctypes.c_uint64), ("timeouts", ctypes.c_uint64),
                ("p50_cycles", ctypes.c_double), ("p99_cycles", ctypes.c_double),
                ("max_cycles", ctypes.c_double), ("hist", ctypes.c_uint64 * SERVE_HIST),
                ("alloc_waits", ctypes.c_uint64), ("grows", ctypes.c_uint64),
                ("grown_bytes", ctypes.c_uint64), ("grow_seconds", ctypes.c_double)]


class _CPhaseRefResult(ctypes.Structure):
    _fields_ = [("kernel_ms", ctypes.c_double), ("alloc_phase_ms", ctypes.c_double),
                ("free_phase_ms", ctypes.c_double), ("acc", ctypes.c_uint64 * 4),
                ("wall_ms", ctypes.c_double)]


class _CLatency(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint64), ("min_cycles", ctypes.c_double),
                ("avg_cycles", ctypes.c_double), ("max_cycles", ctypes.c_double),
                ("p50_cycles", ctypes.c_double), ("p99_cycles", ctypes.c_double)]


class _CDump(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in (
        "tickets", "heads", "cached", "size_infos", "counters", "size_id", "chunk_id",
        "is_head", "chunk_enc", "sets", "bits", "nibbles")]


_vp, _u32, _i64, _int = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int64, ctypes.c_int
_SIGS = {
    "ha_init_c": (_int, [ctypes.POINTER(_COpts)]),
    "ha_shutdown_c": (_int, []),
    "ha_extfrag_c": (ctypes.c_double, [_int]),
    "ha_stats_c": (_int, [ctypes.POINTER(_CStats)]),
    "ha_status_c": (_u32, []),
    "ha_clear_status_c": (_int, []),
    "ha_set_wait_limit_c": (_int, [_u32]),
    "ha_dump_state_c": (_int, [ctypes.POINTER(_CDump)]),
    "ha_l2_persist_c": (_int, [_vp]),
    "ha_debug_set_head_lock_c": (_int, [_u32, _u32]),
    "ha_set_hash_scale_c": (_int, [_u32]),
    "ha_set_heads_c": (_int, [_u32]),
    "ha_set_surge_c": (_int, [ctypes.c_int]),
    "ha_close_surges_c": (_int, [ctypes.c_void_p]),
    "ha_set_growth_c": (_int, [ctypes.c_uint64]),
    "ha_grow_c": (_int, [ctypes.c_uint64, _vp, ctypes.POINTER(ctypes.c_uint64)]),
    "ha_trim_c": (_int, [ctypes.c_uint64, _vp, ctypes.POINTER(ctypes.c_uint64)]),
    "ha_serve_run_c": (_int, [ctypes.POINTER(_CServeCfg), ctypes.POINTER(_CServeResult), _vp]),
    "ha_graph_build_c": (_int, [_u32, _u32, _vp, _u32, _vp, _vp, _vp, _vp]),
    "ha_graph_gather_c": (_int, [_u32, _vp, _vp, _vp, _vp, _vp]),
    "ha_malloc_batch_c": (_int, [_vp, _u32, _u32, _vp, _int, _vp]),
    "ha_free_batch_c": (_int, [_vp, _u32, _u32, _vp]),
    "ha_throughput_c": (_int, [_vp, _u32, _u32, _u32, _u32, _u32, _vp, _vp]),
    "ha_throughput_host_c": (_int, [_vp, _vp, _u32, _u32, _u32, _u32, _u32, _vp, _vp, _vp]),
    "ha_throughput_host_ex_c": (_int, [_vp, _vp, _u32, _u32, _u32, _u32, _u32, _vp, _vp, _u32,
                                       _vp]),
    "ha_cuda_throughput_c": (_int, [_vp, _u32, _u32, _u32, _u32, _u32, _vp, _vp]),
    "ha_trace_c": (_int, [_vp, _i64, _vp, _vp]),
    "ha_phase_round_c": (_int, [_int, _u32, _u32, _u32, _u32, _u32, _vp, _u32, _vp, _vp, _vp,
                                _vp]),
    "ha_phase_run_c": (_int, [_u32, _u32, _u32, _u32, _u32, _u32, ctypes.c_uint64, _u32, _vp,
                              _u32, _vp, _vp, _vp, ctypes.POINTER(_CPhaseResult), _vp]),
    "ha_phase_ref_step_c": (_int, [_u32, _u32, _u32, _u32, _vp, _u32, _u32, _vp, _vp, _vp,
                                   _vp, _int, _vp]),
    "ha_phase_ref_run_c": (_int, [_u32, _u32, _u32, _u32, _vp, _u32, _u32, _vp, _vp, _vp, _vp,
                                  ctypes.POINTER(_CPhaseRefResult), _vp]),
    "ha_atomic_peak_c": (_int, [_vp, _u32, _u32, _u32, _int, _vp]),
    "ha_phase_ref_latency_c": (_int, [_u32, _u32, _u32, _u32, _vp, _u32, _u32, _vp, _vp, _vp,
                                      _vp, _vp, _vp]),
    "ha_atomic_peak_strided_c": (_int, [_vp, _u32, _u32, _u32, _u32, _int, _vp]),
    "ha_grid_insert_c": (_int, [_u32, _u32, _vp, _vp, _vp, _vp, _vp]),
    "ha_grid_check_c": (_int, [_u32, _vp, _vp, _vp, _vp]),
    "ha_grid_free_c": (_int, [_u32, _vp, _int, _vp]),
    "ha_strings_alloc_c": (_int, [_u32, _vp, _vp, _vp, _vp]),
    "ha_strings_concat_c": (_int, [_u32, _vp, _vp, _vp, _vp, _vp]),
    "ha_strings_free_c": (_int, [_u32, _vp, _vp]),
    "ha_strings_check_c": (_int, [_u32, _vp, _vp, _vp, _vp, _vp]),
}

_lib = None


def library_path() -> str:
    return SO_PATH


def load():
    """Loads libhalloc_b200.so (raises HallocError when it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(SO_PATH):
            raise HallocError(f"{SO_PATH} is missing: build it with python -m halloc_b200.build")
        lib = ctypes.CDLL(SO_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def _check(rc: int, what: str):
    if rc != HA_OK:
        raise HallocError(f"{what}: {_ERR.get(rc, rc)}")


def _addr(x) -> int:
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    raise TypeError(f"cannot take the address of {type(x)}")


def _stream(s) -> int:
    if s is None:
        return 0
    if isinstance(s, int):
        return s
    return s.cuda_stream


# ---- init / shutdown / statistics ------------------------------------------

def init(opts: HallocOpts | None = None) -> None:
    """ha_init on the current device (error if already initialised)."""
    o = opts or HallocOpts()
    c = _COpts(o.memory, o.halloc_fraction, o.busy_fraction, o.roomy_fraction,
               o.sparse_fraction, o.sb_sz_sh)
    _check(load().ha_init_c(ctypes.byref(c)), "ha_init_c")


def shutdown() -> None:
    _check(load().ha_shutdown_c(), "ha_shutdown_c")


def extfrag(ideal: bool = False) -> float:
    v = load().ha_extfrag_c(1 if ideal else 0)
    if v < 0:
        raise HallocError("ha_extfrag_c failed")
    return v


def stats() -> dict:
    s = _CStats()
    _check(load().ha_stats_c(ctypes.byref(s)), "ha_stats_c")
    arrays = ("head", "cached", "surge_level")
    d = {f: getattr(s, f) for f, _ in _CStats._fields_ if f not in arrays}
    for f in arrays:
        d[f] = list(getattr(s, f))
    return d


def status() -> int:
    v = load().ha_status_c()
    if v == 0xFFFFFFFF:
        raise HallocError("ha_status_c failed")
    return v


def clear_status() -> None:
    _check(load().ha_clear_status_c(), "ha_clear_status_c")


def set_wait_limit(microseconds: int) -> None:
    _check(load().ha_set_wait_limit_c(microseconds), "ha_set_wait_limit_c")


def dump_state() -> dict:
    """Full device state as numpy arrays (see ha_dump_state_c)."""
    st = stats()
    n, sb = st["nsbs"], st["sb_sz"]
    nw = (n + 31) // 32
    arrs = {
        "tickets": np.zeros(NSIZES, np.uint32), "heads": np.zeros(NSIZES, np.uint32),
        "cached": np.zeros(NSIZES, np.uint32), "size_infos": np.zeros(NSIZES * 8, np.uint32),
        "counters": np.zeros(n, np.uint32), "size_id": np.zeros(n, np.uint32),
        "chunk_id": np.zeros(n, np.uint32), "is_head": np.zeros(n, np.uint32),
        "chunk_enc": np.zeros(n, np.uint32), "sets": np.zeros(NSETS * nw, np.uint32),
        "bits": np.zeros(n * (sb // 512), np.uint32), "nibbles": np.zeros(n * (sb // 128), np.uint32),
    }
    d = _CDump(**{k: a.ctypes.data for k, a in arrs.items()})
    _check(load().ha_dump_state_c(ctypes.byref(d)), "ha_dump_state_c")
    arrs["size_infos"] = arrs["size_infos"].reshape(NSIZES, 8)
    arrs["sets"] = arrs["sets"].reshape(NSETS, nw)
    arrs["bits"] = arrs["bits"].reshape(n, sb // 512)
    arrs["nibbles"] = arrs["nibbles"].reshape(n, sb // 128)
    arrs["pool_base"] = st["pool_base"]
    arrs["nsbs"] = n
    arrs["sb_sz"] = sb
    return arrs


def set_hash_scale(percent: int) -> None:
    """Hash-step scale for the next init (100 = the reference's rule)."""
    _check(load().ha_set_hash_scale_c(percent), "ha_set_hash_scale_c")


def set_heads(nheads: int) -> None:
    """Head slabs per size for the next init (1 = the reference policy)."""
    _check(load().ha_set_heads_c(nheads), "ha_set_heads_c")


def set_surge(on) -> None:
    """Surge head sets for the next init (see ha_set_surge_c): True, False, or
    None for the environment's choice (HALLOC_SURGE, on by default)."""
    _check(load().ha_set_surge_c(-1 if on is None else (1 if on else 0)), "ha_set_surge_c")


def close_surges(stream=None) -> None:
    """Closes every size's surge head sets (see ha_close_surges_c)."""
    _check(load().ha_close_surges_c(_stream(stream)), "ha_close_surges_c")


def debug_set_head_lock(size_id: int, held: bool) -> None:
    """Failure-detection test hook (see ha_debug_set_head_lock_c)."""
    _check(load().ha_debug_set_head_lock_c(size_id, 1 if held else 0),
           "ha_debug_set_head_lock_c")


def l2_persist(stream=None) -> None:
    _check(load().ha_l2_persist_c(_stream(stream)), "ha_l2_persist_c")


# ---- batch entry points ------------------------------------------------------

def malloc_batch(sizes, nthreads: int, nallocs: int, ptrs, tag: bool = False,
                 stream=None) -> None:
    _check(load().ha_malloc_batch_c(_addr(sizes), nthreads, nallocs, _addr(ptrs),
                                    1 if tag else 0, _stream(stream)), "ha_malloc_batch_c")


def free_batch(ptrs, nthreads: int, nallocs: int, stream=None) -> None:
    _check(load().ha_free_batch_c(_addr(ptrs), nthreads, nallocs, _stream(stream)),
           "ha_free_batch_c")


def throughput(out, nthreads: int, nbytes: int = 16, block: int = 128, nallocs: int = 1,
               niters: int = 1, sizes=None, stream=None) -> None:
    _check(load().ha_throughput_c(_addr(sizes), nbytes, nthreads, block, nallocs, niters,
                                  _addr(out), _stream(stream)), "ha_throughput_c")


def cuda_throughput(out, nthreads: int, nbytes: int = 16, block: int = 128, nallocs: int = 1,
                    niters: int = 1, sizes=None, stream=None) -> None:
    _check(load().ha_cuda_throughput_c(_addr(sizes), nbytes, nthreads, block, nallocs, niters,
                                       _addr(out), _stream(stream)), "ha_cuda_throughput_c")


XFER_AUTO, XFER_COPY, XFER_MAPPED = 0, 1, 2


def _load_pyfast():
    """The CPython binding of the host-buffer loop (csrc/ha_pyfast.c), or None
    where it was not built; both call ha_throughput_host_ex_c in
    libhalloc_b200.so."""
    try:
        from . import _pyfast
    except ImportError:
        return None
    return _pyfast


_pyfast = _load_pyfast()


def throughput_host(h_out: np.ndarray, d_out, nthreads: int, nbytes: int = 16,
                    block: int = 128, nallocs: int = 1, niters: int = 1, h_sizes=None,
                    d_sizes=None, stream=None, transfer: int = XFER_AUTO) -> None:
    """End-to-end form: host sizes in, host (checksum, nfail) out.  transfer:
    XFER_AUTO (mapped when both host buffers are pinned), XFER_COPY (copy
    engine, one cached CUDA graph) or XFER_MAPPED (the kernel reads the sizes
    and stores the totals through the pinned buffers).  Called through the
    CPython binding when it is built (about 4 us less per call than ctypes)."""
    args = (_addr(h_sizes), _addr(d_sizes), nbytes, nthreads, block, nallocs, niters,
            _addr(d_out), _addr(h_out), transfer, _stream(stream))
    if _pyfast is not None:
        rc = _pyfast.throughput_host(*args)
    else:
        rc = load().ha_throughput_host_ex_c(*args)
    _check(rc, "ha_throughput_host_ex_c")


def phase_round(kind: int, nthreads: int, nslots: int, seed: int, round_id: int, thr: int,
                slots, slot_sz, acc, size_set=None, nsizes: int = 0, stream=None) -> None:
    """One allocation (kind 0) or free (kind 1) round of the phase workload."""
    _check(load().ha_phase_round_c(kind, nthreads, nslots, seed, round_id, thr,
                                   _addr(size_set), nsizes, _addr(slots), _addr(slot_sz),
                                   _addr(acc), _stream(stream)), "ha_phase_round_c")


PHASE_ACC = ("filled", "failed", "written_sum", "read_sum", "mallocs", "frees")


def phase_run(nthreads: int, nslots: int, seed: int, periods: int, thr_alloc: int,
              thr_free: int, target_filled: int, size_set, nsizes: int, slots, slot_sz, acc,
              max_rounds: int = 64, stream=None) -> dict:
    """The whole phase workload (ha_phase_run_c); device buffers: size_set
    (nsizes u32), slots (nslots*nthreads pointers, all NULL), slot_sz
    (nslots*nthreads u32), acc (6 u64)."""
    r = _CPhaseResult()
    _check(load().ha_phase_run_c(nthreads, nslots, seed, periods, thr_alloc, thr_free,
                                 target_filled, max_rounds, _addr(size_set), nsizes,
                                 _addr(slots), _addr(slot_sz), _addr(acc), ctypes.byref(r),
                                 _stream(stream)), "ha_phase_run_c")
    out = {"alloc_rounds": r.alloc_rounds, "free_rounds": r.free_rounds,
           "kernel_ms": r.kernel_ms, "filled": r.filled}
    out.update(dict(zip(PHASE_ACC, list(r.acc))))
    return out


PHASE_REF_ACC = ("mallocs", "frees", "failed", "bytes")


def _probs(probs) -> ctypes.Array:
    p = (ctypes.c_float * 4)(*[float(x) for x in probs])
    if len(probs) != 4:
        raise HallocError("probs: four transition probabilities expected")
    return p


def phase_ref_step(nthreads: int, nallocs: int, itry: int, niters: int, probs, smin: int,
                   smax: int, states, slots, ctrs, acc, rest: bool = False,
                   stream=None) -> None:
    """One launch of the reference-form phase workload (ha_phase_ref_step_c);
    probs = (p00, p01, p10, p11) as in phase_ref_probabilities; device
    buffers: states (nthreads u32), slots (nallocs*nthreads pointers), ctrs
    (nthreads u32), acc (4 u64, accumulated)."""
    _check(load().ha_phase_ref_step_c(nthreads, nallocs, itry, niters, _probs(probs), smin,
                                      smax, _addr(states), _addr(slots), _addr(ctrs),
                                      _addr(acc), int(rest), _stream(stream)),
           "ha_phase_ref_step_c")


def phase_ref_run(nthreads: int, nallocs: int, ntries: int, niters: int, probs, smin: int,
                  smax: int, states, slots, ctrs, acc, stream=None) -> dict:
    """ntries launches then the final free (ha_phase_ref_run_c)."""
    r = _CPhaseRefResult()
    _check(load().ha_phase_ref_run_c(nthreads, nallocs, ntries, niters, _probs(probs), smin,
                                     smax, _addr(states), _addr(slots), _addr(ctrs),
                                     _addr(acc), ctypes.byref(r), _stream(stream)),
           "ha_phase_ref_run_c")
    out = {"kernel_ms": r.kernel_ms, "alloc_phase_ms": r.alloc_phase_ms,
           "free_phase_ms": r.free_phase_ms, "wall_ms": r.wall_ms}
    out.update(dict(zip(PHASE_REF_ACC, list(r.acc))))
    return out


def phase_ref_latency(nthreads: int, nallocs: int, ntries: int, niters: int, probs,
                      smin: int, smax: int, states, slots, ctrs, acc, stream=None) -> dict:
    """The reference's phase-latency test (ha_phase_ref_latency_c): per-call
    cycles of hamalloc and hafree over ntries tries, then the final free."""
    out = (_CLatency * 2)()
    _check(load().ha_phase_ref_latency_c(nthreads, nallocs, ntries, niters, _probs(probs),
                                         smin, smax, _addr(states), _addr(slots), _addr(ctrs),
                                         _addr(acc), ctypes.cast(out, ctypes.c_void_p),
                                         _stream(stream)), "ha_phase_ref_latency_c")
    f = [k for k, _ in _CLatency._fields_]
    return {"malloc": {k: getattr(out[0], k) for k in f},
            "free": {k: getattr(out[1], k) for k in f}}


def phase_ref_probabilities(alloc_fraction: float, free_fraction: float,
                            exec_fraction: float) -> tuple:
    """Transition probabilities (p00, p01, p10, p11) from the steady-state
    fractions f (after the allocation phase), F (after the free phase) and
    e (threads acting per phase), in float32 as halloc computes them
    (tst/common/common.cu:311-355); p[phase][holding]."""
    f32 = np.float32
    f, F, e = f32(alloc_fraction), f32(free_fraction), f32(exec_fraction)
    one, two = f32(1), f32(2)
    if e + f + F > 2 or e < abs(f - F):
        raise HallocError("phase_ref_probabilities: fractions out of range")
    p00 = (e + f - F) / (two * (one - F)) if F < 1 else one
    p01 = (e - f + F) / (two * F) if F > 0 else one
    p10 = (e - f + F) / (two * (one - f)) if f < 1 else one
    p11 = (e + f - F) / (two * f) if f > 0 else f32(0)
    return tuple(float(f32(x)) for x in (p00, p01, p10, p11))


def grid_insert(n: int, ncells: int, pts, grid, nfail, pre_nodes=None, stream=None) -> None:
    """grid-points sample: point i (pts: 3 float32 each) gets a 16-byte node,
    pushed onto its cell of the ncells^3 grid (ha_grid_insert_c)."""
    _check(load().ha_grid_insert_c(n, ncells, _addr(pts), _addr(grid), _addr(pre_nodes),
                                   _addr(nfail), _stream(stream)), "ha_grid_insert_c")


def grid_check(ncells: int, grid, count, hsum, stream=None) -> None:
    """Per cell: points and sum of mix32(point index) (ha_grid_check_c)."""
    _check(load().ha_grid_check_c(ncells, _addr(grid), _addr(count), _addr(hsum),
                                  _stream(stream)), "ha_grid_check_c")


def grid_free(ncells: int, grid, pre_nodes: bool = False, stream=None) -> None:
    _check(load().ha_grid_free_c(ncells, _addr(grid), int(pre_nodes), _stream(stream)),
           "ha_grid_free_c")


def strings_alloc(n: int, lens, strs, nfail, stream=None) -> None:
    """add-strings sample: strs[i] = lens[i] spaces (ha_strings_alloc_c)."""
    _check(load().ha_strings_alloc_c(n, _addr(lens), _addr(strs), _addr(nfail),
                                     _stream(stream)), "ha_strings_alloc_c")


def strings_concat(n: int, c, a, b, nfail, stream=None) -> None:
    _check(load().ha_strings_concat_c(n, _addr(c), _addr(a), _addr(b), _addr(nfail),
                                      _stream(stream)), "ha_strings_concat_c")


def strings_free(n: int, strs, stream=None) -> None:
    _check(load().ha_strings_free_c(n, _addr(strs), _stream(stream)), "ha_strings_free_c")


def strings_check(n: int, c, la, lb, bad, stream=None) -> None:
    _check(load().ha_strings_check_c(n, _addr(c), _addr(la), _addr(lb), _addr(bad),
                                     _stream(stream)), "ha_strings_check_c")


def set_growth(initial_bytes: int) -> None:
    """Applied by the next init on this process: 0 (default) backs the whole
    slab pool at init; otherwise only initial_bytes, the rest on demand
    (grow) -- ha_set_growth_c."""
    _check(load().ha_set_growth_c(initial_bytes), "ha_set_growth_c")


def grow(nbytes: int, stream=None) -> int:
    """Backs at least nbytes more of the slab pool; returns the bytes added
    (0 when the pool is already fully backed) -- ha_grow_c."""
    added = ctypes.c_uint64(0)
    rc = load().ha_grow_c(nbytes, _stream(stream), ctypes.byref(added))
    if rc == HA_ERANGE:
        return 0
    _check(rc, "ha_grow_c")
    return added.value


def trim(max_bytes: int = 1 << 62, stream=None) -> int:
    """Returns the device memory of wholly free units, up to max_bytes;
    returns the bytes released -- ha_trim_c."""
    released = ctypes.c_uint64(0)
    _check(load().ha_trim_c(max_bytes, _stream(stream), ctypes.byref(released)), "ha_trim_c")
    return released.value


def graph_build(n: int, seed: int, cdf, ncdf: int, arr, deg, acc, stream=None) -> None:
    """Random-graph build with doubling neighbour arrays (ha_graph_build_c)."""
    _check(load().ha_graph_build_c(n, seed, _addr(cdf), ncdf, _addr(arr), _addr(deg),
                                   _addr(acc), _stream(stream)), "ha_graph_build_c")


def graph_gather(n: int, arr, deg, offsets, cols, stream=None) -> None:
    """CSR gather of the graph, freeing every neighbour array."""
    _check(load().ha_graph_gather_c(n, _addr(arr), _addr(deg), _addr(offsets), _addr(cols),
                                    _stream(stream)), "ha_graph_gather_c")


def serve_run(results, njobs: int, lam: float, seed: int = 1, occupancy_limit: float = 0.9,
              mean_life: float = 50.0, block_bytes: int = 256, min_len: int = 64,
              max_len: int = 2 << 20, grow_min: int = 1, grow_max: int = 32,
              cta_threads: int = 256, ctas_per_sm: int = 1, job_ids=None,
              grow_bytes: int = 0, prereleased: bool = False, stream=None) -> dict:
    """Serving loop (ha_serve_run_c).  results: device buffer of 2*njobs
    uint64 (blocks, value sum per job id).  job_ids: optional host sequence
    of ids to release instead of 0..njobs-1.  The default launch, one block
    of 256 job slots per SM, serves 256-B jobs about twice as fast and with
    a several times lower allocation latency than filling every SM: beyond
    that, more slots only add warps contending for the size's head slab.
    grow_bytes: with a growing pool (set_growth), the kernel asks the host
    for that much more backed memory whenever a block cannot be had, and the
    job waits for it instead of failing.  prereleased: every job is handed
    over before the launch (a closed batch; arrival times are not used)."""
    ids = None
    if job_ids is not None:
        ids = np.ascontiguousarray(np.asarray(job_ids, dtype=np.uint32))
    cfg = _CServeCfg(njobs, seed, lam, occupancy_limit, mean_life, block_bytes, min_len,
                     max_len, grow_min, grow_max, cta_threads, ctas_per_sm,
                     ids.ctypes.data if ids is not None else None,
                     len(ids) if ids is not None else 0, _addr(results), grow_bytes,
                     1 if prereleased else 0)
    r = _CServeResult()
    _check(load().ha_serve_run_c(ctypes.byref(cfg), ctypes.byref(r), _stream(stream)),
           "ha_serve_run_c")
    out = {f: getattr(r, f) for f, _ in _CServeResult._fields_ if f != "hist"}
    out["hist"] = np.frombuffer(bytes(r.hist), dtype=np.uint64).copy()
    return out


def trace(ops, n: int, out, stream=None) -> None:
    _check(load().ha_trace_c(_addr(ops), n, _addr(out), _stream(stream)), "ha_trace_c")


def atomic_peak(buf, nwords: int, nthreads: int, reps: int, returning: bool,
                stream=None, stride: int = 1) -> None:
    """L2 atomic throughput probe (ha_atomic_peak_strided_c): buf holds
    nwords x stride 32-bit words."""
    _check(load().ha_atomic_peak_strided_c(_addr(buf), nwords, stride, nthreads, reps,
                                           1 if returning else 0, _stream(stream)),
           "ha_atomic_peak_strided_c")
