"""Oracle for halloc-b200: test infrastructure only.

Two host libraries, both loaded through ctypes:

* ``Model``     -- ``oracle/_build/libhamodel.so``: the C restatement of
  halloc 0.11's small-block policy (``oracle/ha_model.c``).
* ``Reference`` -- ``oracle/_ref/libhalloc_refhost.so``: the reference
  allocator's own sources (src/halloc.cu and the headers it includes)
  compiled unchanged as host C++ (``oracle/refhost``, ``oracle/Makefile``).
  Present only where the reference tree was available at build time.
* ``ref_phase_draws`` -- ``oracle/_ref/libphase_refdraws.so``: the
  decisions and size draws of the reference's phase-throughput test, from
  its own harness header (tst/common/common.h), to pin ``oracle/phase.py``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may use this package; the product path never imports it.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, fields

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MODEL_SO = os.path.join(HERE, "_build", "libhamodel.so")
REF_SO = os.path.join(HERE, "_ref", "libhalloc_refhost.so")
REF_DRAWS_SO = os.path.join(HERE, "_ref", "libphase_refdraws.so")

NSIZES = 16
NSETS = 1 + 4 + 2 * NSIZES  # free, sparse[4], roomy[16], busy[16]
NONE = 0xFFFFFFFF

_vp, _u32, _u64, _i64, _int, _dbl = (ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64,
                                     ctypes.c_int64, ctypes.c_int, ctypes.c_double)
_pu64 = ctypes.POINTER(_u64)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_vp)


@dataclass
class State:
    """Every piece of allocator state, in the reference's own encoding."""

    size_infos: np.ndarray  # (16, 8): nchunks, chunk_sz(enc), chunk_id, ncib, sparse, step, roomy, busy
    tickets: np.ndarray     # (16,)
    heads: np.ndarray       # (16,)
    cached: np.ndarray      # (16,)
    counters: np.ndarray    # (nsbs,) packed counter words
    size_id: np.ndarray     # (nsbs,) slab descriptors
    chunk_id: np.ndarray
    is_head: np.ndarray
    chunk_sz: np.ndarray    # encoded chunk size, 0 for a free slab
    sets: np.ndarray        # (NSETS, ceil(nsbs/32))
    bits: np.ndarray        # (nsbs, bit_words)
    nibbles: np.ndarray     # (nsbs, nib_words)

    def diff(self, other: "State") -> list:
        out = []
        for f in fields(self):
            a, b = getattr(self, f.name), getattr(other, f.name)
            if a.shape != b.shape:
                out.append(f"{f.name}: shape {a.shape} != {b.shape}")
            elif not np.array_equal(a, b):
                idx = np.argwhere(a != b)[:4].tolist()
                out.append(f"{f.name}: differs at {idx}")
        return out


# signatures shared by both libraries, without the model's leading handle
_ACCESSORS = {
    "malloc": (_i64, [_u64]),
    "free": (None, [_i64]),
    "run_ops": (None, [_vp, _i64, _vp]),
    "get_size_infos": (None, [_vp]),
    "get_tickets": (None, [_vp]),
    "get_heads": (None, [_vp, _vp]),
    "get_slabs": (None, [_vp] * 5),
    "get_sets": (None, [_vp, _u32]),
    "get_bits": (None, [_u32, _vp, _u32]),
    "get_alloc_sizes": (None, [_u32, _vp, _u32]),
}


def _bind(lib, prefix, lead):
    for name, (res, args) in _ACCESSORS.items():
        f = getattr(lib, prefix + name)
        f.restype = res
        f.argtypes = lead + args


class _Allocator:
    """Common replay / state interface of Model and Reference."""

    nsbs: int
    bit_words: int
    nib_words: int

    def _call(self, name, *args):  # pragma: no cover - overridden
        raise NotImplementedError

    def malloc(self, nbytes: int) -> int:
        return self._call("malloc", nbytes)

    def free(self, h: int) -> None:
        self._call("free", h)

    def run_ops(self, ops) -> np.ndarray:
        """op >= 0: malloc(op); op < 0: free the result of op -(op+1).
        Returns each op's result (offset, -1 NULL, <= -2 large, 0 for free)."""
        ops = np.ascontiguousarray(ops, dtype=np.int64)
        out = np.zeros(len(ops), dtype=np.int64)
        self._call("run_ops", _ptr(ops), len(ops), _ptr(out))
        return out

    def state(self) -> State:
        nsbs = self.nsbs
        si = np.zeros(NSIZES * 8, np.uint32)
        self._call("get_size_infos", _ptr(si))
        t = np.zeros(NSIZES, np.uint32)
        self._call("get_tickets", _ptr(t))
        h = np.zeros(NSIZES, np.uint32)
        c = np.zeros(NSIZES, np.uint32)
        self._call("get_heads", _ptr(h), _ptr(c))
        sl = [np.zeros(nsbs, np.uint32) for _ in range(5)]
        self._call("get_slabs", *[_ptr(a) for a in sl])
        nw = (nsbs + 31) // 32
        sets = np.zeros(NSETS * nw, np.uint32)
        self._call("get_sets", _ptr(sets), nw)
        bits = np.zeros((nsbs, self.bit_words), np.uint32)
        nib = np.zeros((nsbs, self.nib_words), np.uint32)
        for sb in range(nsbs):
            self._call("get_bits", sb, _ptr(bits[sb]), self.bit_words)
            self._call("get_alloc_sizes", sb, _ptr(nib[sb]), self.nib_words)
        return State(si.reshape(NSIZES, 8), t, h, c, *sl, sets.reshape(NSETS, nw),
                     bits, nib)


_libs: dict = {}


def model_lib():
    if "model" not in _libs:
        if not os.path.exists(MODEL_SO):
            raise FileNotFoundError(f"{MODEL_SO} missing: run make -C oracle model")
        lib = ctypes.CDLL(MODEL_SO)
        lib.ham_create.restype = _vp
        lib.ham_create.argtypes = [_u64, _dbl, _dbl, _dbl, _dbl, _int, _int]
        lib.ham_destroy.restype = None
        lib.ham_destroy.argtypes = [_vp]
        for n in ("nsbs", "nsizes", "bit_words", "nib_words"):
            f = getattr(lib, "ham_" + n)
            f.restype = _u32
            f.argtypes = [_vp]
        lib.ham_size_id.restype = _int
        lib.ham_size_id.argtypes = [_u64]
        lib.ham_plain_run.restype = _dbl
        lib.ham_plain_run.argtypes = [_u64, _int, _u32, _u32, _u32, _int, _pu64, _pu64]
        lib.hostmalloc_plain_run.restype = _dbl
        lib.hostmalloc_plain_run.argtypes = [_u32, _u32, _u32, _int, _pu64, _pu64]
        _bind(lib, "ham_", [_vp])
        _libs["model"] = lib
    return _libs["model"]


class Model(_Allocator):
    """One instance of the C restatement (oracle/ha_model.c)."""

    def __init__(self, memory=512 << 20, halloc_fraction=0.75, busy=0.835,
                 roomy=0.6, sparse=0.012, sb_sz_sh=22, ref_scan_whole_words=False):
        self.lib = model_lib()
        self.h = self.lib.ham_create(memory, halloc_fraction, busy, roomy, sparse,
                                     sb_sz_sh, int(bool(ref_scan_whole_words)))
        if not self.h:
            raise ValueError("invalid model options")
        self.sb_sz_sh = sb_sz_sh
        self.nsbs = self.lib.ham_nsbs(self.h)
        self.bit_words = self.lib.ham_bit_words(self.h)
        self.nib_words = self.lib.ham_nib_words(self.h)

    def _call(self, name, *args):
        return getattr(self.lib, "ham_" + name)(self.h, *args)

    def close(self):
        if getattr(self, "h", None):
            self.lib.ham_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def size_id(nbytes: int) -> int:
    """Size class of a request (-1 above 3072 B)."""
    return model_lib().ham_size_id(nbytes)


def reference_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    if "ref" not in _libs:
        lib = ctypes.CDLL(REF_SO)
        lib.ref_init.restype = _int
        lib.ref_init.argtypes = [_u64, _dbl, _dbl, _dbl, _dbl, _int]
        lib.ref_nsbs.restype = _u32
        lib.ref_nsizes.restype = _u32
        lib.ref_shutdown.restype = None
        lib.ref_plain_run.restype = _dbl
        lib.ref_plain_run.argtypes = [_u32, _u32, _u32, _int, _pu64, _pu64]
        _bind(lib, "ref_", [])
        _libs["ref"] = lib
    return _libs["ref"]


def ref_phase_draws(seeds: np.ndarray, probs, smin: int, smax: int, nallocs: int,
                    ntries: int, niters: int = 1):
    """Runs the reference's phase-test decisions (next_action, next_alloc_sz,
    drandom) for every thread and try, allocations left out.  Returns
    (ctr[ntries, n], sizes[ntries, nallocs, n], final generator states)."""
    if "draws" not in _libs:
        lib = ctypes.CDLL(REF_DRAWS_SO)
        lib.ref_phase_draws.restype = _int
        lib.ref_phase_draws.argtypes = [_vp, _u32, _vp, _u32, _u32, _u32, _u32, _u32, _vp,
                                        _vp, _vp]
        _libs["draws"] = lib
    seeds = np.ascontiguousarray(seeds, np.uint32)
    n = len(seeds)
    ctr = np.zeros((ntries, n), np.uint32)
    sz = np.zeros((ntries, nallocs, n), np.uint32)
    st = np.zeros(n, np.uint32)
    p = (ctypes.c_float * 4)(*[float(x) for x in probs])
    _libs["draws"].ref_phase_draws(_ptr(seeds), n, p, smin, smax, nallocs, ntries, niters,
                                   _ptr(ctr), _ptr(sz), _ptr(st))
    return ctr, sz, st


class Reference(_Allocator):
    """The reference allocator built for the host.  It keeps its state in
    process globals, so only one instance is live at a time."""

    def __init__(self, memory=512 << 20, halloc_fraction=0.75, busy=0.835,
                 roomy=0.6, sparse=0.012, sb_sz_sh=22):
        self.lib = ref_lib()
        n = self.lib.ref_init(memory, halloc_fraction, busy, roomy, sparse, sb_sz_sh)
        if n < 0:
            raise ValueError("configuration not representable by the reference")
        self.nsbs = n
        self.sb_sz_sh = sb_sz_sh
        self.bit_words = (1 << sb_sz_sh) // 512   # one bit per 16 B
        self.nib_words = (1 << sb_sz_sh) // 128   # one nibble per 16-B chunk

    def _call(self, name, *args):
        return getattr(self.lib, "ref_" + name)(*args)


def cpu_plain_run(kind: str, nthreads: int, niters: int, nbytes: int, nworkers: int,
                  memory: int = 512 << 20, sb_sz_sh: int = 22):
    """Times the plain workload (malloc, write 4 words, read back, free) on the
    host cores.  kind: 'reference' (the reference's own code, oracle/_ref,
    shared by all workers), 'port' (one model replica per worker) or 'glibc'.
    Returns (seconds, checksum, nfail)."""
    cs, nf = _u64(), _u64()
    if kind == "reference":
        lib = ref_lib()
        if lib.ref_init(memory, 0.75, 0.835, 0.6, 0.012, sb_sz_sh) < 0:
            raise ValueError("bad configuration")
        dt = lib.ref_plain_run(nthreads, niters, nbytes, nworkers, ctypes.byref(cs),
                               ctypes.byref(nf))
    elif kind == "port":
        dt = model_lib().ham_plain_run(memory, sb_sz_sh, nthreads, niters, nbytes,
                                       nworkers, ctypes.byref(cs), ctypes.byref(nf))
    elif kind == "glibc":
        dt = model_lib().hostmalloc_plain_run(nthreads, niters, nbytes, nworkers,
                                              ctypes.byref(cs), ctypes.byref(nf))
    else:
        raise ValueError(kind)
    return dt, cs.value, nf.value
