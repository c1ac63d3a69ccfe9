"""Shared test helpers: golden fixtures, layout translation between the CUDA
implementation and the oracle, and block invariant checks."""
from __future__ import annotations

import contextlib
import hashlib
import json
import os

import numpy as np

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def load_golden_traces(fname: str = "traces.npz") -> list:
    z = np.load(os.path.join(GOLDEN, fname))
    index = json.loads(bytes(z["index"]).decode())
    cases = []
    for e in index:
        n = e["name"]
        rec = {k.split(".", 1)[1]: z[k] for k in z.files if k.startswith(n + ".")}
        rec.update(e)
        cases.append(rec)
    return cases


def load_size_tables() -> dict:
    with open(os.path.join(GOLDEN, "size_tables.json")) as f:
        return json.load(f)


def digest(a: np.ndarray) -> bytes:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest()


def chunk_bytes(enc: int) -> int:
    """decodes (3 or 1) << 16 | shift"""
    return (enc >> 16) << (enc & 0xFFFF)


def nibbles_to_chunk_layout(nib_dev: np.ndarray, chunk_enc: np.ndarray) -> np.ndarray:
    """The CUDA implementation indexes block-length nibbles by in-slab
    offset / 16; the reference by chunk index.  Returns the device nibbles in
    the reference's layout (same shape: slab size / 128 words per slab)."""
    out = np.zeros_like(nib_dev)
    nsbs, nwords = nib_dev.shape
    for sb in range(nsbs):
        words = nib_dev[sb]
        nz = np.nonzero(words)[0]
        if len(nz) == 0:
            continue
        cb = chunk_bytes(int(chunk_enc[sb]))
        if cb == 0:
            raise AssertionError(f"slab {sb} is free but has size nibbles")
        for w in nz:
            v = int(words[w])
            for k in range(8):
                n = (v >> (4 * k)) & 15
                if n:
                    u = int(w) * 8 + k          # offset / 16
                    c = -(-(u * 16) // cb)      # chunk index of the block start
                    out[sb, c // 8] |= n << (4 * (c % 8))
    return out


def device_state(dump: dict) -> oracle.State:
    """A device dump (halloc_b200.dump_state) as an oracle.State."""
    return oracle.State(
        dump["size_infos"], dump["tickets"], dump["heads"], dump["cached"],
        dump["counters"], dump["size_id"], dump["chunk_id"], dump["is_head"],
        dump["chunk_enc"], dump["sets"], dump["bits"],
        nibbles_to_chunk_layout(dump["nibbles"], dump["chunk_enc"]))


def ptrs_to_results(ops, ptrs: np.ndarray, pool_base: int, pool_bytes: int) -> np.ndarray:
    """Device trace output (raw pointers) in the oracle's result encoding:
    offset from slab 0, -1 for NULL, -2 for a block of the CUDA heap."""
    ops = np.asarray(ops)
    p = ptrs.astype(np.uint64)
    res = np.zeros(len(ops), np.int64)
    m = ops >= 0
    off = p - np.uint64(pool_base)
    inpool = (p >= np.uint64(pool_base)) & (off < np.uint64(pool_bytes))
    res[m & (p == 0)] = -1
    res[m & inpool & (p != 0)] = off[m & inpool & (p != 0)].astype(np.int64)
    res[m & ~inpool & (p != 0)] = -2
    return res


def normalise_large(res: np.ndarray) -> np.ndarray:
    """Maps every large-block handle (<= -2) to -2."""
    r = np.array(res, np.int64)
    r[r <= -2] = -2
    return r


def check_blocks(ptrs: np.ndarray, sizes: np.ndarray, pool_base: int, pool_bytes: int,
                 allow_null: bool = False) -> dict:
    """Invariants of a set of live blocks: non-NULL (unless allowed),
    pairwise non-overlapping, each at least `size` bytes, slab blocks inside
    the pool and aligned to 8 B (16 B for 16-B-chunk sizes)."""
    ptrs = np.asarray(ptrs, np.uint64).ravel()
    sizes = np.asarray(sizes, np.uint64).ravel()
    nn = ptrs != 0
    if not allow_null:
        assert nn.all(), f"{int((~nn).sum())} NULL blocks"
    p, s = ptrs[nn], sizes[nn]
    order = np.argsort(p, kind="stable")
    p, s = p[order], s[order]
    if len(p) > 1:
        gaps = p[1:] - p[:-1]
        bad = np.nonzero(gaps < np.maximum(s[:-1], 1))[0]
        assert len(bad) == 0, (f"{len(bad)} overlapping blocks, first at "
                               f"{hex(int(p[bad[0]]))} size {int(s[bad[0]])} next "
                               f"{hex(int(p[bad[0] + 1]))}")
    inpool = (p >= np.uint64(pool_base)) & (p - np.uint64(pool_base) < np.uint64(pool_bytes))
    small = s <= 3072
    assert inpool[small].all(), "small block outside the slab pool"
    assert (~inpool[~small]).all(), "large block inside the slab pool"
    assert (p[inpool] % 8 == 0).all(), "misaligned slab block"
    # blocks of the power-of-two classes (16-B and 256-B chunks) start on
    # 16-B boundaries; only the 24-B-chunk classes are 8-B aligned
    cls = class_bytes(s[inpool])
    pow2 = (cls & (cls - np.uint64(1))) == 0
    assert (p[inpool][pow2] % 16 == 0).all(), "power-of-two class block not 16-B aligned"
    return {"n": int(nn.sum()), "nnull": int((~nn).sum())}


CLASS_BYTES = np.array([16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768, 1024, 1536,
                        2048, 3072], np.uint64)


def class_bytes(sizes) -> np.ndarray:
    """Block size of the size class serving each request size (<= 3072 B)."""
    sizes = np.maximum(np.asarray(sizes, np.uint64), np.uint64(1))
    return CLASS_BYTES[np.searchsorted(CLASS_BYTES, sizes)]


def expected_slab_state(ptrs, sizes, pool_base: int, sb_sz: int, nsbs: int):
    """Per-slab used-chunk counts, bit arrays and size nibbles (chunk layout)
    that a set of live small blocks implies -- the host model of the state
    after quiescence.  Chunk size of each block from its size class."""
    ptrs = np.asarray(ptrs, np.uint64).ravel()
    sizes = np.asarray(sizes, np.int64).ravel()
    m = (ptrs != 0) & (sizes <= 3072)
    ptrs, sizes = ptrs[m], sizes[m]
    counts = np.zeros(nsbs, np.int64)
    bits = np.zeros((nsbs, sb_sz // 512), np.uint32)
    nib = np.zeros((nsbs, sb_sz // 128), np.uint32)
    cls = np.array([oracle.size_id(int(x)) for x in range(3073)])
    unit = 8 << (np.arange(16) // 2)
    block = np.where(np.arange(16) % 2 == 1, 3, 2) * unit
    cid = (np.arange(16) % 2) + np.where(np.arange(16) < 8, 0, 2)
    cb = np.where(cid % 2 == 1, 3, 2) * np.where(cid >= 2, 128, 8)
    ncib = block // cb
    off = (ptrs - np.uint64(pool_base)).astype(np.int64)
    sb = off // sb_sz
    inslab = off % sb_sz
    sid = cls[sizes]
    chunk = inslab // cb[sid]
    n = ncib[sid]
    np.add.at(counts, sb, n)
    np.bitwise_or.at(bits.reshape(-1), sb * bits.shape[1] + chunk // 32,
                     (((1 << n) - 1) << (chunk % 32)).astype(np.uint32))
    np.bitwise_or.at(nib.reshape(-1), sb * nib.shape[1] + chunk // 8,
                     (n << (4 * (chunk % 8))).astype(np.uint32))
    return counts, bits, nib


def oracle_opts_to_halloc(opts: dict) -> dict:
    """oracle option names -> HallocOpts field names"""
    names = {"busy": "busy_fraction", "roomy": "roomy_fraction", "sparse": "sparse_fraction"}
    return {names.get(k, k): v for k, v in opts.items()}


def plain_checksum(nthreads: int, per_thread: int) -> int:
    """Sum of the words {t^0, t^1, t^2, t^3} over threads t, times the blocks
    each thread writes."""
    t = np.arange(nthreads, dtype=np.int64)
    return int(per_thread * (4 * (t - t % 4) + 6).sum())


@contextlib.contextmanager
def allocator(**opts):
    """Initialises the allocator for a test and shuts it down afterwards."""
    import halloc_b200 as H
    H.init(H.HallocOpts(**opts))
    try:
        yield H
    finally:
        H.shutdown()


def assert_free_count(H) -> dict:
    """The free set's own count of its slabs (kept by the set operations)
    equals the slabs its bits hold, counted by the statistics kernel: to be
    called when no kernel runs."""
    st = H.stats()
    assert st["free_count"] == st["free_slabs"], (st["free_count"], st["free_slabs"])
    return st
