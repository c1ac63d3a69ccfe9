"""Generates the golden fixtures in this directory from the REFERENCE
allocator's own code (halloc 0.11 compiled for the host, oracle/_ref).

    make -C oracle ref && python tests/golden/make_golden.py [traces] [phase]

The reference tree is needed only here; the fixtures are committed so that
tests run where it is absent (e.g. the GPU box).

Fixtures:
* size_tables.json -- the size-class table (src/halloc.cu:363-394) for a
  grid of slab sizes and thresholds.
* traces.npz -- serial hamalloc/hafree traces: for each case its options,
  the op list (op >= 0: malloc(op); op < 0: free the result of op
  -(op+1)), every result (byte offset from slab 0, -1 NULL, <= -2 large)
  and the final allocator state (tickets, heads, cached heads, packed slab
  counters, slab descriptors, slab sets, and SHA-256 digests of the bit
  arrays and size nibbles).
* phase_draws.npz -- the reference's phase-throughput decisions
  (tst/common/common.h next_action / next_alloc_sz / drandom, run by
  oracle/_ref/libphase_refdraws.so): for each case its parameters, the
  initial generator states, every thread's block count and live block
  sizes after every try, and the final generator states.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from tests.trace_gen import make_trace  # noqa: E402

SMALL = [16, 24, 32, 48, 64, 96, 128, 192, 256]
ALL = SMALL + [384, 512, 768, 1024, 1536, 2048, 3072]

# (name, options, trace generator arguments)
CASES = [
    ("plain16", dict(memory=512 << 20), dict(n=3000, sizes=[16], pfree=0.45, seed=1)),
    ("first16_nofree", dict(memory=512 << 20), dict(n=600, sizes=[16], pfree=0.0, seed=2)),
    ("mixed_small", dict(memory=512 << 20), dict(n=4000, sizes=SMALL, pfree=0.4, seed=3)),
    ("mixed_all", dict(memory=256 << 20, sb_sz_sh=21), dict(n=4000, sizes=ALL + [4096, 9000],
                                                          pfree=0.35, seed=4)),
    ("fill_busy", dict(memory=64 << 20, halloc_fraction=0.5, sb_sz_sh=20),
     dict(n=20000, sizes=[3072, 2048], pfree=0.05, seed=5)),
    ("recycle", dict(memory=128 << 20, halloc_fraction=0.5, sb_sz_sh=20, busy=0.745,
                     sparse=0.0125),
     dict(n=15000, sizes=[256, 384, 512, 768], pfree=0.3, seed=6, drain=0.95, tail=3000)),
    # 48 slabs: the reference never hands out slabs 32..47 (its set scan
    # covers whole 32-slab words only); checked against the model's
    # reference-compatible scan, not against the CUDA implementation
    ("h6_partial_word", dict(memory=64 << 20, sb_sz_sh=20),
     dict(n=20000, sizes=[3072, 1536], pfree=0.05, seed=7)),
]


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def state_record(st: oracle.State) -> dict:
    return {
        "tickets": st.tickets, "heads": st.heads, "cached": st.cached,
        "counters": st.counters, "size_id": st.size_id, "chunk_id": st.chunk_id,
        "is_head": st.is_head, "chunk_sz": st.chunk_sz, "sets": st.sets,
        "bits_sha": np.frombuffer(bytes.fromhex(digest(st.bits)), np.uint8),
        "nibbles_sha": np.frombuffer(bytes.fromhex(digest(st.nibbles)), np.uint8),
    }


def size_tables() -> dict:
    out = {}
    for sh in (20, 21, 22, 23, 24):
        for busy, roomy, sparse in ((0.835, 0.6, 0.012), (0.745, 0.6, 0.0125),
                                    (0.91, 0.5, 0.0125)):
            mem = max(512 << 20, 8 << sh)
            r = oracle.Reference(memory=mem, busy=busy, roomy=roomy, sparse=sparse,
                                 sb_sz_sh=sh)
            key = f"sh{sh}_b{busy}_r{roomy}_s{sparse}"
            out[key] = {"sb_sz_sh": sh, "busy": busy, "roomy": roomy, "sparse": sparse,
                        "memory": mem, "table": r.state().size_infos.tolist()}
    return out


# (name, (f, F, e), smin, smax, nallocs, niters, group, seed); 2,048 threads,
# 8 tries each
PHASE_CASES = [
    ("readme_uniform", (0.95, 0.05, 0.91), 16, 256, 4, 1, 1, 1),
    ("readme_groups32", (0.95, 0.05, 0.91), 16, 256, 4, 1, 32, 2),
    ("fixed16_iters3", (0.95, 0.05, 0.91), 16, 16, 4, 3, 1, 3),
    ("skewed", (0.7, 0.2, 0.6), 16, 3072, 2, 2, 1, 4),
    ("always", (1.0, 0.0, 1.0), 24, 24, 1, 1, 1, 5),
]
PHASE_THREADS, PHASE_TRIES = 2048, 8


def phase_draws() -> None:
    from halloc_b200.workloads import group_seeds
    from halloc_b200 import phase_ref_probabilities
    arrays, index = {}, []
    for name, fr, smin, smax, nallocs, niters, group, seed in PHASE_CASES:
        probs = phase_ref_probabilities(*fr)
        seeds = group_seeds(PHASE_THREADS, group, seed)
        ctr, sz, st = oracle.ref_phase_draws(seeds, probs, smin, smax, nallocs, PHASE_TRIES,
                                             niters)
        index.append({"name": name, "fractions": fr, "probs": probs, "smin": smin,
                      "smax": smax, "nallocs": nallocs, "niters": niters, "group": group,
                      "seed": seed, "ntries": PHASE_TRIES})
        arrays[f"{name}.seeds"] = seeds
        arrays[f"{name}.ctr"] = ctr.astype(np.uint8)
        arrays[f"{name}.sizes"] = sz.astype(np.uint16)
        arrays[f"{name}.states"] = st
    arrays["index"] = np.frombuffer(json.dumps(index).encode(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "phase_draws.npz"), **arrays)


def main():
    if not oracle.reference_available():
        sys.exit("oracle/_ref/libhalloc_refhost.so missing: run make -C oracle ref")
    what = set(sys.argv[1:]) or {"traces", "phase"}
    if "phase" in what:
        phase_draws()
    if "traces" not in what:
        return
    with open(os.path.join(HERE, "size_tables.json"), "w") as f:
        json.dump(size_tables(), f, indent=0)
    arrays = {}
    index = []
    for name, opts, targs in CASES:
        ops = make_trace(**targs)
        r = oracle.Reference(**opts)
        res = r.run_ops(ops)
        st = r.state()
        index.append({"name": name, "opts": opts, "nsbs": r.nsbs,
                      "ref_scan_whole_words": r.nsbs % 32 != 0,
                      "nnull": int((res[np.asarray(ops) >= 0] == -1).sum())})
        arrays[f"{name}.ops"] = np.asarray(ops, np.int64)
        arrays[f"{name}.res"] = res
        for k, v in state_record(st).items():
            arrays[f"{name}.{k}"] = v
    arrays["index"] = np.frombuffer(json.dumps(index).encode(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "traces.npz"), **arrays)
    for e in index:
        print(e)


if __name__ == "__main__":
    main()
