"""Where one warp's hamalloc/hafree time goes: the latency breakdown of the
private-throughput loop (hamalloc(16), 16-byte write and read-back, hafree)
run by a single warp, from the instrumented library
(libhalloc_b200_stamps.so, built with -DHA_STAMPS by halloc_b200/build.py).

    python -m halloc_b200.stamps [--nbytes 16] [--iters 10] [--reps 20]

Each lane reads the SM clock after every dependent round trip (the read
waits for the value the round trip returned), so the difference between
consecutive stamps is the time of one step of the chain.  Printed: mean
cycles per step and iteration, over all lanes and reps, with the L2 warm
(metadata resident) and after an L2 flush (a 256 MiB write before each run,
as the benchmark does between steps), and the loop's total time in the
instrumented and the normal library (what the stamps themselves cost).
This process loads only the instrumented library for the stamped runs and
the normal one in a child process for the comparison.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys

import numpy as np

from . import PKG, HallocOpts, _COpts

STAMPS_SO = os.path.join(PKG, "libhalloc_b200_stamps.so")
LANES, SLOTS = 32, 160
WORDS = 32 + 2 * LANES * SLOTS
NAMES = {1: "malloc_in", 2: "ticket+head", 3: "reservation", 4: "count", 5: "malloc_out",
         6: "slow_in", 7: "slow_out", 8: "free_in", 9: "nibble+descriptor", 10: "count_down",
         11: "free_out", 12: "payload_readback"}


def parse(words: np.ndarray, niters: int) -> dict:
    """Mean cycles of each step (a stamp and the one before it in the same
    lane) per iteration, over the lanes; the loop start is the first stamp."""
    words = words.astype(np.uint32)
    steps: dict = {}
    for lane in range(LANES):
        n = min(int(words[lane]), SLOTS)
        base = 32 + 2 * lane * SLOTS
        pts = words[base:base + 2 * n:2]
        clk = words[base + 1:base + 2 * n:2].astype(np.int64)
        for i in range(1, n):
            key = f"{NAMES.get(int(pts[i - 1]), pts[i - 1])} -> {NAMES.get(int(pts[i]), pts[i])}"
            steps.setdefault(key, []).append(int((clk[i] - clk[i - 1]) & 0xFFFFFFFF))
    return {k: {"mean_cycles": float(np.mean(v)), "per_iter": len(v) / LANES / niters}
            for k, v in steps.items()}


def run_stamped(nbytes: int, niters: int, reps: int, flush: bool) -> dict:
    import torch
    lib = ctypes.CDLL(STAMPS_SO)
    lib.ha_init_c.argtypes = [ctypes.POINTER(_COpts)]
    lib.ha_stamps_run_c.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p,
                                    ctypes.c_void_p]
    o = HallocOpts()
    copts = _COpts(o.memory, o.halloc_fraction, o.busy_fraction, o.roomy_fraction,
                   o.sparse_fraction, o.sb_sz_sh)
    torch.cuda.set_device(0)
    out = torch.zeros(WORDS, dtype=torch.int32, device="cuda")
    buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    if lib.ha_init_c(ctypes.byref(copts)) != 0:
        raise RuntimeError("ha_init_c failed in the instrumented library")
    try:
        acc: dict = {}
        total = []
        for r in range(reps + 2):
            if flush:
                buf.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rc = lib.ha_stamps_run_c(nbytes, niters, ctypes.c_void_p(out.data_ptr()),
                                     ctypes.c_void_p(stream.cuda_stream))
            e1.record(stream)
            e1.synchronize()
            if rc != 0:
                raise RuntimeError(f"ha_stamps_run_c: {rc}")
            if r < 2:
                continue  # first touches of the pool and the metadata
            total.append(e0.elapsed_time(e1) * 1e3)
            for k, v in parse(out.cpu().numpy().view(np.uint32), niters).items():
                acc.setdefault(k, []).append(v)
        steps = {k: {"mean_cycles": round(float(np.mean([x["mean_cycles"] for x in v])), 1),
                     "per_iter": round(float(np.mean([x["per_iter"] for x in v])), 3)}
                 for k, v in acc.items()}
        return {"steps": dict(sorted(steps.items(), key=lambda kv: -kv[1]["mean_cycles"]
                                     * kv[1]["per_iter"])),
                "loop_us_median": float(np.median(total))}
    finally:
        lib.ha_shutdown_c()


_PLAIN = """
import sys, numpy as np, torch
sys.path.insert(0, {root!r})
import halloc_b200 as H
torch.cuda.set_device(0)
H.init(H.HallocOpts())
out = torch.zeros(2, dtype=torch.int64, device="cuda")
buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
s = torch.cuda.current_stream()
res = {{}}
for flush in (False, True):
    t = []
    for r in range({reps} + 2):
        if flush:
            buf.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        H.throughput(out, 32, nbytes={nbytes}, block=32, nallocs=1, niters={niters})
        e1.record(s)
        e1.synchronize()
        if r >= 2:
            t.append(e0.elapsed_time(e1) * 1e3)
    res[flush] = float(np.median(t))
H.shutdown()
print("PLAIN", res[False], res[True])
"""


def run_plain(nbytes: int, niters: int, reps: int) -> tuple:
    root = os.path.dirname(PKG)
    p = subprocess.run([sys.executable, "-c", _PLAIN.format(root=root, reps=reps, nbytes=nbytes,
                                                             niters=niters)],
                       capture_output=True, text=True, timeout=600)
    for line in p.stdout.splitlines():
        if line.startswith("PLAIN"):
            a, b = line.split()[1:]
            return float(a), float(b)
    raise RuntimeError(p.stderr[-2000:])


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--nbytes", type=int, default=16)
    ap.add_argument("--iters", type=int, default=10)
    ap.add_argument("--reps", type=int, default=20)
    a = ap.parse_args()
    warm_plain, flushed_plain = run_plain(a.nbytes, a.iters, a.reps)
    out = {"workload": f"1 warp, {a.iters} x (hamalloc({a.nbytes}), 16-B write, read-back, "
                       "hafree), 512 MiB pool, default options",
           "warm": run_stamped(a.nbytes, a.iters, a.reps, False),
           "l2_flushed": run_stamped(a.nbytes, a.iters, a.reps, True),
           "normal_build_loop_us": {"warm": warm_plain, "l2_flushed": flushed_plain}}
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
