"""Benchmark of halloc-b200: 16-byte malloc/free pairs per second.

Workload (the plain-throughput configuration): one kernel of 256 blocks x
128 threads (32,768 threads) over a 512 MiB pool with default options; each
thread runs 10 iterations of hamalloc(16), a 16-byte write of
{tid^0, tid^1, tid^2, tid^3}, a checksummed read-back and hafree.  A step is
one such launch: 327,680 pairs.  The same loop with CUDA's in-kernel
malloc/free is timed beside it, and the reference allocator's own code
(built for the host) is timed on the host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun as independent replicas (one pool per GPU, no
collective on the data path; "weak" scaling): value = all pairs / max time.
Rank 0 prints one JSON line per secondary leg ({"leg": name, "result": ...};
N = 1 only), then the headline JSON line last, a few KB at most, carrying
each leg's one-number summary.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NTHREADS, BLOCK, NITERS, NALLOCS, NBYTES = 32768, 128, 10, 1, 16
POOL = 512 << 20
PAIRS_PER_STEP = NTHREADS * NITERS * NALLOCS
ATOMICS_PER_PAIR = 2  # one bit-array reservation + one release
# DRAM bytes (read + write) of one launch of the plain kernel, from an ncu
# capture of the current build (the bench cannot read DRAM counters itself)
PLAIN_DRAM_BYTES_PER_LAUNCH = 192000
METRIC = "16B malloc/free pairs/s"
WORKLOAD = ("plain: 256 x 128 threads, 10 x (hamalloc(16), 16-B write, read-back, hafree), "
            "512 MiB pool, default halloc_opts_t")


def plain_checksum(nthreads: int, per_thread: int) -> int:
    t = np.arange(nthreads, dtype=np.int64)
    return int(per_thread * (4 * (t - t % 4) + 6).sum())


def reduce_max_over_ranks(torch, values, world: int, device: str) -> list:
    """Element-wise max of per-rank values (the timing rule: the slowest
    replica sets the time); a plain list when there is one rank."""
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def replica_throughput(units_per_rank: float, world: int, max_seconds: float) -> float:
    """Whole-job throughput of independent replicas: every rank processed
    units_per_rank units; the job took as long as its slowest rank."""
    return units_per_rank * world / max_seconds


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


# ---- clocks during the timed region ---------------------------------------

class ClockSampler:
    """nvidia-smi samples (every 50 ms) of SM clock and throttle reasons;
    summary() keeps the rows inside a wall-clock window."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return self
        t0 = time.time()
        while time.time() - t0 < 5 and not self._rows():
            time.sleep(0.05)
        return self

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.proc = None

    def _rows(self):
        import datetime
        rows = []
        if not self.path or not os.path.exists(self.path):
            return rows
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 10 or not f[2].isdigit():
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except ValueError:
                continue
            rows.append((ts, f))
        return rows

    def summary(self, t0: float, t1: float, note: str) -> dict:
        rows = [f for ts, f in self._rows() if t0 - 0.06 <= ts <= t1 + 0.06]
        if self.path and os.path.exists(self.path):
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "window": note}
        reasons = sorted({n for r in rows for n, v in zip(self.REASONS, r[6:10])
                          if v == "Active"})
        return {"sm_mhz": statistics.median(int(r[2]) for r in rows),
                "sm_max_mhz": max(int(r[3]) for r in rows), "reasons": reasons,
                "samples": len(rows), "window": note}


# ---- our arm ----------------------------------------------------------------

def measure_atomic_peak(torch, H, stream) -> dict:
    """Distinct-address 32-bit atomic OR throughput over all SMs (the L2
    atomic roofline denominator), with and without a used return value:
    adjacent threads on adjacent words ("coalesced": L2 applies the eight
    of a 32-byte sector in one operation) and every thread on a sector of
    its own ("per_sector": what the allocator's hashed bit-array probes
    get)."""
    nsm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    nthreads = nsm * 2048
    buf = torch.zeros(nthreads * 8, dtype=torch.int32, device="cuda")
    reps = 256
    out = {}
    for stride, tag in ((1, ""), (8, "per_sector_")):
        for returning in (True, False):
            for _ in range(3):
                H.atomic_peak(buf, nthreads, nthreads, reps, returning, stream, stride=stride)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            best = 0.0
            for _ in range(5):
                e0.record(stream)
                H.atomic_peak(buf, nthreads, nthreads, reps, returning, stream, stride=stride)
                e1.record(stream)
                e1.synchronize()
                best = max(best, nthreads * reps / (e0.elapsed_time(e1) * 1e-3))
            out[tag + ("returning" if returning else "fire_and_forget")] = best / 1e9
    return out


def measure_lone_warp(torch, H, stream, flush) -> float:
    """Device time of the plain loop run by ONE warp (32 threads, the same
    10 iterations, L2 flushed before each run): the latency of one thread's
    chain of dependent round trips, with nothing to contend with."""
    import statistics as stats
    out = torch.zeros(2, dtype=torch.int64, device="cuda")
    times = []
    for r in range(13):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        H.throughput(out, 32, NBYTES, 32, NALLOCS, NITERS, stream=stream)
        e1.record(stream)
        e1.synchronize()
        if r >= 3:
            times.append(e0.elapsed_time(e1) * 1e3)
    return stats.median(times)


def measure_hot_word_rate(torch, H, stream) -> float:
    """Returning 32-bit atomics per second on ONE word, every thread of the
    device hitting it (same-address atomics serialise in their L2 slice)."""
    nsm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    nthreads = nsm * 2048
    buf = torch.zeros(nthreads, dtype=torch.int32, device="cuda")
    reps = 16
    H.atomic_peak(buf, 1, nthreads, reps, True, stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 0.0
    for _ in range(3):
        e0.record(stream)
        H.atomic_peak(buf, 1, nthreads, reps, True, stream)
        e1.record(stream)
        e1.synchronize()
        best = max(best, nthreads * reps / (e0.elapsed_time(e1) * 1e-3))
    return best


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    import halloc_b200 as H

    torch.cuda.set_device(local_rank)
    dev = torch.cuda.current_device()
    stream = torch.cuda.current_stream()
    H.init(H.HallocOpts(memory=POOL))
    H.l2_persist(stream)

    out = torch.zeros(2, dtype=torch.int64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    def step():
        H.throughput(out, NTHREADS, NBYTES, BLOCK, NALLOCS, NITERS, stream=stream)

    clocks = ClockSampler(dev).start()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    out.zero_()

    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t_begin = time.time()
    for e0, e1 in evs:
        flush.zero_()
        e0.record(stream)
        step()
        e1.record(stream)
    torch.cuda.synchronize()
    t_end = time.time()
    if world > 1:
        dist.barrier()
    # a timed region shorter than the sampling period gets the same load
    # (untimed, results discarded) for 0.4 s so the clock samples reflect it
    note = "timed region"
    if t_end - t_begin < 0.4 and not args.only_gpu:
        spare = torch.zeros(2, dtype=torch.int64, device="cuda")
        while time.time() - t_begin < 0.4:
            for _ in range(50):
                flush.zero_()
                H.throughput(spare, NTHREADS, NBYTES, BLOCK, NALLOCS, NITERS, stream=stream)
            torch.cuda.synchronize()
        note = "timed region + the same load, untimed, to 0.4 s"
    clocks.stop()
    clock_summary = clocks.summary(t_begin, time.time(), note)
    step_ms = [e0.elapsed_time(e1) for e0, e1 in evs]
    total_s = sum(step_ms) * 1e-3
    cs, nfail = out.cpu().tolist()
    want = plain_checksum(NTHREADS, NITERS * NALLOCS) * args.steps
    ok = (nfail == 0 and cs == want and H.status() == 0)

    # end to end through the C ABI from host memory (pinned): H2D of the
    # per-thread request sizes, kernel, D2H of (checksum, failures)
    h_sizes = torch.full((NTHREADS,), NBYTES, dtype=torch.int32).pin_memory()
    d_sizes = torch.empty(NTHREADS, dtype=torch.int32, device="cuda")
    h_out = torch.zeros(2, dtype=torch.int64).pin_memory()
    d_out = torch.zeros(2, dtype=torch.int64, device="cuda")

    # the call takes plain addresses, as a C caller would pass them
    h_out_p, h_sizes_p = h_out.data_ptr(), h_sizes.data_ptr()
    d_out_p, d_sizes_p, stream_p = d_out.data_ptr(), d_sizes.data_ptr(), stream.cuda_stream

    def e2e_run(transfer):
        def e2e_step():
            H.throughput_host(h_out_p, d_out_p, NTHREADS, NBYTES, BLOCK, NALLOCS, NITERS,
                              h_sizes=h_sizes_p, d_sizes=d_sizes_p, stream=stream_p,
                              transfer=transfer)

        for _ in range(args.warmup):
            e2e_step()
        secs = 0.0
        good = True
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            h_out.zero_()
            t0 = time.perf_counter()
            e2e_step()
            secs += time.perf_counter() - t0
            good &= (int(h_out[1]) == 0 and
                     int(h_out[0]) == plain_checksum(NTHREADS, NITERS * NALLOCS))
        return secs, good

    # the public call picks mapped transfers for pinned buffers; the copy
    # engine form is timed beside it
    e2e_s, e2e_ok = e2e_run(H.XFER_AUTO)
    e2e_copy_s, copy_ok = e2e_run(H.XFER_COPY)

    # max over ranks
    total_s, e2e_s, e2e_copy_s, bad = reduce_max_over_ranks(
        torch, [total_s, e2e_s, e2e_copy_s, 0.0 if ok and e2e_ok and copy_ok else 1.0], world,
        "cuda")

    res = {"step_ms": step_ms, "total_s": total_s, "e2e_s": e2e_s, "e2e_copy_s": e2e_copy_s,
           "ok": bad == 0.0, "clocks": clock_summary}
    if rank == 0 and not args.only_gpu:
        res["peak"] = measure_atomic_peak(torch, H, stream)
        res["hot_word_rate"] = measure_hot_word_rate(torch, H, stream)
        res["lone_warp_us"] = measure_lone_warp(torch, H, stream, flush)
    H.shutdown()
    return res


def run_cuda_malloc(torch, H, steps: int) -> dict:
    """CUDA's in-kernel malloc/free on the same loop, in a process of its
    own whose device heap is the whole pool size before any kernel runs, as
    halloc's CUDA-malloc wrapper sets it (tst/common/cuda-malloc-wrapper.h:
    10-12)."""
    from cuda.bindings import runtime as rt
    err, = rt.cudaDeviceSetLimit(rt.cudaLimit.cudaLimitMallocHeapSize, POOL)
    if err != rt.cudaError_t.cudaSuccess:
        return {"error": f"cudaDeviceSetLimit: {err}"}
    err, heap = rt.cudaDeviceGetLimit(rt.cudaLimit.cudaLimitMallocHeapSize)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    cout = torch.zeros(2, dtype=torch.int64, device="cuda")
    for _ in range(3):
        H.cuda_throughput(cout, NTHREADS, NBYTES, BLOCK, NALLOCS, NITERS, stream=stream)
    torch.cuda.synchronize()
    cout.zero_()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = 0.0
    for _ in range(steps):
        flush.zero_()
        e0.record(stream)
        H.cuda_throughput(cout, NTHREADS, NBYTES, BLOCK, NALLOCS, NITERS, stream=stream)
        e1.record(stream)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
    cs, nf = cout.cpu().tolist()
    return {"value": PAIRS_PER_STEP * steps / (ms * 1e-3), "unit": "pairs/s", "steps": steps,
            "failed_allocs": nf, "heap_bytes": int(heap),
            "ok": nf == 0 and cs == plain_checksum(NTHREADS, NITERS * NALLOCS) * steps}


def run_atomic_probe(torch, H) -> dict:
    """32-bit atom.or throughput against the number of distinct words all
    threads hit (1 word = every thread on one address)."""
    nsm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    nthreads = nsm * 2048
    buf = torch.zeros(nthreads * 8, dtype=torch.int32, device="cuda")
    out = {}
    cases = [(n, 1) for n in (1, 2, 18, 64, 1024, nthreads)] + [(1024, 8), (nthreads, 8)]
    for nwords, stride in cases:
        reps = 64 if nwords < 100 else 256
        for ret in (True, False):
            H.atomic_peak(buf, nwords, nthreads, reps, ret, stride=stride)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            H.atomic_peak(buf, nwords, nthreads, reps, ret, stride=stride)
            e1.record()
            e1.synchronize()
            key = (f"words={nwords} stride={stride} "
                   f"{'returning' if ret else 'fire_and_forget'}")
            out[key] = nthreads * reps / (e0.elapsed_time(e1) * 1e-3) / 1e9
    return {"unit": "G ops/s", "threads": nthreads, "results": out}


def run_leg(name: str, steps: int = 20) -> dict:
    """A secondary workload in a child process: its own CUDA context, so
    its pool and CUDA-heap sizes are set afresh."""
    try:
        p = subprocess.run([sys.executable, os.path.abspath(__file__), "--leg", name,
                            "--steps", str(steps)],
                           capture_output=True, text=True, timeout=900)
    except subprocess.TimeoutExpired:
        return {"error": "timed out"}
    for line in p.stdout.splitlines():
        if line.startswith("LEG "):
            return json.loads(line[4:])
    return {"error": (p.stderr or p.stdout)[-600:]}


def leg_main(args):
    import torch

    import halloc_b200 as H
    torch.cuda.set_device(0)
    if args.leg == "phase":
        out = run_phase(torch, H, 3, hbm_peak())
        tuned = run_phase(torch, H, 3, hbm_peak(), nheads=4)
        out["tuned_4_heads"] = {"value": tuned["value"], "ms_per_run": tuned["ms_per_run"],
                                "ok": tuned["ok"],
                                "note": "4 head slabs per size (ha_set_heads_c); addresses "
                                        "no longer follow the reference policy"}
        out["reference_form"] = run_phase_ref(torch, H)
        out["reference_form_latency"] = run_phase_ref_latency(torch, H)
    elif args.leg == "graph":
        out = run_graph(torch, H, 3)
    elif args.leg == "serve":
        out = run_serve(torch, H)
    elif args.leg == "atomics":
        out = run_atomic_probe(torch, H)
    elif args.leg == "samples":
        out = run_samples(torch, H, 5)
    elif args.leg == "halloc_programs":
        out = run_halloc_programs()
    elif args.leg == "cuda_malloc":
        out = run_cuda_malloc(torch, H, max(2, min(5, args.steps)))
    else:
        out = run_batched(torch, H, 3, not args.no_tune)
    print("LEG " + json.dumps(out), flush=True)


PHASE_SIZES = [16, 24, 32, 48, 64, 96, 128, 192, 256]
PHASE_THREADS, PHASE_SLOTS, PHASE_PERIODS, PHASE_POOL = 1 << 20, 4, 5, 1 << 30
THR95 = int(0.95 * 2**32)


def run_phase(torch, H, reps: int, hbm_peak_gbs: float | None, nheads: int = 1) -> dict:
    """Mixed-size phase workload: 1,048,576 threads x 4 slots, 1 GiB pool,
    sizes uniform over 16..256 B, 5 periods of (allocation rounds with p=0.95
    until 91 % of the slots are filled; a free round with p=0.95), then the
    rest freed; every block written with a hashed pattern and read back
    before it is freed.  nheads > 1 is the tuned multi-head variant."""
    H.set_heads(nheads)
    H.init(H.HallocOpts(memory=PHASE_POOL))
    H.set_heads(1)
    stream = torch.cuda.current_stream()
    H.l2_persist(stream)
    n = PHASE_THREADS
    size_set = torch.tensor(PHASE_SIZES, dtype=torch.int32, device="cuda")
    slots = torch.zeros(PHASE_SLOTS * n, dtype=torch.int64, device="cuda")
    slot_sz = torch.zeros(PHASE_SLOTS * n, dtype=torch.int32, device="cuda")
    acc = torch.zeros(6, dtype=torch.int64, device="cuda")
    target = int(0.91 * PHASE_SLOTS * n)
    runs = []
    for r in range(reps + 1):  # the first run is warm-up
        res = H.phase_run(n, PHASE_SLOTS, 0x5EED + r, PHASE_PERIODS, THR95, THR95, target,
                          size_set, len(PHASE_SIZES), slots, slot_sz, acc, stream=stream)
        if r:
            runs.append(res)
    ok = all(x["failed"] == 0 and x["written_sum"] == x["read_sum"] and
             x["mallocs"] == x["frees"] for x in runs) and H.status() == 0
    H.shutdown()
    ms = sum(x["kernel_ms"] for x in runs)
    pairs = sum(x["mallocs"] for x in runs)
    mean = sum(PHASE_SIZES) / len(PHASE_SIZES)
    gbs = 2 * pairs * mean / (ms * 1e-3) / 1e9
    out = {"metric": "mixed-size malloc/free pairs/s", "value": pairs / (ms * 1e-3),
           "unit": "pairs/s", "runs": reps, "ms_per_run": ms / reps,
           "pairs_per_run": pairs // reps, "rounds_per_run": runs[0]["alloc_rounds"] +
           runs[0]["free_rounds"], "ok": ok,
           "config": "1,048,576 threads x 4 slots, 1 GiB pool, sizes uniform "
                     f"{PHASE_SIZES}, 5 periods (p=0.95 alloc to 91 % slot occupancy, "
                     "p=0.95 free), hashed payload written and checksummed before free",
           "payload": {"achieved_gbs": gbs, "bytes_per_pair": 2 * mean,
                       "note": "written + read once; expected mean block size"}}
    if hbm_peak_gbs:
        out["payload"]["frac_of_hbm"] = gbs / hbm_peak_gbs
    return out


# The reference's own phase experiments (tst/exp/speed/exp-run.pl:9-101 with
# tst/exp/common.pl): -f0.95 -F0.05 -e0.91 -m512MiB -g5, "spree" = -i1 -t512,
# "private" = -i32 -t16; (name, threads, blocks per thread, smin, smax,
# published Kepler private / spree Mpairs/s with their file:line)
PHASE_REF_CASES = [
    ("mixed_8_256", 1 << 20, 1, 8, 256, (927.18, 795.18),
     "tst/exp/speed/exp-log-combi.csv:4"),
    ("single_16x4", 1 << 20, 4, 16, 16, (1401.70, 1220.15),
     "tst/exp/speed/exp-log-single.csv:2"),
    ("single_16x1", 1 << 20, 1, 16, 16, (1366.76, 940.35),
     "tst/exp/scaling/exp-log-thru.csv:47"),
    ("single_256x1", 1 << 20, 1, 256, 256, (190.58, 557.76),
     "tst/exp/scaling/exp-log-thru.csv:49"),
    # the scaling experiment at 1,024 and 32,768 threads (halloc timed these
    # per launch with the host clock, launch overhead included)
    ("scaling_16x1_1k", 1024, 1, 16, 16, (89.53, 15.43), "tst/exp/scaling/exp-log-thru.csv:17"),
    ("scaling_16x4_1k", 1024, 4, 16, 16, (118.87, 45.02), "tst/exp/scaling/exp-log-thru.csv:18"),
    ("scaling_256x1_1k", 1024, 1, 256, 256, (92.89, 15.51),
     "tst/exp/scaling/exp-log-thru.csv:19"),
    ("scaling_16x1_32k", 32768, 1, 16, 16, (1012.49, 347.03),
     "tst/exp/scaling/exp-log-thru.csv:32"),
    ("scaling_16x4_32k", 32768, 4, 16, 16, (1218.44, 753.21),
     "tst/exp/scaling/exp-log-thru.csv:33"),
    ("scaling_256x1_32k", 32768, 1, 256, 256, (621.78, 312.41),
     "tst/exp/scaling/exp-log-thru.csv:34"),
]


def run_phase_ref(torch, H) -> dict:
    """The phase workload in the reference's own form: per-thread generator
    states seeded per group of 32 threads, Markov transitions with
    p00 = p11 = 0.9526, p01 = p10 = 0.1, one launch per try, the counts
    checked against their balance and the pool left empty."""
    from halloc_b200.workloads import group_seeds
    probs = H.phase_ref_probabilities(0.95, 0.05, 0.91)
    out = {"config": "phase-throughput -f0.95 -F0.05 -e0.91 -m536870912 -g5, as the "
                     "reference's speed experiments run it; device time (CUDA events) "
                     "summed over the launches", "probs": probs}
    def one(n, nallocs, smin, smax, niters, ntries, nheads):
        H.set_heads(nheads)
        try:
            H.init(H.HallocOpts(memory=512 << 20))
        finally:
            H.set_heads(1)
        seeds = group_seeds(n, 32, 0x5EED)
        states = torch.tensor(seeds.view(np.int32), device="cuda")
        slots = torch.zeros(nallocs * n, dtype=torch.int64, device="cuda")
        ctrs = torch.zeros(n, dtype=torch.int32, device="cuda")
        acc = torch.zeros(4, dtype=torch.int64, device="cuda")
        H.phase_ref_run(n, nallocs, 4, niters, probs, smin, smax, states, slots, ctrs,
                        acc)  # warm-up
        states.copy_(torch.tensor(seeds.view(np.int32), device="cuda"))
        r = H.phase_ref_run(n, nallocs, ntries, niters, probs, smin, smax, states, slots,
                            ctrs, acc)
        ok = (r["failed"] == 0 and r["mallocs"] == r["frees"] and H.status() == 0 and
              H.stats()["used_chunks"] == 0)
        H.shutdown()
        return r, ok

    for name, n, nallocs, smin, smax, published, src in PHASE_REF_CASES:
        for form, niters, ntries in (("spree", 1, 512), ("private", 32, 16)):
            r, ok = one(n, nallocs, smin, smax, niters, ntries, 1)
            sec = r["kernel_ms"] * 1e-3
            # the reference's own count: 0.5 x threads x blocks x iterations x tries x e
            formula = 0.5 * n * nallocs * niters * ntries * 0.91
            r4, ok4 = one(n, nallocs, smin, smax, niters, ntries, 4)
            out[f"{name}_{form}"] = {
                "args": f"-n{n} -l{nallocs} -s{smin} -S{smax} -i{niters} -t{ntries}",
                "pairs_per_s": r["mallocs"] / sec,
                "pairs_per_s_reference_formula": formula / sec,
                "pairs_per_s_wall_per_launch": r["mallocs"] / (r["wall_ms"] * 1e-3),
                "mallocs": r["mallocs"], "ms": r["kernel_ms"], "ok": ok,
                "published_kepler_mpairs_s": published[0 if form == "private" else 1],
                "published_source": src,
                "tuned_4_heads": {"pairs_per_s": r4["mallocs"] / (r4["kernel_ms"] * 1e-3),
                                  "ok": ok4}}
    return out


# The reference's latency experiment (tst/exp/scaling/exp-run.pl:56-89):
# phase-latency -f0.95 -F0.05 -e0.91 -m512MiB -g5 -n<threads> -l1 -s<size>
# -i16 -t8; published Kepler malloc / free (min, avg, max) cycles from
# tst/exp/scaling/exp-log-lat.csv:2,3,42,43
PHASE_LAT_CASES = [
    (1, 16, ((2669, 3046.49, 5233), (1966, 2053.32, 2606)), "exp-log-lat.csv:2"),
    (1, 256, ((2664, 3020.17, 5285), (1970, 2051.83, 2578)), "exp-log-lat.csv:3"),
    (1 << 20, 16, ((2805, 3629.24, 14415), (2130, 2455.04, 5298)), "exp-log-lat.csv:42"),
    (1 << 20, 256, ((2683, 42801.76, 250025), (2002, 3734.92, 9445)), "exp-log-lat.csv:43"),
]


def run_phase_ref_latency(torch, H) -> dict:
    """Per-call hamalloc / hafree cycles in the reference's phase-latency
    experiment, beside the figures halloc published for Kepler."""
    from halloc_b200.workloads import group_seeds
    probs = H.phase_ref_probabilities(0.95, 0.05, 0.91)
    out = {"config": "phase-latency -f0.95 -F0.05 -e0.91 -m536870912 -g5 -l1 -i16 -t8; "
                     "clock64() around each call, SM cycles", "cases": []}
    for n, size, published, src in PHASE_LAT_CASES:
        H.init(H.HallocOpts(memory=512 << 20))
        seeds = group_seeds(n, 32, 0x5EED)
        states = torch.tensor(seeds.view(np.int32), device="cuda")
        slots = torch.zeros(n, dtype=torch.int64, device="cuda")
        ctrs = torch.zeros(n, dtype=torch.int32, device="cuda")
        acc = torch.zeros(4, dtype=torch.int64, device="cuda")
        H.phase_ref_latency(n, 1, 1, 16, probs, size, size, states, slots, ctrs, acc)  # warm-up
        states.copy_(torch.tensor(seeds.view(np.int32), device="cuda"))
        lat = H.phase_ref_latency(n, 1, 8, 16, probs, size, size, states, slots, ctrs, acc)
        ok = H.status() == 0 and H.stats()["used_chunks"] == 0 and acc[2].item() == 0
        H.shutdown()
        case = {"threads": n, "size": size, "ok": ok}
        for k, pub in zip(("malloc", "free"), published):
            s = lat[k]
            case[k] = {"n": s["n"], "min": s["min_cycles"], "avg": s["avg_cycles"],
                       "max": s["max_cycles"], "p50": s["p50_cycles"], "p99": s["p99_cycles"],
                       "published_kepler_min_avg_max": pub}
        case["published_source"] = "tst/exp/scaling/" + src
        out["cases"].append(case)
    return out


# ---- halloc's own benchmark programs on this allocator ----------------------
#
# tst/perf/{phase-throughput,phase-latency,priv-throughput} compiled from the
# reference tree unchanged against include/halloc.h + libhalloc.a
# (tests/dropin/Makefile, target ref-tests), run with the arguments of the
# experiment scripts that produced halloc's published figures.  Their numbers
# are the harness's own: host clock around every launch, its pair formula.

HALLOC_BIN = os.path.join(ROOT, "tests", "dropin", "_build", "ref")
PHASE_COMMON = "-f0.95 -F0.05 -e0.91 -m536870912 -g5"  # tst/exp/scaling/exp-run.pl:10-17

# (name, -n -l -s -S arguments, published private pairs, published spree
# pairs, source); spree = -i1 -t512, private = -i32 -t16
# (tst/exp/scaling/exp-run.pl:18-50, tst/exp/speed/exp-run.pl:18-34)
HALLOC_PHASE_CASES = [
    ("scaling 16 B x1, 1M threads", "-n1048576 -l1 -s16", 1366.76, 940.35,
     "tst/exp/scaling/exp-log-thru.csv:47"),
    ("scaling 16 B x4, 1M threads", "-n1048576 -l4 -s16", 1396.75, 1220.92,
     "tst/exp/scaling/exp-log-thru.csv:48"),
    ("scaling 256 B x1, 1M threads", "-n1048576 -l1 -s256", 190.58, 557.76,
     "tst/exp/scaling/exp-log-thru.csv:49"),
    ("scaling 16 B x1, 32K threads", "-n32768 -l1 -s16", 1012.49, 347.03,
     "tst/exp/scaling/exp-log-thru.csv:32"),
    ("scaling 16 B x4, 32K threads", "-n32768 -l4 -s16", 1218.44, 753.21,
     "tst/exp/scaling/exp-log-thru.csv:33"),
    ("scaling 256 B x1, 32K threads", "-n32768 -l1 -s256", 621.78, 312.41,
     "tst/exp/scaling/exp-log-thru.csv:34"),
    ("scaling 16 B x1, 1K threads", "-n1024 -l1 -s16", 89.53, 15.43,
     "tst/exp/scaling/exp-log-thru.csv:17"),
    ("scaling 16 B x4, 1K threads", "-n1024 -l4 -s16", 118.87, 45.02,
     "tst/exp/scaling/exp-log-thru.csv:18"),
    ("scaling 256 B x1, 1K threads", "-n1024 -l1 -s256", 92.89, 15.51,
     "tst/exp/scaling/exp-log-thru.csv:19"),
    ("single size 16 B", "-n1048576 -l4 -s16", 1401.70, 1220.15,
     "tst/exp/speed/exp-log-single.csv:2"),
    ("single size 256 B", "-n838860 -l1 -s256", 194.92, 251.85,
     "tst/exp/speed/exp-log-single.csv:10"),
    ("single size 3072 B", "-n69905 -l1 -s3072", 19.68, 30.02,
     "tst/exp/speed/exp-log-single.csv:17"),
    ("mixed 8..256 B", "-n1048576 -l1 -s8 -S256", 927.18, 795.18,
     "tst/exp/speed/exp-log-combi.csv:4"),
    ("mixed 8..3072 B", "-n139446 -l1 -s8 -S3072", 64.85, 88.33,
     "tst/exp/speed/exp-log-combi.csv:5"),
]

# The private form of mixed 8..3072 B runs out of slabs at 512 MiB on a B200,
# where all 139,446 threads are resident at once (about 28 K on the Kepler),
# so about 243 MB are live at an allocation phase's peak; halloc's harness
# then stops.  It is run as published and again with this pool.
MIXED_3072_POOL = 805306368

# (name, full arguments, published pairs, source): halloc against CUDA's
# allocator (tst/exp/halloc-vs-scatter/exp-run.pl:12-86) and slab settings
# (tst/exp/settings/exp-run.pl:7-37)
HALLOC_OTHER_CASES = [
    ("spree 4x16 B, 640K threads, halloc",
     "-f0.9 -F0.2 -e0.71 -m536870912 -g5 -ahalloc -n655360 -l4 -s16 -i1 -t16", 736.18,
     "tst/exp/halloc-vs-scatter/exp-log-spree.csv:29"),
    ("spree 4x16 B, 640K threads, CUDA malloc",
     "-f0.9 -F0.2 -e0.71 -m536870912 -g5 -acuda -n655360 -l4 -s16 -i1 -t16", 0.19,
     "tst/exp/halloc-vs-scatter/exp-log-spree.csv:31"),
    ("private 4x16 B, 640K threads, halloc",
     "-e0.75 -m536870912 -g5 -ahalloc -n655360 -l4 -s16 -f0.9 -F0.35 -e0.75 -i16 -t8", 990.06,
     "tst/exp/halloc-vs-scatter/exp-log-priv.csv:29"),
    ("private 4x16 B, 640K threads, CUDA malloc",
     "-e0.75 -m536870912 -g5 -acuda -n655360 -l4 -s16 -f0.9 -F0.35 -e0.75 -i16 -t1", 1.09,
     "tst/exp/halloc-vs-scatter/exp-log-priv.csv:31"),
    ("settings 4x16 B, 4 MiB slabs, busy 0.745",
     "-f0.95 -F0.05 -e0.91 -n524288 -m536870912 -g5 -i31 -t31 -b22 -B0.745 -s16 -l4", 1441.52,
     "tst/exp/settings/exp-log.csv:86"),
    ("settings 4x16 B, 4 MiB slabs, busy 0.835",
     "-f0.95 -F0.05 -e0.91 -n524288 -m536870912 -g5 -i31 -t31 -b22 -B0.835 -s16 -l4", 1369.94,
     "tst/exp/settings/exp-log.csv:104"),
    ("settings 4x16 B, 4 MiB slabs, busy 0.915",
     "-f0.95 -F0.05 -e0.91 -n524288 -m536870912 -g5 -i31 -t31 -b22 -B0.915 -s16 -l4", 1287.82,
     "tst/exp/settings/exp-log.csv:120"),
    ("settings 1x256 B, 2 MiB slabs, busy 0.835",
     "-f0.95 -F0.05 -e0.91 -n524288 -m536870912 -g5 -i31 -t31 -b21 -B0.835 -s256 -l1", 140.04,
     "tst/exp/settings/exp-log.csv:63"),
    ("settings 1x256 B, 4 MiB slabs, busy 0.835",
     "-f0.95 -F0.05 -e0.91 -n524288 -m536870912 -g5 -i31 -t31 -b22 -B0.835 -s256 -l1", 319.74,
     "tst/exp/settings/exp-log.csv:105"),
    ("settings 1x256 B, 8 MiB slabs, busy 0.835",
     "-f0.95 -F0.05 -e0.91 -n524288 -m536870912 -g5 -i31 -t31 -b23 -B0.835 -s256 -l1", 814.79,
     "tst/exp/settings/exp-log.csv:147"),
]


def _halloc_program(prog: str, args: str, timeout: int = 300) -> dict:
    """Runs one of halloc's programs on GPU 0 and parses what it prints."""
    import re
    try:
        p = subprocess.run([os.path.join(HALLOC_BIN, prog), "-D0"] + args.split(),
                           capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return {"error": "timed out"}
    out = {}
    for line in p.stdout.splitlines():
        m = re.match(r"(malloc|free|pair) throughput ([0-9.]+)", line)
        if m:
            out[m.group(1) + "_mops"] = float(m.group(2))
        m = re.match(r"(min|avg|max) (malloc|free) latency ([0-9.]+) cycles", line)
        if m:
            out.setdefault(m.group(2) + "_cycles", {})[m.group(1)] = float(m.group(3))
    if p.returncode != 0:
        out["error"] = (p.stderr or p.stdout)[-300:]
    return out


def run_halloc_programs() -> dict:
    """halloc's published experiments re-run by halloc's own programs, on
    this allocator, beside the published (Kepler) figures."""
    if not os.path.exists(os.path.join(HALLOC_BIN, "phase-throughput")):
        return {"skipped": "halloc's programs are built where the reference tree is present "
                           "(make -C tests/dropin ref-tests)"}
    out = {"unit": "M pairs/s (the harness's formula, host clock per launch)",
           "how": "tst/perf programs from the reference tree, unchanged, compiled against "
                  "include/halloc.h and linked with libhalloc.a", "cases": []}
    r = _halloc_program("priv-throughput", "-n32768 -T128 -s16 -l1 -i10 -m536870912")
    out["plain"] = {"args": "-n32768 -T128 -s16 -l1 -i10 -m536870912", **r}
    for name, args, pub_priv, pub_spree, src in HALLOC_PHASE_CASES:
        for form, extra, pub in (("spree", "-i1 -t512", pub_spree),
                                 ("private", "-i32 -t16", pub_priv)):
            a = f"{PHASE_COMMON} {args} {extra}"
            r = _halloc_program("phase-throughput", a)
            got = r.get("pair_mops")
            case = {"name": f"{name}, {form}", "args": a, **r,
                    "published_kepler_pair_mops": pub, "published_source": src,
                    "vs_published": got / pub if got else None}
            if "-S3072" in args and form == "private":
                case["note"] = ("all 139,446 threads resident at once: the live set at a "
                                "phase peak (about 243 MB in 16 size classes) can exceed "
                                "the 512 MiB pool, and the harness stops at a NULL")
                a2 = a.replace("-m536870912", f"-m{MIXED_3072_POOL}")
                r2 = _halloc_program("phase-throughput", a2)
                case["with_larger_pool"] = {"args": a2, **r2}
            out["cases"].append(case)
    for name, args, pub, src in HALLOC_OTHER_CASES:
        r = _halloc_program("phase-throughput", args)
        got = r.get("pair_mops")
        out["cases"].append({"name": name, "args": args, **r,
                             "published_kepler_pair_mops": pub, "published_source": src,
                             "vs_published": got / pub if got else None})
    out["latency"] = []
    for n, size, published, src in PHASE_LAT_CASES:
        a = f"{PHASE_COMMON} -n{n} -l1 -s{size} -i16 -t8"
        r = _halloc_program("phase-latency", a)
        out["latency"].append({"args": a, **r, "published_kepler_malloc_free_min_avg_max":
                               published, "published_source": "tst/exp/scaling/" + src})
    ratios = [c["vs_published"] for c in out["cases"]
              if c["vs_published"] and "CUDA" not in c["name"]]
    out["ok"] = (all("error" not in c or "note" in c for c in out["cases"]) and
                 "error" not in out["plain"])
    out["vs_published_min_max"] = [min(ratios), max(ratios)] if ratios else None
    return out


BATCH_POOL, BATCH_HF = 4 << 30, 0.5
# launch shape of the persistent form: 32 warps per block, 8,192 requests per
# task (the fastest of a 3 x 3 x 3 sweep of block, task size and blocks per SM)
PERSIST_BLOCK, PERSIST_ITEMS = 1024, 8192


def run_batched(torch, H, reps: int, tune: bool) -> dict:
    """Batched request stream (64 batches, log-uniform 1,024..1,048,576
    requests, geometric size classes p=0.3, 1 % large 4..64 KiB, lifetimes
    1..8 batches) served by per-batch launches and by one graph-captured
    persistent launch; then the autotuner sweep."""
    from halloc_b200.autotune import autotune
    from halloc_b200.workloads import BatchedRunner, batched_plan
    plan = batched_plan(seed=1)
    runner = BatchedRunner(plan, torch)
    stream = torch.cuda.current_stream()
    H.init(H.HallocOpts(memory=BATCH_POOL, halloc_fraction=BATCH_HF))
    H.l2_persist(stream)

    def timed(fn) -> list:
        fn()
        torch.cuda.synchronize()
        runner.verify()
        out = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            runner.verify()
            out.append(e0.elapsed_time(e1))
        return out

    plain = timed(lambda: runner.plain(block=256, stream=stream))
    try:
        h = runner.prepare(block=PERSIST_BLOCK, task_items=PERSIST_ITEMS, graph=True)
        pers = timed(lambda: runner.launch(h, stream))
    except Exception as e:  # report the plain form even so
        runner.release()
        H.shutdown()
        return {"error": f"persistent form: {e}", "plain_ms": plain}
    runner.release()
    ok = H.status() == 0 and H.stats()["used_chunks"] == 0
    H.shutdown()
    n = plan.nreq
    res = {"metric": "batched malloc/free pairs/s", "unit": "pairs/s", "requests": n,
           "batches": plan.nbatch, "large_requests": int((plan.req_size > 3072).sum()),
           "plain": {"value": n / (min(plain) * 1e-3), "ms": plain,
                     "launches": int(np.count_nonzero(np.diff(plan.free_start))) +
                     int(np.count_nonzero(np.diff(plan.batch_start)))},
           "persistent_graph": {"value": n / (min(pers) * 1e-3), "ms": pers, "launches": 1,
                                "block": PERSIST_BLOCK, "task_items": PERSIST_ITEMS},
           "speedup": min(plain) / min(pers), "ok": ok,
           "pool": {"memory": BATCH_POOL, "halloc_fraction": BATCH_HF}}
    if tune:
        t = autotune(torch, runner, BATCH_POOL, BATCH_HF, reps=2)
        t["best"]["value"] = n / (t["best"]["ms"] * 1e-3)
        t["best"]["speedup_vs_plain"] = min(plain) / t["best"]["ms"]
        res["autotune"] = t
    res["small_only"] = run_batched_small_only(torch, H, reps, tune)
    return res


def run_batched_small_only(torch, H, reps: int, tune: bool = False) -> dict:
    """The same stream without its 1 % of large requests (same seed, sizes
    and lifetimes otherwise): what the slabs alone sustain, without CUDA's
    in-kernel malloc for the 4..64 KiB requests; then the autotuner on it,
    where the allocator's own settings decide the time."""
    from halloc_b200.autotune import autotune
    from halloc_b200.workloads import BatchedRunner, batched_plan
    plan = batched_plan(seed=1, large_frac=0.0)
    runner = BatchedRunner(plan, torch)
    stream = torch.cuda.current_stream()
    H.init(H.HallocOpts(memory=BATCH_POOL, halloc_fraction=BATCH_HF))
    H.l2_persist(stream)
    out = {}
    try:
        for name, fn in (("plain", lambda: runner.plain(block=256, stream=stream)),):
            fn()
            torch.cuda.synchronize()
            runner.verify()
            ms = []
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn()
                e1.record(stream)
                e1.synchronize()
                runner.verify()
                ms.append(e0.elapsed_time(e1))
            out[name] = {"value": plan.nreq / (min(ms) * 1e-3), "ms": ms}
        h = runner.prepare(block=PERSIST_BLOCK, task_items=PERSIST_ITEMS, graph=True)
        runner.launch(h, stream)
        torch.cuda.synchronize()
        runner.verify()
        ms = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            runner.launch(h, stream)
            e1.record(stream)
            e1.synchronize()
            runner.verify()
            ms.append(e0.elapsed_time(e1))
        out["persistent_graph"] = {"value": plan.nreq / (min(ms) * 1e-3), "ms": ms}
        out["speedup"] = min(out["plain"]["ms"]) / min(ms)
        out["ok"] = H.status() == 0 and H.stats()["used_chunks"] == 0
    finally:
        runner.release()
        H.shutdown()
    out["requests"] = plan.nreq
    if tune and "plain" in out:
        t = autotune(torch, runner, BATCH_POOL, BATCH_HF, reps=2)
        t["best"]["value"] = plan.nreq / (t["best"]["ms"] * 1e-3)
        t["best"]["speedup_vs_plain"] = min(out["plain"]["ms"]) / t["best"]["ms"]
        out["autotune"] = t
    return out


SERVE_POOL = 16 << 30
SERVE_POINTS = ((1e6, 1_000_000), (1e7, 2_000_000), (1e8, 10_000_000))


def run_serve(torch, H) -> dict:
    """Serving loop: Poisson arrivals at rate lambda of jobs that grow by 1..32
    blocks of 256 B per step up to ceil(L/256), L log-uniform 64 B..2 MiB,
    and live Exp(mean 50 steps); admission refused while the 12 GiB slab
    pool of a 16 GiB pool is over 90 % full; one persistent kernel of one
    256-slot block per SM.  The launch with every SM full is reported
    beside it at the highest rate."""
    H.init(H.HallocOpts(memory=SERVE_POOL))
    out = {"metric": "serving jobs/s and hamalloc latency", "points": []}
    ok = True
    for lam, njobs in SERVE_POINTS:
        res = torch.zeros(2 * njobs, dtype=torch.int64, device="cuda")
        r = H.serve_run(res, njobs, lam, seed=7)
        ok &= r["jobs_done"] == njobs and r["timeouts"] == 0
        cpn = r["cycles_per_ns"] or 1.0
        out["points"].append({
            "lambda": lam, "jobs": njobs, "jobs_per_s": r["jobs_done"] / r["seconds"],
            "seconds": r["seconds"], "allocs": r["allocs"],
            "allocs_per_s": r["allocs"] / r["seconds"],
            "alloc_failures": r["alloc_failures"], "refusals": r["refusals"],
            "peak_occupancy": r["peak_live_blocks"] * 256 / H.stats()["pool_bytes"],
            "p50_ns": r["p50_cycles"] / cpn, "p99_ns": r["p99_cycles"] / cpn,
            "max_ns": r["max_cycles"] / cpn, "p50_cycles": r["p50_cycles"],
            "p99_cycles": r["p99_cycles"], "sm_ghz": cpn})
        del res
    # the same at the highest rate, every SM filled with job slots
    lam, njobs = SERVE_POINTS[-1]
    res = torch.zeros(2 * njobs, dtype=torch.int64, device="cuda")
    r = H.serve_run(res, njobs, lam, seed=7, ctas_per_sm=0)
    cpn = r["cycles_per_ns"] or 1.0
    ok &= r["jobs_done"] == njobs and r["timeouts"] == 0
    out["full_occupancy_launch"] = {
        "lambda": lam, "jobs": njobs, "jobs_per_s": r["jobs_done"] / r["seconds"],
        "allocs_per_s": r["allocs"] / r["seconds"], "p50_ns": r["p50_cycles"] / cpn,
        "p99_ns": r["p99_cycles"] / cpn,
        "note": "as many 256-slot blocks per SM as fit: more warps contend for the "
                "one head slab of the 256-B size"}
    del res
    ok &= H.status() == 0 and H.stats()["used_chunks"] == 0
    H.shutdown()
    # the same rate on a growing pool: 1 GiB of the 12 GiB of slabs backed at
    # init, 1 GiB more whenever the kernel finds none left; trimmed afterwards
    H.set_growth(1 << 30)
    try:
        H.init(H.HallocOpts(memory=SERVE_POOL))
    finally:
        H.set_growth(0)
    res = torch.zeros(2 * njobs, dtype=torch.int64, device="cuda")
    st0 = H.stats()
    r = H.serve_run(res, njobs, lam, seed=7, grow_bytes=1 << 30)
    st1 = H.stats()
    cpn = r["cycles_per_ns"] or 1.0
    gok = r["jobs_done"] == njobs and r["timeouts"] == 0 and r["alloc_failures"] == 0
    released = H.trim()
    st2 = H.stats()
    gok &= st1["used_chunks"] == 0 and (H.status() & ~H.ST_GROW) == 0
    out["growing_pool"] = {
        "lambda": lam, "jobs": njobs, "jobs_per_s": r["jobs_done"] / r["seconds"],
        "allocs_per_s": r["allocs"] / r["seconds"], "p50_ns": r["p50_cycles"] / cpn,
        "p99_ns": r["p99_cycles"] / cpn, "alloc_waits": r["alloc_waits"],
        "grows": r["grows"], "grow_seconds": r["grow_seconds"],
        "backed_bytes_start": st0["committed_slabs"] * st0["sb_sz"],
        "backed_bytes_end": st1["committed_slabs"] * st1["sb_sz"],
        "released_by_trim": released,
        "backed_bytes_after_trim": st2["committed_slabs"] * st2["sb_sz"],
        "slab_pool_bytes": st0["pool_bytes"], "ok": gok,
        "note": "ha_set_growth_c(1 GiB) + serve grow_bytes 1 GiB: slabs backed by "
                "cuMemCreate/cuMemMap while the kernel runs, released by ha_trim_c"}
    ok &= gok
    del res
    H.shutdown()
    # tuned variant: four head slabs per size
    H.set_heads(4)
    H.init(H.HallocOpts(memory=SERVE_POOL))
    H.set_heads(1)
    lam, njobs = SERVE_POINTS[-1]
    res = torch.zeros(2 * njobs, dtype=torch.int64, device="cuda")
    r = H.serve_run(res, njobs, lam, seed=7)
    cpn = r["cycles_per_ns"] or 1.0
    out["tuned_4_heads"] = {"lambda": lam, "jobs": njobs,
                            "jobs_per_s": r["jobs_done"] / r["seconds"],
                            "allocs_per_s": r["allocs"] / r["seconds"],
                            "alloc_failures": r["alloc_failures"],
                            "p50_ns": r["p50_cycles"] / cpn, "p99_ns": r["p99_cycles"] / cpn,
                            "ok": r["jobs_done"] == njobs and r["timeouts"] == 0,
                            "note": "4 head slabs per size (ha_set_heads_c)"}
    del res
    H.shutdown()
    out["ok"] = ok
    out["config"] = ("jobs of ceil(L/256) 256-B blocks, L log-uniform 64 B..2 MiB, growing "
                     "1..32 blocks per step, lifetime Exp(mean 50 steps), Poisson arrivals, "
                     "admission refused above 0.9 occupancy of the slab pool (16 GiB pool, "
                     "12 GiB of slabs), one persistent kernel of 148 x 256 job slots, host-fed "
                     "through mapped memory")
    return out


GRAPH_N, GRAPH_POOL = 1 << 20, 1 << 30

SAMPLE_POINTS, SAMPLE_CELLS, SAMPLE_STRINGS, SAMPLE_STRLEN = 1_000_000, 32, 1_000_000, 31


def run_samples(torch, H, reps: int) -> dict:
    """The reference's sample programs at their own sizes (512 MiB pool):
    grid-points, 1,000,000 points into a 32^3 grid, and add-strings,
    1,000,000 pairs of 31-character strings concatenated; each kernel timed
    with CUDA events (median of reps, L2 flushed before each), results
    checked on the device."""
    import statistics as stats

    from halloc_b200.workloads import sample_lengths, sample_points
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def timed(fn) -> float:
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    H.init(H.HallocOpts(memory=512 << 20))
    out = {"config": "samples/grid-points and samples/add-strings at the sizes their main() "
                     "uses, 512 MiB pool, device time per kernel (median of "
                     f"{reps}, L2 flushed before each)"}
    # grid-points
    n, nc = SAMPLE_POINTS, SAMPLE_CELLS
    pts = torch.tensor(sample_points(n, seed=5), device="cuda")
    grid = torch.zeros(nc ** 3, dtype=torch.int64, device="cuda")
    nodes = torch.zeros(2 * n, dtype=torch.int64, device="cuda")
    nfail = torch.zeros(1, dtype=torch.int64, device="cuda")
    ins, fre, pre = [], [], []
    for r in range(reps + 1):
        t_ins = timed(lambda: H.grid_insert(n, nc, pts, grid, nfail, stream=stream))
        used = H.stats()["used_chunks"]
        t_fre = timed(lambda: H.grid_free(nc, grid, stream=stream))
        t_pre = timed(lambda: H.grid_insert(n, nc, pts, grid, nfail, pre_nodes=nodes,
                                            stream=stream))
        H.grid_free(nc, grid, pre_nodes=True, stream=stream)
        if r:
            ins.append(t_ins), fre.append(t_fre), pre.append(t_pre)
    torch.cuda.synchronize()
    grid_ok = nfail.item() == 0 and used == n and H.stats()["used_chunks"] == 0
    out["grid_points"] = {
        "points": n, "cells": nc ** 3,
        "insert_mpoints_s": n / (stats.median(ins) * 1e-3) / 1e6,
        "free_mpoints_s": n / (stats.median(fre) * 1e-3) / 1e6,
        "insert_preallocated_mpoints_s": n / (stats.median(pre) * 1e-3) / 1e6,
        "insert_ms": stats.median(ins), "free_ms": stats.median(fre), "ok": grid_ok}
    del pts, grid, nodes
    # add-strings
    n = SAMPLE_STRINGS
    la = torch.full((n,), SAMPLE_STRLEN, dtype=torch.int32, device="cuda")
    a, b, c = (torch.zeros(n, dtype=torch.int64, device="cuda") for _ in range(3))
    bad = torch.zeros(1, dtype=torch.int64, device="cuda")
    t_a, t_c, t_f = [], [], []
    for r in range(reps + 1):
        ta = timed(lambda: H.strings_alloc(n, la, a, nfail, stream=stream))
        ta += timed(lambda: H.strings_alloc(n, la, b, nfail, stream=stream))
        tc = timed(lambda: H.strings_concat(n, c, a, b, nfail, stream=stream))
        H.strings_check(n, c, la, la, bad, stream=stream)
        tf = sum(timed(lambda s=s: H.strings_free(n, s, stream=stream)) for s in (a, b, c))
        if r:
            t_a.append(ta / 2), t_c.append(tc), t_f.append(tf / 3)
    torch.cuda.synchronize()
    str_ok = nfail.item() == 0 and bad.item() == 0 and H.stats()["used_chunks"] == 0
    out["add_strings"] = {
        "strings": n, "length": SAMPLE_STRLEN,
        "alloc_mstrings_s": n / (stats.median(t_a) * 1e-3) / 1e6,
        "concat_mstrings_s": n / (stats.median(t_c) * 1e-3) / 1e6,
        "free_mstrings_s": n / (stats.median(t_f) * 1e-3) / 1e6, "ok": str_ok}
    out["ok"] = grid_ok and str_ok and H.status() == 0
    H.shutdown()
    return out


def run_graph(torch, H, reps: int) -> dict:
    """Random-graph build: 1,048,576 vertices, Poisson(16) out-degree from a
    seed, one thread per vertex growing an int32 neighbour array by doubling
    (malloc new, copy, hafree old); then a CSR gather that frees every
    array."""
    from halloc_b200.workloads import poisson_thresholds
    t = poisson_thresholds(16.0)
    H.init(H.HallocOpts(memory=GRAPH_POOL))
    stream = torch.cuda.current_stream()
    n = GRAPH_N
    cdf = torch.from_numpy(t.view(np.int32)).cuda()
    arr = torch.zeros(n, dtype=torch.int64, device="cuda")
    deg = torch.zeros(n, dtype=torch.int32, device="cuda")
    acc = torch.zeros(3, dtype=torch.int64, device="cuda")
    off = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    cols = torch.zeros(20 * n, dtype=torch.int32, device="cuda")
    build_ms, gather_ms, edges, ok = [], [], 0, True
    for r in range(reps + 1):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        H.graph_build(n, 0xC0FFEE + r, cdf, len(t), arr, deg, acc, stream)
        e1.record(stream)
        off[1:] = torch.cumsum(deg.to(torch.int64), 0)
        e1b = torch.cuda.Event(enable_timing=True)
        e1b.record(stream)
        H.graph_gather(n, arr, deg, off, cols, stream)
        e2.record(stream)
        e2.synchronize()
        failed, grows, ne = acc.cpu().tolist()
        ok &= failed == 0 and ne == int(off[-1])
        if r:
            build_ms.append(e0.elapsed_time(e1))
            gather_ms.append(e1b.elapsed_time(e2))
            edges += ne
    ok &= H.status() == 0 and H.stats()["used_chunks"] == 0
    H.shutdown()
    return {"metric": "graph-build edges/s", "unit": "edges/s",
            "value": edges / (sum(build_ms) * 1e-3), "build_ms": build_ms,
            "gather_free_ms": gather_ms, "edges_per_run": edges // reps, "ok": ok,
            "config": "n=1,048,576, Poisson(16) out-degree from a seed on the device, "
                      "int32 arrays from capacity 2 doubling (malloc new, copy, hafree old); "
                      "gather = CSR copy + hafree of every array"}


def hbm_peak() -> float | None:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, ValueError, KeyError):
        return None


def cpu_sample(kind: str, seconds: float) -> dict:
    """The plain workload replayed on the host cores; repeats the full
    workload until about `seconds` have passed."""
    import oracle
    cores = os.cpu_count() or 1
    dt1, _, _ = oracle.cpu_plain_run(kind, NTHREADS, NITERS, NBYTES, cores)
    reps = max(1, int(seconds / max(dt1, 1e-3)))
    tot, pairs = 0.0, 0
    for _ in range(reps):
        dt, cs, nf = oracle.cpu_plain_run(kind, NTHREADS, NITERS, NBYTES, cores)
        if nf or cs != plain_checksum(NTHREADS, NITERS):
            raise RuntimeError(f"CPU {kind} run failed")
        tot += dt
        pairs += PAIRS_PER_STEP
    return {"value": pairs / tot, "unit": "pairs/s", "cores": cores,
            "sample": f"{reps} x the full workload ({PAIRS_PER_STEP} pairs) on {cores} threads"}


def cpu_add_strings() -> dict | None:
    """The reference's own CPU twin of its add-strings sample
    (samples/add-strings/add-strings.c, OpenMP over every host core, built
    unchanged into oracle/_ref): 500,000 strings of 31 characters."""
    exe = os.path.join(ROOT, "oracle", "_ref", "add_strings_cpu")
    if not os.path.exists(exe):
        return None
    try:
        p = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    except subprocess.TimeoutExpired:
        return None
    out = {"cores": os.cpu_count() or 1, "strings": 500000, "kind": "reference"}
    for line in p.stdout.splitlines():
        for key, tag in (("alloc_mstrings_s", "allocation performance"),
                         ("concat_mstrings_s", "concatenation performance"),
                         ("free_mstrings_s", "freeing performance")):
            if tag in line:
                out[key] = float(line.split(":")[1].split()[0])
    return out


def hot_word_bound(res: dict, pairs_per_s: float) -> dict:
    """What bounds the plain workload: each thread's 10 iterations are a
    chain of dependent L2 round trips (ticket, reservation, count, payload
    read-back, nibble, count-down), and one warp running the same loop alone
    (no contention at all) takes nearly as long as the whole 1,024-warp grid.
    Floor = that lone warp's launch; frac = floor / the grid's launch.  Also
    given: the one-word atomic floor of the head slab's counter, which every
    warp's malloc and free hit (2 per warp-iteration)."""
    lone = res.get("lone_warp_us")
    launch_s = PAIRS_PER_STEP / pairs_per_s
    out = None
    if lone:
        out = {"resource": "latency of one thread's dependent L2 round trips (10 iterations "
                           "of malloc, 16-B write, read-back, free)",
               "floor_us": lone, "launch_us": launch_s * 1e6, "frac": lone * 1e-6 / launch_s,
               "how": "the same kernel run by one warp alone, L2 flushed, CUDA events"}
    rate = res.get("hot_word_rate")
    if rate and out is not None:
        ops = 2 * (NTHREADS // 32) * NITERS * NALLOCS
        out["head_counter_word"] = {"ops_per_launch": ops, "rate_gops_measured": rate / 1e9,
                                    "floor_us": ops / rate * 1e6,
                                    "frac": ops / rate / launch_s}
    return out


def reference_kind():
    import oracle
    return "reference" if oracle.reference_available() else "port"


def _get(d, *path):
    """d[path[0]][path[1]]... or None where any step is missing."""
    for k in path:
        if isinstance(d, dict):
            d = d.get(k)
        elif isinstance(d, list) and isinstance(k, int) and -len(d) <= k < len(d):
            d = d[k]
        else:
            return None
    return d


def leg_summary(name: str, out: dict) -> dict:
    """The one-number summaries of a secondary leg that the headline line
    carries; the leg's full result is on its own line before it."""
    if not isinstance(out, dict) or "error" in out:
        return {"error": str(_get(out, "error"))[:120]}
    if name == "phase":
        return {"pairs_per_s": out.get("value"), "ok": out.get("ok"),
                "tuned_4_heads_pairs_per_s": _get(out, "tuned_4_heads", "value"),
                "payload_frac_of_hbm": _get(out, "payload", "frac_of_hbm")}
    if name == "batched":
        return {"persistent_pairs_per_s": _get(out, "persistent_graph", "value"),
                "persistent_vs_plain": out.get("speedup"),
                "small_only_persistent_vs_plain": _get(out, "small_only", "speedup"),
                "ok": out.get("ok")}
    if name == "graph":
        return {"edges_per_s": out.get("value"), "ok": out.get("ok")}
    if name == "serve":
        pts = out.get("points") or []
        top = max(pts, key=lambda q: q.get("lambda", 0)) if pts else {}
        return {"lambda": top.get("lambda"), "jobs_per_s": top.get("jobs_per_s"),
                "p50_us": (top.get("p50_ns") or 0) / 1e3, "p99_us": (top.get("p99_ns") or 0) / 1e3,
                "ok": out.get("ok")}
    if name == "samples":
        return {"ok": out.get("ok")}
    if name == "halloc_programs":
        cases = out.get("cases") or []
        return {"rows": len(cases),
                "rows_ahead_of_published": sum(1 for c in cases
                                               if (c.get("vs_published") or 0) > 1.0)}
    return {}


def rounded(x, digits: int = 5):
    """x with every float rounded to `digits` significant digits (keeps the
    headline line short enough for a log tail)."""
    if isinstance(x, float):
        return float(f"{x:.{digits}g}")
    if isinstance(x, dict):
        return {k: rounded(v, digits) for k, v in x.items()}
    if isinstance(x, list):
        return [rounded(v, digits) for v in x]
    return x


def print_leg(name: str, out) -> None:
    print(json.dumps({"leg": name, "result": out}), flush=True)


def headline(args, world: int, res: dict, cpu, glibc, cuda_malloc, legs: dict) -> dict:
    """The last line of a run: the contract's keys for the plain workload,
    floats rounded, the secondary legs as one-number summaries."""
    value = replica_throughput(PAIRS_PER_STEP * args.steps, world, res["total_s"])
    e2e = replica_throughput(PAIRS_PER_STEP * args.steps, world, res["e2e_s"])
    e2e_copy = replica_throughput(PAIRS_PER_STEP * args.steps, world, res["e2e_copy_s"])
    peak = res["peak"]["per_sector_returning"] * 1e9
    peak_coalesced = max(res["peak"]["returning"], res["peak"]["fire_and_forget"]) * 1e9
    achieved = value / world * ATOMICS_PER_PAIR
    binding = hot_word_bound(res, value / world) or {}
    cm_value = _get(cuda_malloc, "value")
    line = {
        "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": res["total_s"] * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "threads": NTHREADS, "iters": NITERS,
                   "block_bytes": NBYTES, "pool_bytes": POOL,
                   "pairs_per_step": PAIRS_PER_STEP, "parallelism": f"replicas{world}",
                   "l2": "flushed between steps (256 MiB write)"},
        "ok": res["ok"],
        "e2e": {"value": e2e, "unit": "pairs/s", "h2d_bytes_per_step": NTHREADS * 4,
                "d2h_bytes_per_step": 16,
                "how": "ha_throughput_host_c, wall clock per step: sizes in and result out "
                       "through pinned host memory (pinned once, before timing)",
                "copy_engine_value": e2e_copy},
        "roofline": {"bound": "l2_atomic", "achieved": achieved / 1e9, "peak": peak / 1e9,
                     "unit": "Gatomic/s", "frac": achieved / peak,
                     "traffic": PLAIN_DRAM_BYTES_PER_LAUNCH,
                     "peak_how": "live: returning u32 atomicOr, a 32-B sector per thread",
                     "frac_vs_coalesced_peak": achieved / peak_coalesced,
                     "atomics_per_pair": ATOMICS_PER_PAIR,
                     "lone_warp_floor_us": binding.get("floor_us"),
                     "frac_of_lone_warp_floor": binding.get("frac")},
        "cpu_baseline": cpu,
        "host_malloc_baseline": ({"value": glibc["value"], "unit": "pairs/s",
                                  "cores": glibc["cores"]} if glibc else None),
        "cuda_malloc_baseline": ({"value": cm_value, "unit": "pairs/s",
                                  "heap_bytes": _get(cuda_malloc, "heap_bytes"),
                                  "ok": _get(cuda_malloc, "ok")} if cuda_malloc else None),
        "vs_cuda_malloc": value / world / cm_value if cm_value else None,
        "legs": legs,
        "gpu_launches": args.steps,
        "clocks": res["clocks"],
    }
    return rounded(line)


def main_ours(args):
    rank, world, local_rank = dist_env()
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    res = run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return
    if args.only_gpu:
        value = replica_throughput(PAIRS_PER_STEP * args.steps, world, res["total_s"])
        e2e = replica_throughput(PAIRS_PER_STEP * args.steps, world, res["e2e_s"])
        print(json.dumps({"metric": METRIC, "value": value, "e2e": e2e, "ok": res["ok"],
                          "note": "GPU legs only (profiling run)"}), flush=True)
        return
    # the comparator and the secondary legs are one-GPU workloads, each in a
    # process of its own (fresh pool and CUDA-heap sizes): N=1 line only
    legs = {}
    cuda_malloc = None
    if world == 1:
        cuda_malloc = run_leg("cuda_malloc", args.steps)
        print_leg("cuda_malloc", cuda_malloc)
        for name, skip in (("phase", args.skip_phase), ("batched", args.skip_batched),
                           ("graph", args.skip_graph), ("serve", args.skip_serve),
                           ("samples", args.skip_samples),
                           ("halloc_programs", args.skip_halloc_programs)):
            if skip:
                continue
            out = run_halloc_programs() if name == "halloc_programs" else run_leg(name)
            if name == "samples" and isinstance(out, dict):
                out["add_strings_cpu_baseline"] = cpu_add_strings()
            print_leg(name, out)
            legs[name] = leg_summary(name, out)
    kind = reference_kind()
    cpu = cpu_sample(kind, args.cpu_seconds) if world == 1 else None
    if cpu:
        cpu["kind"] = kind
    glibc = cpu_sample("glibc", min(3.0, args.cpu_seconds)) if world == 1 else None
    line = headline(args, world, res, cpu, glibc, cuda_malloc, legs)
    print(json.dumps(line), flush=True)


def main_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle
    kind = reference_kind()
    cores = os.cpu_count() or 1
    for _ in range(args.warmup):
        oracle.cpu_plain_run(kind, NTHREADS, NITERS, NBYTES, cores)
    tot = 0.0
    for _ in range(args.steps):
        dt, cs, nf = oracle.cpu_plain_run(kind, NTHREADS, NITERS, NBYTES, cores)
        if nf or cs != plain_checksum(NTHREADS, NITERS):
            raise RuntimeError("reference run failed")
        tot += dt
    value = PAIRS_PER_STEP * args.steps / tot
    sample = (f"{args.steps} runs of the full workload ({PAIRS_PER_STEP} pairs each) through "
              + ("the reference allocator's own code built for the host (oracle/_ref)"
                 if kind == "reference" else "the host replay model (oracle port)")
              + f" on {cores} host threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tot * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "threads": NTHREADS, "iters": NITERS,
                   "block_bytes": NBYTES, "pool_bytes": POOL},
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--cpu-seconds", type=float, default=10.0)
    p.add_argument("--skip-phase", action="store_true", help="skip the mixed-size phase leg")
    p.add_argument("--skip-batched", action="store_true", help="skip the batched leg")
    p.add_argument("--no-tune", action="store_true", help="batched leg without the autotuner")
    p.add_argument("--skip-graph", action="store_true", help="skip the random-graph leg")
    p.add_argument("--skip-serve", action="store_true", help="skip the serving leg")
    p.add_argument("--skip-samples", action="store_true",
                   help="skip the grid-points / add-strings sample leg")
    p.add_argument("--skip-halloc-programs", action="store_true",
                   help="skip halloc's own benchmark programs")
    p.add_argument("--leg", choices=["phase", "batched", "graph", "serve", "atomics", "samples",
                                     "halloc_programs", "cuda_malloc"],
                   help=argparse.SUPPRESS)
    p.add_argument("--only-gpu", action="store_true",
                   help="skip the CPU and CUDA-malloc legs (profiling runs)")
    args = p.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.leg:
        leg_main(args)
    elif args.impl == "reference":
        main_reference(args)
    else:
        main_ours(args)


if __name__ == "__main__":
    main()
