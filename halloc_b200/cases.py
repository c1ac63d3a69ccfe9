"""Small instances of the workload kernels, each launched once, for
profiling one kernel at a time and as short usage examples:

    python -m halloc_b200.cases phase_ref|phase|batched|batched_small|graph|samples|storm|serve|all

Every case holds at most about 1.1 GB on the device and checks its
result the way the tests do (counts, checksums, an empty pool at the end);
a failed check raises.
"""
from __future__ import annotations

import sys

import numpy as np

import halloc_b200 as H


def _torch():
    import torch
    assert torch.cuda.is_available(), "the cases need a CUDA device"
    torch.cuda.set_device(0)
    return torch


def _done(name: str) -> None:
    st = H.stats()
    if st["used_chunks"] != 0 or H.status() != 0:
        raise RuntimeError(f"{name}: pool not empty or status {H.status():#x}")
    H.shutdown()
    print(f"{name}: ok", flush=True)


def phase_ref(torch) -> None:
    """halloc's phase experiment (8..256 B, -f0.95 -F0.05 -e0.91 -g5),
    1,048,576 threads, 4 tries and the final free: ha_phase_ref_k."""
    from halloc_b200.workloads import group_seeds
    n = 1 << 20
    H.init(H.HallocOpts(memory=512 << 20))
    probs = H.phase_ref_probabilities(0.95, 0.05, 0.91)
    states = torch.tensor(group_seeds(n, 32, 0x5EED).view(np.int32), device="cuda")
    slots = torch.zeros(n, dtype=torch.int64, device="cuda")
    ctrs = torch.zeros(n, dtype=torch.int32, device="cuda")
    acc = torch.zeros(4, dtype=torch.int64, device="cuda")
    r = H.phase_ref_run(n, 1, 4, 1, probs, 8, 256, states, slots, ctrs, acc)
    if r["failed"] or r["mallocs"] != r["frees"]:
        raise RuntimeError(f"phase_ref: {r}")
    _done("phase_ref")


def phase(torch) -> None:
    """The mixed-size phase workload, two periods: 1,048,576 threads x 4
    slots, 1 GiB pool, 16..256 B, allocation rounds (p=0.95) until 91 % of
    the slots are filled, a free round; then the rest freed: ha_phase_alloc_k,
    ha_phase_free_k."""
    n, nslots = 1 << 20, 4
    sizes = [16, 24, 32, 48, 64, 96, 128, 192, 256]
    thr = int(0.95 * 2**32)
    H.init(H.HallocOpts(memory=1 << 30))
    size_set = torch.tensor(sizes, dtype=torch.int32, device="cuda")
    slots = torch.zeros(nslots * n, dtype=torch.int64, device="cuda")
    slot_sz = torch.zeros(nslots * n, dtype=torch.int32, device="cuda")
    acc = torch.zeros(6, dtype=torch.int64, device="cuda")
    r = H.phase_run(n, nslots, 0x5EED, 2, thr, thr, int(0.91 * nslots * n), size_set,
                    len(sizes), slots, slot_sz, acc)
    if r["failed"] or r["written_sum"] != r["read_sum"] or r["mallocs"] != r["frees"]:
        raise RuntimeError(f"phase: {r}")
    print(f"phase: {r['mallocs']} pairs in {r['alloc_rounds']} allocation and "
          f"{r['free_rounds']} free rounds, {r['kernel_ms']:.3f} ms of kernels")
    _done("phase")


def batched(torch) -> None:
    """8 batches of 1,024..65,536 requests (1 % large): per-batch launches
    (ha_bmalloc_k, ha_bfree_k) and one persistent launch (ha_bpersist_k)."""
    from halloc_b200.workloads import BatchedRunner, batched_plan
    plan = batched_plan(seed=3, nbatch=8, max_batch=1 << 16)
    runner = BatchedRunner(plan, torch)
    H.init(H.HallocOpts(memory=1 << 30, halloc_fraction=0.5))
    stream = torch.cuda.current_stream()
    runner.plain(block=256, stream=stream)
    torch.cuda.synchronize()
    runner.verify()
    h = runner.prepare(block=256, task_items=2048, graph=False)
    runner.launch(h, stream)
    torch.cuda.synchronize()
    runner.verify()
    runner.release()
    _done("batched")


def batched_small(torch) -> None:
    """The batched stream without its large requests: 16 batches of
    1,024..262,144 requests, sizes geometric over the 16 classes; per-batch
    launches, then one persistent launch with the benchmark's launch shape
    (1,024 threads, 8,192 requests per task)."""
    from halloc_b200.workloads import BatchedRunner, batched_plan
    plan = batched_plan(seed=3, nbatch=16, max_batch=1 << 18, large_frac=0.0)
    runner = BatchedRunner(plan, torch)
    H.init(H.HallocOpts(memory=1 << 30, halloc_fraction=0.5))
    stream = torch.cuda.current_stream()
    runner.plain(block=256, stream=stream)
    torch.cuda.synchronize()
    runner.verify()
    h = runner.prepare(block=1024, task_items=8192, graph=False)
    runner.launch(h, stream)
    torch.cuda.synchronize()
    runner.verify()
    runner.release()
    _done("batched_small")


def graph(torch) -> None:
    """Random graph of 262,144 vertices, Poisson(16) out-degree, doubling
    neighbour arrays: ha_graph_build_k, then the CSR gather."""
    from halloc_b200.workloads import poisson_thresholds
    n = 1 << 18
    t = poisson_thresholds(16.0)
    H.init(H.HallocOpts(memory=1 << 30))
    cdf = torch.tensor(np.asarray(t, np.uint32).view(np.int32), device="cuda")
    arr = torch.zeros(n, dtype=torch.int64, device="cuda")
    deg = torch.zeros(n, dtype=torch.int32, device="cuda")
    acc = torch.zeros(3, dtype=torch.int64, device="cuda")
    H.graph_build(n, 7, cdf, len(t), arr, deg, acc)
    torch.cuda.synchronize()
    d = deg.cpu().numpy().astype(np.int64)
    off = np.zeros(n + 1, np.int64)
    off[1:] = np.cumsum(d)
    d_off = torch.tensor(off, device="cuda")
    edges = torch.zeros(max(1, int(off[-1])), dtype=torch.int32, device="cuda")
    H.graph_gather(n, arr, deg, d_off, edges)
    torch.cuda.synchronize()
    if acc[0].item():
        raise RuntimeError("graph: failed allocations")
    _done("graph")


def samples(torch) -> None:
    """grid-points (1,000,000 points, 32^3 cells: ha_grid_insert_k,
    ha_grid_free_k) and add-strings (1,000,000 pairs of 31-character
    strings: ha_strings_alloc_k, ha_strings_concat_k, ha_strings_free_k)."""
    from halloc_b200.workloads import sample_points
    H.init(H.HallocOpts(memory=512 << 20))
    n, nc = 1_000_000, 32
    pts = torch.tensor(sample_points(n, seed=5), device="cuda")
    grid = torch.zeros(nc ** 3, dtype=torch.int64, device="cuda")
    nfail = torch.zeros(1, dtype=torch.int64, device="cuda")
    H.grid_insert(n, nc, pts, grid, nfail)
    H.grid_free(nc, grid)
    lens = torch.full((n,), 31, dtype=torch.int32, device="cuda")
    a, b, c = (torch.zeros(n, dtype=torch.int64, device="cuda") for _ in range(3))
    bad = torch.zeros(1, dtype=torch.int64, device="cuda")
    H.strings_alloc(n, lens, a, nfail)
    H.strings_alloc(n, lens, b, nfail)
    H.strings_concat(n, c, a, b, nfail)
    H.strings_check(n, c, lens, lens, bad)
    for s in (a, b, c):
        H.strings_free(n, s)
    torch.cuda.synchronize()
    if nfail.item() or bad.item():
        raise RuntimeError("samples: failed allocations or bad strings")
    _done("samples")


def storm(torch) -> None:
    """1,048,576 threads each allocating, writing, reading back and freeing
    one 256-B block, twice (ha_throughput_k): every resident warp contends
    for the 256-B size's head slab, which fills every 13,680 blocks."""
    H.init(H.HallocOpts(memory=1 << 30))
    n = 1 << 20
    out = torch.zeros(2, dtype=torch.int64, device="cuda")
    H.throughput(out, n, nbytes=256, block=128, nallocs=1, niters=2)
    torch.cuda.synchronize()
    cs, nfail = out.cpu().tolist()
    # every block holds {t^0, t^1, t^2, t^3} and is read back into the sum
    t = np.arange(n, dtype=np.int64)
    if nfail or cs != int(2 * (4 * (t - t % 4) + 6).sum()):
        raise RuntimeError(f"storm: checksum {cs} failures {nfail}")
    _done("storm")


def serve(torch) -> None:
    """The serving kernel on a closed batch of 20,000 jobs, all handed over
    before the launch (ha_serve_k waits on nothing from the host)."""
    H.init(H.HallocOpts(memory=1 << 30))
    n = 20000
    res = torch.zeros(2 * n, dtype=torch.int64, device="cuda")
    r = H.serve_run(res, n, 1e8, seed=7, max_len=64 << 10, prereleased=True)
    if r["jobs_done"] != n or r["alloc_failures"] or r["timeouts"]:
        raise RuntimeError(f"serve: {r['jobs_done']} jobs, {r['alloc_failures']} failures")
    print(f"serve: {r['seconds'] * 1e3:.2f} ms wall, {r['allocs']} allocations, "
          f"p50 {r['p50_cycles']:.0f} / p99 {r['p99_cycles']:.0f} cycles per hamalloc")
    _done("serve")


CASES = {"phase_ref": phase_ref, "phase": phase, "batched": batched,
         "batched_small": batched_small, "graph": graph,
         "samples": samples, "storm": storm, "serve": serve}


def main(argv) -> None:
    torch = _torch()
    names = list(CASES) if not argv or argv[0] == "all" else argv
    for name in names:
        CASES[name](torch)


if __name__ == "__main__":
    main(sys.argv[1:])
