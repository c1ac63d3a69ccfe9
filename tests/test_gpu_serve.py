"""Serving loop: a host-fed Poisson stream of jobs served by continuous
batching in one persistent kernel.  Every job completes, nothing fails,
each block's payload survives to the job's end (the value sum equals the
host recomputation), the pool is empty afterwards, and a job's result is
the same served alone as in the mix."""
import numpy as np
import pytest

from oracle.phase import mix32
from tests.helpers import allocator

pytestmark = pytest.mark.gpu

CFG = dict(lam=2e6, seed=11, mean_life=20.0, min_len=64, max_len=64 << 10)


def value_sums(ids: np.ndarray, blocks: np.ndarray) -> np.ndarray:
    """Sum over k < blocks of mix32(id * 0x27D4EB2F + k), per job."""
    out = np.zeros(len(ids), np.uint64)
    for i, (j, b) in enumerate(zip(ids, blocks)):
        k = np.arange(int(b), dtype=np.uint32)
        out[i] = mix32(np.uint32((int(j) * 0x27D4EB2F) & 0xFFFFFFFF) + k).astype(np.uint64).sum()
    return out


def test_serving_stream_and_alone_vs_mix(torch_cuda):
    import halloc_b200 as H
    torch = torch_cuda
    n = 3000
    with allocator(memory=1 << 30):
        res = torch.zeros(2 * n, dtype=torch.int64, device="cuda")
        r = H.serve_run(res, n, **CFG)
        assert r["jobs_done"] == n and r["alloc_failures"] == 0 and r["timeouts"] == 0
        assert r["allocs"] > n and r["p99_cycles"] >= r["p50_cycles"] > 0
        assert int(r["hist"].sum()) == r["allocs"]
        mix = res.view(-1, 2).cpu().numpy().astype(np.uint64)
        assert (mix[:, 0] >= 1).all()
        ids = np.arange(n)
        assert np.array_equal(mix[:, 1], value_sums(ids, mix[:, 0]))
        st = H.stats()
        assert st["used_chunks"] == 0 and st["status"] == 0
        # the same jobs, each served alone
        for j in (0, 7, 1234, n - 1):
            alone = torch.zeros(2 * n, dtype=torch.int64, device="cuda")
            r1 = H.serve_run(alone, n, job_ids=[j], **CFG)
            assert r1["jobs_done"] == 1
            a = alone.view(-1, 2)[j].cpu().numpy().astype(np.uint64)
            assert np.array_equal(a, mix[j]), j
        assert H.stats()["used_chunks"] == 0


def test_admission_gate_refuses_and_recovers(torch_cuda):
    """With a tiny occupancy limit most admissions are refused at first;
    jobs still all complete once memory frees up."""
    import halloc_b200 as H
    torch = torch_cuda
    n = 800
    with allocator(memory=1 << 30):
        res = torch.zeros(2 * n, dtype=torch.int64, device="cuda")
        r = H.serve_run(res, n, occupancy_limit=0.0005, **CFG)
        assert r["refusals"] > 0
        assert r["jobs_done"] == n and r["alloc_failures"] == 0 and r["timeouts"] == 0
        assert H.stats()["used_chunks"] == 0 and H.status() == 0


def test_serving_on_a_growing_pool(torch_cuda):
    """The pool backs one unit at init and grows on the kernel's requests
    while the stream runs: every job completes with the same result as on a
    fully backed pool, nothing fails, the pool grew, and a trim afterwards
    gives the memory back."""
    import halloc_b200 as H
    torch = torch_cuda
    n = 3000
    ref = torch.zeros(2 * n, dtype=torch.int64, device="cuda")
    with allocator(memory=1 << 30):
        r0 = H.serve_run(ref, n, **CFG)
        assert r0["jobs_done"] == n and r0["alloc_failures"] == 0
    H.set_growth(8 << 20)
    try:
        H.init(H.HallocOpts(memory=1 << 30))
    finally:
        H.set_growth(0)
    try:
        st0 = H.stats()
        res = torch.zeros(2 * n, dtype=torch.int64, device="cuda")
        r = H.serve_run(res, n, grow_bytes=16 << 20, **CFG)
        assert r["jobs_done"] == n and r["alloc_failures"] == 0 and r["timeouts"] == 0
        assert r["grows"] >= 1 and r["alloc_waits"] >= 1
        assert r["grown_bytes"] == r["grows"] * (16 << 20)
        assert torch.equal(res, ref)
        st = H.stats()
        assert st["committed_slabs"] > st0["committed_slabs"]
        assert st["used_chunks"] == 0
        assert H.status() & ~H.ST_GROW == 0
        released = H.trim()
        assert released % st["unit_bytes"] == 0
        assert H.stats()["committed_slabs"] == st["committed_slabs"] - released // st["sb_sz"]
    finally:
        H.shutdown()


def test_closed_batch_gives_the_streamed_results(torch_cuda):
    """All jobs handed over before the launch (prereleased): every job's
    result equals the streamed run's."""
    import halloc_b200 as H
    torch = torch_cuda
    n = 2000
    with allocator(memory=1 << 30):
        a = torch.zeros(2 * n, dtype=torch.int64, device="cuda")
        b = torch.zeros(2 * n, dtype=torch.int64, device="cuda")
        ra = H.serve_run(a, n, **CFG)
        rb = H.serve_run(b, n, prereleased=True, **CFG)
        assert ra["jobs_done"] == rb["jobs_done"] == n
        assert rb["alloc_failures"] == 0 and rb["timeouts"] == 0
        assert torch.equal(a, b)
        assert H.stats()["used_chunks"] == 0 and H.status() == 0


def test_serving_at_the_benchmark_rate(torch_cuda):
    """One point of the benchmark's sweep: 1 M jobs at lambda = 1e8 jobs/s,
    256-B blocks, job lengths log-uniform 64 B..2 MiB, 16 GiB pool.  Every
    job completes with no failure or timeout, the latency histogram holds
    every allocation, a sample of jobs' value sums equals the host
    recomputation, and the pool is empty at the end."""
    import halloc_b200 as H
    torch = torch_cuda
    n = 1_000_000
    with allocator(memory=16 << 30):
        res = torch.zeros(2 * n, dtype=torch.int64, device="cuda")
        r = H.serve_run(res, n, 1e8, seed=7)
        assert r["jobs_done"] == n and r["alloc_failures"] == 0 and r["timeouts"] == 0
        assert int(r["hist"].sum()) == r["allocs"] and r["allocs"] > 100 * n
        assert r["p99_cycles"] >= r["p50_cycles"] > 0
        got = res.view(-1, 2).cpu().numpy().astype(np.uint64)
        ids = np.random.default_rng(3).choice(n, 300, replace=False)
        assert np.array_equal(got[ids, 1], value_sums(ids, got[ids, 0]))
        st = H.stats()
        assert st["used_chunks"] == 0 and st["status"] == 0
