"""Concurrent use: many threads allocating and freeing at once.  Checks the
reference's own invariants (non-NULL while space is left, no overlap,
halloc tst/common/common.cu:412-529), the ones it lacked (alignment, pool
range, payload checksum), and that after quiescence the device's per-slab
used-chunk counts, bit arrays and size nibbles equal what the host model
derives from the live blocks."""
import numpy as np
import pytest

from tests.helpers import (allocator, assert_free_count, check_blocks, expected_slab_state,
                           nibbles_to_chunk_layout, plain_checksum)

pytestmark = pytest.mark.gpu

SMALL = [16, 24, 32, 48, 64, 96, 128, 192, 256]


def malloc_batch(torch, H, sizes: np.ndarray, nthreads: int, nallocs: int):
    d_sizes = torch.tensor(sizes.astype(np.int32), device="cuda")
    ptrs = torch.zeros(nthreads * nallocs, dtype=torch.int64, device="cuda")
    H.malloc_batch(d_sizes, nthreads, nallocs, ptrs, tag=True)
    torch.cuda.synchronize()
    return ptrs


def assert_state_matches_live(H, ptrs: np.ndarray, sizes: np.ndarray):
    dump = H.dump_state()
    counts, bits, nib = expected_slab_state(ptrs, sizes, dump["pool_base"], dump["sb_sz"],
                                            dump["nsbs"])
    assert np.array_equal(dump["counters"] >> 12, counts), "per-slab used-chunk counts"
    assert np.array_equal(dump["bits"], bits), "bit arrays"
    assert np.array_equal(nibbles_to_chunk_layout(dump["nibbles"], dump["chunk_enc"]), nib)
    return dump


def assert_empty(H):
    dump = H.dump_state()
    assert (dump["counters"] >> 12 == 0).all()
    assert not dump["bits"].any() and not dump["nibbles"].any()


def test_plain_config_blocks(torch_cuda):
    """256 x 128 threads, 4 blocks of 16 B each, held at once."""
    torch = torch_cuda
    n, k = 32768, 4
    sizes = np.full(n * k, 16, np.int64)
    with allocator(memory=512 << 20) as H:
        st = H.stats()
        ptrs = malloc_batch(torch, H, sizes, n, k)
        p = ptrs.cpu().numpy()
        check_blocks(p, sizes, st["pool_base"], st["pool_bytes"])
        assert_state_matches_live(H, p, sizes)
        H.free_batch(ptrs, n, k)
        torch.cuda.synchronize()
        assert_empty(H)
        assert H.status() == 0


def test_mixed_sizes_1m_blocks(torch_cuda):
    """262144 threads x 4 blocks drawn uniformly from 16..256 B (seeded)."""
    torch = torch_cuda
    n, k = 262144, 4
    rng = np.random.default_rng(7)
    sizes = rng.choice(SMALL, n * k)
    with allocator(memory=1 << 30) as H:
        st = H.stats()
        ptrs = malloc_batch(torch, H, sizes, n, k)
        p = ptrs.cpu().numpy()
        check_blocks(p, sizes, st["pool_base"], st["pool_bytes"])
        assert_state_matches_live(H, p, sizes)
        # free half, check again, free the rest
        half = torch.tensor(np.where(np.arange(n * k) % 2 == 0, p, 0), device="cuda")
        H.free_batch(half, n, k)
        torch.cuda.synchronize()
        rest = np.where(np.arange(n * k) % 2 == 1, p, 0)
        assert_state_matches_live(H, rest, sizes)
        H.free_batch(torch.tensor(rest, device="cuda"), n, k)
        torch.cuda.synchronize()
        assert_empty(H)
        assert H.status() == 0


def test_large_blocks_go_to_cuda_heap(torch_cuda):
    torch = torch_cuda
    n, k = 4096, 2
    rng = np.random.default_rng(8)
    sizes = rng.choice([16, 100, 3072, 3073, 4096, 20000], n * k)
    with allocator(memory=512 << 20) as H:
        st = H.stats()
        ptrs = malloc_batch(torch, H, sizes, n, k)
        p = ptrs.cpu().numpy()
        check_blocks(p, sizes, st["pool_base"], st["pool_bytes"])
        assert_state_matches_live(H, p, sizes)
        H.free_batch(ptrs, n, k)
        torch.cuda.synchronize()
        assert_empty(H)
        assert H.status() == 0


def test_exhaustion_returns_null_and_recovers(torch_cuda):
    """A 32-slab pool asked for twice its size: some requests get NULL, the
    blocks handed out are still valid, and after freeing everything the same
    request succeeds again."""
    torch = torch_cuda
    n = 65536
    sizes = np.full(n, 1024, np.int64)
    with allocator(memory=64 << 20, halloc_fraction=0.5, sb_sz_sh=20) as H:
        st = H.stats()
        ptrs = malloc_batch(torch, H, sizes, n, 1)
        p = ptrs.cpu().numpy()
        r = check_blocks(p, sizes, st["pool_base"], st["pool_bytes"], allow_null=True)
        assert r["nnull"] > 0 and r["n"] > 20000
        assert H.stats()["n_null"] >= r["nnull"]
        assert_state_matches_live(H, p, sizes)
        H.free_batch(ptrs, n, 1)
        torch.cuda.synchronize()
        assert_empty(H)
        ptrs2 = malloc_batch(torch, H, np.full(20000, 1024, np.int64), 20000, 1)
        check_blocks(ptrs2.cpu().numpy(), np.full(20000, 1024), st["pool_base"],
                     st["pool_bytes"])
        H.free_batch(ptrs2, 20000, 1)
        torch.cuda.synchronize()
        assert H.status() == 0


def test_freed_slabs_are_reused_across_sizes(torch_cuda):
    """The reference's freeslabs test (tst/corr/freeslabs/freeslabs.cu:43-70):
    sizes 16..1024, each allocating 40 % of the memory and freeing it; it only
    passes if slabs released by one size serve the next."""
    torch = torch_cuda
    memory = 512 << 20
    sizes_swept = []
    s, step = 16, 8
    while s <= 1024:
        sizes_swept.append(s)
        s += step
        step = 128 if s >= 256 else 16 if s >= 64 else 8
    with allocator(memory=memory) as H:
        st = H.stats()
        for sz in sizes_swept:
            n = min(1 << 20, int(0.4 * memory / sz))
            sizes = np.full(n, sz, np.int64)
            ptrs = malloc_batch(torch, H, sizes, n, 1)
            check_blocks(ptrs.cpu().numpy(), sizes, st["pool_base"], st["pool_bytes"])
            H.free_batch(ptrs, n, 1)
            torch.cuda.synchronize()
        assert_empty(H)
        # every slab is in the free set or serves as a head or prefetched
        # slab (surge sets of the sizes that stormed may still hold some);
        # closing the surge sets leaves at most the head and prefetched slab
        # of each size
        end = assert_free_count(H)
        assert end["free_slabs"] + end["head_slabs"] == st["nsbs"]
        H.close_surges()
        torch.cuda.synchronize()
        assert assert_free_count(H)["free_slabs"] >= st["nsbs"] - 2 * 16
        assert H.stats()["surge_level"] == [0] * 16
        assert H.status() == 0


@pytest.mark.parametrize("nallocs,niters", [(1, 10), (4, 3)])
def test_throughput_loop_checksum(torch_cuda, nallocs, niters):
    """The private-throughput loop writes {t^0..t^3} into every block and
    reads it back: any overlap between live blocks breaks the checksum."""
    torch = torch_cuda
    n = 32768
    with allocator(memory=512 << 20) as H:
        out = torch.zeros(2, dtype=torch.int64, device="cuda")
        H.throughput(out, n, nbytes=16, block=128, nallocs=nallocs, niters=niters)
        torch.cuda.synchronize()
        cs, nfail = out.cpu().tolist()
        assert nfail == 0
        assert cs == plain_checksum(n, nallocs * niters)
        st = H.stats()
        assert st["used_chunks"] == 0 and st["status"] == 0


def test_throughput_loop_mixed_sizes_host_api(torch_cuda):
    torch = torch_cuda
    n = 65536
    rng = np.random.default_rng(9)
    h_sizes = rng.choice(SMALL + [512, 3072], n).astype(np.uint32)
    with allocator(memory=1 << 30) as H:
        d_sizes = torch.zeros(n, dtype=torch.int32, device="cuda")
        d_out = torch.zeros(2, dtype=torch.int64, device="cuda")
        h_out = np.zeros(2, np.uint64)
        H.throughput_host(h_out, d_out, n, nallocs=2, niters=4, h_sizes=h_sizes,
                          d_sizes=d_sizes)
        assert int(h_out[1]) == 0
        assert int(h_out[0]) == plain_checksum(n, 8)
        assert H.stats()["used_chunks"] == 0


@pytest.mark.parametrize("transfer", [0, 1, 2])
def test_throughput_loop_host_api_pinned_transfers(torch_cuda, transfer):
    """Pinned host buffers: the automatic choice (mapped), the copy engine and
    the mapped form give the same totals, in h_out and in d_out, call after
    call (the mapped form's device totals start from zero each launch)."""
    torch = torch_cuda
    n = 40000  # not a multiple of the block
    rng = np.random.default_rng(11)
    sizes = rng.choice(SMALL + [512, 3072], n).astype(np.int32)
    with allocator(memory=1 << 30) as H:
        h_sizes = torch.from_numpy(sizes).pin_memory()
        h_out = torch.zeros(2, dtype=torch.int64).pin_memory()
        d_sizes = torch.zeros(n, dtype=torch.int32, device="cuda")
        d_out = torch.zeros(2, dtype=torch.int64, device="cuda")
        for niters in (3, 3, 1):
            h_out.zero_()
            H.throughput_host(h_out.data_ptr(), d_out, n, nallocs=2, niters=niters,
                              h_sizes=h_sizes.data_ptr(), d_sizes=d_sizes, transfer=transfer)
            want = plain_checksum(n, 2 * niters)
            assert h_out.tolist() == [want, 0]
            assert d_out.cpu().tolist() == [want, 0]
        # a fixed size, no sizes buffer at all
        H.throughput_host(h_out.data_ptr(), d_out, n, nbytes=48, niters=2, transfer=transfer)
        assert h_out.tolist() == [plain_checksum(n, 2), 0]
        assert H.stats()["used_chunks"] == 0 and H.status() == 0


def test_throughput_loop_mapped_needs_pinned_buffers(torch_cuda):
    """The mapped form refuses pageable host buffers before any launch."""
    torch = torch_cuda
    import halloc_b200 as H
    n = 1024
    with allocator(memory=512 << 20):
        d_sizes = torch.zeros(n, dtype=torch.int32, device="cuda")
        d_out = torch.zeros(2, dtype=torch.int64, device="cuda")
        h_out = np.zeros(2, np.uint64)
        h_sizes = np.full(n, 16, np.uint32)
        with pytest.raises(H.HallocError):
            H.throughput_host(h_out, d_out, n, h_sizes=h_sizes, d_sizes=d_sizes,
                              transfer=H.XFER_MAPPED)
        # the automatic choice falls back to the copy engine for them
        H.throughput_host(h_out, d_out, n, h_sizes=h_sizes, d_sizes=d_sizes)
        assert int(h_out[0]) == plain_checksum(n, 1) and int(h_out[1]) == 0


def test_cuda_malloc_comparator_checksum(torch_cuda):
    torch = torch_cuda
    n = 4096
    with allocator(memory=512 << 20) as H:
        out = torch.zeros(2, dtype=torch.int64, device="cuda")
        H.cuda_throughput(out, n, nbytes=16, niters=2)
        torch.cuda.synchronize()
        cs, nfail = out.cpu().tolist()
        assert nfail == 0 and cs == plain_checksum(n, 2)


def test_stats_and_extfrag(torch_cuda):
    with allocator(memory=512 << 20) as H:
        st = H.stats()
        assert st["nsbs"] == 96 and st["sb_sz"] == 4 << 20
        assert st["free_slabs"] == 96 and st["used_chunks"] == 0
        assert st["pool_base"] % (4 << 20) == 0
        f = H.extfrag(False)
        assert 0.0 <= f <= 1.0


@pytest.mark.parametrize("nheads", [2, 8])
def test_multi_head_variant(torch_cuda, nheads):
    """The tuned variant with several head slabs per size keeps every
    invariant and the exact slab state.  Each (head, size) pair holds a head
    and a prefetched slab, so the pool is sized for 2 x nheads x 12 sizes
    slabs beside the data."""
    import halloc_b200
    torch = torch_cuda
    n, k = 131072, 4
    rng = np.random.default_rng(nheads)
    sizes = rng.choice(SMALL + [384, 1024, 3072], n * k)
    halloc_b200.set_heads(nheads)
    try:
        with allocator(memory=4 << 30) as H:
            st = H.stats()
            ptrs = malloc_batch(torch, H, sizes, n, k)
            p = ptrs.cpu().numpy()
            check_blocks(p, sizes, st["pool_base"], st["pool_bytes"])
            assert_state_matches_live(H, p, sizes)
            H.free_batch(ptrs, n, k)
            torch.cuda.synchronize()
            assert_empty(H)
            out = torch.zeros(2, dtype=torch.int64, device="cuda")
            H.throughput(out, 32768, nbytes=16, block=128, nallocs=2, niters=5)
            torch.cuda.synchronize()
            assert out.cpu().tolist() == [plain_checksum(32768, 10), 0]
            assert H.status() == 0
    finally:
        halloc_b200.set_heads(1)


def test_empty_inputs_are_no_ops(torch_cuda):
    """Zero threads, zero ops, zero points, zero strings: every entry point
    returns success, touches nothing and leaves the pool empty (the
    reference's harness launches with n >= 1 only)."""
    import halloc_b200
    torch = torch_cuda
    with allocator(memory=256 << 20) as H:
        d = torch.zeros(8, dtype=torch.int64, device="cuda")
        sizes = torch.zeros(1, dtype=torch.int32, device="cuda")
        H.malloc_batch(sizes, 0, 1, d)
        H.free_batch(d, 0, 1)
        H.throughput(d, 0, nbytes=16)
        H.trace(d, 0, d)
        H.phase_round(0, 0, 4, 1, 0, 1 << 31, d, sizes, d, sizes, 1)
        probs = halloc_b200.phase_ref_probabilities(0.95, 0.05, 0.91)
        H.phase_ref_step(0, 1, 0, 1, probs, 16, 16, sizes, d, sizes, d)
        pts = torch.zeros(3, dtype=torch.float32, device="cuda")
        H.grid_insert(0, 8, pts, d, d)
        H.strings_alloc(0, sizes, d, d)
        H.strings_free(0, d)
        torch.cuda.synchronize()
        assert not d.any().item()
        st = H.stats()
        assert st["used_chunks"] == 0 and st["status"] == 0


def test_kernels_on_concurrent_streams(torch_cuda):
    """hamalloc / hafree called at once from kernels of different streams
    (halloc's README: thread-safe across kernels): two private-throughput
    loops and a batch allocation run side by side; every checksum holds, the
    blocks left live are valid and disjoint, and the pool ends empty."""
    torch = torch_cuda
    n = 65536
    rng = np.random.default_rng(21)
    sizes = rng.choice(SMALL + [512, 3072], n * 2)
    with allocator(memory=1 << 30) as H:
        st = H.stats()
        streams = [torch.cuda.Stream() for _ in range(3)]
        outs = [torch.zeros(2, dtype=torch.int64, device="cuda") for _ in range(2)]
        d_sizes = torch.tensor(sizes.astype(np.int32), device="cuda")
        ptrs = torch.zeros(n * 2, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        for rep in range(3):
            for o in outs:
                o.zero_()
            torch.cuda.synchronize()
            H.throughput(outs[0], n, nbytes=16, block=128, nallocs=2, niters=4,
                         stream=streams[0].cuda_stream)
            H.throughput(outs[1], n, nbytes=96, block=256, nallocs=1, niters=6,
                         stream=streams[1].cuda_stream)
            H.malloc_batch(d_sizes, n, 2, ptrs, tag=True, stream=streams[2].cuda_stream)
            torch.cuda.synchronize()
            assert outs[0].cpu().tolist() == [plain_checksum(n, 8), 0]
            assert outs[1].cpu().tolist() == [plain_checksum(n, 6), 0]
            p = ptrs.cpu().numpy()
            check_blocks(p, sizes, st["pool_base"], st["pool_bytes"])
            assert_state_matches_live(H, p, sizes)
            H.free_batch(ptrs, n, 2, stream=streams[2].cuda_stream)
            torch.cuda.synchronize()
            assert_empty(H)
        assert H.status() == 0


_HEADS_PROBE = """
import sys
sys.path.insert(0, {root!r})
import torch
import halloc_b200 as H
torch.cuda.set_device(0)
H.init(H.HallocOpts(memory=512 << 20))
out = torch.zeros(2, dtype=torch.int64, device="cuda")
H.throughput(out, 1 << 18, nbytes=16, block=128, nallocs=4, niters=2)
torch.cuda.synchronize()
st = H.stats()
assert int(out[1]) == 0 and st["used_chunks"] == 0 and H.status() == 0
print("head_slabs", st["head_slabs"])
H.shutdown()
"""


@pytest.mark.parametrize("env,many", [(None, False), ("4", True), ("3", False)])
def test_heads_from_environment(torch_cuda, env, many):
    """HALLOC_HEADS reaches programs that only use halloc.h: with 4 head slabs
    per size a 16-B workload spread over every SM flags more than the one head
    and one prefetched slab of the reference policy; an invalid value is
    reported and ignored."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    e = dict(os.environ)
    e.pop("HALLOC_HEADS", None)
    e["HALLOC_SURGE"] = "0"  # fixed heads only: no surge sets under this storm
    if env is not None:
        e["HALLOC_HEADS"] = env
    r = subprocess.run([sys.executable, "-c", _HEADS_PROBE.format(root=root)], env=e,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    n = int(r.stdout.split("head_slabs")[1])
    assert (n > 2) if many else (n <= 2), n
    if env == "3":
        assert "HALLOC_HEADS=3 ignored" in r.stderr
