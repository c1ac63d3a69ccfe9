"""Slab growth and release: a pool whose slabs are backed by device memory
on demand (ha_set_growth_c / ha_grow_c) and given back when wholly free
(ha_trim_c).  The allocator must behave exactly as over a fully backed pool
for the slabs it has, return NULL with HA_ST_GROW when it runs out of backed
slabs, serve again after a grow, and keep every block valid and every
payload intact across grows and trims."""
import numpy as np
import pytest

from tests.helpers import assert_free_count, check_blocks, expected_slab_state, plain_checksum

pytestmark = pytest.mark.gpu

MiB = 1 << 20


@pytest.fixture
def growing():
    import halloc_b200 as H
    H.set_growth(64 * MiB)
    try:
        H.init(H.HallocOpts(memory=4 << 30, halloc_fraction=0.75))
    finally:
        H.set_growth(0)
    try:
        yield H
    finally:
        H.shutdown()


def malloc_batch(torch, H, sizes, n, k=1):
    d_sizes = torch.tensor(np.asarray(sizes, np.int32), device="cuda")
    ptrs = torch.zeros(n * k, dtype=torch.int64, device="cuda")
    H.malloc_batch(d_sizes, n, k, ptrs, tag=True)
    torch.cuda.synchronize()
    return ptrs


def test_growth_init_backs_only_the_first_units(torch_cuda, growing):
    H = growing
    st = H.stats()
    assert st["growth"] == 1
    assert st["unit_bytes"] % st["sb_sz"] == 0
    per_unit = st["unit_bytes"] // st["sb_sz"]
    want = -(-(64 * MiB) // st["unit_bytes"]) * per_unit
    assert st["committed_slabs"] == want == st["free_slabs"]
    assert st["nsbs"] == (3 << 30) // st["sb_sz"]
    assert st["pool_base"] % st["unit_bytes"] == 0


def test_exhaustion_raises_grow_then_grow_serves(torch_cuda, growing):
    """256-B blocks for 3x the backed slabs: NULLs and HA_ST_GROW, no other
    status; after a grow the same request is served in full, blocks valid
    and the slab state exact."""
    torch, H = torch_cuda, growing
    st = H.stats()
    n = 3 * st["committed_slabs"] * (st["sb_sz"] // 256)
    sizes = np.full(n, 256, np.int64)
    ptrs = malloc_batch(torch, H, sizes, n)
    p = ptrs.cpu().numpy()
    r = check_blocks(p, sizes, st["pool_base"], st["pool_bytes"], allow_null=True)
    assert r["nnull"] > 0
    assert H.status() == H.ST_GROW
    H.free_batch(ptrs, n, 1)
    torch.cuda.synchronize()
    H.clear_status()
    added = H.grow(4 * n * 256)
    assert added >= 4 * n * 256 - st["unit_bytes"] and added % st["unit_bytes"] == 0
    torch.cuda.synchronize()
    st2 = H.stats()
    assert st2["committed_slabs"] == st["committed_slabs"] + added // st["sb_sz"]
    ptrs = malloc_batch(torch, H, sizes, n)
    p = ptrs.cpu().numpy()
    check_blocks(p, sizes, st2["pool_base"], st2["pool_bytes"])
    dump = H.dump_state()
    counts, bits, _ = expected_slab_state(p, sizes, dump["pool_base"], dump["sb_sz"],
                                          dump["nsbs"])
    assert np.array_equal(dump["counters"] >> 12, counts)
    assert np.array_equal(dump["bits"], bits)
    # every block lies in a backed slab
    assert ((p - st2["pool_base"]) // st2["sb_sz"] < st2["committed_slabs"]).all()
    H.free_batch(ptrs, n, 1)
    torch.cuda.synchronize()
    assert H.stats()["used_chunks"] == 0 and H.status() == 0


def test_payload_through_grow_and_trim(torch_cuda, growing):
    """The private-throughput loop (payload written and read back) before a
    grow, after two grows, after a trim that returned the untouched chunk,
    and after growing again; the trim gives back whole chunks only."""
    torch, H = torch_cuda, growing
    out = torch.zeros(2, dtype=torch.int64, device="cuda")

    def loop(nbytes, n=65536):
        out.zero_()
        H.throughput(out, n, nbytes=nbytes, block=128, nallocs=4, niters=3)
        torch.cuda.synchronize()
        return out.cpu().tolist()

    assert loop(16) == [plain_checksum(65536, 12), 0]
    assert H.grow(256 * MiB) == 256 * MiB
    assert H.grow(1 << 30) == 1 << 30
    torch.cuda.synchronize()
    # 16,384 threads x 4 blocks of 1 KiB: the slabs come lowest first, so the
    # 1 GiB chunk is never touched
    assert loop(1024, 16384) == [plain_checksum(16384, 12), 0]
    before = H.stats()
    released = H.trim()
    after = H.stats()
    assert released >= 1 << 30 and released % before["unit_bytes"] == 0
    assert after["committed_slabs"] == before["committed_slabs"] - released // before["sb_sz"]
    assert after["used_chunks"] == 0 and H.status() == 0
    assert_free_count(H)
    assert loop(16, 32768) == [plain_checksum(32768, 12), 0]
    H.grow(256 * MiB)
    torch.cuda.synchronize()
    assert loop(512) == [plain_checksum(65536, 12), 0]
    assert H.stats()["used_chunks"] == 0 and H.status() == 0
    assert_free_count(H)


def test_trim_keeps_units_with_live_blocks(torch_cuda, growing):
    """Blocks stay live across a trim: only units with no live chunk are
    released, and the live blocks (1,023-character strings) keep their
    contents."""
    torch, H = torch_cuda, growing
    H.grow(256 * MiB)
    H.grow(512 * MiB)
    torch.cuda.synchronize()
    n = 100000
    lens = torch.full((n,), 1023, dtype=torch.int32, device="cuda")
    zeros = torch.zeros_like(lens)
    strs = torch.zeros(n, dtype=torch.int64, device="cuda")
    nfail = torch.zeros(1, dtype=torch.int64, device="cuda")
    bad = torch.zeros(1, dtype=torch.int64, device="cuda")
    H.strings_alloc(n, lens, strs, nfail)
    torch.cuda.synchronize()
    assert nfail.item() == 0
    p = strs.cpu().numpy()
    st = H.stats()
    check_blocks(p, np.full(n, 1024), st["pool_base"], st["pool_bytes"])
    live_units = set(((p - st["pool_base"]) // st["unit_bytes"]).tolist())
    released = H.trim()
    assert released >= 512 * MiB
    st2 = H.stats()
    assert st2["committed_slabs"] * st2["sb_sz"] >= len(live_units) * st2["unit_bytes"]
    H.strings_check(n, strs, lens, zeros, bad)
    torch.cuda.synchronize()
    assert bad.item() == 0
    H.strings_free(n, strs)
    torch.cuda.synchronize()
    assert H.stats()["used_chunks"] == 0 and H.status() == 0
    assert_free_count(H)


def test_grow_and_trim_need_growth_mode(torch_cuda):
    import halloc_b200 as H
    H.init(H.HallocOpts(memory=256 << 20))
    try:
        with pytest.raises(H.HallocError):
            H.grow(1 << 20)
        with pytest.raises(H.HallocError):
            H.trim()
        assert H.stats()["growth"] == 0
        assert H.stats()["committed_slabs"] == H.stats()["nsbs"]
    finally:
        H.shutdown()


def test_trim_closes_surge_sets_first(torch_cuda, growing):
    """A storm on a grown pool opens surge head sets; once everything is
    freed, trim closes them before it looks for wholly free units, so the
    memory their heads held goes back too: what stays backed is at most the
    head and prefetched slab of each size, and the free set's count of its
    slabs still matches its bits."""
    torch, H = torch_cuda, growing
    H.grow(1 << 30)
    torch.cuda.synchronize()
    n = 1 << 20
    out = torch.zeros(2, dtype=torch.int64, device="cuda")
    H.throughput(out, n, nbytes=256, block=256, nallocs=1, niters=2)
    torch.cuda.synchronize()
    assert out.cpu().tolist() == [plain_checksum(n, 2), 0]
    st = assert_free_count(H)
    assert st["n_surge_changes"] > 0 and st["used_chunks"] == 0
    H.trim()
    st = assert_free_count(H)
    assert st["surge_level"] == [0] * 16
    # every slab still backed is free or one of the single head / prefetched
    # slab of a size
    assert st["committed_slabs"] - st["free_slabs"] <= 2 * 16
    assert st["head_slabs"] <= 2 * 16
    assert H.status() & ~H.ST_GROW == 0
