"""The mixed-size phase workload: 5 periods of occupancy-driven allocation
rounds and free rounds over 16..256-byte blocks, every block filled with a
hashed pattern and read back before it is freed.  The device's counts and
payload sums must equal the host replay of the same hashed decisions, and
the slab state after an allocation round must equal what the live blocks
imply."""
import numpy as np
import pytest

from oracle.phase import PhaseReplay
from tests.helpers import allocator, check_blocks, expected_slab_state, nibbles_to_chunk_layout

pytestmark = pytest.mark.gpu

SIZES = [16, 24, 32, 48, 64, 96, 128, 192, 256]
THR95 = int(0.95 * 2**32)


def buffers(torch, n, nslots):
    size_set = torch.tensor(SIZES, dtype=torch.int32, device="cuda")
    slots = torch.zeros(nslots * n, dtype=torch.int64, device="cuda")
    slot_sz = torch.zeros(nslots * n, dtype=torch.int32, device="cuda")
    acc = torch.zeros(6, dtype=torch.int64, device="cuda")
    return size_set, slots, slot_sz, acc


@pytest.mark.parametrize("n,memory", [(65536, 256 << 20), (1 << 20, 1 << 30)])
def test_phase_run_matches_replay(torch_cuda, n, memory):
    torch = torch_cuda
    nslots, seed, periods = 4, 0x5EED, 5
    target = int(0.91 * nslots * n)
    want = PhaseReplay(n, nslots, seed, SIZES).run(periods, THR95, THR95, target, 64)
    with allocator(memory=memory) as H:
        size_set, slots, slot_sz, acc = buffers(torch, n, nslots)
        got = H.phase_run(n, nslots, seed, periods, THR95, THR95, target, size_set,
                          len(SIZES), slots, slot_sz, acc)
        assert got["failed"] == 0
        for k in ("alloc_rounds", "free_rounds", "filled", "mallocs", "frees"):
            assert got[k] == want[k], k
        assert got["written_sum"] == want["wsum"] and got["read_sum"] == want["rsum"]
        assert got["written_sum"] == got["read_sum"]
        st = H.stats()
        assert st["used_chunks"] == 0 and st["status"] == 0


def test_phase_state_after_alloc_round(torch_cuda):
    """After an allocation round and a free round, the live blocks are valid
    and the slab state is exactly what they imply."""
    torch = torch_cuda
    n, nslots, seed = 1 << 18, 4, 77
    with allocator(memory=512 << 20) as H:
        size_set, slots, slot_sz, acc = buffers(torch, n, nslots)
        H.phase_round(0, n, nslots, seed, 0, THR95, slots, slot_sz, acc, size_set, len(SIZES))
        H.phase_round(1, n, nslots, seed, 1, THR95 // 2, slots, slot_sz, acc)
        H.phase_round(0, n, nslots, seed, 2, THR95, slots, slot_sz, acc, size_set, len(SIZES))
        torch.cuda.synchronize()
        p = slots.cpu().numpy()
        sz = slot_sz.cpu().numpy().astype(np.int64)
        st = H.stats()
        check_blocks(p, np.where(p != 0, sz, 0), st["pool_base"], st["pool_bytes"],
                     allow_null=True)
        dump = H.dump_state()
        counts, bits, nib = expected_slab_state(p, np.where(p != 0, sz, 0), dump["pool_base"],
                                                dump["sb_sz"], dump["nsbs"])
        assert np.array_equal(dump["counters"] >> 12, counts)
        assert np.array_equal(dump["bits"], bits)
        assert np.array_equal(nibbles_to_chunk_layout(dump["nibbles"], dump["chunk_enc"]), nib)
        a = acc.cpu().numpy()
        assert a[1] == 0 and a[2] - a[3] > 0  # live blocks still hold their payload
        H.phase_round(1, n, nslots, seed, 3, 0xFFFFFFFF, slots, slot_sz, acc)
        torch.cuda.synchronize()
        a = acc.cpu().numpy()
        assert a[2] == a[3] and a[4] == a[5]
        assert H.stats()["used_chunks"] == 0 and H.status() == 0


# ---- the reference's own form (Markov transitions, per-thread generator) ----

def ref_buffers(torch, seeds, n, nallocs):
    states = torch.tensor(seeds.view(np.int32), device="cuda")
    slots = torch.zeros(nallocs * n, dtype=torch.int64, device="cuda")
    ctrs = torch.zeros(n, dtype=torch.int32, device="cuda")
    acc = torch.zeros(4, dtype=torch.int64, device="cuda")
    return states, slots, ctrs, acc


@pytest.mark.parametrize("group,niters,smax", [(1, 1, 256), (32, 1, 256), (1, 3, 256),
                                               (1, 1, 4096)])
def test_phase_ref_tries_match_replay(torch_cuda, group, niters, smax):
    """Try by try: every thread's block count, which of its slots hold a
    block, the blocks' validity and the exact slab state equal the replay
    of the reference's draws (phase-throughput.cu:17-48)."""
    import halloc_b200
    from halloc_b200.workloads import group_seeds
    from oracle.phase import PhaseRefReplay
    torch = torch_cuda
    n, nallocs, ntries, smin = 65536, 4, 10, 16
    probs = halloc_b200.phase_ref_probabilities(0.95, 0.05, 0.91)
    seeds = group_seeds(n, group, 7 + group)
    r = PhaseRefReplay(seeds, nallocs, probs, smin, smax, niters)
    # Blocks above 3 KiB come from CUDA's heap, whose size is fixed by the
    # first in-kernel malloc of the process (an earlier test may have set it
    # smaller than asked here): NULL is allowed for those blocks only.
    with allocator(memory=2 << 30, halloc_fraction=0.5) as H:
        states, slots, ctrs, acc = ref_buffers(torch, seeds, n, nallocs)
        st = H.stats()
        for t in range(ntries):
            H.phase_ref_step(n, nallocs, t, niters, probs, smin, smax, states, slots, ctrs, acc)
            r.step(t)
            torch.cuda.synchronize()
            assert np.array_equal(ctrs.cpu().numpy().astype(np.uint32), r.ctr), t
            p = slots.cpu().numpy()
            sz = r.sizes.reshape(-1).astype(np.int64)
            small = sz <= 3072
            assert np.array_equal((p != 0)[small], (sz != 0)[small]), t
            assert not p[sz == 0].any(), t
            if t in (0, 5, ntries - 1):
                check_blocks(p, sz, st["pool_base"], st["pool_bytes"], allow_null=True)
                dump = H.dump_state()
                counts, bits, nib = expected_slab_state(p, sz, dump["pool_base"], dump["sb_sz"],
                                                        dump["nsbs"])
                assert np.array_equal(dump["counters"] >> 12, counts)
                assert np.array_equal(dump["bits"], bits)
                assert np.array_equal(nibbles_to_chunk_layout(dump["nibbles"],
                                                              dump["chunk_enc"]), nib)
        assert np.array_equal(states.cpu().numpy().view(np.uint32), r.st)
        a = acc.cpu().numpy()
        assert a[0] + a[2] == r.mallocs and a[1] == r.frees
        if smax <= 3072:
            assert a[2] == 0 and a[3] == r.bytes
        H.phase_ref_step(n, nallocs, ntries, niters, probs, smin, smax, states, slots, ctrs,
                         acc, rest=True)
        r.rest()
        torch.cuda.synchronize()
        a = acc.cpu().numpy()
        assert a[1] == r.frees
        assert not slots.any().item() and not ctrs.any().item()
        assert H.stats()["used_chunks"] == 0 and H.status() == 0


def test_phase_ref_run_readme_config(torch_cuda):
    """1,048,576 threads x 4 blocks, sizes 16..256, -f0.95 -F0.05 -e0.91,
    16 tries: the run's counts equal the replay's."""
    import halloc_b200
    from halloc_b200.workloads import group_seeds
    from oracle.phase import PhaseRefReplay
    torch = torch_cuda
    n, nallocs, ntries = 1 << 20, 4, 16
    probs = halloc_b200.phase_ref_probabilities(0.95, 0.05, 0.91)
    seeds = group_seeds(n, 1, 0x5EED)
    r = PhaseRefReplay(seeds, nallocs, probs, 16, 256)
    for t in range(ntries):
        r.step(t)
    r.rest()
    with allocator(memory=1 << 30) as H:
        states, slots, ctrs, acc = ref_buffers(torch, seeds, n, nallocs)
        got = H.phase_ref_run(n, nallocs, ntries, 1, probs, 16, 256, states, slots, ctrs, acc)
        assert got["failed"] == 0
        assert got["mallocs"] == r.mallocs and got["frees"] == r.frees
        assert got["bytes"] == r.bytes
        assert got["kernel_ms"] > 0
        assert H.stats()["used_chunks"] == 0 and H.status() == 0


def test_phase_ref_latency_counts_every_call(torch_cuda):
    """The timed form files one sample per hamalloc and hafree call of the
    tries: the counts equal the replay's, and min <= p50 <= p99 <= max."""
    import halloc_b200
    from halloc_b200.workloads import group_seeds
    from oracle.phase import PhaseRefReplay
    torch = torch_cuda
    n, nallocs, ntries, niters = 65536, 2, 4, 4
    probs = halloc_b200.phase_ref_probabilities(0.95, 0.05, 0.91)
    seeds = group_seeds(n, 32, 5)
    r = PhaseRefReplay(seeds, nallocs, probs, 16, 256, niters)
    for t in range(ntries):
        r.step(t)
    with allocator(memory=512 << 20) as H:
        states, slots, ctrs, acc = ref_buffers(torch, seeds, n, nallocs)
        lat = H.phase_ref_latency(n, nallocs, ntries, niters, probs, 16, 256, states, slots,
                                  ctrs, acc)
        assert lat["malloc"]["n"] == r.mallocs and lat["free"]["n"] == r.frees
        for k in ("malloc", "free"):
            s = lat[k]
            assert 0 < s["min_cycles"] <= s["p50_cycles"] <= s["p99_cycles"]
            assert s["min_cycles"] <= s["avg_cycles"] <= s["max_cycles"]
            assert s["p99_cycles"] <= 2 * s["max_cycles"]
        assert not ctrs.any().item()
        assert H.stats()["used_chunks"] == 0 and H.status() == 0
