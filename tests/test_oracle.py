"""The oracle (oracle/ha_model.c) against the reference allocator's own code
built for the host (oracle/_ref) and against the golden fixtures generated
from it.  CPU only."""
import os

import numpy as np
import pytest

import oracle
from tests.helpers import load_golden_traces, load_size_tables
from tests.trace_gen import make_trace

SMALL = [16, 24, 32, 48, 64, 96, 128, 192, 256]
ALL = SMALL + [384, 512, 768, 1024, 1536, 2048, 3072]
EDGES = [0, 1, 15, 16, 17, 24, 25, 33, 47, 49, 255, 257, 383, 385, 1025, 3071, 3072, 3073,
         4096]

needs_ref = pytest.mark.skipif(not oracle.reference_available(),
                               reason="reference host build (oracle/_ref) absent")


# ---- known answers --------------------------------------------------------

def test_size_class_rule():
    """bytes -> class: blocks of 2 or 3 units of 8 << k (src/halloc.cu:53-67)."""
    blocks = [(2 if s % 2 == 0 else 3) * (8 << (s // 2)) for s in range(16)]
    for n in range(0, 3073):
        want = next(s for s in range(16) if blocks[s] >= max(n, 16))
        assert oracle.size_id(n) == want, n
    for n in (3073, 4096, 1 << 20):
        assert oracle.size_id(n) == -1


def test_default_size_table_known_values():
    """Spot values of the default table (4 MiB slabs, busy .835, roomy .6,
    sparse .012), computed by hand from src/halloc.cu:363-394."""
    t = oracle.Model().state().size_infos
    # nchunks, chunk_sz(enc), chunk_id, ncib, sparse, hash_step, roomy, busy
    assert t[0].tolist() == [262144, 65540, 0, 1, 3145, 5119, 157286, 218890]
    assert t[1].tolist() == [174760, 196611, 1, 1, 2097, 3407, 104856, 145924]
    assert t[8].tolist() == [16384, 65544, 2, 1, 196, 317, 9830, 13680]
    assert t[15].tolist() == [10920, 196615, 3, 8, 131, 184, 6552, 9118]


def test_first_16b_chunks():
    """A single thread's first 16-B blocks: tickets 0x0B0B0B0B + k hash to
    chunks 96603, 96644, 96645, 96646 of head slab 0 (src/halloc.cu:107-122)."""
    m = oracle.Model()
    offs = [m.malloc(16) for _ in range(4)]
    assert [(o >> 22, (o & ((1 << 22) - 1)) // 16) for o in offs] == [
        (0, 96603), (0, 96644), (0, 96645), (0, 96646)]
    st = m.state()
    assert st.tickets[0] == 0x0B0B0B0B + 4
    assert st.heads[0] == 0 and st.cached[0] == 1


def test_empty_and_null_ops():
    m = oracle.Model()
    assert len(m.run_ops([])) == 0
    m.free(-1)  # hafree(NULL)
    assert m.malloc(0) >= 0  # zero bytes still gets a 16-B block
    assert m.malloc(5000) <= -2  # large -> CUDA heap


# ---- golden fixtures (generated from the reference) ------------------------

def test_golden_size_tables():
    for key, rec in load_size_tables().items():
        m = oracle.Model(memory=rec["memory"], busy=rec["busy"], roomy=rec["roomy"],
                         sparse=rec["sparse"], sb_sz_sh=rec["sb_sz_sh"])
        assert m.state().size_infos.tolist() == rec["table"], key


@pytest.mark.parametrize("case", load_golden_traces(), ids=lambda c: c["name"])
def test_golden_traces(case):
    m = oracle.Model(ref_scan_whole_words=case["ref_scan_whole_words"], **case["opts"])
    res = m.run_ops(case["ops"])
    assert np.array_equal(res, case["res"])
    st = m.state()
    for k in ("tickets", "heads", "cached", "counters", "size_id", "chunk_id", "is_head",
              "chunk_sz", "sets"):
        assert np.array_equal(getattr(st, k), case[k]), k
    from tests.helpers import digest
    assert digest(st.bits) == bytes(case["bits_sha"])
    assert digest(st.nibbles) == bytes(case["nibbles_sha"])


# ---- against the reference build --------------------------------------------

@needs_ref
@pytest.mark.parametrize("sb_sz_sh", [20, 21, 22, 23, 24])
@pytest.mark.parametrize("fr", [(0.835, 0.6, 0.012), (0.745, 0.6, 0.0125), (0.91, 0.5, 0.0125)])
def test_size_tables_vs_reference(sb_sz_sh, fr):
    mem = max(512 << 20, 8 << sb_sz_sh)
    a = oracle.Model(memory=mem, busy=fr[0], roomy=fr[1], sparse=fr[2], sb_sz_sh=sb_sz_sh)
    b = oracle.Reference(memory=mem, busy=fr[0], roomy=fr[1], sparse=fr[2], sb_sz_sh=sb_sz_sh)
    assert a.nsbs == b.nsbs
    assert np.array_equal(a.state().size_infos, b.state().size_infos)


REF_CASES = [
    # (options, trace arguments)
    (dict(memory=512 << 20), dict(n=20000, sizes=[16], pfree=0.45, seed=11)),
    (dict(memory=512 << 20), dict(n=20000, sizes=SMALL, pfree=0.4, seed=12)),
    (dict(memory=512 << 20), dict(n=20000, sizes=ALL + [5000], pfree=0.3, seed=13)),
    (dict(memory=64 << 20, halloc_fraction=0.5, sb_sz_sh=20),
     dict(n=40000, sizes=[3072, 2048, 1536], pfree=0.02, seed=14, drain=0.9, tail=5000)),
    (dict(memory=128 << 20, halloc_fraction=0.5, sb_sz_sh=20),
     dict(n=80000, sizes=[256, 384, 512], pfree=0.2, seed=15, drain=0.9, tail=20000)),
    (dict(memory=128 << 20, halloc_fraction=0.5, sb_sz_sh=21, busy=0.91, roomy=0.5),
     dict(n=80000, sizes=[16, 24, 32], pfree=0.05, seed=16, drain=0.95, tail=20000)),
    (dict(memory=256 << 20, sb_sz_sh=23, halloc_fraction=1.0),
     dict(n=40000, sizes=[16, 3072], pfree=0.2, seed=17)),
    # pools with nsbs % 32 != 0: the reference's scan stops at the last whole
    # set word, the model follows with ref_scan_whole_words
    (dict(memory=64 << 20, sb_sz_sh=20), dict(n=20000, sizes=[3072], pfree=0.05, seed=18)),
    (dict(memory=40 << 20, sb_sz_sh=20), dict(n=5000, sizes=SMALL, pfree=0.3, seed=19)),
    # size-class edges: zero bytes, one byte, either side of every unit
    # boundary up to the 3 KiB limit and past it
    (dict(memory=256 << 20), dict(n=20000, sizes=EDGES, pfree=0.35, seed=20)),
    # other busy / roomy / sparse thresholds on 1 MiB slabs of large blocks
    # (the same traces run on the device in test_gpu_parity)
    (dict(memory=128 << 20, halloc_fraction=0.5, sb_sz_sh=20, busy=0.745, roomy=0.6,
          sparse=0.0125),
     dict(n=40000, sizes=[1536, 2048, 3072], pfree=0.45, seed=106, drain=0.7, tail=5000)),
    (dict(memory=64 << 20, halloc_fraction=0.5, sb_sz_sh=20, busy=0.91, roomy=0.5,
          sparse=0.0125),
     dict(n=40000, sizes=[768, 3072], pfree=0.4, seed=107, drain=0.9, tail=6000)),
]


@needs_ref
@pytest.mark.parametrize("opts,targs", REF_CASES)
def test_model_matches_reference(opts, targs):
    ops = make_trace(**targs)
    r = oracle.Reference(**opts)
    m = oracle.Model(ref_scan_whole_words=r.nsbs % 32 != 0, **opts)
    assert m.nsbs == r.nsbs
    rr, mr = r.run_ops(ops), m.run_ops(ops)
    first = np.nonzero(oracle_norm(rr) != oracle_norm(mr))[0]
    assert len(first) == 0, f"first difference at op {first[0]}"
    assert m.state().diff(r.state()) == []


def oracle_norm(res):
    r = np.array(res, np.int64)
    r[r <= -2] = -2
    return r


@needs_ref
def test_partial_word_deviation_is_only_the_scan():
    """With 48 slabs the reference never uses slabs 32..47; the CUDA
    implementation (and the model without the compat flag) does, so it
    returns NULL later.  Up to the first slab >= 32 they agree."""
    opts = dict(memory=64 << 20, sb_sz_sh=20)
    ops = make_trace(n=20000, sizes=[3072], pfree=0.05, seed=21)
    r = oracle.Reference(**opts)
    fixed = oracle.Model(**opts)
    rr, fr = r.run_ops(ops), fixed.run_ops(ops)
    assert (rr == -1).sum() > (fr == -1).sum()
    used_late = np.nonzero((fr >= 0) & ((fr >> 20) >= 32))[0]
    assert len(used_late) > 0
    k = used_late[0]
    assert np.array_equal(oracle_norm(rr[:k]), oracle_norm(fr[:k]))


@needs_ref
def test_reference_multithreaded_plain_run():
    """The reference code on several host threads at once (the CPU
    baseline) keeps the checksum and never fails at this load."""
    n, iters = 4096, 5
    dt, cs, nf = oracle.cpu_plain_run("reference", n, iters, 16, 4)
    expect = iters * sum(4 * (t - t % 4) + 6 for t in range(n))
    assert nf == 0 and cs == expect and dt > 0


def test_port_and_glibc_plain_runs():
    n, iters = 2048, 3
    expect = iters * sum(4 * (t - t % 4) + 6 for t in range(n))
    for kind in ("port", "glibc"):
        dt, cs, nf = oracle.cpu_plain_run(kind, n, iters, 16, 2)
        assert nf == 0 and cs == expect, kind


# ---- the reference's phase test: transition probabilities and draws ---------

def test_phase_ref_probabilities():
    """-f0.95 -F0.05 -e0.91 (halloc README): p00 = p11 = 1.81 / 1.9,
    p01 = p10 = 0.1 (tst/common/common.cu:311-355, float32)."""
    from halloc_b200 import HallocError, phase_ref_probabilities
    p00, p01, p10, p11 = phase_ref_probabilities(0.95, 0.05, 0.91)
    f32 = np.float32
    num = f32(0.91) + f32(0.95) - f32(0.05)
    assert p00 == float(num / (f32(2) * (f32(1) - f32(0.05))))
    assert p11 == float(num / (f32(2) * f32(0.95)))
    assert abs(p00 - 0.9526316) < 1e-6 and abs(p01 - 0.1) < 1e-6 and abs(p10 - 0.1) < 1e-6
    assert phase_ref_probabilities(1.0, 0.0, 1.0) == (1.0, 1.0, 1.0, 1.0)
    with pytest.raises(HallocError):
        phase_ref_probabilities(0.9, 0.9, 0.9)   # e + f + F > 2
    with pytest.raises(HallocError):
        phase_ref_probabilities(0.9, 0.1, 0.5)   # e < |f - F|


def test_wang_hash_vector_and_scalar_agree():
    from oracle.phase import wang_next, wang_next_scalar
    x = np.random.default_rng(3).integers(0, 1 << 32, 1000, dtype=np.uint64).astype(np.uint32)
    assert wang_next(x).tolist() == [wang_next_scalar(int(v)) for v in x]


@pytest.mark.parametrize("case", load_golden_traces("phase_draws.npz"),
                         ids=lambda c: c["name"])
def test_phase_replay_matches_golden_draws(case):
    """The host replay's decisions, sizes and generator states equal the
    reference's own, try by try (fixtures from tst/common/common.h)."""
    from oracle.phase import PhaseRefReplay
    r = PhaseRefReplay(case["seeds"], case["nallocs"], case["probs"], case["smin"],
                       case["smax"], case["niters"])
    for t in range(case["ntries"]):
        r.step(t)
        assert np.array_equal(r.ctr, case["ctr"][t]), t
        assert np.array_equal(r.sizes, case["sizes"][t]), t
    assert np.array_equal(r.st, case["states"])


@pytest.mark.skipif(not os.path.exists(oracle.REF_DRAWS_SO),
                    reason="reference host build (oracle/_ref) absent")
def test_phase_replay_matches_reference_draws():
    from halloc_b200 import phase_ref_probabilities
    from halloc_b200.workloads import group_seeds
    from oracle.phase import PhaseRefReplay
    probs = phase_ref_probabilities(0.9, 0.1, 0.85)
    seeds = group_seeds(20000, 4, 99)
    ctr, sz, st = oracle.ref_phase_draws(seeds, probs, 16, 1000, 3, 20, 2)
    r = PhaseRefReplay(seeds, 3, probs, 16, 1000, 2)
    for t in range(20):
        r.step(t)
        assert np.array_equal(r.ctr, ctr[t]) and np.array_equal(r.sizes, sz[t]), t
    assert np.array_equal(r.st, st)
