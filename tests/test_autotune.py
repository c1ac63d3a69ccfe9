"""The autotuner of the batched persistent form (halloc_b200/autotune.py).

CPU: the sweep order with a stub timer -- slab size x busy fraction first
(as the reference's settings experiment sweeps them,
tst/exp/settings/exp-run.pl:27-44), then block x hash scale at the best of
those, then head slabs at the best so far; `best` is the fastest point.
GPU: a reduced sweep on a small plan, every point verified, the knobs back
at the reference's values afterwards.
"""
import numpy as np
import pytest

from halloc_b200 import autotune as A


def test_sweep_order_and_best_with_a_stub_timer():
    calls = []

    def fake(torch, runner, opts, block, items, hash_pct, reps, nheads):
        calls.append((opts.sb_sz_sh, opts.busy_fraction, block, hash_pct, nheads))
        # fastest: 4-MiB slabs, busy 0.745, block 512, hash 200, 2 heads
        ms = 10.0
        ms -= 1.0 if opts.sb_sz_sh == 22 else 0.0
        ms -= 0.5 if opts.busy_fraction == 0.745 else 0.0
        ms -= 0.25 if block == 512 else 0.0
        ms -= 0.125 if hash_pct == 200 else 0.0
        ms -= 0.0625 if nheads == 2 else 0.0
        return ms

    out = A.autotune(None, None, memory=1 << 30, halloc_fraction=0.5, reps=1, time_point=fake)
    stage1 = [(sh, b, 256, 100, 1) for sh in A.SLAB_SHIFTS for b in A.BUSY_FRACTIONS]
    stage2 = [(22, 0.745, blk, hp, 1) for blk in A.BLOCKS for hp in A.HASH_PCTS
              if (blk, hp) != (256, 100)]
    stage3 = [(22, 0.745, 512, 200, nh) for nh in A.HEADS]
    assert calls == stage1 + stage2 + stage3
    assert len(out["points"]) == len(calls)
    best = out["best"]
    assert (best["sb_sz_sh"], best["busy"], best["block"], best["hash_pct"],
            best["nheads"]) == (22, 0.745, 512, 200, 2)
    assert best["ms"] == min(p["ms"] for p in out["points"])
    assert all("nheads" in p for p in out["points"])


def test_sparse_fraction_follows_busy():
    seen = {}

    def fake(torch, runner, opts, block, items, hash_pct, reps, nheads):
        seen[opts.busy_fraction] = opts.sparse_fraction
        return 1.0

    A.autotune(None, None, memory=1 << 30, halloc_fraction=0.5, time_point=fake,
               slab_shifts=(22,), blocks=(256,), hash_pcts=(100,), heads=())
    assert seen == {0.745: 0.012, 0.835: 0.012, 0.91: 0.0125}


@pytest.mark.gpu
def test_reduced_sweep_on_a_small_plan(torch_cuda):
    import halloc_b200 as H
    from halloc_b200.workloads import BatchedRunner, batched_plan
    from tests.helpers import allocator
    torch = torch_cuda
    plan = batched_plan(seed=11, nbatch=8, max_batch=1 << 13)
    runner = BatchedRunner(plan, torch)
    verified = []
    real_verify = runner.verify

    def counting_verify(acc=None):
        verified.append(real_verify(acc))
        return verified[-1]

    runner.verify = counting_verify
    # 512 MiB of 2-MiB slabs: room for two head sets per size (4 slabs each)
    out = A.autotune(torch, runner, memory=1 << 30, halloc_fraction=0.5, reps=1,
                     slab_shifts=(21, 22), busy_fractions=(0.835,), blocks=(128, 256),
                     hash_pcts=(100,), heads=(2,))
    # 2 + 1 + 1 points, each verified after its warm-up launch and its replay
    assert len(out["points"]) == 4
    assert len(verified) == 2 * 4
    assert all(p["ms"] > 0 for p in out["points"])
    assert out["best"]["ms"] == min(p["ms"] for p in out["points"])
    # the knobs are back at the reference's values: the default size table
    # (hash steps of the reference rule) and a single head per size
    with allocator(memory=512 << 20) as H2:
        infos = H2.dump_state()["size_infos"]
        assert int(infos[0][5]) == 5119 and int(infos[8][5]) == 317  # Appendix-A hash steps
        d_sizes = torch.full((32768,), 16, dtype=torch.int32, device="cuda")
        ptrs = torch.zeros(32768, dtype=torch.int64, device="cuda")
        H2.malloc_batch(d_sizes, 32768, 1, ptrs)
        torch.cuda.synchronize()
        assert H2.stats()["head_slabs"] <= 2
        H2.free_batch(ptrs, 32768, 1)
        torch.cuda.synchronize()
        assert H2.status() == 0
    assert np.asarray(plan.req_size).size == plan.nreq
