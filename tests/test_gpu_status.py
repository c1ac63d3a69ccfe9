"""Failure detection without a GPU fault: every device-side wait is bounded
and reports a status bit; misuse is reported instead of corrupting state.
Each failure is made on the host (a lock that nobody releases, a second
free of the same block)."""
import numpy as np
import pytest

from tests.helpers import allocator

pytestmark = pytest.mark.gpu


def batch(torch, H, n, size=16):
    sizes = torch.full((n,), size, dtype=torch.int32, device="cuda")
    ptrs = torch.zeros(n, dtype=torch.int64, device="cuda")
    H.malloc_batch(sizes, n, 1, ptrs)
    torch.cuda.synchronize()
    return ptrs


def test_double_free_is_reported_and_harmless(torch_cuda):
    torch = torch_cuda
    with allocator() as H:
        ptrs = batch(torch, H, 64)
        H.free_batch(ptrs, 64, 1)
        torch.cuda.synchronize()
        assert H.status() == 0
        H.free_batch(ptrs, 64, 1)  # second free of every block
        torch.cuda.synchronize()
        assert H.status() & H.ST_BAD_FREE
        dump = H.dump_state()
        assert (dump["counters"] >> 12 == 0).all() and not dump["bits"].any()
        H.clear_status()
        assert H.status() == 0


def test_head_lock_wait_times_out(torch_cuda):
    """A size's head lock held by a holder that never releases it: the
    first hamalloc of that size must wait for a new head, gives up at the
    wait limit, returns NULL and raises HA_ST_TIMEOUT; the context stays
    usable and allocation works once the lock is free."""
    torch = torch_cuda
    with allocator() as H:
        H.set_wait_limit(20_000)  # 20 ms
        H.debug_set_head_lock(0, True)
        ptrs = batch(torch, H, 64, 16)
        assert not ptrs.cpu().numpy().any()
        assert H.status() & H.ST_TIMEOUT
        # other sizes are unaffected
        other = batch(torch, H, 64, 48)
        assert other.cpu().numpy().all()
        H.debug_set_head_lock(0, False)
        H.clear_status()
        ptrs = batch(torch, H, 64, 16)
        assert ptrs.cpu().numpy().all()
        assert H.status() == 0
        H.free_batch(ptrs, 64, 1)
        H.free_batch(other, 64, 1)
        torch.cuda.synchronize()
        assert H.status() == 0


def test_uninitialised_and_double_init_are_errors(torch_cuda):
    import halloc_b200 as H
    with pytest.raises(H.HallocError):
        H.shutdown()  # not initialised
    H.init()
    try:
        with pytest.raises(H.HallocError):
            H.init()  # already initialised
    finally:
        H.shutdown()


def test_invalid_options_rejected(torch_cuda):
    import halloc_b200 as H
    for bad in (dict(sb_sz_sh=19), dict(sb_sz_sh=25), dict(halloc_fraction=0.0),
                dict(busy_fraction=1.5), dict(memory=0), dict(memory=1 << 20)):
        with pytest.raises(H.HallocError):
            H.init(H.HallocOpts(**bad))
    H.init()
    H.shutdown()
    _ = np
