"""Batched request stream served by per-batch launches and by one persistent
kernel (plain and graph-replayed): every request is allocated and freed
exactly once, every block still holds its request id when freed, and the
pool is empty afterwards."""
import numpy as np
import pytest

from tests.helpers import allocator

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_plan():
    from halloc_b200.workloads import batched_plan
    return batched_plan(seed=3, nbatch=12, max_batch=1 << 15)


def test_batched_plain_form(torch_cuda, small_plan):
    from halloc_b200.workloads import BatchedRunner
    torch = torch_cuda
    with allocator(memory=1 << 30, halloc_fraction=0.5) as H:
        r = BatchedRunner(small_plan, torch)
        r.plain(block=256)
        torch.cuda.synchronize()
        r.verify()
        assert H.stats()["used_chunks"] == 0 and H.status() == 0


@pytest.mark.parametrize("graph,block,items", [(True, 256, 2048), (False, 128, 256),
                                               (True, 64, 64)])
def test_batched_persistent_form(torch_cuda, small_plan, graph, block, items):
    from halloc_b200.workloads import BatchedRunner
    torch = torch_cuda
    with allocator(memory=1 << 30, halloc_fraction=0.5) as H:
        r = BatchedRunner(small_plan, torch)
        h = r.prepare(block=block, task_items=items, graph=graph)
        for _ in range(2):  # a replay starts from the state the last run left
            r.launch(h)
            torch.cuda.synchronize()
            r.verify()
            assert H.stats()["used_chunks"] == 0
        r.release()
        assert H.status() == 0


def test_full_batched_config_both_forms_agree(torch_cuda):
    """The full configuration the benchmark serves: 64 batches of
    log-uniform 1,024..1,048,576 requests (about 10 M), sizes geometric over
    the 16 classes, 1 % large (4..64 KiB, CUDA's heap), lifetimes of 1..8
    batches.  Per-batch launches and the graph-captured persistent kernel
    give the same exact totals: every request allocated and freed once,
    every block still carrying its id, no failure."""
    from halloc_b200.workloads import BatchedRunner, batched_plan
    torch = torch_cuda
    plan = batched_plan(seed=1)
    assert plan.nbatch == 64
    counts = np.diff(plan.batch_start.astype(np.int64))
    assert counts.min() >= 1024 and counts.max() <= 1 << 20
    large = plan.req_size > 3072
    assert 0.008 < large.mean() < 0.012
    assert plan.req_size[large].min() >= 4096 and plan.req_size[large].max() <= 65536
    with allocator(memory=4 << 30, halloc_fraction=0.5) as H:
        r = BatchedRunner(plan, torch)
        r.plain(block=256)
        torch.cuda.synchronize()
        plain = r.verify()
        h = r.prepare(block=256, task_items=2048, graph=True)
        r.launch(h)
        torch.cuda.synchronize()
        persistent = r.verify()
        r.release()
        assert plain == persistent
        assert plain["mallocs"] == plan.nreq and plain["failed"] == 0
        assert H.stats()["used_chunks"] == 0 and H.status() == 0
