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
