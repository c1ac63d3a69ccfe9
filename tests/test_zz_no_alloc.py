"""The batched persistent form that allocates nothing
(ha_batched_run_noalloc_c).

It exists for callers that cannot call cudaMalloc: programs that have given
all device memory to their own pool, where cudaMalloc would fail, and
latency-bound serving loops that must not call cudaMalloc/cudaFree because
those calls synchronise the whole device.  It keeps its scratch in one fixed
device array instead, so it has to give exactly what the allocating entry
point gives -- here on two calls in a row, since every call reuses the array
the previous call left behind.  This file is collected last so that, if it
fails, a run that stops at the first failure has already run every other
test; it also passes alone in a fresh process.
"""
import pytest

from tests.helpers import allocator

pytestmark = pytest.mark.gpu


def test_noalloc_entry_point_matches_allocating_one(torch_cuda):
    import halloc_b200 as H
    from halloc_b200.workloads import BatchedRunner, batched_plan
    torch = torch_cuda
    plan = batched_plan(seed=5, nbatch=10, max_batch=1 << 14)
    with allocator(memory=1 << 30, halloc_fraction=0.5):
        runner = BatchedRunner(plan, torch)
        h = runner.prepare(block=256, task_items=1024, graph=False)
        runner.launch(h)
        torch.cuda.synchronize()
        want = runner.verify()
        runner.release()
        for _ in range(2):
            assert runner.run_noalloc(block=256, task_items=1024) == H.HA_OK
            torch.cuda.synchronize()
            got = runner.verify()
            assert got == want  # integer counts and id sums: exact
        assert H.stats()["used_chunks"] == 0 and H.status() == 0


def test_noalloc_entry_point_rejects_plans_beyond_its_limit(torch_cuda):
    import halloc_b200 as H
    from halloc_b200.workloads import BatchedRunner, batched_plan
    torch = torch_cuda
    plan = batched_plan(seed=6, nbatch=4, min_batch=40000, max_batch=40000)
    with allocator(memory=1 << 30, halloc_fraction=0.5):
        runner = BatchedRunner(plan, torch)
        # one request per task: 2 x 160,000 tasks > 65,536
        assert runner.run_noalloc(block=256, task_items=1) == H.HA_ERANGE
        assert runner.run_noalloc(block=256, task_items=4096) == H.HA_OK
        torch.cuda.synchronize()
        runner.verify()


def test_noalloc_entry_point_with_one_task_per_step(torch_cuda):
    """A task size near 2^32 makes each non-empty step one task; the task
    table is counted in 64 bits on the host and on the device, so both
    entry points give the same run as with small tasks."""
    import halloc_b200 as H
    from halloc_b200.workloads import BatchedRunner, batched_plan
    torch = torch_cuda
    plan = batched_plan(seed=7, nbatch=6, max_batch=1 << 12)
    with allocator(memory=1 << 30, halloc_fraction=0.5):
        runner = BatchedRunner(plan, torch)
        h = runner.prepare(block=256, task_items=1024, graph=False)
        runner.launch(h)
        torch.cuda.synchronize()
        want = runner.verify()
        runner.release()
        h = runner.prepare(block=256, task_items=0xFFFFFFF0, graph=False)
        runner.launch(h)
        torch.cuda.synchronize()
        assert runner.verify() == want
        runner.release()
        assert runner.run_noalloc(block=256, task_items=0xFFFFFFF0) == H.HA_OK
        torch.cuda.synchronize()
        assert runner.verify() == want
        assert H.stats()["used_chunks"] == 0 and H.status() == 0
