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


_FULL_PLAN = """
import json, sys
import numpy as np
sys.path.insert(0, {root!r})
import torch
import halloc_b200 as H
from halloc_b200.workloads import BatchedRunner, batched_plan
torch.cuda.set_device(0)
plan = batched_plan(seed=1)
counts = np.diff(plan.batch_start.astype(np.int64))
large = plan.req_size > 3072
shape = dict(nbatch=plan.nbatch, nreq=plan.nreq, min=int(counts.min()), max=int(counts.max()),
             large=float(large.mean()), large_min=int(plan.req_size[large].min()),
             large_max=int(plan.req_size[large].max()))
H.init(H.HallocOpts(memory=4 << 30, halloc_fraction=0.5))
r = BatchedRunner(plan, torch)
r.plain(block=256)
torch.cuda.synchronize()
plain = r.acc()
h = r.prepare(block=1024, task_items=8192, graph=True)
r.launch(h)
torch.cuda.synchronize()
persistent = r.acc()
r.release()
st = H.stats()
print("RESULT", json.dumps(dict(shape=shape, plain=plain, persistent=persistent,
                                used=st["used_chunks"], status=H.status())))
H.shutdown()
"""


def test_full_batched_config_both_forms_agree(torch_cuda):
    """The full configuration the benchmark serves: 64 batches of
    log-uniform 1,024..1,048,576 requests (about 10 M), sizes geometric over
    the 16 classes, 1 % large (4..64 KiB, CUDA's heap), lifetimes of 1..8
    batches.  Per-batch launches and the graph-captured persistent kernel
    give the same exact totals: every request allocated and freed once,
    every block still carrying its id, no failure.  It runs in a process of
    its own: the CUDA heap that serves the large requests (2 GiB here) can
    only be sized before the first kernel of a process uses in-kernel
    malloc."""
    import json
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    p = subprocess.run([sys.executable, "-c", _FULL_PLAN.format(root=root)],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    res = json.loads(p.stdout.split("RESULT", 1)[1])
    shape = res["shape"]
    assert shape["nbatch"] == 64
    assert shape["min"] >= 1024 and shape["max"] <= 1 << 20
    assert 0.008 < shape["large"] < 0.012
    assert shape["large_min"] >= 4096 and shape["large_max"] <= 65536
    n = shape["nreq"]
    for acc in (res["plain"], res["persistent"]):
        assert acc["failed"] == 0 and acc["mismatches"] == 0 and acc["late"] == 0
        assert acc["mallocs"] == n and acc["frees"] == n
        assert acc["id_sum"] == n * (n - 1) // 2
    assert res["plain"] == res["persistent"]
    assert res["used"] == 0 and res["status"] == 0
