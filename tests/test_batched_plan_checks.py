"""Argument checks of the batched entry points (include/halloc_c.h), CPU only.

Every case here is rejected before the library touches the device, so the
calls run without a GPU: a plan whose step offsets decrease or run past
nreq, a no-alloc plan beyond its batch or task limits, a task size of 0.
The plan's device buffers are placeholders that a rejected call never
reads, so no case here may ever be one that gets as far as a launch.
"""
import ctypes

import numpy as np
import pytest

import halloc_b200 as H
from halloc_b200.workloads import _CPlan

FAKE = 0x1000  # a non-NULL placeholder for device buffers; never dereferenced


def c_plan(batch_start, free_start, nreq):
    bs = np.ascontiguousarray(batch_start, dtype=np.uint32)
    fs = np.ascontiguousarray(free_start, dtype=np.uint32)
    nbatch = len(bs) - 1
    assert len(fs) == nbatch + 2
    plan = _CPlan(nbatch, nreq, FAKE, FAKE, FAKE, bs.ctypes.data, fs.ctypes.data, FAKE)
    return plan, (bs, fs)  # keep the arrays alive beside the struct


@pytest.fixture(scope="module")
def lib():
    lib = H.load()
    lib.ha_batched_run_noalloc_c.restype = ctypes.c_int
    lib.ha_batched_run_noalloc_c.argtypes = [ctypes.POINTER(_CPlan), ctypes.c_uint32,
                                             ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p]
    lib.ha_batched_prepare_c.restype = ctypes.c_int
    lib.ha_batched_prepare_c.argtypes = [ctypes.POINTER(_CPlan), ctypes.c_uint32,
                                         ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_void_p)]
    lib.ha_batched_plain_c.restype = ctypes.c_int
    lib.ha_batched_plain_c.argtypes = [ctypes.POINTER(_CPlan), ctypes.c_uint32, ctypes.c_void_p]
    return lib


def all_forms(lib, plan, task_items=1024):
    out = ctypes.c_void_p()
    return (lib.ha_batched_run_noalloc_c(ctypes.byref(plan), 256, 0, task_items, None),
            lib.ha_batched_prepare_c(ctypes.byref(plan), 256, 0, task_items, 0,
                                     ctypes.byref(out)),
            lib.ha_batched_plain_c(ctypes.byref(plan), 256, None))


def test_decreasing_batch_offsets_are_rejected(lib):
    plan, _keep = c_plan([0, 10, 5, 20], [0, 0, 5, 10, 20], nreq=20)
    assert all_forms(lib, plan) == (H.HA_EINVAL,) * 3


def test_decreasing_free_offsets_are_rejected(lib):
    plan, _keep = c_plan([0, 10, 20], [0, 8, 4, 20], nreq=20)
    assert all_forms(lib, plan) == (H.HA_EINVAL,) * 3


def test_offsets_past_nreq_are_rejected(lib):
    plan, _keep = c_plan([0, 10, 30], [0, 0, 10, 30], nreq=20)
    assert all_forms(lib, plan) == (H.HA_EINVAL,) * 3
    plan, _keep = c_plan([0, 10, 20], [0, 0, 10, 25], nreq=20)
    assert all_forms(lib, plan) == (H.HA_EINVAL,) * 3


def test_noalloc_rejects_more_than_1024_batches(lib):
    nbatch = 1025
    bs = np.arange(nbatch + 1, dtype=np.uint32)
    fs = np.concatenate([[0, 0], np.arange(1, nbatch + 1)]).astype(np.uint32)
    plan, _keep = c_plan(bs, fs, nreq=nbatch)
    assert lib.ha_batched_run_noalloc_c(ctypes.byref(plan), 256, 0, 1024, None) == H.HA_ERANGE


def test_noalloc_rejects_more_than_65536_tasks(lib):
    # 2 batches of 40,000 requests, freed at the end: with one request per
    # task that is 160,000 tasks
    plan, _keep = c_plan([0, 40000, 80000], [0, 0, 0, 80000], nreq=80000)
    assert lib.ha_batched_run_noalloc_c(ctypes.byref(plan), 256, 0, 1, None) == H.HA_ERANGE


def test_noalloc_rejects_task_size_zero(lib):
    plan, _keep = c_plan([0, 40000, 80000], [0, 0, 0, 80000], nreq=80000)
    assert lib.ha_batched_run_noalloc_c(ctypes.byref(plan), 256, 0, 0, None) == H.HA_EINVAL
