"""Host-side input generators of the workloads (halloc_b200/workloads.py):
the batched request plan, the Poisson degree table, the phase generator
seeds and the sample inputs have the shapes and distributions their
workloads promise.  CPU only."""
import numpy as np

from halloc_b200.workloads import (CLASS_BYTES, batched_plan, group_seeds, poisson_thresholds,
                                   sample_lengths, sample_points)


def test_batched_plan_frees_every_request_once_within_its_lifetime():
    p = batched_plan(seed=3, nbatch=12, max_batch=1 << 15)
    assert p.batch_start[0] == 0 and p.batch_start[-1] == p.nreq == p.free_start[-1]
    assert (np.diff(p.batch_start.astype(np.int64)) >= 1).all()
    assert np.array_equal(np.sort(p.free_ids), np.arange(p.nreq, dtype=np.uint32))
    batch_of = np.repeat(np.arange(p.nbatch), np.diff(p.batch_start.astype(np.int64)))
    step_of = np.empty(p.nreq, np.int64)
    for s in range(p.nbatch + 1):
        step_of[p.free_ids[p.free_start[s]:p.free_start[s + 1]]] = s
    life = step_of - batch_of
    assert life.min() >= 1 and life.max() <= 8
    # freed no later than the final step
    assert step_of.max() <= p.nbatch


def test_batched_plan_sizes():
    p = batched_plan(seed=1)
    small = p.req_size[p.req_size <= 3072]
    assert set(np.unique(small)) <= set(CLASS_BYTES)
    large = p.req_size[p.req_size > 3072]
    assert large.min() >= 4096 and large.max() <= 65536
    assert abs(len(large) / p.nreq - 0.01) < 0.002
    # geometric over classes with p = 0.3: class 0 takes about 30 %
    assert abs((p.req_size == 16).mean() / 0.99 - 0.3) < 0.01
    assert 1024 <= np.diff(p.batch_start.astype(np.int64)).min()
    assert np.diff(p.batch_start.astype(np.int64)).max() <= 1 << 20
    assert np.array_equal(batched_plan(seed=1).req_size, p.req_size)  # seeded


def test_poisson_thresholds_shape():
    t = poisson_thresholds(16.0)
    assert (np.diff(t.astype(np.int64)) >= 0).all() and t[-1] == 2**32 - 1
    cdf = t.astype(np.float64) / 2**32
    pmf = np.diff(np.concatenate([[0.0], cdf]))
    assert abs((pmf * np.arange(len(t))).sum() - 16.0) < 1e-3


def test_group_seeds():
    s = group_seeds(1000, 32, 7)
    assert s.dtype == np.uint32 and len(s) == 1000
    g = s[: 992].reshape(-1, 32)
    assert (g == g[:, :1]).all()                      # one seed per group
    assert len(np.unique(g[:, 0])) == len(g)          # distinct across groups
    assert np.array_equal(group_seeds(1000, 32, 7), s)
    assert len(np.unique(group_seeds(64, 1, 1))) == 64


def test_sample_inputs():
    pts = sample_points(10000, seed=5)
    assert pts.shape == (10000, 3) and pts.dtype == np.float32
    assert pts.min() >= 0 and pts.max() < 1
    assert np.array_equal(pts * 65536, np.floor(pts * 65536))  # the 1/65536 lattice
    lens = sample_lengths(100, 32, 0, 100, seed=1)
    assert lens.dtype == np.int32 and lens.min() >= 0 and lens.max() <= 100
    assert (lens[:96].reshape(-1, 32) == lens[:96].reshape(-1, 32)[:, :1]).all()
