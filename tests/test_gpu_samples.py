"""The reference's sample programs as workloads: grid-points (every point's
16-byte list node in its grid cell, checked cell by cell against the host
binning) and add-strings (every concatenation checked byte by byte), both
ending with the pool empty."""
import numpy as np
import pytest

from halloc_b200.workloads import sample_lengths, sample_points
from oracle.samples import grid_expect
from tests.helpers import allocator

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,ncells,pre", [(10000, 8, False), (1000000, 32, False),
                                          (200000, 7, False), (200000, 32, True)])
def test_grid_points_cells_match_host(torch_cuda, n, ncells, pre):
    torch = torch_cuda
    pts = sample_points(n, seed=n + ncells)
    want_count, want_hsum = grid_expect(pts, ncells)
    with allocator(memory=512 << 20) as H:
        d_pts = torch.tensor(pts, device="cuda")
        grid = torch.zeros(ncells ** 3, dtype=torch.int64, device="cuda")
        nodes = torch.zeros(2 * n, dtype=torch.int64, device="cuda") if pre else None
        nfail = torch.zeros(1, dtype=torch.int64, device="cuda")
        H.grid_insert(n, ncells, d_pts, grid, nfail, pre_nodes=nodes)
        count = torch.zeros(ncells ** 3, dtype=torch.int32, device="cuda")
        hsum = torch.zeros(ncells ** 3, dtype=torch.int64, device="cuda")
        H.grid_check(ncells, grid, count, hsum)
        torch.cuda.synchronize()
        assert nfail.item() == 0
        assert np.array_equal(count.cpu().numpy().view(np.uint32), want_count)
        assert np.array_equal(hsum.cpu().numpy().view(np.uint64), want_hsum)
        st = H.stats()
        assert st["used_chunks"] == (0 if pre else n)
        H.grid_free(ncells, grid, pre_nodes=pre)
        torch.cuda.synchronize()
        assert not grid.any().item()
        assert H.stats()["used_chunks"] == 0 and H.status() == 0


@pytest.mark.parametrize("n,lo,hi", [(1000000, 31, 31), (100000, 0, 100), (5000, 0, 3100)])
def test_add_strings_concatenations(torch_cuda, n, lo, hi):
    """1,000,000 strings of 31 characters (the sample's sizes), then random
    lengths in groups of 32, up to lengths whose blocks come from CUDA's
    heap."""
    torch = torch_cuda
    la = sample_lengths(n, 32, lo, hi, seed=1)
    lb = sample_lengths(n, 32, lo, hi, seed=2)
    with allocator(memory=1 << 30, halloc_fraction=0.5) as H:
        d_la = torch.tensor(la, device="cuda")
        d_lb = torch.tensor(lb, device="cuda")
        a, b, c = (torch.zeros(n, dtype=torch.int64, device="cuda") for _ in range(3))
        nfail = torch.zeros(1, dtype=torch.int64, device="cuda")
        bad = torch.zeros(1, dtype=torch.int64, device="cuda")
        H.strings_alloc(n, d_la, a, nfail)
        H.strings_alloc(n, d_lb, b, nfail)
        H.strings_check(n, a, d_la, torch.zeros_like(d_la), bad)
        H.strings_concat(n, c, a, b, nfail)
        H.strings_check(n, c, d_la, d_lb, bad)
        torch.cuda.synchronize()
        assert nfail.item() == 0 and bad.item() == 0
        for s in (a, b, c):
            H.strings_free(n, s)
        torch.cuda.synchronize()
        assert not c.any().item()
        assert H.stats()["used_chunks"] == 0 and H.status() == 0
