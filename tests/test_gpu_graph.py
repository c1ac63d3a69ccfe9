"""Random-graph build with doubling hamalloc'd neighbour arrays: the device
edge set, gathered into a CSR, is bit-exact against the CPU-built CSR from
the same seed, and every array is freed afterwards."""
import numpy as np
import pytest

from oracle.graph import graph_csr
from tests.helpers import allocator

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1 << 16, 1 << 20])
def test_graph_build_is_bit_exact(torch_cuda, n):
    import halloc_b200 as H
    from halloc_b200.workloads import poisson_thresholds
    torch = torch_cuda
    seed = 0xC0FFEE
    t = poisson_thresholds(16.0)
    want_off, want_cols = graph_csr(n, seed, t)
    with allocator(memory=1 << 30):
        cdf = torch.from_numpy(t.view(np.int32)).cuda()
        arr = torch.zeros(n, dtype=torch.int64, device="cuda")
        deg = torch.zeros(n, dtype=torch.int32, device="cuda")
        acc = torch.zeros(3, dtype=torch.int64, device="cuda")
        H.graph_build(n, seed, cdf, len(t), arr, deg, acc)
        torch.cuda.synchronize()
        failed, grows, edges = acc.cpu().tolist()
        assert failed == 0 and edges == want_off[-1] and grows > 0
        off = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
        off[1:] = torch.cumsum(deg.to(torch.int64), 0)
        cols = torch.zeros(max(edges, 1), dtype=torch.int32, device="cuda")
        H.graph_gather(n, arr, deg, off, cols)
        torch.cuda.synchronize()
        assert np.array_equal(off.cpu().numpy(), want_off)
        assert np.array_equal(cols[:edges].cpu().numpy().view(np.uint32), want_cols)
        st = H.stats()
        assert st["used_chunks"] == 0 and st["status"] == 0
