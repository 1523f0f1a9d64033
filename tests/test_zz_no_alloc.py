"""gtc_count_noalloc: the counting entry point for callers that cannot
allocate device memory when they count.  It must give exactly what gtc_count
gives (integer counts bit-exact, lcc bit-identical), call after call, while
its scratch lives in the library's fixed device array.

Collected last on purpose: if it fails, a run that stops at the first
failure has already run every other test.  It loads everything it needs
itself, so it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest
import torch

from gputrianglecounting_b200 import _lib, graphs as G

pytestmark = pytest.mark.gpu

GTC_ERR_CAPACITY = 8
SCRATCH_BYTES = 32 << 20


def _outputs(n, dev):
    return (torch.full((n,), -7, dtype=torch.int64, device=dev),
            torch.full((n,), -7, dtype=torch.int64, device=dev),
            torch.full((n,), float("nan"), dtype=torch.float64, device=dev),
            torch.full((3,), -7, dtype=torch.int64, device=dev))


def _host(outs):
    torch.cuda.synchronize()
    r, t, lcc, g = (o.cpu().numpy() for o in outs)
    return r, t, lcc.view(np.int64), g


def test_noalloc_matches_gtc_count_twice():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    for make in (lambda: G.rmat(14, 16, 5), lambda: G.erdos_renyi(5000, 20, 6)):
        g = make().to(dev)
        n, nnz = g.n, g.nnz
        for off, bits in ((g.off, 64), (g.off.to(torch.int32), 32)):
            # the existing entry point, with a caller-allocated workspace
            need = ctypes.c_size_t(0)
            assert lib.gtc_workspace_size(n, nnz, bits, 0, ctypes.byref(need)) == 0
            assert need.value <= SCRATCH_BYTES
            ws = torch.empty(need.value, dtype=torch.uint8, device=dev)
            ref = _outputs(n, dev)
            assert lib.gtc_count(off.data_ptr(), bits, g.ind.data_ptr(), n, nnz, 0,
                                 *(o.data_ptr() for o in ref), ws.data_ptr(), ws.numel(),
                                 None) == 0
            want = _host(ref)
            # the allocation-free entry point, twice in a row
            for _ in range(2):
                got = _outputs(n, dev)
                assert lib.gtc_count_noalloc(off.data_ptr(), bits, g.ind.data_ptr(), n, nnz,
                                             0, *(o.data_ptr() for o in got), None) == 0
                have = _host(got)
                for a, b in zip(want, have):
                    assert np.array_equal(a, b)
            # global-count mode as well
            glob = torch.full((3,), -7, dtype=torch.int64, device=dev)
            assert lib.gtc_count_noalloc(off.data_ptr(), bits, g.ind.data_ptr(), n, nnz, 1,
                                         None, None, None, glob.data_ptr(), None) == 0
            torch.cuda.synchronize()
            assert np.array_equal(glob.cpu().numpy(), want[3])


def test_noalloc_rejects_graphs_beyond_its_scratch():
    lib = _lib.load()
    dummy = ctypes.c_void_p(256)   # never dereferenced: rejected before any device work
    assert lib.gtc_count_noalloc(dummy, 64, dummy, 1 << 20, 1 << 24, 0, dummy, None, None,
                                 None, None) == GTC_ERR_CAPACITY
