"""GPU test of hb_search_noalloc, the search entry point that allocates no
device memory.

It exists for callers that cannot allocate while serving a query -- a process
whose device memory belongs to another allocator or a fixed pool, where a
cudaMalloc can fail or fragment the pool, or a latency-bound process where
cudaFree would synchronise the whole device.  Its results must be those of the
ordinary hb_search (exact FP32 search, ORIGINAL mode), call after call, even
though every call reuses the same fixed scratch array.  Collected last, so a
run that stops at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from tests.parity import assert_topk_parity

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def built():
    import torch
    from harmony_b200 import Index, SearchMode, datasets
    base, q = datasets.config2(seed=31, nb=60_000, nq=300, ncomp=200)
    ix = Index(128, 128, 12)
    ix.train(base.shape[0], base)
    ix.add(base.shape[0], base)
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.ORIGINAL), "")
    qd = torch.from_numpy(q).cuda()
    return ix, q, qd


def _noalloc(ix, qd, k):
    import torch
    from harmony_b200 import lib
    nq = qd.shape[0]
    D = torch.full((nq, k), -1.0, dtype=torch.float32, device="cuda")
    I = torch.full((nq, k), -7, dtype=torch.int64, device="cuda")
    L = lib()
    rc = L.hb_search_noalloc(ix._h, nq, qd.data_ptr(), k, D.data_ptr(), I.data_ptr())
    assert rc == 0, L.hb_last_error().decode()
    return D.cpu().numpy(), I.cpu().numpy()


@pytest.mark.parametrize("k", [10, 100])
def test_noalloc_matches_search_on_two_calls_in_a_row(built, k):
    import torch
    ix, q, qd = built
    nq = qd.shape[0]
    D0 = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    I0 = torch.empty((nq, k), dtype=torch.int64, device="cuda")
    ix.search(nq, qd, k, D0, I0)
    D0, I0 = D0.cpu().numpy(), I0.cpu().numpy()
    first = _noalloc(ix, qd, k)
    second = _noalloc(ix, qd, k)
    for D, I in (first, second):
        assert_topk_parity(D, I, D0, I0, label=f"noalloc k={k}")
        # Same kernels and tie rule as hb_search: identical output.
        assert np.array_equal(D.view(np.uint32), D0.view(np.uint32)) and np.array_equal(I, I0)


def test_noalloc_allocates_nothing(built):
    """The reason the entry point exists: after the first call (which looks the
    fixed array's address up), a call makes no device allocation -- the
    library's own allocation counter and the device's free memory are the same
    before and after it, with the caller's buffers allocated beforehand."""
    import torch
    from harmony_b200 import lib
    ix, q, qd = built
    L = lib()
    k = 10
    nq = qd.shape[0]
    D = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    I = torch.empty((nq, k), dtype=torch.int64, device="cuda")
    assert L.hb_search_noalloc(ix._h, nq, qd.data_ptr(), k, D.data_ptr(), I.data_ptr()) == 0
    torch.cuda.synchronize()
    allocs0 = L.hb_device_allocations()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert L.hb_search_noalloc(ix._h, nq, qd.data_ptr(), k, D.data_ptr(), I.data_ptr()) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert L.hb_device_allocations() == allocs0
    assert free1 == free0
    assert allocs0 > 0  # the counter counts: building the index allocated


def test_noalloc_smaller_call_after_larger_one(built):
    """The scratch keeps the previous call's contents; a smaller search after
    a larger one must not see them."""
    import torch
    ix, q, qd = built
    _noalloc(ix, qd, 100)
    sub = qd[:17].contiguous()
    D, I = _noalloc(ix, sub, 5)
    D0 = torch.empty((17, 5), dtype=torch.float32, device="cuda")
    I0 = torch.empty((17, 5), dtype=torch.int64, device="cuda")
    ix.search(17, sub, 5, D0, I0)
    assert np.array_equal(I, I0.cpu().numpy())


def test_noalloc_rejects_host_pointers_and_oversize(built):
    import torch
    from harmony_b200 import lib
    ix, q, qd = built
    L = lib()
    D = np.empty((q.shape[0], 10), np.float32)
    I = np.empty((q.shape[0], 10), np.int64)
    rc = L.hb_search_noalloc(ix._h, q.shape[0], q.ctypes.data, 10, D.ctypes.data, I.ctypes.data)
    assert rc == 1 and b"device pointers" in L.hb_last_error()
    big = torch.zeros((65000, 128), dtype=torch.float32, device="cuda")
    Db = torch.empty((65000, 10), dtype=torch.float32, device="cuda")
    Ib = torch.empty((65000, 10), dtype=torch.int64, device="cuda")
    rc = L.hb_search_noalloc(ix._h, 65000, big.data_ptr(), 10, Db.data_ptr(), Ib.data_ptr())
    assert rc == 1 and b"scratch" in L.hb_last_error()
