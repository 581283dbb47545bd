"""GPU test of the bounded device waits.

Every mbarrier wait in the tensor-core kernels gives up after a clock budget,
records an error code in a device flag and lets its kernel return; the host
reports HB_ERR_CUDA.  hb_selftest_bounded_wait runs that give-up path on its
own: one thread waits on an mbarrier nothing arrives on, with no copy or MMA
in flight, so the wait must run out, and the index must search correctly
afterwards."""
import ctypes

import numpy as np
import pytest

from harmony_b200 import Index, Precision, SearchMode, datasets, lib

pytestmark = pytest.mark.gpu


def _search(ix, q, k, precision):
    ix.search_params.precision = precision
    D = np.empty((q.shape[0], k), np.float32)
    I = np.empty((q.shape[0], k), np.int64)
    try:
        ix.search(q.shape[0], q, k, D, I)
    finally:
        ix.search_params.precision = Precision.FP32
    return D, I


@pytest.mark.parametrize("budget", [100_000, 2_000_000])
def test_wait_gives_up_within_budget_and_index_stays_usable(budget):
    base, q = datasets.config2(seed=7, nb=20_000, nq=64, ncomp=50)
    ix = Index(128, 64, 8)
    ix.train(base.shape[0], base)
    ix.add(base.shape[0], base)
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.ORIGINAL), "")
    before = {p: _search(ix, q, 10, p) for p in (Precision.FP32, Precision.BF16)}
    L = lib()
    waited = ctypes.c_int64(0)
    rc = L.hb_selftest_bounded_wait(ix._h, budget, ctypes.byref(waited))
    assert rc == 2, rc  # HB_ERR_CUDA
    assert b"gave up waiting (code 99)" in L.hb_last_error()
    # It ran out at its budget (plus one poll), not earlier and not much later.
    assert budget <= waited.value < budget + 1_000_000, waited.value
    after = {p: _search(ix, q, 10, p) for p in (Precision.FP32, Precision.BF16)}
    for p in before:
        assert np.array_equal(before[p][0], after[p][0]) and np.array_equal(before[p][1], after[p][1])
