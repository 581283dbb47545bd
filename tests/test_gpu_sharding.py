"""GPU tests of list sharding on one B200.  The ranks' shards are separate
Index objects searched one after another (no kernel waits on another), their
rows stacked as the all-gather stacks them, and merged on the device; a
one-rank NCCL group runs the ListShard path itself."""
import datetime
import socket

import numpy as np
import pytest
import torch

from harmony_b200 import HarmonyError, Index, Precision, SearchMode, datasets
from harmony_b200.sharding import ListShard, list_range
from tests.parity import FLT_MAX, assert_topk_parity

pytestmark = pytest.mark.gpu

NLIST = 64


@pytest.fixture(scope="module")
def saved(tmp_path_factory):
    base, q = datasets.config2(seed=81, nb=60_000, nq=300, ncomp=200)
    ix = Index(128, NLIST, 8)
    ix.train(base.shape[0], base)
    ix.add(base.shape[0], base)
    p = str(tmp_path_factory.mktemp("shard") / "full.index")
    ix.save_index(p)
    return base, q, p


def load(p):
    ix = Index()
    ix.load_index(p)
    ix.preSearch(0, 0, 0, 0, 0, Index.Param(mode=SearchMode.ORIGINAL), "")
    return ix


def search_dev(ix, q, k, nprobe, precision=Precision.FP32):
    ix.nprobe = nprobe
    ix.search_params.precision = precision
    D = torch.empty((q.shape[0], k), dtype=torch.float32, device="cuda")
    I = torch.empty((q.shape[0], k), dtype=torch.int64, device="cuda")
    try:
        ix.search(q.shape[0], torch.from_numpy(q).cuda(), k, D, I)
    finally:
        ix.search_params.precision = Precision.FP32
    return D, I


@pytest.mark.parametrize("world", [2, 3, 8])
def test_sharded_search_equals_one_index(saved, restated, world):
    base, q, p = saved
    full = load(p)
    sizes = full.list_sizes()
    k = 10
    De, Ie = search_dev(full, q, k, 8)
    parts = []
    for r in range(world):
        ix = load(p)
        first, count = list_range(NLIST, world, r)
        ix.retain_lists(first, count)
        got = ix.list_sizes()
        assert np.array_equal(got[first:first + count], sizes[first:first + count])
        assert got.sum() == sizes[first:first + count].sum()
        parts.append(search_dev(ix, q, k, 8))
    gD = torch.stack([d for d, _ in parts]).contiguous()
    gI = torch.stack([i for _, i in parts]).contiguous()
    D = torch.empty_like(De)
    I = torch.empty_like(Ie)
    full.merge_topk(gD, gI, D, I)
    assert_topk_parity(D.cpu().numpy(), I.cpu().numpy(), De.cpu().numpy(), Ie.cpu().numpy(),
                       lambda qi, i: restated.l2(q[qi], base[i]), f"world {world}")
    # BF16 shards: every shard's bounded scan returns its exact rows, so the
    # merged rows are the exact merge's.
    parts = []
    for r in range(world):
        ix = load(p)
        ix.retain_lists(*list_range(NLIST, world, r))
        parts.append(search_dev(ix, q, k, 8, Precision.BF16))
    full.merge_topk(torch.stack([d for d, _ in parts]).contiguous(), torch.stack([i for _, i in parts]).contiguous(),
                    D, I)
    assert_topk_parity(D.cpu().numpy(), I.cpu().numpy(), De.cpu().numpy(), Ie.cpu().numpy(),
                       lambda qi, i: restated.l2(q[qi], base[i]), f"bf16 world {world}")


def test_merge_is_the_reference_master_heap(saved, restated):
    """Device merge against the oracle's heap (pinned to the reference's
    heap.hpp): parts in order, strict admission, heap sort -- bit for bit,
    ids included, with many exact ties."""
    base, q, p = saved
    ix = load(p)
    rng = np.random.default_rng(4)
    for parts, nq, k in ((3, 50, 10), (1, 7, 1), (8, 20, 33), (2, 5, 100)):
        vals = np.round(rng.uniform(0, 20, (parts, nq, k))).astype(np.float32)  # coarse grid: many ties
        vals[0, :, -2:] = FLT_MAX  # padding rows as searches leave them
        ids = np.arange(parts * nq * k, dtype=np.int64).reshape(parts, nq, k)
        D = torch.empty((nq, k), dtype=torch.float32, device="cuda")
        I = torch.empty((nq, k), dtype=torch.int64, device="cuda")
        ix.merge_topk(torch.from_numpy(vals).cuda(), torch.from_numpy(ids).cuda(), D, I)
        Dg, Ig = D.cpu().numpy(), I.cpu().numpy()
        for qi in range(nq):
            hv, hp = restated.heap_topk(vals[:, qi, :].reshape(-1), k)
            want_i = np.where(hp >= 0, ids[:, qi, :].reshape(-1)[np.maximum(hp, 0)], -1)
            assert np.array_equal(Dg[qi].view(np.uint32), hv.view(np.uint32)), (parts, nq, k, qi)
            assert np.array_equal(Ig[qi], want_i), (parts, nq, k, qi)


def test_retain_lists_edges(saved):
    base, q, p = saved
    ix = load(p)
    ix.retain_lists(5, 0)  # nothing kept: every result is padding
    assert ix.list_sizes().sum() == 0
    D, I = search_dev(ix, q[:4], 5, 8)
    assert (I.cpu().numpy() == -1).all() and (D.cpu().numpy() == FLT_MAX).all()
    ix = load(p)
    with pytest.raises(HarmonyError):
        ix.retain_lists(60, 10)
    full = load(p)
    ix.retain_lists(0, NLIST)  # everything kept: the same index
    for a, b in zip(search_dev(ix, q, 10, 8), search_dev(full, q, 10, 8)):
        assert torch.equal(a, b)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_list_shard_one_rank_nccl(saved):
    import torch.distributed as dist
    base, q, p = saved
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        shard = ListShard(load(p))
        assert (shard.first, shard.count) == (0, NLIST)
        shard.index.nprobe = 8
        D = torch.empty((q.shape[0], 10), dtype=torch.float32, device="cuda")
        I = torch.empty((q.shape[0], 10), dtype=torch.int64, device="cuda")
        shard.search(q.shape[0], torch.from_numpy(q).cuda(), 10, D, I)
        De, Ie = search_dev(load(p), q, 10, 8)
        # One part re-sorted by the master's heap: the same distances; equal
        # distances may come out in another order.
        assert torch.equal(D, De)
        assert_topk_parity(D.cpu().numpy(), I.cpu().numpy(), De.cpu().numpy(), Ie.cpu().numpy())
    finally:
        dist.destroy_process_group()
