"""Host-side logic of the list-sharded search (harmony_b200.sharding) on CPU:
the reference's list partition, and the gather + master merge across two
gloo ranks, each scanning only its own lists with the CPU oracle (the GPU
scan and the device merge are covered by tests/test_gpu_sharding.py)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from harmony_b200.sharding import gather_results, list_range
from tests.parity import assert_topk_parity


@pytest.mark.parametrize("nlist,world", [(100, 1), (100, 2), (100, 3), (1024, 8), (7, 4), (3, 3)])
def test_list_range_is_the_reference_partition(nlist, world):
    ranges = [list_range(nlist, world, r) for r in range(world)]
    # src/Index.cpp:81-83: worker r (1-based) starts at (r - 1) * (nlist / W); the
    # last one takes the remainder.
    for r, (first, count) in enumerate(ranges):
        assert first == r * (nlist // world)
        assert count == (nlist - first if r == world - 1 else nlist // world)
    assert sum(c for _, c in ranges) == nlist
    assert all(ranges[r][0] + ranges[r][1] == ranges[r + 1][0] for r in range(world - 1))
    with pytest.raises(ValueError):
        list_range(nlist, world, world)


def _data():
    rng = np.random.default_rng(7)
    cent = rng.standard_normal((24, 16)).astype(np.float32) * 4
    x = (cent[rng.integers(0, 24, 3000)] + rng.standard_normal((3000, 16))).astype(np.float32)
    q = (cent[rng.integers(0, 24, 40)] + rng.standard_normal((40, 16))).astype(np.float32)
    return cent, x, q


def _heap_merge(restated, gD, gI, k):
    """The reference master's merge (src/Index.cpp:1327-1341) with the oracle's
    heap: parts in rank order, entries in order, ids by position."""
    world, nq, _ = gD.shape
    D = np.empty((nq, k), np.float32)
    I = np.empty((nq, k), np.int64)
    for q in range(nq):
        vals = gD[:, q, :].reshape(-1)
        hv, hp = restated.heap_topk(vals, k)
        D[q] = hv
        I[q] = np.where(hp >= 0, gI[:, q, :].reshape(-1)[np.maximum(hp, 0)], -1)
    return D, I


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    import oracle
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        restated = oracle.restated()
        cent, x, q = _data()
        ix = restated.add(x, cent)
        k, P = 10, 6
        _, probes = restated.coarse(q, cent, P)
        first, count = list_range(cent.shape[0], world, rank)
        mine = np.where((probes >= first) & (probes < first + count), probes, -1)
        D, I = restated.search_probes(ix, q, mine, k)
        gD, gI = gather_results(torch.from_numpy(D), torch.from_numpy(I))
        assert tuple(gD.shape) == (world, q.shape[0], k)
        Dm, Im = _heap_merge(restated, gD.numpy(), gI.numpy(), k)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), D=Dm, I=Im)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_gather_and_master_merge_equal_one_index(restated, tmp_path, world):
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    cent, x, q = _data()
    ix = restated.add(x, cent)
    De, Ie = restated.search(ix, q, 10, 6)
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npz")
        assert_topk_parity(got["D"], got["I"], De, Ie, lambda qi, i: restated.l2(q[qi], x[i]), f"rank {r}")
