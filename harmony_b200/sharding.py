"""List-sharded search across GPUs: the reference's DIVIDE_IVF layout
(src/Index.cpp:79-123, 1279-1347) with one process per GPU, NCCL in place of
MPI, and the master's merge run on the device by every rank.

Every rank holds the same trained index (the centroids are shared) and keeps
one contiguous range of lists (``list_range``).  A search runs the full
coarse quantizer on every rank, so all ranks probe the same lists, and each
rank scans only the probed lists it holds.  The per-rank (nq x k) result rows
are all-gathered -- nq x k x 12 bytes per rank, the only exchange -- and merged
with the reference master's heap rule (``Index.merge_topk``), parts in rank
order.  The merged rows hold the same distances as one index holding every
list; among equal distances at the k-th place the ids kept may differ, as they
do between the reference's own modes.

Every rank must make the same calls in the same order with the same queries
and k (the gather is a collective).
"""
from __future__ import annotations

from typing import Tuple


def list_range(nlist: int, world: int, rank: int) -> Tuple[int, int]:
    """(first, count) of the lists rank owns: ranks 0..world-2 take
    nlist // world consecutive lists each and the last rank the rest, the
    partition of src/Index.cpp:81-83 (whose worker ranks count from 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base = nlist // world
    first = rank * base
    count = nlist - first if rank == world - 1 else base
    return first, count


def gather_results(D, I, group=None):
    """All-gather this rank's result rows: D (nq, k) float32 and I (nq, k)
    int64 become (world, nq, k) tensors in rank order."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    D, I = D.contiguous(), I.contiguous()
    if dist.get_backend(group) == "nccl":
        gD = torch.empty((world,) + tuple(D.shape), dtype=D.dtype, device=D.device)
        gI = torch.empty((world,) + tuple(I.shape), dtype=I.dtype, device=I.device)
        dist.all_gather_into_tensor(gD, D, group=group)
        dist.all_gather_into_tensor(gI, I, group=group)
        return gD, gI
    parts_D = [torch.empty_like(D) for _ in range(world)]
    parts_I = [torch.empty_like(I) for _ in range(world)]
    dist.all_gather(parts_D, D, group=group)
    dist.all_gather(parts_I, I, group=group)
    return torch.stack(parts_D), torch.stack(parts_I)


class ListShard:
    """One rank's share of a list-sharded index.

    ``index`` is this rank's copy of the trained, filled index (every rank
    loads the same one, e.g. with ``load_index``); the constructor keeps this
    rank's list range and empties the rest.  ``search`` takes the same
    arguments on every rank and leaves the merged result in D, I on every
    rank.
    """

    def __init__(self, index, group=None):
        import torch.distributed as dist
        self.index = index
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        _, nlist, _, _ = index._info()
        self.first, self.count = list_range(nlist, self.world, self.rank)
        index.retain_lists(self.first, self.count)

    def search(self, n: int, queries, k: int, D, I):
        """Search this rank's lists, gather every rank's rows and merge them into
        D, I (CUDA tensors of shape (n, k)).  Index.preSearch settings and
        search_params apply to the per-rank search."""
        import torch
        dev = D.device
        D_local = torch.empty((n, k), dtype=torch.float32, device=dev)
        I_local = torch.empty((n, k), dtype=torch.int64, device=dev)
        self.index.search(n, queries, k, D_local, I_local)
        gD, gI = gather_results(D_local, I_local, self.group)
        self.index.merge_topk(gD, gI, D, I)
        return D, I
