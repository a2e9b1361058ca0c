"""Multi-process plumbing of the weak-scaling path (one process per GPU, torch.distributed): the split of science
segments over ranks, the max-over-ranks step time and the gather of the ranks' peak tables at the end.

(detector, segment) units are independent in the reference (the loop at fp_filter.py:728-730) and so are science
segments here: each rank filters its own share against the full bank, and the only exchange is one gather of the
consolidated tables (host records, gathered as objects). The step time of a multi-rank run is the maximum over the
ranks of each rank's device-timed step."""
import heapq

import numpy as np
import torch
import torch.distributed as dist


def world_rank():
    """(world size, rank); (1, 0) when no process group is initialised."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def shard_by_length(lengths, world):
    """Indices of the segments each rank filters: longest first, each to the rank with the least work so far (ties to
    the lower rank). Deterministic; every segment goes to exactly one rank; returns world lists in ascending order."""
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    order = sorted(range(len(lengths)), key=lambda i: (-int(lengths[i]), i))
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(lengths[i]), r))
    return [sorted(o) for o in out]


def max_over_ranks(value, device=None):
    """The maximum of a float over the ranks (all_reduce MAX on the process group's device)."""
    w, _ = world_rank()
    if w == 1:
        return float(value)
    if device is None:
        device = 'cuda' if dist.get_backend() == 'nccl' else 'cpu'
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_tables(tables, dst=0):
    """Every rank's {segment index: table} merged on rank dst (None elsewhere); the tables are host numpy records."""
    w, r = world_rank()
    if w == 1:
        return dict(tables)
    host = {int(k): {f: np.asarray(v) for f, v in t.items()} for k, t in tables.items()}
    got = [None] * w if r == dst else None
    dist.gather_object(host, got, dst=dst)
    if r != dst:
        return None
    merged = {}
    for part in got:
        for k, t in part.items():
            assert k not in merged, 'segment %d filtered on two ranks' % k
            merged[k] = t
    return merged
