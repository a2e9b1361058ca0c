"""The multi-rank host path (gwb200.dist) on two gloo ranks on the CPU: the segment split covers every segment once and
balances the work, the step time is the maximum over ranks, and the gathered tables equal a one-process run (each
rank consolidating its own segments' peaks with the oracle)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from gwb200 import dist as gd
from oracle import consolidate as oc


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _segments(seed=5):
    """Peaks of 7 segments of different lengths: (lengths, per segment (ti, snr, chi, dof))."""
    rng = np.random.default_rng(seed)
    lengths = rng.integers(64, 4096, 7) * 2048
    segs = []
    for n in lengths:
        k = int(rng.integers(100, 3000))
        ti = rng.integers(0, n, k).astype(np.int64)
        snr = np.round(rng.uniform(3.9, 9.0, k), 2).astype(np.float32)
        dof = np.where(rng.uniform(size=k) < 0.5, 30, 0).astype(np.int32)
        chi = np.where(dof > 0, np.round(rng.uniform(0, 80, k), 1), 0).astype(np.float32)
        segs.append((ti, snr, chi, dof))
    return lengths, segs


def _table(i, seg, gps):
    ti, snr, chi, dof = seg
    t = gps + ti / 2048.0
    keep, _ = oc.consolidate(snr, chi, dof, t, [], gps, 2048.0, 4.0, 1.072, 5, 5.0)
    return oc.peak_table(np.full(keep.sum(), i), t[keep], snr[keep], np.zeros(keep.sum(), np.float32),
                         np.ones(keep.sum()), dof[keep] > 0, chi[keep], dof[keep], [], None)


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        lengths, segs = _segments()
        mine = gd.shard_by_length(lengths, world)[rank]
        tables = {i: _table(i, segs[i], 1e9 + 1e5 * i) for i in mine}
        ms = gd.max_over_ranks(10.0 + rank)
        merged = gd.gather_tables(tables)
        q.put((rank, mine, ms, None if merged is None else {k: {f: v.tolist() for f, v in t.items()}
                                                            for k, t in merged.items()}))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_time_and_gather():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        rank, mine, ms, merged = q.get(timeout=120)
        out[rank] = (mine, ms, merged)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    lengths, segs = _segments()
    shards = [out[0][0], out[1][0]]
    assert sorted(shards[0] + shards[1]) == list(range(len(lengths)))
    loads = [int(np.sum(lengths[s])) for s in shards]
    assert abs(loads[0] - loads[1]) <= int(lengths.max())
    assert out[0][1] == out[1][1] == 11.0
    assert out[1][2] is None
    merged = out[0][2]
    assert sorted(merged) == list(range(len(lengths)))
    for i in range(len(lengths)):
        ref = _table(i, segs[i], 1e9 + 1e5 * i)
        for f, v in ref.items():
            assert np.array_equal(np.asarray(merged[i][f]), v), (i, f)


@pytest.mark.parametrize('world', [1, 2, 3, 8])
def test_shard_by_length_covers_and_balances(world):
    rng = np.random.default_rng(world)
    lengths = rng.integers(1, 1000, 50)
    sh = gd.shard_by_length(lengths, world)
    assert sorted(i for s in sh for i in s) == list(range(50))
    loads = [int(lengths[s].sum()) for s in sh]
    assert max(loads) - min(loads) <= int(lengths.max())
