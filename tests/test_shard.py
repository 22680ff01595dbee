"""Sharding one image by first-level child (fastsar_b200.shard), on the CPU: the partition, the restricted plans, and
a world-size-2 run over gloo in which the oracle stands in for the per-rank former (each rank forms its children's
tiles with the oracle's driver, fastsar/ffbp_cpu.py:278-291's first-level groups), the ranks' images are summed by
an all-reduce, and the result equals the single-process image exactly."""
import os
import socket

import numpy as np
import pytest

from fastsar_b200 import plan as P_
from fastsar_b200 import shard
from fastsar_b200.sim import Collect


def test_child_ranges_cover_every_child_once():
    for G in (1, 7, 64, 56):
        for world in range(1, min(G, 9) + 1):
            r = shard.child_ranges(G, world)
            assert len(r) == world and r[0][0] == 0 and r[-1][1] == G
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            sizes = [b - a for a, b in r]
            assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
    with pytest.raises(ValueError):
        shard.child_ranges(4, 0)


def _plan(golden, nlev=3):
    g = golden('image_small')
    fmin, df, K = g['scal']
    col = Collect(fmin=float(fmin), df=float(df), K=int(K), ant=g['ant'], res=0.5)
    return g, P_.make_plan(col, 128, 128, 0.5, 0.5, T=16, nlev=nlev, pmax=0.4, e1=(1.0, 0.0, 0.0), e2=(0.0, 1.0, 0.0))


@pytest.mark.parametrize('nlev', [2, 3])
def test_restricted_plans_partition_the_tiles(golden, nlev):
    """The restricted plans' final tiles are disjoint, together the whole plan's, in its order; every level's parents
    are the descendants of the rank's children."""
    _, plan = _plan(golden, nlev)
    G = plan['levels'][0]['C']
    firsts, cens = [], []
    for g0, g1 in shard.child_ranges(G, 3):
        sub = shard.restrict_plan(plan, g0, g1)
        assert sub['levels'][0]['C'] == g1 - g0 and sub['partial']
        np.testing.assert_array_equal(sub['levels'][0]['cen'][0], plan['levels'][0]['cen'][0, g0:g1])
        B = g1 - g0
        for l in range(1, nlev):
            assert sub['levels'][l]['ref'].shape[0] == B
            B *= plan['levels'][l]['C']
        assert sub['final']['cen'].shape[0] == B
        firsts.append(sub['final']['first'])
        cens.append(sub['final']['cen'])
    np.testing.assert_array_equal(np.concatenate(firsts), plan['final']['first'])
    np.testing.assert_array_equal(np.concatenate(cens), plan['final']['cen'])
    with pytest.raises(ValueError):
        shard.restrict_plan(plan, 3, 3)


def _rank(rank, world, port, S, plan, coll, q):
    import torch
    import torch.distributed as dist
    import oracle as O
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        g0, g1 = shard.child_ranges(plan['levels'][0]['C'], world)[rank]
        img = O.make_ffbp(plan, coll, 'port')(S, ng=2, children=range(g0, g1))
        t = torch.from_numpy(np.ascontiguousarray(img))
        dist.all_reduce(t)
        if rank == 0:
            q.put(t.numpy())
    finally:
        dist.destroy_process_group()


def test_two_ranks_sum_to_the_whole_image(golden, oracle_lib):
    import torch.multiprocessing as mp
    g, plan = _plan(golden, 3)
    coll = P_.collection_arrays(plan, g['ant'])
    from fastsar_b200.api import _window
    wp, wk = _window(*g['S'].shape)
    S = (g['S'] * (wp[:, None] * wk[None, :]).astype(np.float32)).astype(np.complex64)
    whole = oracle_lib.make_ffbp(plan, coll, 'port')(S, ng=2)
    with socket.socket() as s_:
        s_.bind(('127.0.0.1', 0))
        port = s_.getsockname()[1]
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, S, plan, coll, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert np.array_equal(got, whole)
