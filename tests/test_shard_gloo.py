"""Multi-GPU host logic on CPU: whole-world shards and the cross-rank
bookkeeping (max step time, sums, gathers) over gloo with two ranks."""
import os
import socket

import numpy as np
import pytest

from omi_physics_b200.shard import plan_shards


def test_plan_shards_partition_and_balance():
    rng = np.random.default_rng(0)
    sizes = np.exp(rng.uniform(np.log(16), np.log(2048), size=101)).astype(int)
    for n in (1, 2, 3, 8):
        sh = plan_shards(sizes, n)
        flat = sorted(i for s in sh for i in s)
        assert flat == list(range(len(sizes)))            # disjoint, complete
        loads = [int(sizes[s].sum()) for s in sh]
        assert max(loads) - min(loads) <= int(sizes.max())  # LPT bound
        assert plan_shards(sizes, n) == sh                # deterministic


def test_plan_shards_edge_cases():
    assert plan_shards([], 3) == [[], [], []]
    assert plan_shards([5], 2) == [[0], []]
    with pytest.raises(ValueError):
        plan_shards([1, 2], 0)


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world_size, port, sizes, out):
    import datetime
    import torch.distributed as dist
    from omi_physics_b200 import shard
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world_size,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mine = shard.local_shard(sizes, rank, world_size)
        bodies = int(np.asarray(sizes)[mine].sum())
        fake_ms = 10.0 + rank            # rank 1 is the slow one
        shard.barrier(world_size)
        t = shard.max_over_ranks(fake_ms, world_size)
        total = shard.sum_over_ranks(bodies, world_size)
        got = shard.gather_to_rank0(mine, world_size)
        out.put((rank, t, total, got))
    finally:
        dist.destroy_process_group()


def test_two_ranks_over_gloo():
    import torch.multiprocessing as mp
    sizes = [300, 17, 2048, 64, 999, 128, 5, 700]
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r, t, total, got = q.get(timeout=120)
        res[r] = (t, total, got)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][0] == res[1][0] == 11.0
    assert res[0][1] == res[1][1] == float(sum(sizes))
    assert res[1][2] is None
    gathered = res[0][2]
    assert sorted(i for s in gathered for i in s) == list(range(len(sizes)))
    assert gathered == plan_shards(sizes, 2)


def test_plan_groups_complete_and_balanced():
    from omi_physics_b200.groups import plan_groups
    rng = np.random.default_rng(3)
    sizes = np.exp(rng.uniform(np.log(16), np.log(2048), size=257)).astype(int)
    for g in (1, 2, 4, 8):
        plan = plan_groups(sizes, g)
        assert sorted(i for grp in plan for i in grp) == list(range(len(sizes)))
        loads = [int(sizes[grp].sum()) for grp in plan]
        assert max(loads) - min(loads) <= 2 * int(sizes.max())
    assert plan_groups([5, 3], 4) == [[0], [1]]        # no empty groups


def _pack_rank_main(rank, world_size, port, out):
    """Each rank builds and packs only its shard of a fixed 24-world serving
    mix (no GPU: ``load=False``), then sends rank 0 every local world's
    packed body rows keyed by global world index."""
    import datetime
    import torch.distributed as dist
    from omi_physics_b200 import scenes, shard
    from omi_physics_b200.arena import pack_worlds
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world_size,
                            timeout=datetime.timedelta(seconds=60))
    try:
        reqs = scenes.serving_requests(24, seed=3, n_max=300)
        build = lambda i: (lambda r: (r[0], r[1]['dt']))(scenes.serving_world(reqs[i]))
        sw = shard.ShardedWorlds([r['bodies'] + 1 for r in reqs], build, rank, world_size, load=False)
        assert sw.indices == shard.shard_requests(reqs, rank, world_size)
        P = pack_worlds(sw.worlds, sw.dts)
        rows = {}
        for j, gi in enumerate(sw.indices):
            b0, b1 = P.body_off[j], P.body_off[j + 1]
            rows[gi] = {k: P.arrays[k][b0:b1].copy() for k in ('pos', 'q', 'inv_mass', 'inv_inertia',
                                                               'motion_type')}
        ticks = shard.merge_ticks([1.0 + rank, 5.0 - rank, 2.0], world_size)
        got = shard.gather_to_rank0((rows, sw.local_bodies), world_size)
        out.put((rank, got, ticks))
    finally:
        dist.destroy_process_group()


def test_two_ranks_pack_disjoint_shards_that_make_up_the_whole_mix():
    import torch.multiprocessing as mp
    from omi_physics_b200 import scenes
    from omi_physics_b200.arena import pack_worlds
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_pack_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r, got, ticks = q.get(timeout=180)
        res[r] = (got, ticks)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] == res[1][1] == [2.0, 5.0, 2.0]        # per-tick max over ranks
    parts = res[0][0]
    merged = {}
    for rows, _ in parts:
        assert not set(rows) & set(merged)                  # disjoint shards
        merged.update(rows)
    reqs = scenes.serving_requests(24, seed=3, n_max=300)
    assert sorted(merged) == list(range(len(reqs)))         # complete
    worlds = [scenes.serving_world(r) for r in reqs]
    P = pack_worlds([w for w, _ in worlds], [m['dt'] for _, m in worlds])
    for i in range(len(reqs)):                              # the same rows as one rank packing all
        b0, b1 = P.body_off[i], P.body_off[i + 1]
        for k, v in merged[i].items():
            assert np.array_equal(v, P.arrays[k][b0:b1]), (i, k)
    total = sum(int(np.count_nonzero(w.motion_type == 2)) for w, _ in worlds)
    assert sum(b for _, b in parts) == total
