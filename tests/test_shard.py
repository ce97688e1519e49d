"""Sharding of independent systems across ranks: the assignment itself, the
host-side bookkeeping run as two gloo ranks on the CPU, and a sharded batch
whose ranks each solve their share (with the oracle, on the CPU) and whose
union equals the one-rank results system by system."""
import hashlib
import os


import pytest
import torch.multiprocessing as mp

from mfix_b200 import shard
from mfix_b200 import systems as S


def test_assign_covers_every_system_once_and_balances():
    sizes = S.batch_sizes(512, 0)
    cells = [(i + 2) * (j + 2) * (k + 2) for i, j, k in sizes]
    for world in (1, 2, 3, 4, 8):
        parts = shard.assign(cells, world)
        flat = sorted(q for p in parts for q in p)
        assert flat == list(range(len(cells)))
        loads = [sum(cells[q] for q in p) for p in parts]
        assert max(loads) <= sum(cells) / world + max(cells)
    assert shard.assign([5, 1], 4)[2:] == [[], []]
    with pytest.raises(ValueError):
        shard.assign([1], 0)


def _rank(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        cells = [(i + 2) * (j + 2) * (k + 2) for i, j, k in S.batch_sizes(64, 1)]
        mine = shard.assign(cells, world)[rank]
        got = [None] * world
        dist.all_gather_object(got, mine)
        t_max = shard.max_over_ranks(1.0 + rank)
        n_tot = shard.sum_over_ranks(len(mine))
        q.put((rank, got, t_max, n_tot))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_the_batch():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, t_max, n_tot in res:
        assert sorted(got[0] + got[1]) == list(range(64)) and not set(got[0]) & set(got[1])
        assert t_max == 2.0 and n_tot == 64


# small uneven systems: a sharded batch solved on the CPU in seconds
SHARD_DIMS = [(6, 9, 5), (12, 7, 10), (5, 14, 6), (9, 9, 9), (16, 6, 4), (7, 11, 8), (4, 20, 5), (10, 5, 12)]


def _solve_share(indices):
    import oracle as O

    out = {}
    for q in indices:
        s = S.conv_diff(*SHARD_DIMS[q], seed=100 + q)
        st = O.leq_bicgs(s)
        out[q] = (st["ier"], st["iterations"], hashlib.sha256(s.x.tobytes()).hexdigest())
    return out


def _solve_rank(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), OMP_NUM_THREADS="2")
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=120))
    try:
        cells = [(i + 2) * (j + 2) * (k + 2) for i, j, k in SHARD_DIMS]
        mine = shard.assign(cells, world)[rank]
        res = _solve_share(mine)  # no collective while solving
        got = [None] * world
        dist.all_gather_object(got, res)
        n_tot = shard.sum_over_ranks(len(mine))
        q.put((rank, got, n_tot))
    finally:
        dist.destroy_process_group()


def test_sharded_batch_equals_one_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30500 + os.getpid() % 1000
    ps = [ctx.Process(target=_solve_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=300) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    one_rank = _solve_share(range(len(SHARD_DIMS)))
    assert all(v[0] == 0 for v in one_rank.values())
    for rank, got, n_tot in res:
        assert n_tot == len(SHARD_DIMS)
        union = {}
        for part in got:
            assert not set(part) & set(union)  # every system solved by one rank only
            union.update(part)
        assert union == one_rank  # same IER, iterations and solution bits per system
