"""Multi-GPU sharding logic on CPU: two gloo ranks split systems by cost, together cover every
system exactly once, and agree on the max-over-ranks time."""
import os
import socket

import numpy as np
import pytest

from surfmol_b200.shard import assign_by_cost, block_range, system_cost


def test_block_range_covers_all():
    for n in (0, 1, 7, 4096, 16385):
        for w in (1, 2, 3, 8):
            parts = [block_range(n, r, w) for r in range(w)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[k][1] == parts[k + 1][0] for k in range(w - 1))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        block_range(10, 2, 2)


def test_assign_by_cost_balanced_and_deterministic():
    rng = np.random.default_rng(5)
    n = np.exp(rng.uniform(np.log(20), np.log(400), 2000)).astype(int)
    c = system_cost(n)
    for w in (2, 4, 8):
        a = assign_by_cost(c, w)
        b = assign_by_cost(c, w)
        assert all(np.array_equal(x, y) for x, y in zip(a, b))
        allidx = np.sort(np.concatenate(a))
        assert np.array_equal(allidx, np.arange(len(c)))
        loads = np.array([c[x].sum() for x in a])
        assert loads.max() - loads.min() <= c.max()          # LPT bound


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, costs, out_q):
    import torch.distributed as dist
    from surfmol_b200.shard import assign_by_cost, max_over_ranks
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        mine = assign_by_cost(costs, world)[rank]
        t = max_over_ranks(float(10 + rank))                  # a per-rank "device time"
        dist.barrier()
        out_q.put((rank, mine.tolist(), t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    costs = system_cost(np.arange(20, 120))
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    got = sorted(res[0][1] + res[1][1])
    assert got == list(range(len(costs)))
    assert not set(res[0][1]) & set(res[1][1])
    assert res[0][2] == res[1][2] == 11.0
