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


def test_grid_slabs_partition():
    from surfmol_b200.shard import gather_slabs, grid_slabs
    for nx, world in ((28, 1), (28, 3), (226, 8), (904, 8), (5, 4)):
        w, slabs = grid_slabs(nx, world)
        assert slabs[0][0] == 0 and all(slabs[k][1] == slabs[k + 1][0] for k in range(world - 1))
        assert slabs[-1][1] >= nx and w * world - nx < world
        ny, nz = 3, 2
        full = np.arange(3 * nx * ny * nz, dtype=np.float64)
        pad = np.concatenate([full, -np.ones(3 * (w * world - nx) * ny * nz)])
        chunks = [pad[3 * x0 * ny * nz:3 * x1 * ny * nz] for x0, x1 in slabs]
        assert np.array_equal(gather_slabs(chunks, nx, ny, nz), full)


def _slab_rank(rank, world, port, nx, ny, nz, out_q):
    import torch
    import torch.distributed as dist
    from surfmol_b200.shard import grid_slabs
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        w, slabs = grid_slabs(nx, world)
        x0, x1 = slabs[rank]
        # this rank's raw slab: voxel-major triples whose values encode (plane, y, z, channel)
        x = np.arange(x0, x1)[:, None, None, None]
        y = np.arange(ny)[None, :, None, None]
        z = np.arange(nz)[None, None, :, None]
        c = np.arange(3)[None, None, None, :]
        local = torch.from_numpy((1000 * x + 100 * y + 10 * z + c).astype(np.float64).reshape(-1))
        parts = [torch.empty_like(local) for _ in range(world)]
        dist.all_gather(parts, local)
        full = torch.cat(parts)[:3 * nx * ny * nz]
        out_q.put((rank, full.numpy().tolist()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_grid_slabs():
    """The raw slabs of two ranks, gathered in rank order, are the voxel-major raw array of the
    whole grid (the exchange step of the sharded grid build)."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    nx, ny, nz = 7, 3, 4
    ps = [ctx.Process(target=_slab_rank, args=(r, 2, port, nx, ny, nz, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    x = np.arange(nx)[:, None, None, None]
    y = np.arange(ny)[None, :, None, None]
    z = np.arange(nz)[None, None, :, None]
    c = np.arange(3)[None, None, None, :]
    want = (1000 * x + 100 * y + 10 * z + c).reshape(-1)
    assert np.array_equal(res[0], want) and np.array_equal(res[1], want)
