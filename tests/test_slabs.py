"""z-slab halo exchange on CPU: the planes each rank receives, with one rank (periodic self-exchange)
and with two gloo ranks, against the global periodic field."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from public_b200.slabs import ZSlabs


def _global(n, nf=5, seed=0):
    return np.random.default_rng(seed).standard_normal(n + (nf,))


def _check_rank(n, H, rank, world, g, nf):
    sl = ZSlabs(n, H, rank, world)
    want = sl.local_state(g)
    loc = want.copy()
    loc[:, :, :H] = -7.0                       # stale halos
    loc[:, :, -H:] = 9.0
    flat = torch.from_numpy(np.ascontiguousarray(loc.ravel(order="F"))).clone()
    sl.exchange(flat, nf)
    got = flat.numpy().reshape(loc.shape, order="F")
    return np.array_equal(got, want)


def test_self_exchange_is_periodic_wrap():
    n, H = (4, 3, 10), 3
    g = _global(n)
    assert _check_rank(n, H, 0, 1, g, 5)
    sl = ZSlabs(n, H, 0, 1)
    s = sl.local_settings({"n": n, "x0": (0, 0, 0.0), "x1": (1, 1, 2.0)})
    assert s["n"] == (4, 3, 16) and np.isclose(s["x1"][2] - s["x0"][2], 16 * 0.2) and np.isclose(s["x0"][2], -0.6)


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        n, H = (4, 3, 12), 2
        g = _global(n, nf=3, seed=5)
        q.put((rank, _check_rank(n, H, rank, world, g, 3)))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("world", [2, 3])
def test_two_and_three_gloo_ranks_receive_their_neighbours_planes(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert all(res[r] for r in range(world)), res
