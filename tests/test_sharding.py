"""Host logic of the multi-GPU batched form on CPU: the instance partition
covers every instance exactly once, and the gather reassembles per-rank
series in global order, with world size 2 and 3 gloo ranks on 127.0.0.1."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ptha_b200.sharding import gather_instance_series, instance_range


@pytest.mark.parametrize("nbatch", [0, 1, 7, 256])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_instance_range_partition(nbatch, world):
    seen = []
    for r in range(world):
        f, c = instance_range(nbatch, world, r)
        seen.extend(range(f, f + c))
        assert c in (nbatch // world, nbatch // world + 1)
    assert seen == list(range(nbatch))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, nbatch, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        f, c = instance_range(nbatch, world, rank)
        T, G = 4, 3
        # series value = 1000 * instance + 10 * record + gauge
        local = (1000.0 * np.arange(f, f + c)[None, :, None] + 10.0 * np.arange(T)[:, None, None]
                 + np.arange(G)[None, None, :])
        out = gather_instance_series(local, nbatch, world, rank)
        expect = (1000.0 * np.arange(nbatch)[None, :, None] + 10.0 * np.arange(T)[:, None, None]
                  + np.arange(G)[None, None, :])
        q.put((rank, bool(np.array_equal(out, expect))))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nbatch", [(2, 7), (3, 256)])
def test_gather_gloo(world, nbatch):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, nbatch, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    assert sorted(res) == [(r, True) for r in range(world)]


def _oracle_instance_series(q, nsteps=8):
    """Instance q of a small batched-linear case advanced by the oracle:
    (nsteps, gauges) stage series."""
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    if here not in sys.path:
        sys.path.insert(0, here)
    from pairs import oracle_from_kw
    from ptha_b200 import workloads
    kw, U = workloads.spherical_patch(nx=40, ny=30, seed=6)
    kw = dict(kw, timestepping_method="linear")
    rng = np.random.default_rng(100 + q)
    X, Y = np.meshgrid(np.arange(40), np.arange(30))
    cx, cy = rng.uniform(12, 28), rng.uniform(10, 20)
    U = U.copy()
    U[0] = np.where(U[3] < 0, rng.uniform(0.5, 2.0) * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / 8.0), 0.0)
    o = oracle_from_kw(kw)
    o.U[:] = U
    dt = o.linear_timestep_max()
    sites = [(8, 7), (20, 15), (31, 22), (15, 24)]
    out = np.zeros((nsteps, len(sites)))
    for n in range(nsteps):
        o.evolve_one_step(dt)
        out[n] = [o.U[0][j, i] for i, j in sites]
    return out


def _oracle_worker(rank, world, port, nbatch, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        f, c = instance_range(nbatch, world, rank)
        local = np.stack([_oracle_instance_series(b) for b in range(f, f + c)], axis=1) if c else \
            np.zeros((8, 0, 4))
        out = gather_instance_series(local, nbatch, world, rank)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_sharded_instances_with_the_oracle_equal_one_rank():
    """Two gloo ranks each advance their range of 5 instances with the
    oracle and gather the gauge series; the result equals one process
    advancing all 5 instances, bit for bit."""
    world, nbatch = 2, 5
    ctx = mp.get_context("spawn")
    qu = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_oracle_worker, args=(r, world, port, nbatch, qu)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(qu.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    single = np.stack([_oracle_instance_series(b) for b in range(nbatch)], axis=1)
    assert single.shape == (8, nbatch, 4) and np.any(single != 0)
    for r in range(world):
        np.testing.assert_array_equal(res[r], single)
