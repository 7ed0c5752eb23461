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
