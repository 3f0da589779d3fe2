"""Shot sharding and the FP64 all-reduce of the misfit, data norm and
gradient over two gloo ranks on CPU (the reduction the sharded objective
uses over NCCL on GPUs)."""
import multiprocessing as mp
import socket

import numpy as np

from fwi3d_b200 import distributed


def test_shards_cover_every_shot_once():
    for ns in (1, 5, 16):
        for world in (1, 2, 3, 8):
            got = sorted(s for r in range(world) for s in distributed.shard(ns, r, world))
            assert got == list(range(ns))
    assert distributed.shard(5, 1, 2) == [1, 3]  # rank-strided, as the reference's loop


def _worker(rank, world, port, q):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        shape = (3, 2, 2, 2)
        g = np.full(shape, rank + 1.0, dtype=np.float32) if rank == 0 else None  # rank 1 has no shot
        f, gr = distributed.reduce_objective(10.0 * (rank + 1), 2.0 + rank, g, shape, "cpu")
        q.put((rank, f, gr))
    finally:
        dist.destroy_process_group()


def test_reduce_objective_over_gloo():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
    for rank, f, g in out:
        assert abs(f - 30.0 / 5.0) < 1e-12
        assert np.allclose(g, 1.0 / 5.0)
