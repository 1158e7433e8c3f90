"""The multi-rank paths of bench.py on CPU ranks (gloo, world size 2): the
batched leg's scene shards partition the batch and balance its triangles,
and the timed region is reduced as the maximum over ranks."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, sizes, out):
    import torch

    import scenes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    mine = scenes.shard_scenes(sizes, world, rank)
    mask = torch.zeros(len(sizes), dtype=torch.int64)
    mask[torch.from_numpy(mine)] = 1
    counts = [torch.zeros_like(mask) for _ in range(world)]
    dist.all_gather(counts, mask)
    t = torch.tensor([float(10 + rank)])          # a rank's device time
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    out[rank] = (torch.stack(counts).numpy(), float(t.item()), int(sizes[mine].sum()))
    dist.barrier()
    dist.destroy_process_group()


def test_batched_shards_partition_and_balance():
    import scenes
    b = scenes.BatchedScenes(num_scenes=64, t_min=200, t_max=20_000, seed=3)
    sizes = np.diff(b.tri_offsets)
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, sizes, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    masks, tmax, tris = out[0][0], out[0][1], [out[r][2] for r in range(world)]
    assert np.array_equal(masks, out[1][0])
    assert np.array_equal(masks.sum(axis=0), np.ones(len(sizes)))      # every scene on exactly one rank
    assert tmax == 11.0 and out[1][1] == 11.0                            # max over ranks
    assert sum(tris) == sizes.sum()
    assert max(tris) - min(tris) <= sizes.max()                          # greedy balance bound
