"""Multi-rank host logic on CPU (gloo, world size 2): the sample ranges of the ranks are disjoint and
cover the frame's samples, and combining the ranks' images gives the image of all their samples."""

import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from math_b200 import distributed

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        spp = 8
        rng = np.random.default_rng(100 + rank)
        per_sample = rng.random((2, spp, 5, 3))  # two passes of spp samples for 5 pixels
        mean = per_sample.reshape(-1, 5, 3).mean(axis=0).astype(np.float32)
        offsets = [distributed.sample_offset(rank, k, spp, world) for k in range(2)]
        img, total = distributed.combine(mean, 2 * spp)
        out[rank] = (offsets, img, total, per_sample)
    finally:
        dist.destroy_process_group()


def test_two_ranks_combine_and_shard():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    offsets = sorted(o for r in range(world) for o in out[r][0])
    assert offsets == [0, 8, 16, 24]
    allsamples = np.concatenate([out[r][3].reshape(-1, 5, 3) for r in range(world)])
    expect = allsamples.mean(axis=0)
    for r in range(world):
        _, img, total, _ = out[r]
        assert total == 32
        assert np.allclose(img, expect, rtol=1e-5)
