"""The multi-GPU path is replicas (no data-path collective): the router's assignment and the gather of results, run as
world-size-2 gloo process groups on the CPU, with a host stand-in for the per-image encode."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from av1gpu_b200 import replicas


def test_assign_covers_and_balances():
    areas = [12_000_000, 300_000, 5_000_000, 5_000_000, 180_000, 24_000_000, 700_000]
    parts = replicas.assign(areas, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(areas)))
    loads = [sum(areas[i] for i in p) for p in parts]
    assert max(loads) == 24_000_000   # the largest image alone bounds the makespan here
    assert replicas.assign(areas, 3) == parts   # deterministic


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rng = np.random.default_rng(5)
    images = [(rng.integers(0, 256, (h, w), dtype=np.uint8),) for h, w in ((64, 96), (128, 32), (8, 8), (200, 100), (16, 16))]
    res = replicas.run(images, lambda i, im: (i, int(im[0].sum()), os.getpid()), rank, world)
    out[rank] = {k: v[:2] for k, v in res.items()}
    dist.destroy_process_group()


def test_replicas_gloo_world2():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    manager = mp.Manager()
    out = manager.dict()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    assert out[0] == out[1]
    assert sorted(out[0]) == [0, 1, 2, 3, 4]


def _worker_own(rank, world, port, out):
    """Each rank loads only the images assign() gives it; the areas are known beforehand."""
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    shapes = ((64, 96), (128, 32), (8, 8), (200, 100), (16, 16))
    areas = [h * w for h, w in shapes]
    mine = set(replicas.assign(areas, world)[rank])
    images = [(np.full(s, i, np.uint8),) if i in mine else None for i, s in enumerate(shapes)]
    res = replicas.run(images, lambda i, im: (i, int(im[0].sum())), rank, world, areas=areas)
    out[rank] = dict(res)
    dist.destroy_process_group()


def test_replicas_gloo_world2_own_images_only():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    manager = mp.Manager()
    out = manager.dict()
    mp.spawn(_worker_own, args=(2, port, out), nprocs=2, join=True)
    assert out[0] == out[1]
    assert out[0] == {i: (i, i * h * w) for i, (h, w) in enumerate(((64, 96), (128, 32), (8, 8), (200, 100), (16, 16)))}


def test_replicas_missing_own_image_raises():
    import pytest
    with pytest.raises(ValueError):
        replicas.run([None, (np.zeros((4, 4), np.uint8),)], lambda i, im: i, 0, 1, areas=[16, 16])
