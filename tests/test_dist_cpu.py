"""Multi-rank sharding of the reconstruction, on CPU with gloo (world size 2).

Each rank builds the partial Fourier grids (X, W after SYMPLANE0, the BP 3F P
output) of its SETPART block with the CPU oracle; an all-reduce sums them.
The sum equals the grids of one process over all images: the exchange step
the GPU ranks perform on their own grids before finishing.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from spider_b200 import dist as sdist
from spider_b200 import synth


def test_setpart_matches_reference_partition():
    assert sdist.setpart(10, 3) == ([4, 3, 3], [0, 4, 7])
    assert sdist.setpart(2, 4) == ([1, 1, 0, 0], [0, 1, 2, 2])
    for n in (0, 1, 7, 100):
        for p in (1, 2, 3, 8):
            ps, nb = sdist.setpart(n, p)
            assert sum(ps) == n and nb[0] == 0 and max(ps) - min(ps) <= 1


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, imgs, ang, out_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import oracle
    start, count = sdist.shard(imgs.shape[0], rank, world)
    x, w = oracle.bp3f_partial(imgs[start:start + count], ang[start:start + count], prec=1, nthreads=1)
    tx = torch.from_numpy(np.stack([x.real, x.imag], -1).copy())
    tw = torch.from_numpy(w.copy())
    sdist.allreduce_grids([tx, tw])
    if rank == 0:
        np.savez(out_path, x=tx.numpy(), w=tw.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_grid_allreduce(tmp_path):
    import oracle
    rng = np.random.default_rng(3)
    nx, n = 16, 30
    vol = synth.blob_phantom(nx, 5, sigma=(1.5, 3), radius=5, rng=rng)
    ang = synth.so3_angles(n, rng)
    imgs = oracle.pj3q(vol, ang)
    out = str(tmp_path / "sum.npz")
    mp.start_processes(_worker, args=(2, _port(), imgs, ang, out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    x, w = oracle.bp3f_partial(imgs, ang, prec=1, nthreads=1)
    gx = got["x"][..., 0] + 1j * got["x"][..., 1]
    assert np.linalg.norm(gx - x) / np.linalg.norm(x) < 1e-12
    assert np.linalg.norm(got["w"] - w) / np.linalg.norm(w) < 1e-12
