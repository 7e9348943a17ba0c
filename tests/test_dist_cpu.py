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


class _FakeLib:
    """The two grid entry points sharded_bp32f calls, on host memory."""

    def __init__(self):
        self.ptrs = (None, None)

    def spi_bp_grid_bytes(self, nx, out):
        out._obj.value = (nx + 1) * (2 * nx) * (2 * nx) * 16
        return 0

    def spi_bp_attach_grids(self, h, g0, g1):
        self.ptrs = (g0, g1)
        return 0


class _RecordingContext:
    """A context whose insertion writes the oracle's partial grids (X, W of
    its images, FP64 rounded to FP32) into the attached grids as float4
    {Re X, Im X, W, 0}, and whose finish returns the grids it then holds; it
    records the order of the calls sharded_bp32f makes."""

    def __init__(self):
        self._L = _FakeLib()
        self.handle = None
        self.device = 0
        self.calls = []

    def _grid(self, g):
        import ctypes
        n = 2 * self.nx
        size = n * n * (self.nx + 1) * 4
        p = self._L.ptrs[g]
        return np.ctypeslib.as_array((ctypes.c_float * size).from_address(p.value)).reshape(n, n, self.nx + 1, 4)

    def bp_open(self, nx, ngrids):
        self.calls.append("open")
        self.nx = nx
        for g in range(2):
            self._grid(g)[...] = 0.0

    def bp_insert(self, imgs, angles, half):
        import oracle
        self.calls.append(("insert", int(imgs.shape[0])))
        for g, sel in ((0, half != 0), (1, half == 0)):
            if sel.any():
                x, w = oracle.bp3f_partial(imgs[sel], angles[sel], prec=1, nthreads=1)
                a = self._grid(g)
                a[..., 0] += x.real
                a[..., 1] += x.imag
                a[..., 2] += w

    def bp_flush(self):
        self.calls.append("flush")

    def bp_finish(self, want):
        self.calls.append("finish")
        g0, g1 = self._grid(0).copy(), self._grid(1).copy()
        return {"all": g0 + g1, "1": g0, "2": g1}

    def bp_close(self):
        self.calls.append("close")


def _shard_worker(rank, world, port, imgs, ang, half, out_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ctx = _RecordingContext()
    v_all, v1, v2 = sdist.sharded_bp32f(ctx, imgs, ang, half, rank, world, device="cpu")
    np.savez(out_path + f".{rank}.npz", all=v_all, first=v1, second=v2,
             calls=np.array([str(c) for c in ctx.calls]))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_bp32f_gloo_two_ranks(tmp_path):
    """sharded_bp32f's own orchestration over two gloo ranks: each rank
    inserts exactly its SETPART block, completes its grids before the
    all-reduce and finishes after it; both ranks end with the grids of all
    images."""
    import oracle
    rng = np.random.default_rng(13)
    nx, n = 12, 25
    vol = synth.blob_phantom(nx, 4, sigma=(1.5, 3), radius=4, rng=rng)
    ang = synth.so3_angles(n, rng)
    imgs = oracle.pj3q(vol, ang)
    half = synth.half_mask(n, rng)
    out = str(tmp_path / "shard")
    mp.start_processes(_shard_worker, args=(2, _port(), imgs, ang, half, out), nprocs=2, join=True,
                       start_method="spawn")
    x1, w1 = oracle.bp3f_partial(imgs[half != 0], ang[half != 0], prec=1, nthreads=1)
    x2, w2 = oracle.bp3f_partial(imgs[half == 0], ang[half == 0], prec=1, nthreads=1)
    sizes, _ = sdist.setpart(n, 2)
    for r in range(2):
        got = np.load(out + f".{r}.npz")
        assert list(got["calls"]) == ["open", str(("insert", sizes[r])), "flush", "finish", "close"]
        for key, x, w in (("first", x1, w1), ("second", x2, w2)):
            g = got[key]
            assert np.linalg.norm(g[..., 0] + 1j * g[..., 1] - x) <= 1e-6 * np.linalg.norm(x)
            assert np.linalg.norm(g[..., 2] - w) <= 1e-6 * np.linalg.norm(w)

