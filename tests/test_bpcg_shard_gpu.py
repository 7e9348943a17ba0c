"""BP CG over several processes (spi_bpcg_shard, the reference's MPI form
bpcg.f:522-672, 855-1080): each rank back-projects its block of images and
applies the normal operator to its block of HIANG's merged angles, and CB,
the image statistics and BCKE are summed over the ranks through the
caller's all-reduce.

Two ranks are emulated on one GPU by two contexts on two host threads whose
all-reduce sums on the host behind a barrier (no kernel waits on another);
the result is the single-process solve up to the grouping of the sums.
"""
import os
import socket
import threading

import numpy as np
import pytest

from spider_b200 import dist as sdist
from spider_b200 import ops, synth

pytestmark = pytest.mark.gpu


def _data(n, nang, seed):
    import oracle
    rng = np.random.default_rng(seed)
    vol = synth.blob_phantom(n, 8, sigma=(1.5, 3.5), radius=0.3 * n, rng=rng)
    ang = synth.so3_angles(nang, rng)
    ang[nang // 2: nang // 2 + 6] = ang[0:6]   # duplicates: HIANG merges them (LB > 1)
    pr = synth.add_noise(oracle.pj3q(vol, ang), 1.0, rng)
    return pr, ang


def _two_ranks(pr, ang, kw):
    world = 2
    ctxs = [ops.Context(0) for _ in range(world)]
    bar = threading.Barrier(world, timeout=120)
    bufs = [None] * world
    out = [None] * world
    errs = []

    def make_sum(r):
        def sum_inplace(t):
            bufs[r] = t.cpu()
            bar.wait()
            total = bufs[0] + bufs[1]   # the same order on both ranks
            bar.wait()
            t.copy_(total.to(t.device))
            calls[r] += 1
        return sum_inplace

    calls = [0] * world

    def worker(r):
        try:
            start, count = sdist.shard(len(ang), r, world)
            out[r] = ops.bpcg_shard(pr[start:start + count], start, ang, rank=r, world=world,
                                    sum_inplace=make_sum(r), ctx=ctxs[r], **kw)
        except Exception as e:   # pragma: no cover - reported below
            errs.append(e)
            bar.abort()

    th = [threading.Thread(target=worker, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for c in ctxs:
        c.close()
    if errs:
        raise errs[0]
    return out, calls


def test_one_rank_equals_bpcg(ctx):
    pr, ang = _data(32, 70, 1)
    kw = dict(ri=12.0, errm=1e-9, maxit=5, mode=1, lam=0.5)
    ref, rlog = ops.bpcg(pr, ang, ctx=ctx, **kw)
    v, log = ops.bpcg_shard(pr, 0, ang, ctx=ctx, **kw)
    assert synth.rel_l2(v, ref) <= 1e-9
    np.testing.assert_allclose(log, rlog, rtol=1e-6)
    calls = []
    v2, log2 = ops.bpcg_shard(pr, 0, ang, ctx=ctx, sum_inplace=lambda t: calls.append(t.numel()), **kw)
    assert synth.rel_l2(v2, ref) <= 1e-9
    assert len(calls) == 2 + len(log2)                 # CB, the statistics, then BCKE per iteration
    assert calls[0] == 32 ** 3 and calls[1] == 3 and calls[2] == 32 ** 3


@pytest.mark.parametrize("fp64,interp", [("mixed", "linear"), (True, "linear"), (True, "fbs")])
def test_two_ranks_match_one_process(ctx, fp64, interp):
    pr, ang = _data(32, 70, 2)
    kw = dict(ri=12.0, errm=1e-9, maxit=5, mode=2, lam=0.5, fp64=fp64, interp=interp)
    ref, rlog = ops.bpcg(pr, ang, ctx=ctx, **kw)
    (v0, log0), (v1, log1) = _two_ranks(pr, ang, kw)[0]
    e = synth.rel_l2(v0, ref)
    print(f"BP CG 2 ranks ({fp64}, {interp}): rel-err vs one process {e:.3e}")
    assert np.array_equal(v0, v1) and np.array_equal(log0, log1)   # replicated iteration
    assert e <= 1e-6
    np.testing.assert_allclose(log0, rlog, rtol=1e-4)


def _nccl_worker(rank, port, pr, ang, kw, path):
    import torch
    import torch.distributed as tdist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    tdist.init_process_group("nccl", rank=0, world_size=1)
    try:
        c = ops.Context(0)
        v, log = ops.bpcg_shard(pr, 0, ang, rank=0, world=1, sum_inplace=lambda t: tdist.all_reduce(t), ctx=c,
                                **kw)
        np.save(path, v)
        c.close()
    finally:
        tdist.destroy_process_group()


def test_nccl_allreduce_plumbing(ctx, tmp_path):
    """The torch.distributed (NCCL) all-reduce reaches the library's device
    arrays through the callback (one rank, in a process of its own)."""
    import torch.multiprocessing as mp
    pr, ang = _data(32, 40, 3)
    kw = dict(ri=12.0, errm=1e-9, maxit=3, mode=1, lam=0.5)
    ref, _ = ops.bpcg(pr, ang, ctx=ctx, **kw)
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    path = str(tmp_path / "v.npy")
    mp.spawn(_nccl_worker, args=(port, pr, ang, kw, path), nprocs=1, join=True)
    assert synth.rel_l2(np.load(path), ref) <= 1e-9
