"""The product's sharded BP 32F (dist.sharded_bp32f: SETPART blocks,
caller-owned grids, spi_bp_flush, a sum over the ranks, finish on every
rank), the reference's MPI form (setpart.f:4-29, bp32f.f:720-774).

Two ranks are emulated on one GPU by two contexts on two host threads whose
all-reduce sums the grids on the host behind a barrier (no kernel waits on
another rank's).  Every rank's volumes must equal one process's BP 32F of all
images and the oracle's."""
import threading

import numpy as np
import pytest

from spider_b200 import dist as sdist
from spider_b200 import ops, synth

pytestmark = pytest.mark.gpu

TOL = 1e-5


def test_sharded_bp32f_two_ranks_one_gpu(orc):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(71)
    nx, nimg = 32, 301
    vol = synth.blob_phantom(nx, 10, sigma=(1.5, 4.0), radius=0.35 * nx, rng=rng)
    ang = synth.so3_angles(nimg, rng)
    pr = synth.add_noise(orc.pj3q(vol, ang), 0.5, rng)
    half = synth.half_mask(nimg, rng)
    world = 2
    ctxs = [ops.Context(0) for _ in range(world)]
    bar = threading.Barrier(world, timeout=120)
    bufs = [None] * world
    out = [None] * world
    errs = []
    calls = [0] * world

    def make_allreduce(r):
        def allreduce(tensors):
            calls[r] += 1
            bufs[r] = [t.cpu() for t in tensors]
            bar.wait()
            total = [a + b for a, b in zip(bufs[0], bufs[1])]   # the same order on both ranks
            bar.wait()
            for t, v in zip(tensors, total):
                t.copy_(v.to(t.device))
        return allreduce

    def run(r):
        try:
            out[r] = sdist.sharded_bp32f(ctxs[r], pr, ang, half, r, world, allreduce=make_allreduce(r))
        except Exception as e:  # pragma: no cover
            errs.append(e)
            bar.abort()

    th = [threading.Thread(target=run, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for c in ctxs:
        c.close()
    assert not errs, errs
    assert calls == [1, 1]
    one = ops.bp32f(pr, ang, half)
    ref = orc.bp32f(pr, ang, half, prec=1)
    for r in range(world):
        for a, b, c in zip(out[r], one, ref):
            assert synth.rel_l2(a, b) <= TOL
            assert synth.rel_l2(a, c) <= TOL
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
