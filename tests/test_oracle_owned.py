"""The oracle's owner-computes insertion schedule (each thread owns a range
of z planes and walks every image and row in the serial order) must give the
grids of the one-thread loop bit for bit, for any thread count: it is the
parallel checker of the GPU insertion at configuration sizes, where the
serial loop is too slow and the reference's own OpenMP row striping races
(oneline.f:59-66,118-150 under bp3f.f:468-474)."""
import numpy as np
import pytest

import oracle
from spider_b200 import synth


@pytest.mark.parametrize("nx", [32, 33])
@pytest.mark.parametrize("prec", [0, 1])
def test_owned_schedule_equals_serial(nx, prec):
    rng = np.random.default_rng(100 + nx + 10 * prec)
    imgs = rng.standard_normal((50, nx, nx)).astype(np.float32)
    ang = synth.so3_angles(50, rng)
    x1, w1 = oracle.bp3f_partial(imgs, ang, prec=prec, nthreads=1)
    for nt in (2, 5, 8):
        xt, wt = oracle.bp3f_partial(imgs, ang, prec=prec, nthreads=nt)
        assert np.array_equal(x1, xt) and np.array_equal(w1, wt), nt


def test_owned_schedule_bp32f_symmetry_and_rb():
    rng = np.random.default_rng(7)
    nx = 24
    imgs = rng.standard_normal((40, nx, nx)).astype(np.float32)
    ang = synth.so3_angles(40, rng)
    half = synth.half_mask(40, rng)
    sym = np.array([[0, 0, 0], [0, 0, 90], [0, 0, 180], [0, 0, 270]], np.float32)
    a = oracle.bp32f(imgs, ang, half, sym=sym, prec=1, nthreads=1)
    b = oracle.bp32f(imgs, ang, half, sym=sym, prec=1, nthreads=6)
    assert all(np.array_equal(p, q) for p, q in zip(a, b))
    inplane = np.stack([rng.uniform(-180, 180, 40), rng.uniform(-3, 3, 40), rng.uniform(-3, 3, 40)], 1)
    inplane = inplane.astype(np.float32)
    a = oracle.rb3f(imgs, ang, inplane, half, nthreads=1)
    b = oracle.rb3f(imgs, ang, inplane, half, nthreads=6)
    assert all(np.array_equal(p, q) for p, q in zip(a, b))
