"""The oracle's FBS restatement (fbs2.f, fbs3.f: Fourier-based bicubic and
tricubic interpolation) pinned against plane waves, whose derivatives the
FFT gives exactly: grid points are reproduced exactly, points between them
to the accuracy of cubic Hermite interpolation; and BP CG with FBS
interpolation runs (FP32 and FP64 agree)."""
import numpy as np
import pytest

import oracle


def test_fbs2_grid_points_and_plane_wave():
    n = 32
    y, x = np.mgrid[0:n, 0:n].astype(np.float64)
    f = np.cos(2 * np.pi * (2 * x + 3 * y) / n + 0.3)
    grid = np.array([[5, 7], [10, 3], [32, 1]], np.float32)   # 1-based X, Y
    v = oracle.fbs2(f.astype(np.float32), grid)
    assert np.allclose(v, [f[6, 4], f[2, 9], f[0, 31]], atol=1e-6)
    pts = np.random.default_rng(0).uniform(1, n, (300, 2))
    v = oracle.fbs2(f.astype(np.float32), pts)
    ref = np.cos(2 * np.pi * (2 * (pts[:, 0] - 1) + 3 * (pts[:, 1] - 1)) / n + 0.3)
    assert np.abs(v - ref).max() < 1e-3
    # periodic wrap: X = n + 0.5 sits between the last and the first pixel
    w = oracle.fbs2(f.astype(np.float32), np.array([[n + 0.5, 4.0]], np.float32))
    assert abs(w[0] - np.cos(2 * np.pi * (2 * (n - 0.5) + 3 * 3) / n + 0.3)) < 1e-3


@pytest.mark.parametrize("k", [(2, 1, 0), (0, 0, 2), (1, 2, 0)])
def test_fbs3_plane_wave(k):
    n = 24
    z, y, x = np.mgrid[0:n, 0:n, 0:n].astype(np.float64)
    f = np.cos(2 * np.pi * (k[0] * x + k[1] * y + k[2] * z) / n)
    pts = np.random.default_rng(1).uniform(1, n, (200, 3))
    v = oracle.fbs3(f.astype(np.float32), pts)
    ref = np.cos(2 * np.pi * (k[0] * (pts[:, 0] - 1) + k[1] * (pts[:, 1] - 1) + k[2] * (pts[:, 2] - 1)) / n)
    assert np.abs(v - ref).max() < 5e-4


def test_bpcg_fbs_runs_fp32_and_fp64_agree():
    from spider_b200 import synth
    rng = np.random.default_rng(3)
    n = 16
    vol = synth.blob_phantom(n, 4, sigma=(1.5, 3.0), radius=4, rng=rng)
    ang = synth.so3_angles(12, rng)
    pr = oracle.pj3q(vol, ang)
    v64, log64, _, _ = oracle.bpcg(pr, ang, 5.0, errm=1e-9, maxit=3, mode=1, lam=0.5, prec=1, fbs=True)
    v32, _, _, _ = oracle.bpcg(pr, ang, 5.0, errm=1e-9, maxit=3, mode=1, lam=0.5, prec=0, fbs=True)
    vl, _, _, _ = oracle.bpcg(pr, ang, 5.0, errm=1e-9, maxit=3, mode=1, lam=0.5, prec=1)
    assert np.isfinite(v64).all() and len(log64) == 3
    assert synth.rel_l2(v32, v64) < 1e-4
    # a different interpolation, the same problem: close to the linear solution, not equal
    assert 1e-6 < synth.rel_l2(v64, vl) < 0.5
