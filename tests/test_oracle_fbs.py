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


def test_rtsf_identity_and_integer_shifts():
    """RTSF (rtsf.f:109-205) with no rotation reproduces integer shifts exactly
    (circularly), since FBS2 at grid points returns the pixel itself."""
    rng = np.random.default_rng(3)
    img = rng.standard_normal((24, 24)).astype(np.float32)
    assert np.array_equal(oracle.rtsf(img, 0.0, 0.0, 0.0), img)
    assert np.array_equal(oracle.rtsf(img, 0.0, 3.0, 0.0), np.roll(img, 3, axis=1))
    assert np.array_equal(oracle.rtsf(img, 0.0, 0.0, -5.0), np.roll(img, -5, axis=0))
    assert np.array_equal(oracle.rtsf(img, 0.0, 27.0, 0.0), np.roll(img, 3, axis=1))   # MODULO(SHX, NX)


def test_rtsf_rotates_band_limited_image():
    """A band-limited image rotated by RTSF matches the analytic rotation
    (about the centre NX/2+1) to the accuracy of the cubic interpolation; a
    quarter turn is a transposition up to float rounding of COS(90)."""
    n = 32
    y, x = np.mgrid[1:n + 1, 1:n + 1].astype(np.float64)
    c = n // 2 + 1

    def f(xx, yy):
        return np.cos(2 * np.pi * (2 * xx + 1 * yy) / n + 0.4) + 0.5 * np.sin(2 * np.pi * (xx - 3 * yy) / n)

    img = f(x, y).astype(np.float32)
    for th in (17.0, -63.0):
        t = np.deg2rad(th)
        # RTSF reads the source at XOLD = cos*FX - sin*FY + CX, YOLD = sin*FX + cos*FY + CY
        xs = np.cos(t) * (x - c) - np.sin(t) * (y - c) + c
        ys = np.sin(t) * (x - c) + np.cos(t) * (y - c) + c
        ref = f(xs, ys)
        got = oracle.rtsf(img, th, 0.0, 0.0)
        assert np.abs(got - ref).max() < 2e-3, th
    q = oracle.rtsf(img, 90.0, 0.0, 0.0)
    xs = -(y - c) + c
    ys = (x - c) + c
    assert np.abs(q - f(xs, ys)).max() < 1e-4


def test_rb3f_fbs_mode_uses_rtsf():
    """RB 3F in FBS mode equals BP 3F of the RTSF-rotated images."""
    from spider_b200 import synth
    rng = np.random.default_rng(4)
    n, nimg = 24, 12
    imgs = rng.standard_normal((nimg, n, n)).astype(np.float32)
    ang = synth.so3_angles(nimg, rng)
    inplane = np.stack([rng.uniform(-180, 180, nimg), rng.uniform(-3, 3, nimg), rng.uniform(-3, 3, nimg)], 1)
    inplane = inplane.astype(np.float32)
    rot = np.stack([oracle.rtsf(imgs[i], *inplane[i]) for i in range(nimg)])
    a = oracle.rb3f(imgs, ang, inplane, fbs=True, nthreads=1)
    b = oracle.bp3f(rot, ang, nthreads=1)
    assert np.array_equal(a, b)
    c = oracle.rb3f(imgs, ang, inplane, nthreads=1)
    assert not np.array_equal(a, c)
