"""Pins of the oracle's sub-functions against independent implementations.

The reference cannot be built here (Fortran + FFTW3) and ships no golden data
for this path, so the oracle is pinned piece by piece:
  * FILLBESSIL's Kaiser-Bessel table (fillbessi0.f:88-125) against the same
    formula evaluated with scipy.special.i1 in float64;
  * WINDKB2A's |WKB| (bp32f.f:964-1005) against scipy.special.iv(1.5, .);
  * the FFT against numpy.fft (forward and backward, powers of two and the
    mixed radices 3, 5, 7 the box sizes use);
  * CANG (cang.f:44-81) against the rotation Rz(psi) Ry(theta) Rz(phi);
  * the fixtures in tests/golden/ (made by tests/golden/make_golden.py with
    scipy and numpy only).
"""
import os

import numpy as np
import pytest
import scipy.special as sp

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("n2", [64, 128, 256, 512])
def test_kb_table_against_scipy(n2):
    tab, fltb, alpha, aaaa = oracle.kb_table(n2)
    assert fltb == np.float32(4999.0) / np.float32(3.0)
    assert alpha == np.float32(6.5)
    i = np.arange(5000)
    s = (i.astype(np.float32) / np.float32(fltb)) / np.float32(n2)
    inside = s <= np.float32(aaaa)
    x = np.sqrt(1.0 - (s[inside].astype(np.float64) / aaaa) ** 2)
    ref = np.sqrt(alpha * x) * sp.i1(alpha * x) / (np.sqrt(alpha) * sp.i1(alpha))
    np.testing.assert_allclose(tab[inside], ref, rtol=2e-6, atol=1e-7)
    assert np.all(tab[~inside] == 0)
    # the window ends at 1.8 grid units (0.9 * 2 / N2 in frequency)
    last = np.nonzero(tab)[0].max()
    assert abs(last / fltb - 1.8) < 1e-3


def test_kb_table_golden():
    g = np.load(os.path.join(GOLDEN, "kb_table_n2_128.npy"))
    tab, _, _, _ = oracle.kb_table(128)
    np.testing.assert_allclose(tab, g, rtol=2e-6, atol=1e-7)


@pytest.mark.parametrize("nx", [32, 64, 128, 256])
def test_windkb_against_scipy(nx):
    w = oracle.windkb_table(nx)
    tab, fltb, alpha, aaaa = oracle.kb_table(2 * nx)
    qrt = (np.float32(2.0) * np.float32(np.pi) * np.float32(aaaa)) ** 2
    lr = np.arange((nx // 2) ** 2 + 1, dtype=np.float64)
    sigma = qrt * lr - alpha * alpha
    art = np.sqrt(np.abs(sigma))
    nu = 1.5
    wkb0 = alpha ** nu / sp.iv(nu, alpha)
    ref = np.where(sigma > 0, wkb0 * sp.jv(nu, art) / art ** nu, wkb0 * sp.iv(nu, art) / art ** nu)
    np.testing.assert_allclose(w, np.abs(ref), rtol=2e-6)
    assert w[0] == pytest.approx(1.0, rel=1e-6)


@pytest.mark.parametrize("n", [8, 64, 128, 192, 320, 448, 512])
def test_fft_against_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    np.testing.assert_allclose(oracle.fft_c2c(x, -1), np.fft.fft(x), atol=1e-10 * n)
    np.testing.assert_allclose(oracle.fft_c2c(x, +1), np.fft.ifft(x) * n, atol=1e-10 * n)


def _rz(a):
    c, s = np.cos(a), np.sin(a)
    return np.array([[c, s, 0], [-s, c, 0], [0, 0, 1.0]])


def _ry(a):
    c, s = np.cos(a), np.sin(a)
    return np.array([[c, 0, -s], [0, 1.0, 0], [s, 0, c]])


def test_cang_is_zyz_rotation():
    rng = np.random.default_rng(1)
    for _ in range(20):
        phi, theta, psi = rng.uniform(0, 360, 3)
        # DM(1:9) read row by row (the Fortran DM(3,3) transposed) is Rz(psi) Ry(theta) Rz(phi)
        dm = oracle.cang(phi, theta, psi).reshape(3, 3).astype(np.float64)
        d = np.radians([phi, theta, psi])
        r = _rz(d[2]) @ _ry(d[1]) @ _rz(d[0])
        np.testing.assert_allclose(dm, r, atol=2e-6)
        np.testing.assert_allclose(dm @ dm.T, np.eye(3), atol=1e-6)


def test_stage_image_matches_numpy():
    """PADD2 + forward FFT with SPIDER's sign + (-1)^(I+J) phase."""
    rng = np.random.default_rng(5)
    nx = 16
    img = rng.standard_normal((nx, nx)).astype(np.float32)
    bi = oracle.stage_image(img)
    n = 2 * nx
    g = np.arange(nx) - nx // 2
    outside = (g[:, None] ** 2 + g[None, :] ** 2) > (nx // 2) ** 2
    qs = img[outside].astype(np.float64).mean()
    pad = np.zeros((n, n))
    ip = (n - nx) // 2
    pad[ip:ip + nx, ip:ip + nx] = (img.astype(np.float64) - qs).astype(np.float32)
    f = np.conj(np.fft.rfft2(pad))                       # SPIDER forward sign
    ky, kx = np.meshgrid(np.arange(n), np.arange(nx + 1), indexing="ij")
    f *= np.where((kx + ky) % 2 == 0, 1.0, -1.0)
    np.testing.assert_allclose(bi, f, atol=1e-4)


def test_rtsq_shift_and_rotation():
    """RTSQ (rtsq.f:56-140): a (sx, sy) shift moves content by (+sx, +sy); a
    zero transform is the identity; 90 degrees maps the x axis onto y."""
    nx = 32
    g = np.arange(nx) - nx // 2
    img = np.exp(-((g[None, :] - 3) ** 2 + (g[:, None] + 2) ** 2) / 8.0).astype(np.float32)
    assert np.array_equal(oracle.rtsq(img, 0.0, 0.0, 0.0), img)
    out = oracle.rtsq(img, 0.0, 2.0, -1.0)
    np.testing.assert_allclose(out, np.roll(np.roll(img, 2, axis=1), -1, axis=0), atol=1e-6)
    r = oracle.rtsq(img, 90.0, 0.0, 0.0)
    p0 = np.unravel_index(np.argmax(img), img.shape)
    p1 = np.unravel_index(np.argmax(r), r.shape)
    # centre (16, 16): offset (dy, dx) = (-2, 3) -> (-3, -2) under a 90 degree turn
    assert (p1[0] - 16, p1[1] - 16) == (-(p0[1] - 16), (p0[0] - 16))
