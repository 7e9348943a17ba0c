"""Seeded synthetic inputs with the shapes of the reconstruction workloads.

No public dataset is named for this path; the phantoms are sums of isotropic
Gaussian blobs, the angles are uniform on SO(3) and written in SPIDER's
angle-document order (psi, theta, phi in degrees), the half-set assignment is
an explicit Bernoulli(1/2) mask.
"""
from __future__ import annotations

import numpy as np


def rng_for(config_index: int) -> np.random.Generator:
    return np.random.default_rng(1000 + config_index)


def blob_phantom(nx: int, nblobs: int, sigma=(2.0, 5.0), amp=(0.5, 1.0), radius=None,
                 rng: np.random.Generator | None = None) -> np.ndarray:
    """Volume [nz, ny, nx] float32: sum of A*exp(-|r-c|^2/(2 s^2)).

    Centres uniform inside a ball of `radius` (default 0.375*nx) around the
    SPIDER centre nx//2 (0-based), sigma and amplitude uniform in the ranges.
    """
    rng = rng or np.random.default_rng(0)
    if radius is None:
        radius = 0.375 * nx
    c0 = nx // 2
    g = np.arange(nx, dtype=np.float64) - c0
    vol = np.zeros((nx, nx, nx), np.float64)
    for _ in range(nblobs):
        while True:
            p = rng.uniform(-radius, radius, 3)
            if np.dot(p, p) <= radius * radius:
                break
        s = rng.uniform(*sigma)
        a = rng.uniform(*amp)
        ez = np.exp(-((g - p[2]) ** 2) / (2 * s * s))
        ey = np.exp(-((g - p[1]) ** 2) / (2 * s * s))
        ex = np.exp(-((g - p[0]) ** 2) / (2 * s * s))
        vol += a * ez[:, None, None] * ey[None, :, None] * ex[None, None, :]
    return vol.astype(np.float32)


def so3_angles(n: int, rng: np.random.Generator | None = None) -> np.ndarray:
    """[n, 3] float32 (psi, theta, phi) in degrees, uniform on SO(3)."""
    rng = rng or np.random.default_rng(0)
    psi = rng.uniform(0.0, 360.0, n)
    phi = rng.uniform(0.0, 360.0, n)
    theta = np.degrees(np.arccos(rng.uniform(-1.0, 1.0, n)))
    return np.stack([psi, theta, phi], axis=1).astype(np.float32)


def add_noise(projs: np.ndarray, snr: float, rng: np.random.Generator | None = None) -> np.ndarray:
    """Additive white Gaussian noise with variance var(clean)/snr per image."""
    rng = rng or np.random.default_rng(0)
    out = np.empty_like(projs)
    for i in range(projs.shape[0]):
        v = float(projs[i].var())
        sd = np.sqrt(v / snr) if v > 0 else 0.0
        out[i] = projs[i] + rng.normal(0.0, sd, projs[i].shape).astype(np.float32)
    return out


def half_mask(n: int, rng: np.random.Generator | None = None) -> np.ndarray:
    """Bernoulli(1/2) half-set assignment: 1 = first sample, 0 = second."""
    rng = rng or np.random.default_rng(0)
    return (rng.random(n) < 0.5).astype(np.uint8)


def fourier_shift(imgs: np.ndarray, shifts: np.ndarray) -> np.ndarray:
    """Circularly shift each image by (sx, sy) pixels through a Fourier phase."""
    n = imgs.shape[-1]
    k = np.fft.fftfreq(n)
    out = np.empty_like(imgs)
    for i in range(imgs.shape[0]):
        ph = np.exp(-2j * np.pi * (k[None, :] * shifts[i, 0] + k[:, None] * shifts[i, 1]))
        out[i] = np.real(np.fft.ifft2(np.fft.fft2(imgs[i]) * ph)).astype(np.float32)
    return out


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.linalg.norm((a - b).ravel())
    r = np.linalg.norm(b.ravel())
    return float(d / r) if r > 0 else float(d)


def fsc(v1: np.ndarray, v2: np.ndarray) -> np.ndarray:
    """Fourier shell correlation per integer shell radius 0..n//2."""
    f1 = np.fft.fftshift(np.fft.fftn(np.asarray(v1, np.float64)))
    f2 = np.fft.fftshift(np.fft.fftn(np.asarray(v2, np.float64)))
    n = v1.shape[0]
    g = np.arange(n) - n // 2
    r = np.sqrt(g[:, None, None] ** 2 + g[None, :, None] ** 2 + g[None, None, :] ** 2)
    ri = np.rint(r).astype(np.int64).ravel()
    m = ri <= n // 2
    ri = ri[m]
    a, b = f1.ravel()[m], f2.ravel()[m]
    nb = n // 2 + 1
    num = np.bincount(ri, weights=(a * np.conj(b)).real, minlength=nb)
    d1 = np.bincount(ri, weights=np.abs(a) ** 2, minlength=nb)
    d2 = np.bincount(ri, weights=np.abs(b) ** 2, minlength=nb)
    den = np.sqrt(d1 * d2)
    out = np.ones(nb)
    ok = den > 0
    out[ok] = num[ok] / den[ok]
    return out


def projection_stack(ctx, vol: np.ndarray, angles: np.ndarray, snr: float | None = None, shifts=None,
                     seed: int = 0, chunk: int = 4096):
    """Noisy, shifted PJ 3Q projections as a CUDA tensor [n, ny, nx] float32.

    The clean projections come from this library's PJ 3Q (``ops.pj3q``) in
    chunks; ``shifts`` [n, 2] = (sx, sy) pixels moves each image circularly by
    a Fourier phase (+x by +sx, the direction RTSQ shifts); ``snr`` adds white
    Gaussian noise of variance var(image)/snr from a seeded torch generator.
    Test and benchmark data only: the inputs of every path come from here and
    go to the GPU path and the oracle alike.
    """
    import torch

    from . import ops
    dev = torch.device("cuda", ctx.device)
    gen = torch.Generator(device=dev)
    gen.manual_seed(int(seed))
    n = int(angles.shape[0])
    ny, nx = int(vol.shape[1]), int(vol.shape[2])
    out = torch.empty((n, ny, nx), dtype=torch.float32, device=dev)
    dvol = torch.from_numpy(np.ascontiguousarray(vol, np.float32)).to(dev)
    for a0 in range(0, n, chunk):
        a1 = min(n, a0 + chunk)
        pr = ops.pj3q(dvol, angles[a0:a1], ctx=ctx)
        if shifts is not None:
            ky = torch.fft.fftfreq(ny, device=dev, dtype=torch.float64)[:, None]
            kx = torch.fft.fftfreq(nx, device=dev, dtype=torch.float64)[None, :]
            sh = torch.as_tensor(np.asarray(shifts[a0:a1], np.float64), device=dev)
            ph = torch.exp(-2j * np.pi * (kx[None] * sh[:, 0, None, None] + ky[None] * sh[:, 1, None, None]))
            pr = torch.fft.ifft2(torch.fft.fft2(pr.double()) * ph).real.float()
        if snr:
            sd = torch.sqrt(pr.var(dim=(1, 2), keepdim=True) / snr)
            pr = pr + torch.randn(pr.shape, device=dev, generator=gen) * sd
        out[a0:a1] = pr
    return out
