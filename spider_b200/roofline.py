"""Algorithmic byte counts for the gridding insertion (roofline numerator).

A gridding tap of ONELINE (oneline.f:76-150) reads and writes one voxel of
the Fourier grid: 8 bytes of complex X and 4 bytes of weight W each way, so
24 bytes per nonzero tap.  The insertion also reads the image spectrum once.
The nonzero-tap count of an image depends on its orientation; it is counted
here exactly, with the same float arithmetic as the kernel, for a sample of
orientations.
"""
from __future__ import annotations

import numpy as np

BYTES_PER_TAP = 24


def _nint(v: np.ndarray) -> np.ndarray:
    f = np.floor(v)
    return (f + ((v - f) >= np.float32(0.5))).astype(np.int64)


def taps_for_slice(nx: int, dm: np.ndarray, tab: np.ndarray, fltb: float) -> int:
    """Number of nonzero taps ONELINE adds for one slice (dm = DMS(1:6))."""
    N, N2, LN2 = 2 * nx, nx, 2
    f32 = np.float32
    J = np.arange(-nx + 1, nx + 1)
    I = np.arange(0, nx + 1)
    II, JJ = np.meshgrid(I, J, indexing="xy")
    ok = (II * II + JJ * JJ < (N * N) // 4) & ~((II == 0) & (JJ < 0))
    fi = II[ok].astype(f32)
    fj = JJ[ok].astype(f32)
    d = dm.astype(f32)
    x = fi * d[0] + fj * d[3]
    y = fi * d[1] + fj * d[4]
    z = fi * d[2] + fj * d[5]
    neg = x < 0
    x = np.where(neg, -x, x)
    y = np.where(neg, -y, y)
    z = np.where(neg, -z, z)
    fN = f32(N)
    ixn = ((x + f32(0.5)) + fN).astype(np.int64) - N
    iyn = ((y + f32(0.5)) + fN).astype(np.int64) - N
    izn = ((z + f32(0.5)) + fN).astype(np.int64) - N
    inb = (ixn <= N2 - LN2 - 1) & (iyn >= -N2 + 2 + LN2) & (iyn <= N2 - LN2 - 1) & \
          (izn >= -N2 + 2 + LN2) & (izn <= N2 - LN2 - 1)
    x, y, z, ixn, iyn, izn = x[inb], y[inb], z[inb], ixn[inb], iyn[inb], izn[inb]
    fl = f32(fltb)
    off = np.arange(-2, 3)
    tz = tab[_nint(np.abs(z[:, None] - (izn[:, None] + off).astype(f32)) * fl)] != 0
    ty = tab[_nint(np.abs(y[:, None] - (iyn[:, None] + off).astype(f32)) * fl)] != 0
    tx = tab[_nint(np.abs(x[:, None] - (ixn[:, None] + off).astype(f32)) * fl)] != 0
    nyz = tz.sum(1) * ty.sum(1)
    lb = -np.minimum(ixn, LN2)
    main_x = (tx & ((off[None, :]) >= lb[:, None])).sum(1)
    refl_x = (tx & ((ixn[:, None] + off[None, :]) <= -1)).sum(1) * (ixn < LN2)
    return int((nyz * (main_x + refl_x)).sum())


def kb_table(n2: int):
    """FILLBESSIL table from the CUDA library's host code: (tab[5000], fltb)."""
    import ctypes
    from . import _lib
    tab = np.zeros(5000, np.float32)
    fl = ctypes.c_float()
    _lib.check(_lib.load().spi_kb_table(n2, tab.ctypes.data_as(ctypes.c_void_p), ctypes.cast(ctypes.byref(fl), ctypes.c_void_p)))
    return tab, fl.value


def mean_taps(nx: int, dms: np.ndarray, tab: np.ndarray, fltb: float) -> float:
    return float(np.mean([taps_for_slice(nx, dm, tab, fltb) for dm in dms]))


def spectrum_bytes(nx: int, bf16: bool = False) -> int:
    return (nx + 1) * 2 * nx * (4 if bf16 else 8)
