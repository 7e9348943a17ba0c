"""CPU oracle for SPIDER's reconstruction path -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper over ``oracle/_build/liboracle.so`` (built from
``oracle/spider_oracle.cpp`` by ``oracle/Makefile``), a C++ restatement of the
reference Fortran: BP 3F / BP 32F (bp3f.f, bp32f.f, oneline.f, fillbessi0.f),
PJ 3Q (pj3q_n.f, prepcub.f, wpro_n.f) and BP CG (bpcg.f, prjcq.f, bckpj.f,
prepcub_s.f, hiang.f).

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of
``bench.py`` may import this package, and only as the checker or as the timed
CPU baseline; the product (``spider_b200``) never calls it.

Parity against outputs of the reference itself is UNPINNED (the Fortran +
FFTW3 reference cannot be built on this machine and ships no golden data for
this path); the sub-functions are pinned to scipy / numpy implementations in
``tests/test_oracle_pins.py``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_i32p = ctypes.POINTER(ctypes.c_int)


def build() -> str:
    """Compile the oracle library (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = ctypes.CDLL(_SO)
        L.orc_fillbessil.argtypes = [ctypes.c_int, _f32p, _f32p, _f32p, _f32p]
        L.orc_windkb_table.argtypes = [ctypes.c_int, _f32p]
        L.orc_cang.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_float, _f32p]
        L.orc_fft_c2c.argtypes = [_f64p, _f64p, ctypes.c_int, ctypes.c_int]
        L.orc_stage_image.argtypes = [_f32p, ctypes.c_int, _f64p]
        L.orc_bp3f.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, _f32p, _f32p, ctypes.c_int,
                               _u8p, ctypes.c_int, ctypes.c_int, _f32p, _f32p, _f32p,
                               _f64p, _f64p, ctypes.c_int]
        L.orc_bp3f.restype = ctypes.c_int
        L.orc_rb3f.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, _f32p, _f32p, _u8p, ctypes.c_int,
                               _f32p, _f32p, _f32p, ctypes.c_int, ctypes.c_int]
        L.orc_rb3f.restype = ctypes.c_int
        L.orc_symvol.argtypes = [_f32p, _f32p, ctypes.c_int, _f32p, ctypes.c_int]
        L.orc_rtsf.argtypes = [_f32p, _f32p, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float]
        L.orc_rtsf.restype = None
        L.orc_rtsq.argtypes = [_f32p, _f32p, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                               ctypes.c_float]
        L.orc_bp_insert_only.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, _f32p, _u8p, ctypes.c_int]
        L.orc_bp_insert_only.restype = ctypes.c_int
        L.orc_bp_session_open.argtypes = [ctypes.c_int]
        L.orc_bp_session_open.restype = ctypes.c_void_p
        L.orc_bp_session_free.argtypes = [ctypes.c_void_p]
        L.orc_bp_session_insert.argtypes = [ctypes.c_void_p, _f32p, ctypes.c_int, _f32p, _u8p, ctypes.c_int]
        L.orc_bp_session_insert.restype = ctypes.c_int
        L.orc_pj3f.argtypes = [_f32p, ctypes.c_int, ctypes.c_float, _f32p, ctypes.c_int, ctypes.c_int, _f32p,
                               ctypes.c_int]
        L.orc_pj3f.restype = None
        L.orc_pj3q.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                               _f32p, ctypes.c_int, ctypes.c_int, _f32p, ctypes.c_int]
        L.orc_prepcub_count.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float]
        L.orc_prepcub_count.restype = ctypes.c_int
        L.orc_bpcg.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, _f32p, ctypes.c_float, ctypes.c_float,
                               ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                               _f32p, _f32p, _i32p, _i32p, _f64p, ctypes.c_int]
        L.orc_bpcg.restype = ctypes.c_int
        L.orc_bpcg_fbs.argtypes = L.orc_bpcg.argtypes
        L.orc_bpcg_fbs.restype = ctypes.c_int
        L.orc_fbs2.argtypes = [_f32p, ctypes.c_int, _f32p, ctypes.c_int, ctypes.c_int, _f64p]
        L.orc_fbs3.argtypes = [_f32p, ctypes.c_int, _f32p, ctypes.c_int, _f64p]
        L.orc_prjcq_fbs3.argtypes = [_f32p, ctypes.c_int, _f32p, ctypes.c_int, ctypes.c_int, _f32p]
        L.orc_prjcq.argtypes = [_f32p, ctypes.c_int, ctypes.c_float, _f32p, ctypes.c_int, ctypes.c_int, _f32p]
        L.orc_bckpj.argtypes = [_f32p, ctypes.c_int, ctypes.c_float, _f32p, ctypes.c_int, ctypes.c_int, _f32p]
        L.orc_hiang.argtypes = [_f32p, ctypes.c_int, _f32p, _i32p, _f32p]
        L.orc_hiang.restype = ctypes.c_int
        L.orc_fixedge.argtypes = [_f32p, ctypes.c_int, ctypes.c_float, ctypes.c_int]
        L.orc_fslice_insert.argtypes = [_f64p, ctypes.c_int, _f32p, ctypes.c_int, _f64p, ctypes.c_int]
        L.orc_fslice_insert.restype = None
        L.orc_fslice_extract.argtypes = [_f64p, ctypes.c_int, _f32p, ctypes.c_int, _f64p, ctypes.c_int]
        L.orc_fslice_extract.restype = None
        L.orc_prepcub_s_count.argtypes = [ctypes.c_int, ctypes.c_float]
        L.orc_prepcub_s_count.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a, t):
    if a is None:
        return None
    return a.ctypes.data_as(t)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def kb_table(n2: int):
    """FILLBESSIL (fillbessi0.f:88-125): returns (tabi[5000], fltb, alpha, aaaa)."""
    tab = np.zeros(5000, np.float32)
    f, a, aa = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    lib().orc_fillbessil(n2, _p(tab, _f32p), ctypes.byref(f), ctypes.byref(a), ctypes.byref(aa))
    return tab, f.value, a.value, aa.value


def windkb_table(nx: int) -> np.ndarray:
    """|WKB| of WINDKB2A (bp32f.f:964-1005) per integer squared radius 0..(nx/2)^2."""
    out = np.zeros((nx // 2) ** 2 + 1, np.float32)
    lib().orc_windkb_table(nx, _p(out, _f32p))
    return out


def cang(phi: float, theta: float, psi: float) -> np.ndarray:
    """CANG (cang.f:44-81): DM(9), column-major 3x3."""
    dm = np.zeros(9, np.float32)
    lib().orc_cang(phi, theta, psi, _p(dm, _f32p))
    return dm


def fft_c2c(x: np.ndarray, sign: int = -1) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.zeros_like(x)
    lib().orc_fft_c2c(x.ctypes.data_as(_f64p), out.ctypes.data_as(_f64p), x.size, sign)
    return out


def stage_image(img: np.ndarray) -> np.ndarray:
    """PADD2 + forward FFT (SPIDER sign) + phase: complex128 [2nx, nx+1]."""
    img = _f32(img)
    nx = img.shape[0]
    out = np.zeros((2 * nx, nx + 1), np.complex128)
    lib().orc_stage_image(_p(img, _f32p), nx, out.ctypes.data_as(_f64p))
    return out


def bp3f(imgs, angles, *, sym=None, prec=0, nthreads=0):
    """BP 3F: imgs [nang, nx, nx] float32, angles [nang, 3] = (psi, theta, phi) deg."""
    imgs = _f32(imgs)
    ang = _f32(angles)
    nang, nx = imgs.shape[0], imgs.shape[1]
    vol = np.zeros((nx, nx, nx), np.float32)
    sym_a = _f32(sym) if sym is not None else None
    nsym = 0 if sym is None else sym_a.shape[0]
    rc = lib().orc_bp3f(_p(imgs, _f32p), nx, nang, _p(ang, _f32p), _p(sym_a, _f32p), nsym,
                        None, 0, prec, _p(vol, _f32p), None, None, None, None, nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle bp3f failed: {rc}")
    return vol


def bp3f_partial(imgs, angles, *, sym=None, prec=0, nthreads=0):
    """BP 3F P: returns (X complex128 [2nx, 2nx, nx+1], W float64 [2nx, 2nx, nx+1])."""
    imgs = _f32(imgs)
    ang = _f32(angles)
    nang, nx = imgs.shape[0], imgs.shape[1]
    n = 2 * nx
    x = np.zeros((n, n, nx + 1), np.complex128)
    w = np.zeros((n, n, nx + 1), np.float64)
    sym_a = _f32(sym) if sym is not None else None
    nsym = 0 if sym is None else sym_a.shape[0]
    rc = lib().orc_bp3f(_p(imgs, _f32p), nx, nang, _p(ang, _f32p), _p(sym_a, _f32p), nsym,
                        None, 1, prec, None, None, None, x.ctypes.data_as(_f64p),
                        w.ctypes.data_as(_f64p), nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle bp3f partial failed: {rc}")
    return x, w


def bp32f(imgs, angles, half, *, sym=None, prec=0, nthreads=0):
    """BP 32F: returns (vol_all, vol_1, vol_2); half[i] != 0 routes image i to set 1."""
    imgs = _f32(imgs)
    ang = _f32(angles)
    h = np.ascontiguousarray(half, dtype=np.uint8)
    nang, nx = imgs.shape[0], imgs.shape[1]
    vols = [np.zeros((nx, nx, nx), np.float32) for _ in range(3)]
    sym_a = _f32(sym) if sym is not None else None
    nsym = 0 if sym is None else sym_a.shape[0]
    rc = lib().orc_bp3f(_p(imgs, _f32p), nx, nang, _p(ang, _f32p), _p(sym_a, _f32p), nsym,
                        _p(h, _u8p), 0, prec, _p(vols[0], _f32p), _p(vols[1], _f32p),
                        _p(vols[2], _f32p), None, None, nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle bp32f failed: {rc}")
    return tuple(vols)


def symvol(vol, sym):
    """SYMVOL (symvol.f:39-180): sum of the volume rotated by each symmetry."""
    vol = _f32(vol)
    sa = _f32(sym)
    out = np.zeros_like(vol)
    lib().orc_symvol(_p(vol, _f32p), _p(out, _f32p), vol.shape[0], _p(sa, _f32p), sa.shape[0])
    return out


def rtsq(img, theta, shx, shy):
    """RTSQ (rtsq.f:56-140) of one image [ny, nx]: rotate by theta degrees, shift."""
    img = _f32(img)
    out = np.zeros_like(img)
    lib().orc_rtsq(_p(img, _f32p), _p(out, _f32p), img.shape[1], img.shape[0], theta, shx, shy)
    return out


def rtsf(img, theta, shx, shy):
    """RTSF (rtsf.f:109-205, SCLI = 1) of one square image: FBS rotate and shift."""
    img = _f32(img)
    out = np.zeros_like(img)
    lib().orc_rtsf(_p(img, _f32p), _p(out, _f32p), img.shape[1], theta, shx, shy)
    return out


def rb3f(imgs, angles, inplane, half=None, *, prec=0, nthreads=0, fbs=False):
    """RB 3F / RB 32F: RTSQ (RTSF with ``fbs``, SPIDER's FBS mode) with inplane
    [n, 3] = (angle, sx, sy), then BP 3F (half None) or BP 32F (returns three volumes)."""
    imgs = _f32(imgs)
    ang = _f32(angles)
    ip = _f32(inplane)
    nang, nx = imgs.shape[0], imgs.shape[1]
    vols = [np.zeros((nx, nx, nx), np.float32) for _ in range(3)]
    h = None if half is None else np.ascontiguousarray(half, dtype=np.uint8)
    rc = lib().orc_rb3f(_p(imgs, _f32p), nx, nang, _p(ang, _f32p), _p(ip, _f32p), _p(h, _u8p), prec,
                        _p(vols[0], _f32p), _p(vols[1], _f32p) if h is not None else None,
                        _p(vols[2], _f32p) if h is not None else None, nthreads, 1 if fbs else 0)
    if rc != 0:
        raise RuntimeError(f"oracle rb3f failed: {rc}")
    return vols[0] if h is None else tuple(vols)


def bp32f_insert_only(imgs, angles, half, *, nthreads=0):
    """BP 32F insertion (PADD2 + FFT + ONELINE) of a sample, FP32, timing use."""
    imgs = _f32(imgs)
    ang = _f32(angles)
    h = np.ascontiguousarray(half, dtype=np.uint8)
    rc = lib().orc_bp_insert_only(_p(imgs, _f32p), imgs.shape[1], imgs.shape[0], _p(ang, _f32p), _p(h, _u8p),
                                  nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle insert failed: {rc}")


class BpSession:
    """Two FP32 grids zeroed once; insert() times the per-image work only."""

    def __init__(self, nx: int):
        self.nx = nx
        self._h = lib().orc_bp_session_open(nx)

    def insert(self, imgs, angles, half, nthreads=0):
        imgs = _f32(imgs)
        ang = _f32(angles)
        h = np.ascontiguousarray(half, dtype=np.uint8)
        lib().orc_bp_session_insert(self._h, _p(imgs, _f32p), imgs.shape[0], _p(ang, _f32p), _p(h, _u8p), nthreads)

    def close(self):
        if self._h:
            lib().orc_bp_session_free(self._h)
            self._h = None

    def __del__(self):
        self.close()


def pj3f(vol, angles, ri=None, *, prec=0, nthreads=0):
    """PJ 3F (PJ 3Q with FBS interpolation): cubic vol [n, n, n] -> projections [nang, n, n]."""
    vol = _f32(vol)
    n = vol.shape[0]
    if vol.shape != (n, n, n):
        raise ValueError("PJ 3F: cubic volume expected")
    if ri is None:
        ri = float(n // 2 - 2)
    ang = _f32(angles)
    nang = ang.shape[0]
    out = np.zeros((nang, n, n), np.float32)
    lib().orc_pj3f(_p(vol, _f32p), n, ri, _p(ang, _f32p), nang, prec, _p(out, _f32p), nthreads)
    return out


def pj3q(vol, angles, ri=None, *, prec=0, nthreads=0):
    """PJ 3Q: vol [nz, ny, nx] float32 -> projections [nang, ny, nx]."""
    vol = _f32(vol)
    nz, ny, nx = vol.shape
    if ri is None:
        ri = float(min(nx, ny, nz) // 2 - 2)
    ang = _f32(angles)
    nang = ang.shape[0]
    out = np.zeros((nang, ny, nx), np.float32)
    lib().orc_pj3q(_p(vol, _f32p), nx, ny, nz, ri, _p(ang, _f32p), nang, prec, _p(out, _f32p), nthreads)
    return out


def prepcub_count(nx, ny, nz, ri):
    return lib().orc_prepcub_count(nx, ny, nz, ri)


def bpcg(projs, angles, ri, *, errm=5e-5, chim=0.0, maxit=20, mode=1, lam=2000.0, prec=0, nthreads=0, fbs=False):
    """BP CG (linear, or FBS with ``fbs``): returns (vol [n,n,n], log [niter,3], nang_eff, stats[4])."""
    projs = _f32(projs)
    ang = _f32(angles)
    nang, n = projs.shape[0], projs.shape[1]
    vol = np.zeros((n, n, n), np.float32)
    logv = np.zeros((max(maxit, 1), 3), np.float32)
    niter = ctypes.c_int(0)
    neff = ctypes.c_int(0)
    stats = np.zeros(4, np.float64)
    fn = lib().orc_bpcg_fbs if fbs else lib().orc_bpcg
    rc = fn(_p(projs, _f32p), n, nang, _p(ang, _f32p), ri, errm, chim, maxit, mode, lam,
            prec, _p(vol, _f32p), _p(logv, _f32p), ctypes.byref(niter), ctypes.byref(neff),
            stats.ctypes.data_as(_f64p), nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle bpcg failed: {rc}")
    return vol, logv[: niter.value].copy(), neff.value, stats


def prjcq(vol, angles, ri, *, prec=0):
    """PRJCQ_N (prjcq.f:48-82) of vol for each (psi,theta,phi): [nang, n, n]."""
    vol = _f32(vol)
    n = vol.shape[0]
    ang = _f32(angles)
    out = np.zeros((ang.shape[0], n, n), np.float32)
    lib().orc_prjcq(_p(vol, _f32p), n, ri, _p(ang, _f32p), ang.shape[0], prec, _p(out, _f32p))
    return out


def bckpj(projs, angles, ri, *, prec=0):
    """Sum over images of BCKPJ_LIN (bckpj.f:59-94) via PROJT: [n, n, n]."""
    projs = _f32(projs)
    n = projs.shape[1]
    ang = _f32(angles)
    out = np.zeros((n, n, n), np.float32)
    lib().orc_bckpj(_p(projs, _f32p), n, ri, _p(ang, _f32p), ang.shape[0], prec, _p(out, _f32p))
    return out


def hiang(angles):
    """HIANG (hiang.f:40-112): returns (phi_theta [lo,2], lb [lo], dm [lo,9])."""
    ang = _f32(angles)
    nang = ang.shape[0]
    pt = np.zeros((nang, 2), np.float32)
    lb = np.zeros(nang, np.int32)
    dm = np.zeros((nang, 9), np.float32)
    lo = lib().orc_hiang(_p(ang, _f32p), nang, _p(pt, _f32p), lb.ctypes.data_as(_i32p), _p(dm, _f32p))
    return pt[:lo].copy(), lb[:lo].copy(), dm[:lo].copy()


def fixedge(p, ri, mode):
    p = _f32(p).copy()
    lib().orc_fixedge(_p(p, _f32p), p.shape[0], ri, mode)
    return p


def prepcub_s_count(n, ri):
    return lib().orc_prepcub_s_count(n, ri)


def fbs2(img, xy, prec=1):
    """FBS2_PREP + FBS2 (fbs2.f) of an n x n image at points xy [m, 2] (1-based X, Y)."""
    img = _f32(img)
    xy = _f32(xy)
    out = np.zeros(xy.shape[0], np.float64)
    lib().orc_fbs2(_p(img, _f32p), img.shape[0], _p(xy, _f32p), xy.shape[0], prec, out.ctypes.data_as(_f64p))
    return out


def fbs3(vol, xyz):
    """FBS3_PREP + FBS3 (fbs3.f, FP64) of an n^3 volume at points xyz [m, 3] (1-based)."""
    vol = _f32(vol)
    xyz = _f32(xyz)
    out = np.zeros(xyz.shape[0], np.float64)
    lib().orc_fbs3(_p(vol, _f32p), vol.shape[0], _p(xyz, _f32p), xyz.shape[0], out.ctypes.data_as(_f64p))
    return out


def prjcq_fbs3(vol, angles, prec=1):
    """PRJCQ_FBS3 (prjcq.f:97-167) of vol for each (psi, theta, phi): [nang, n, n]."""
    vol = _f32(vol)
    ang = _f32(angles)
    n = vol.shape[0]
    out = np.zeros((ang.shape[0], n, n), np.float32)
    lib().orc_prjcq_fbs3(_p(vol, _f32p), n, _p(ang, _f32p), ang.shape[0], prec, _p(out, _f32p))
    return out


def fslice_extract(grid, angles, *, nthreads=0):
    """FourierSlice forward in FP64: complex grid [2nx, 2nx, nx+1] -> slices
    [nang, 2nx, nx+1] (the adjoint of ONELINE's insertion without weights)."""
    X = np.ascontiguousarray(grid, dtype=np.complex128)
    n, nx = X.shape[0], X.shape[2] - 1
    ang = _f32(angles)
    out = np.zeros((ang.shape[0], n, nx + 1), np.complex128)
    lib().orc_fslice_extract(X.ctypes.data_as(_f64p), nx, _p(ang, _f32p), ang.shape[0], out.ctypes.data_as(_f64p),
                             nthreads)
    return out


def fslice_insert(slices, angles, *, nthreads=0):
    """FourierSlice adjoint in FP64: slices [nang, 2nx, nx+1] -> grid
    [2nx, 2nx, nx+1] (ONELINE's insertion of X without weights)."""
    T = np.ascontiguousarray(slices, dtype=np.complex128)
    n, nx = T.shape[1], T.shape[2] - 1
    ang = _f32(angles)
    out = np.zeros((n, n, nx + 1), np.complex128)
    lib().orc_fslice_insert(T.ctypes.data_as(_f64p), nx, _p(ang, _f32p), ang.shape[0], out.ctypes.data_as(_f64p),
                            nthreads)
    return out
