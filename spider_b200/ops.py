"""Host-side mirror of SPIDER's reconstruction operations on the CUDA library.

Each function carries the name of the SPIDER operation it replaces and takes
the values that operation prompts for, in the same order and meaning:

=================  ==================================================  =========================
function           SPIDER operation (dispatch in vtil2.f)              reference subroutine
=================  ==================================================  =========================
``bp3f``           ``BP 3F``        (vtil2.f:301-313)                  BP3F, bp3f.f:79
``bp3f_partial``   ``BP 3F P``      partial Fourier volume + weights   BP3F(HALT), bp3f.f:191-248
``bp3f_merge``     ``BP 3F M``      merge partial volumes              BP3F_MERGE, bp3f.f:531
``bp32f``          ``BP 32F``       (vtil2.f:316-322)                  BP32F, bp32f.f:57
``rb3f``/``rb32f`` ``RB 3F/RB 32F`` RTSQ pre-rotation (vtil2.f:88-95)  BP3F(.TRUE.), bp3f.f:406-425
``pj3q``           ``PJ 3Q``        (vtil2.f:218-220)                  PJ3Q_N, pj3q_n.f:41
``bpcg``           ``BP CG``        (vtil2.f:324)                      BPCG, bpcg.f:70
=================  ==================================================  =========================

Arrays are numpy (host) or torch CUDA tensors (device, no host copy).  Images
are ``[nimg, nx, nx]`` float32 (x fastest), volumes ``[nz, ny, nx]``, angles
``[nimg, 3]`` = (psi, theta, phi) in degrees (angle-document registers 1-3).
Errors raise :class:`spider_b200._lib.SpiderError` carrying the IRTFLG-style
code (101 invalid argument, 102 missing data / radius too large, 46 memory).
"""
from __future__ import annotations

import ctypes
import threading

import numpy as np

from . import _lib
from ._lib import SpiderError, check

try:  # torch is plumbing for device memory; optional for host use
    import torch
except Exception:  # pragma: no cover
    torch = None

__all__ = ["Context", "default_context", "bp3f", "bp32f", "rb3f", "rb32f", "bp3f_partial", "bp3f_merge", "pj3q",
           "pj3q_adjoint", "bpcg", "cg_project", "cg_backproject", "SpiderError"]


def _is_dev(a) -> bool:
    return torch is not None and isinstance(a, torch.Tensor) and a.is_cuda


def _ptr(a):
    if a is None:
        return None
    if _is_dev(a):
        if a.dtype != torch.float32 and a.dtype != torch.uint8:
            raise SpiderError(101, f"device tensor dtype {a.dtype} (float32 expected)")
        if not a.is_contiguous():
            raise SpiderError(101, "device tensor must be contiguous")
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)


def _host_f32(a):
    if torch is not None and isinstance(a, torch.Tensor):
        a = a.detach().cpu().numpy()
    return np.ascontiguousarray(a, dtype=np.float32)


class Context:
    """One CUDA device + stream + reusable buffers (an ``spi_ctx``)."""

    def __init__(self, device: int = 0):
        L = _lib.load()
        h = ctypes.c_void_p()
        check(L.spi_ctx_create(device, ctypes.byref(h)))
        self._h = h
        self.device = device
        self._L = L
        self.fbs = False

    def set_fbs(self, on: bool):
        """SPIDER's ``MD`` FBS mode: RB 3F / RB 32F rotate with RTSF (on) or RTSQ."""
        check(self._L.spi_ctx_set_rb_interpolation(self._h, 1 if on else 0))
        self.fbs = bool(on)

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            self._L.spi_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    @property
    def launches(self) -> int:
        return int(self._L.spi_ctx_launch_count(self._h))

    @property
    def device_bytes(self) -> int:
        return int(self._L.spi_ctx_device_bytes(self._h))

    # -------- streaming back-projection (BP 3F / BP 32F) --------
    def bp_open(self, nx: int, ngrids: int = 1, sym=None, bf16: bool = False):
        sym_a = None if sym is None else _host_f32(sym)
        nsym = 0 if sym_a is None else sym_a.shape[0]
        check(self._L.spi_bp_open(self._h, nx, ngrids, _ptr(sym_a), nsym))
        check(self._L.spi_bp_set_spectrum_precision(self._h, 1 if bf16 else 0))
        self._nx = nx
        self._ngrids = ngrids

    KERNELS = {0: "insert_tile_kernel", 1: "insert_kernel", 2: "insert_xlane_kernel", 3: "insert_x4_kernel"}

    def bp_autotune(self, force: bool = False) -> dict:
        """Pick the insertion kernel and launch shape for the open
        reconstruction by timing them (call right after bp_open)."""
        check(self._L.spi_bp_autotune(self._h, 1 if force else 0))
        return self.bp_launch()

    def bp_launch(self) -> dict:
        k, t, b, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        check(self._L.spi_bp_get_launch(self._h, ctypes.byref(k), ctypes.byref(t), ctypes.byref(b), ctypes.byref(ms)))
        return {"kernel": self.KERNELS.get(k.value, str(k.value)), "threads": t.value, "blocks_per_sm": b.value,
                "tuned_ms": ms.value}

    def bp_insert(self, imgs, angles, half=None, inplane=None):
        """Insert images; with ``inplane`` [n, 3] = (angle, sx, sy) every image is
        first rotated and shifted by RTSQ (RB 3F / RB 32F)."""
        ang = _host_f32(angles)
        h = None if half is None else np.ascontiguousarray(
            half.detach().cpu().numpy() if (torch is not None and isinstance(half, torch.Tensor)) else half,
            dtype=np.uint8)
        dev = _is_dev(imgs)
        if not dev:
            imgs = _host_f32(imgs)
        n = int(imgs.shape[0])
        if ang.shape[0] != n:
            raise SpiderError(101, f"{n} images but {ang.shape[0]} angle triples")
        if inplane is None:
            check(self._L.spi_bp_insert(self._h, _ptr(imgs), n, _ptr(ang), _ptr(h), 1 if dev else 0))
        else:
            ip = _host_f32(inplane)
            if ip.shape != (n, 3):
                raise SpiderError(101, f"in-plane parameters must be [{n}, 3]")
            check(self._L.spi_bp_insert_rb(self._h, _ptr(imgs), n, _ptr(ang), _ptr(ip), _ptr(h), 1 if dev else 0))

    def bp_finish(self, want=("all",), device: bool = False):
        nx = self._nx
        outs = {}
        for k in want:
            if device:
                outs[k] = torch.empty((nx, nx, nx), dtype=torch.float32, device=f"cuda:{self.device}")
            else:
                outs[k] = np.zeros((nx, nx, nx), np.float32)
        check(self._L.spi_bp_finish(self._h, _ptr(outs.get("all")), _ptr(outs.get("1")), _ptr(outs.get("2")),
                                    1 if device else 0))
        return outs

    def bp_partial_out(self, g: int = 0):
        nx = self._nx
        n = 2 * nx
        x = np.zeros((n, n, nx + 1, 2), np.float32)
        w = np.zeros((n, n, nx + 1), np.float32)
        check(self._L.spi_bp_partial_out(self._h, g, _ptr(x), _ptr(w)))
        return x, w

    def bp_partial_add(self, x, w, g: int = 0):
        x = _host_f32(x)
        w = _host_f32(w)
        check(self._L.spi_bp_partial_add(self._h, g, _ptr(x), _ptr(w)))

    def bp_close(self):
        check(self._L.spi_bp_close(self._h))

    def set_accumulation(self, compensated: bool = True, fold_every: int = 0):
        """Grid accumulation of the next bp_open: compensated (two-sum folds
        of a partial grid every ``fold_every`` images, 0 = default) or plain
        FP32 atomics into the grid."""
        check(self._L.spi_bp_set_accumulation(self._h, 1 if compensated else 0, int(fold_every)))

    def bp_flush(self):
        """Fold pending sums and the compensation into the grids (before an
        exchange of caller-owned grids); synchronises the library stream."""
        check(self._L.spi_bp_flush(self._h))


_tls = threading.local()


def default_context(device: int = 0) -> Context:
    ctxs = getattr(_tls, "ctxs", None)
    if ctxs is None:
        ctxs = _tls.ctxs = {}
    if device not in ctxs:
        ctxs[device] = Context(device)
    return ctxs[device]


def _nx_of(imgs) -> int:
    if imgs.ndim != 3 or imgs.shape[1] != imgs.shape[2]:
        raise SpiderError(101, "ONLY WORKS ON SQUARE IMAGES")  # bp3f.f:135-138
    return int(imgs.shape[1])


def bp3f(imgs, angles, sym=None, *, ctx: Context | None = None, device_out: bool = False):
    """``BP 3F``: Fourier gridding back-projection -> volume [nx, nx, nx]."""
    ctx = ctx or default_context()
    nx = _nx_of(imgs)
    ctx.bp_open(nx, 1, sym)
    try:
        ctx.bp_insert(imgs, angles)
        return ctx.bp_finish(("all",), device=device_out)["all"]
    finally:
        ctx.bp_close()


def bp32f(imgs, angles, half, sym=None, *, ctx: Context | None = None, bf16: bool = False,
          device_out: bool = False):
    """``BP 32F``: returns (reconstructed volume, first sample volume, second sample volume)."""
    ctx = ctx or default_context()
    nx = _nx_of(imgs)
    ctx.bp_open(nx, 2, sym, bf16=bf16)
    try:
        ctx.bp_insert(imgs, angles, half)
        o = ctx.bp_finish(("all", "1", "2"), device=device_out)
        return o["all"], o["1"], o["2"]
    finally:
        ctx.bp_close()


def bp32f_multiclass(classes, sym=None, *, device: int = 0, bf16: bool = False, concurrent: bool = True,
                     device_out: bool = False, autotune: bool = False, one_launch: bool = True, ctxs=None):
    """``BP 32F`` of several classes of one image stream: ``classes`` is a list
    of (images [n_k, nx_k, nx_k], angles [n_k, 3], half mask [n_k]) with any
    box sizes.  Each class has its own context (grids, FFT plans).  With
    ``one_launch`` (default) all classes go through spi_bp_insert_multi: one
    insertion launch per round over every class's slices, on one stream.
    Otherwise, with ``concurrent`` the classes are inserted from one host
    thread each, so that their launches share the GPU.  Returns a list of
    (vol, vol1, vol2).  ``ctxs``: one context per class to use (and keep
    open) instead of new ones, so that repeated calls reuse their buffers
    and FFT plans."""
    import concurrent.futures as cf
    own = ctxs is None
    if own:
        ctxs = [Context(device) for _ in classes]
    elif len(ctxs) != len(classes):
        raise SpiderError(101, "one context per class")
    try:
        for c, (imgs, _, _) in zip(ctxs, classes):
            c.bp_open(_nx_of(imgs), 2, sym, bf16=bf16)
            if autotune and not one_launch:   # launch shape per box size (cached per process)
                c.bp_autotune()

        def finish_all():
            out = []
            for c in ctxs:
                o = c.bp_finish(("all", "1", "2"), device=device_out)
                out.append((o["all"], o["1"], o["2"]))
                if own:   # caller contexts stay open: a same-size bp_open keeps their buffers and plans
                    c.bp_close()
            return out

        if one_launch:
            bp_insert_multi(ctxs, classes)
            return finish_all()

        def insert(k):
            imgs, ang, half = classes[k]
            ctxs[k].bp_insert(imgs, ang, half)

        if concurrent and len(classes) > 1:
            with cf.ThreadPoolExecutor(max_workers=len(classes)) as ex:
                for f in [ex.submit(insert, k) for k in range(len(classes))]:
                    f.result()
        else:
            for k in range(len(classes)):
                insert(k)
        return finish_all()
    finally:
        if own:
            for c in ctxs:
                c.close()


def bp_insert_multi(ctxs, classes):
    """spi_bp_insert_multi: insert (images, angles, half) of every class into
    its open context, all classes in one insertion launch per round."""
    k = len(ctxs)
    if k != len(classes):
        raise SpiderError(101, "one context per class")
    keep = []
    dev = None
    P = ctypes.c_void_p * k
    pi, pa, ph = P(), P(), P()
    counts = (ctypes.c_int * k)()
    for i, (imgs, ang, half) in enumerate(classes):
        d = _is_dev(imgs)
        if dev is None:
            dev = d
        elif d != dev:
            raise SpiderError(101, "all classes' images must be on the host or all on the device")
        if not d:
            imgs = _host_f32(imgs)
        a = _host_f32(ang)
        if a.shape[0] != imgs.shape[0]:
            raise SpiderError(101, f"class {i}: {imgs.shape[0]} images but {a.shape[0]} angle triples")
        h = None if half is None else np.ascontiguousarray(
            half.detach().cpu().numpy() if (torch is not None and isinstance(half, torch.Tensor)) else half,
            dtype=np.uint8)
        keep += [imgs, a, h]
        pi[i] = _ptr(imgs).value if int(imgs.shape[0]) else None
        pa[i] = _ptr(a).value if int(a.shape[0]) else None
        ph[i] = None if h is None else _ptr(h).value
        counts[i] = int(imgs.shape[0])
    handles = P(*[c.handle.value for c in ctxs])
    check(ctxs[0]._L.spi_bp_insert_multi(handles, k, pi, counts, pa, ph, 1 if dev else 0))


def _rb_mode(ctx, fbs):
    """fbs None keeps the context's mode (SPIDER's ``MD`` FBS setting)."""
    if fbs is not None:
        ctx.set_fbs(bool(fbs))


def rb3f(imgs, angles, inplane, sym=None, *, ctx: Context | None = None, fbs=None):
    """``RB 3F``: RTSQ (RTSF with ``fbs`` or the context's FBS mode) by
    (angle, sx, sy) per image, then BP 3F."""
    ctx = ctx or default_context()
    _rb_mode(ctx, fbs)
    nx = _nx_of(imgs)
    ctx.bp_open(nx, 1, sym)
    try:
        ctx.bp_insert(imgs, angles, inplane=inplane)
        return ctx.bp_finish(("all",))["all"]
    finally:
        ctx.bp_close()


def rb32f(imgs, angles, inplane, half, sym=None, *, ctx: Context | None = None, fbs=None):
    """``RB 32F``: RTSQ (RTSF with ``fbs`` or the context's FBS mode) by
    (angle, sx, sy) per image, then BP 32F."""
    ctx = ctx or default_context()
    _rb_mode(ctx, fbs)
    nx = _nx_of(imgs)
    ctx.bp_open(nx, 2, sym)
    try:
        ctx.bp_insert(imgs, angles, half, inplane=inplane)
        o = ctx.bp_finish(("all", "1", "2"))
        return o["all"], o["1"], o["2"]
    finally:
        ctx.bp_close()


def bp3f_partial(imgs, angles, sym=None, *, ctx: Context | None = None):
    """``BP 3F P``: returns (X [2nx, 2nx, nx+1, 2] re/im, W [2nx, 2nx, nx+1]) after plane-0 symmetry."""
    ctx = ctx or default_context()
    nx = _nx_of(imgs)
    ctx.bp_open(nx, 1, sym)
    try:
        ctx.bp_insert(imgs, angles)
        return ctx.bp_partial_out(0)
    finally:
        ctx.bp_close()


def bp3f_merge(partials, sym=None, *, ctx: Context | None = None):
    """``BP 3F M``: sum partial (X, W) pairs and finish -> volume [nx, nx, nx]
    (symmetrised in real space when a symmetry list is given, bp3f.f:701-728)."""
    ctx = ctx or default_context()
    partials = list(partials)
    if not partials:
        raise SpiderError(101, "no partial volumes")
    nx = int(partials[0][1].shape[2]) - 1
    ctx.bp_open(nx, 1, sym)
    try:
        for x, w in partials:
            ctx.bp_partial_add(x, w)
        return ctx.bp_finish(("all",))["all"]
    finally:
        ctx.bp_close()


def _vol_shape(vol):
    if vol.ndim != 3:
        raise SpiderError(101, "volume must be 3-D")
    return int(vol.shape[2]), int(vol.shape[1]), int(vol.shape[0])


def pj3q(vol, angles, ri=None, *, ctx: Context | None = None):
    """``PJ 3Q``: trilinear projections [nang, ny, nx] of vol [nz, ny, nx]."""
    ctx = ctx or default_context()
    nx, ny, nz = _vol_shape(vol)
    if ri is None:
        ri = float(min(nx, ny, nz) // 2 - 2)  # pj3q_n.f:82
    ang = _host_f32(angles)
    nang = ang.shape[0]
    dev = _is_dev(vol)
    if dev:
        out = torch.empty((nang, ny, nx), dtype=torch.float32, device=vol.device)
    else:
        vol = _host_f32(vol)
        out = np.zeros((nang, ny, nx), np.float32)
    check(ctx._L.spi_pj3q(ctx.handle, _ptr(vol), nx, ny, nz, float(ri), _ptr(ang), nang, _ptr(out), 1 if dev else 0))
    return out


def pj3f(vol, angles, ri=None, *, ctx: Context | None = None):
    """``PJ 3F``: FBS (tricubic, FFT-derivative) projections [nang, n, n] of a
    cubic vol [n, n, n]; host arrays or CUDA tensors, as :func:`pj3q`."""
    ctx = ctx or default_context()
    nx, ny, nz = _vol_shape(vol)
    if ri is None:
        ri = float(min(nx, ny, nz) // 2 - 2)  # pj3q_n.f:82
    ang = _host_f32(angles)
    nang = ang.shape[0]
    dev = _is_dev(vol)
    if dev:
        out = torch.empty((nang, ny, nx), dtype=torch.float32, device=vol.device)
    else:
        vol = _host_f32(vol)
        out = np.zeros((nang, ny, nx), np.float32)
    check(ctx._L.spi_pj3f(ctx.handle, _ptr(vol), nx, ny, nz, float(ri), _ptr(ang), nang, _ptr(out), 1 if dev else 0))
    return out


def pj3q_adjoint(projs, angles, shape, ri=None, *, ctx: Context | None = None):
    """Exact adjoint of :func:`pj3q`: volume [nz, ny, nx] from projections [nang, ny, nx]."""
    ctx = ctx or default_context()
    nz, ny, nx = shape
    if ri is None:
        ri = float(min(nx, ny, nz) // 2 - 2)
    ang = _host_f32(angles)
    nang = ang.shape[0]
    dev = _is_dev(projs)
    if dev:
        out = torch.empty((nz, ny, nx), dtype=torch.float32, device=projs.device)
    else:
        projs = _host_f32(projs)
        out = np.zeros((nz, ny, nx), np.float32)
    check(ctx._L.spi_pj3q_adjoint(ctx.handle, _ptr(projs), nx, ny, nz, float(ri), _ptr(ang), nang, _ptr(out),
                                  1 if dev else 0))
    return out


def _set_cg_modes(ctx, fp64, interp):
    """BP CG precision mode and interpolation of the context (see bpcg)."""
    if isinstance(fp64, str):
        modes = {"mixed": 2, "fast": 3, "mixed64": 4}
        if fp64 not in modes:
            raise SpiderError(101, f"unknown BP CG precision {fp64!r}")
        prec = modes[fp64]
    else:
        prec = 1 if fp64 else 0
    check(ctx._L.spi_ctx_set_cg_precision(ctx.handle, prec))
    interps = {"linear": 0, "l": 0, "fbs": 1, "f": 1}
    if str(interp).lower() not in interps:
        raise SpiderError(101, f"unknown BP CG interpolation {interp!r}")
    check(ctx._L.spi_ctx_set_cg_interpolation(ctx.handle, interps[str(interp).lower()]))


def bpcg(projs, angles, ri=None, errm=5e-5, chim=0.0, maxit=20, mode=1, lam=2000.0, *,
         ctx: Context | None = None, fp64="mixed", interp="linear"):
    """``BP CG``.  Prompts in reference order: radius (default n/2-2),
    error & chi^2 limits, iteration limit & mode, lambda.
    ``interp``: "linear" (the 'L' answer) or "fbs" (the 'F' answer: FBS
    interpolation through FFT derivatives, BPCG_3_FBS); with "fbs", True
    and "mixed64" are FP64 throughout, "mixed" and "fast" keep FP64 vectors
    and arithmetic with FP32 interpolation tables, False is FP32.
    ``fp64``: "mixed" (default) keeps the CG vectors in FP64 and the
    projections in 47-bit fixed point with FP32 PROJT tables, "mixed64" the
    same with FP64 tables, "fast" 31-bit fixed point, True keeps everything
    in FP64, False uses the reference's REAL.
    Returns (volume [n,n,n], log [niter, 3] of (iteration, difference, chisq))."""
    ctx = ctx or default_context()
    _set_cg_modes(ctx, fp64, interp)
    projs = _host_f32(projs)
    n = _nx_of(projs)
    if ri is None:
        ri = float(n // 2 - 2)  # bpcg.f:161
    ang = _host_f32(angles)
    vol = np.zeros((n, n, n), np.float32)
    logv = np.zeros((max(maxit, 1), 3), np.float32)
    niter = ctypes.c_int(0)
    check(ctx._L.spi_bpcg(ctx.handle, _ptr(projs), n, projs.shape[0], _ptr(ang), float(ri), float(errm),
                          float(chim), int(maxit), int(mode), float(lam), _ptr(vol), _ptr(logv),
                          ctypes.cast(ctypes.byref(niter), ctypes.c_void_p)))
    return vol, logv[: niter.value].copy()


class _DeviceArray:
    """A device array the library passes to an all-reduce callback, as a
    zero-copy torch tensor through __cuda_array_interface__."""

    def __init__(self, ptr, count, fp64):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<f8" if fp64 else "<f4",
                                         "data": (int(ptr), False), "version": 3, "strides": None}


def allreduce_callback(sum_inplace):
    """Wrap ``sum_inplace(tensor)`` (sums a CUDA tensor over the ranks in
    place, e.g. ``torch.distributed.all_reduce``) as the library's
    spi_allreduce_fn.  The library's stream is synchronised before the call
    and the device after it, so the sum is complete when the callback returns."""
    def cb(ptr, count, fp64, stream, user):
        try:
            t = torch.as_tensor(_DeviceArray(ptr, count, fp64), device="cuda")
            torch.cuda.ExternalStream(stream, device=t.device).synchronize()
            sum_inplace(t)
            torch.cuda.synchronize(t.device)
            return 0
        except Exception:   # reported by the library as a failed all-reduce
            return 1
    return _lib.ALLREDUCE_FN(cb)


def bpcg_shard(projs, first, angles, ri=None, errm=5e-5, chim=0.0, maxit=20, mode=1, lam=2000.0, *,
               rank=0, world=1, sum_inplace=None, ctx: Context | None = None, fp64="mixed", interp="linear"):
    """One rank's BP CG over several processes (the reference's MPI form):
    ``projs`` are images first .. first+len(projs)-1 of the full ``angles``
    list; ``sum_inplace(tensor)`` sums a CUDA tensor over the ranks in place
    (CB, the image statistics, then BCKE every iteration).  Every rank returns
    the same (volume, log)."""
    ctx = ctx or default_context()
    _set_cg_modes(ctx, fp64, interp)
    projs = _host_f32(projs)
    ang = _host_f32(angles)
    count = int(projs.shape[0])
    n = int(projs.shape[-1])
    if ri is None:
        ri = float(n // 2 - 2)  # bpcg.f:161
    vol = np.zeros((n, n, n), np.float32)
    logv = np.zeros((max(maxit, 1), 3), np.float32)
    niter = ctypes.c_int(0)
    cb = allreduce_callback(sum_inplace) if sum_inplace is not None else ctypes.cast(None, _lib.ALLREDUCE_FN)
    check(ctx._L.spi_bpcg_shard(ctx.handle, _ptr(projs) if count else None, int(first), count, n, ang.shape[0],
                                _ptr(ang), float(ri), float(errm), float(chim), int(maxit), int(mode), float(lam),
                                int(rank), int(world), cb, None, _ptr(vol), _ptr(logv),
                                ctypes.cast(ctypes.byref(niter), ctypes.c_void_p)))
    return vol, logv[: niter.value].copy()


def bpcg3(projs, angles, half_mask, ri=None, errm=5e-5, chim=0.0, maxit=20, mode=1, lam=2000.0, *,
          ctx: Context | None = None, fp64="mixed", interp="linear"):
    """``BP CG 3``: the overall solution and one for each of two sample sets,
    as three independent CG solves (bpcg.f:139-160,300-400).  ``half_mask[i]``
    = 1 puts image i in the first sample (the reference draws the two lists
    with MAKETWOLISTS, bpcg.f:1593-1632, or reads them for ``BP CG 3L``).
    Returns (vol, vol1, vol2, (log, log1, log2))."""
    projs = _host_f32(projs)
    ang = _host_f32(angles)
    m = np.asarray(half_mask).astype(bool).reshape(-1)
    if m.shape[0] != projs.shape[0]:
        raise SpiderError(101, "half mask length differs from the number of images")
    v, lg = bpcg(projs, ang, ri, errm, chim, maxit, mode, lam, ctx=ctx, fp64=fp64, interp=interp)
    v1, lg1 = bpcg(projs[m], ang[m], ri, errm, chim, maxit, mode, lam, ctx=ctx, fp64=fp64, interp=interp)
    v2, lg2 = bpcg(projs[~m], ang[~m], ri, errm, chim, maxit, mode, lam, ctx=ctx, fp64=fp64, interp=interp)
    return v, v1, v2, (lg, lg1, lg2)


def cg_project(vol, angles, ri, *, ctx: Context | None = None):
    """PRJCQ_N (the BP CG projector A) of vol [n,n,n] -> [nang, n, n]."""
    ctx = ctx or default_context()
    ang = _host_f32(angles)
    n = int(vol.shape[0])
    dev = _is_dev(vol)
    if dev:
        out = torch.empty((ang.shape[0], n, n), dtype=torch.float32, device=vol.device)
    else:
        vol = _host_f32(vol)
        out = np.zeros((ang.shape[0], n, n), np.float32)
    check(ctx._L.spi_cg_project(ctx.handle, _ptr(vol), n, float(ri), _ptr(ang), ang.shape[0], _ptr(out),
                                1 if dev else 0))
    return out


def cg_backproject(projs, angles, ri, *, ctx: Context | None = None):
    """BCKPJ_LIN (the BP CG back-projector A^T) of [nang, n, n] -> [n, n, n]."""
    ctx = ctx or default_context()
    ang = _host_f32(angles)
    n = int(projs.shape[1])
    dev = _is_dev(projs)
    if dev:
        out = torch.empty((n, n, n), dtype=torch.float32, device=projs.device)
    else:
        projs = _host_f32(projs)
        out = np.zeros((n, n, n), np.float32)
    check(ctx._L.spi_cg_backproject(ctx.handle, _ptr(projs), n, float(ri), _ptr(ang), ang.shape[0], _ptr(out),
                                    1 if dev else 0))
    return out
