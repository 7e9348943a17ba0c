"""PJ 3Q as a differentiable operator.

``PJ3Q`` is a ``torch.autograd.Function``: forward is the trilinear
projection of ``spi_pj3q`` (WPRO_N, wpro_n.f:44-150), backward is its exact
adjoint ``spi_pj3q_adjoint`` -- the trilinear insertion that spreads each
projection value back onto the 8 voxels around the same sample position.  The
backward recomputes the rotated sample positions from the angles instead of
storing them, so the autograd graph holds only the angles.
"""
from __future__ import annotations

import numpy as np
import torch

from . import ops


class PJ3Q(torch.autograd.Function):
    @staticmethod
    def forward(fctx, vol: torch.Tensor, angles: np.ndarray, ri: float, lib_ctx):
        if not vol.is_cuda:
            raise ops.SpiderError(101, "PJ3Q needs a CUDA volume (there is no CPU path)")
        fctx.angles = angles
        fctx.ri = ri
        fctx.lib_ctx = lib_ctx
        fctx.shape = tuple(vol.shape)
        return ops.pj3q(vol.detach().contiguous().float(), angles, ri, ctx=lib_ctx)

    @staticmethod
    def backward(fctx, grad: torch.Tensor):
        g = ops.pj3q_adjoint(grad.detach().contiguous().float(), fctx.angles, fctx.shape, fctx.ri,
                             ctx=fctx.lib_ctx)
        return g, None, None, None


def pj3q(vol: torch.Tensor, angles, ri: float | None = None, ctx: ops.Context | None = None) -> torch.Tensor:
    """Differentiable ``PJ 3Q`` of a CUDA volume [nz, ny, nx] -> [nang, ny, nx]."""
    if ri is None:
        ri = float(min(vol.shape) // 2 - 2)
    ang = np.ascontiguousarray(angles, dtype=np.float32)
    return PJ3Q.apply(vol, ang, float(ri), ctx or ops.default_context(vol.device.index or 0))


# ---------------------------------------------------------------------------
# Capturable operator pair and a differentiable CG reconstruction on it.
class PJ3QPlan:
    """PJ 3Q (forward) and its exact adjoint for one volume shape, radius and
    angle list, with the voxel runs and rotations uploaded once
    (``spi_pj3q_plan_*``).  Both launch on torch's current CUDA stream,
    allocate nothing in the library and do not synchronise, so they can be
    captured in a CUDA graph."""

    def __init__(self, shape, angles, ri: float | None = None, ctx: ops.Context | None = None, device: int = 0):
        import ctypes
        nz, ny, nx = (int(v) for v in shape)
        self.shape = (nz, ny, nx)
        self.ri = float(min(shape) // 2 - 2) if ri is None else float(ri)
        self.angles = np.ascontiguousarray(angles, dtype=np.float32)
        self.nang = int(self.angles.shape[0])
        self.ctx = ctx or ops.default_context(device)
        self.device = torch.device("cuda", self.ctx.device)
        self._L = self.ctx._L
        h = ctypes.c_void_p()
        ops.check(self._L.spi_pj3q_plan_create(self.ctx.handle, nx, ny, nz, self.ri,
                                               self.angles.ctypes.data_as(ctypes.c_void_p), self.nang,
                                               ctypes.byref(h)))
        self._h = h

    def _stream(self):
        import ctypes
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def forward(self, vol: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        import ctypes
        if out is None:
            out = torch.empty((self.nang,) + self.shape[1:], dtype=torch.float32, device=self.device)
        ops.check(self._L.spi_pj3q_plan_forward(self._h, ctypes.c_void_p(vol.data_ptr()),
                                                ctypes.c_void_p(out.data_ptr()), self._stream()))
        return out

    def adjoint(self, proj: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        import ctypes
        if out is None:
            out = torch.empty(self.shape, dtype=torch.float32, device=self.device)
        ops.check(self._L.spi_pj3q_plan_adjoint(self._h, ctypes.c_void_p(proj.data_ptr()),
                                                ctypes.c_void_p(out.data_ptr()), self._stream()))
        return out

    def close(self):
        if getattr(self, "_h", None) and self._h:
            self._L.spi_pj3q_plan_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# FourierSlice: the central-slice pair on ONELINE's geometry.
class FourierSlicePlan:
    """The FourierSlice operator pair (``spi_fslice_*``) for one box size and
    angle list: ``forward`` extracts central slices from a Fourier grid (the
    exact adjoint of ONELINE's insertion, oneline.f:38-200, without the weight
    grid), ``adjoint`` inserts slices into a grid (that insertion), ``normal``
    applies E^T E + lam I in one fused pass.  Grids are float32 tensors
    [2nx, 2nx, nx+1, 2] (complex as (re, im) pairs), slices [nang, 2nx, nx+1, 2]
    in the layout and sign of the staged image spectra (``stage``).  forward,
    adjoint and normal run on torch's current stream, allocate nothing in the
    library and do not synchronise, so they can be captured in a CUDA graph."""

    def __init__(self, nx: int, angles, ctx: ops.Context | None = None, device: int = 0):
        import ctypes
        self.nx = int(nx)
        self.n = 2 * self.nx
        self.angles = np.ascontiguousarray(angles, dtype=np.float32)
        self.nang = int(self.angles.shape[0])
        self.ctx = ctx or ops.default_context(device)
        self.device = torch.device("cuda", self.ctx.device)
        self._L = self.ctx._L
        self.shape = (self.n, self.n, self.nx + 1, 2)
        self.range_shape = (self.nang, self.n, self.nx + 1, 2)
        h = ctypes.c_void_p()
        ops.check(self._L.spi_fslice_plan_create(self.ctx.handle, self.nx,
                                                 self.angles.ctypes.data_as(ctypes.c_void_p), self.nang,
                                                 ctypes.byref(h)))
        self._h = h

    def _stream(self):
        import ctypes
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    @staticmethod
    def _p(t):
        import ctypes
        if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
            raise ops.SpiderError(101, "FourierSlice needs contiguous float32 CUDA tensors")
        return ctypes.c_void_p(t.data_ptr())

    def stage(self, imgs: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        """Slices of CUDA images [nang, nx, nx]: PADD2, phase, 2D transform."""
        if out is None:
            out = torch.empty(self.range_shape, dtype=torch.float32, device=self.device)
        ops.check(self._L.spi_fslice_stage(self._h, self._p(imgs), self._p(out), self._stream()))
        return out

    def forward(self, grid: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        if out is None:
            out = torch.empty(self.range_shape, dtype=torch.float32, device=self.device)
        ops.check(self._L.spi_fslice_forward(self._h, self._p(grid), self._p(out), self._stream()))
        return out

    def adjoint(self, slices: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        if out is None:
            out = torch.empty(self.shape, dtype=torch.float32, device=self.device)
        ops.check(self._L.spi_fslice_adjoint(self._h, self._p(slices), self._p(out), self._stream()))
        return out

    def normal(self, grid: torch.Tensor, lam: float, out: torch.Tensor | None = None) -> torch.Tensor:
        if out is None:
            out = torch.empty(self.shape, dtype=torch.float32, device=self.device)
        ops.check(self._L.spi_fslice_normal(self._h, self._p(grid), float(lam), self._p(out), self._stream()))
        return out

    def normal64(self, grid: torch.Tensor, lam: float, out: torch.Tensor | None = None) -> torch.Tensor:
        """E^T E + lam I on FP64 grids: FP64 sums and scatter, FP32 table weights."""
        import ctypes
        if out is None:
            out = torch.empty(self.shape, dtype=torch.float64, device=self.device)
        for t in (grid, out):
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                raise ops.SpiderError(101, "normal64 needs contiguous float64 CUDA tensors")
        ops.check(self._L.spi_fslice_normal64(self._h, ctypes.c_void_p(grid.data_ptr()), float(lam),
                                              ctypes.c_void_p(out.data_ptr()), self._stream()))
        return out

    def forward64(self, grid: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        """E on an FP64 grid into FP64 slices (FP64 sums of the same taps)."""
        import ctypes
        if out is None:
            out = torch.empty(self.range_shape, dtype=torch.float64, device=self.device)
        for t in (grid, out):
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                raise ops.SpiderError(101, "forward64 needs contiguous float64 CUDA tensors")
        ops.check(self._L.spi_fslice_forward64(self._h, ctypes.c_void_p(grid.data_ptr()),
                                               ctypes.c_void_p(out.data_ptr()), self._stream()))
        return out

    def adjoint64(self, slices: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        """E^T slices into an FP64 grid (FP64 scatter): the CG's right-hand side."""
        import ctypes
        if out is None:
            out = torch.empty(self.shape, dtype=torch.float64, device=self.device)
        if not (out.is_cuda and out.dtype == torch.float64 and out.is_contiguous()):
            raise ops.SpiderError(101, "adjoint64 needs a contiguous float64 CUDA output")
        ops.check(self._L.spi_fslice_adjoint64(self._h, self._p(slices), ctypes.c_void_p(out.data_ptr()),
                                               self._stream()))
        return out

    def volume(self, grid: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        """Real-space volume [nx, nx, nx] of a grid of spectrum coefficients."""
        if out is None:
            out = torch.empty((self.nx,) * 3, dtype=torch.float32, device=self.device)
        ops.check(self._L.spi_fslice_volume(self._h, self._p(grid), self._p(out), self._stream()))
        return out

    def close(self):
        if getattr(self, "_h", None) and self._h:
            self._L.spi_fslice_plan_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


class FourierSlice(torch.autograd.Function):
    """Differentiable central-slice extraction: forward E (grid -> slices),
    backward the insertion E^T (ONELINE without weights), recomputing every
    tap's voxel and weight from the plan's angles instead of storing them."""

    @staticmethod
    def forward(fctx, grid: torch.Tensor, plan: FourierSlicePlan):
        fctx.plan = plan
        return plan.forward(grid.detach().contiguous().float())

    @staticmethod
    def backward(fctx, grad: torch.Tensor):
        return fctx.plan.adjoint(grad.detach().contiguous().float()), None


def fourier_slice(grid: torch.Tensor, plan: FourierSlicePlan) -> torch.Tensor:
    """Differentiable FourierSlice of a CUDA grid [2nx, 2nx, nx+1, 2]."""
    if not grid.is_cuda:
        raise ops.SpiderError(101, "fourier_slice needs a CUDA grid (there is no CPU path)")
    return FourierSlice.apply(grid, plan)


class NormalCG:
    """Conjugate gradients on (A^T A + lam I) x = rhs, in fixed device
    buffers; A is the plan's operator (PJ 3Q with PJ3QPlan, the FourierSlice
    extraction with FourierSlicePlan, whose E^T E + lam I is one fused pass).
    With ``graph`` one iteration is captured once as a CUDA graph and
    replayed.  Dot products and step lengths are FP64; with ``fp64_vectors``
    (the default for the FourierSlice pair, whose eigenvalues spread over
    many orders of magnitude) x, r and p are FP64 too, and with
    ``fp64_operator`` (the default with FP64 vectors on the FourierSlice
    pair) the normal operator sums in FP64 as well (``normal64``): a late
    direction p has ||E^T E p|| << ||E^T E|| ||p||, and FP32 sums would lose
    that many digits.  Otherwise the operator's input and output are FP32.
    ``solve`` returns x in FP32."""

    def __init__(self, plan, lam: float, iters: int, graph: bool = True, fp64_vectors: bool | None = None,
                 fp64_operator: bool | None = None):
        self.plan, self.lam, self.iters, self.graph = plan, float(lam), int(iters), graph
        self.fused = hasattr(plan, "normal")
        self.vec64 = self.fused if fp64_vectors is None else bool(fp64_vectors)
        # FP64 normal operator (FourierSlice pair with FP64 vectors): no FP32 copies at all
        self.op64 = (self.vec64 and hasattr(plan, "normal64")) if fp64_operator is None else bool(fp64_operator)
        if self.op64 and not (self.vec64 and hasattr(plan, "normal64")):
            raise ops.SpiderError(101, "an FP64 operator needs FP64 vectors and a plan with normal64")
        vt = torch.float64 if self.vec64 else torch.float32
        z = lambda shape, dt=torch.float32: torch.zeros(shape, dtype=dt, device=plan.device)  # noqa: E731
        self.x, self.r, self.p = (z(plan.shape, vt) for _ in range(3))
        self.ap = None if self.op64 else z(plan.shape)                    # operator output (FP32)
        self.p32 = z(plan.shape) if (self.vec64 and not self.op64) else None  # operator input (FP32)
        self.ap64 = z(plan.shape, vt) if self.vec64 else None
        self.q = None if self.fused else z((plan.nang,) + tuple(plan.shape[1:]))
        self.rs = torch.zeros((), dtype=torch.float64, device=plan.device)
        self._g = None

    def _iteration(self):
        if self.op64:
            self.plan.normal64(self.p, self.lam, out=self.ap64)
            self._update(self.ap64)
            return
        pin = self.p
        if self.vec64:
            self.p32.copy_(self.p)
            pin = self.p32
        if self.fused:
            self.plan.normal(pin, self.lam, out=self.ap)
        else:
            self.plan.forward(pin, out=self.q)
            self.plan.adjoint(self.q, out=self.ap)
            self.ap.add_(pin, alpha=self.lam)
        ap = self.ap
        if self.vec64:
            self.ap64.copy_(self.ap)
            ap = self.ap64
        self._update(ap)

    def _update(self, ap):
        pap = (self.p.double() * ap.double()).sum()
        alpha = torch.where(pap > 0, self.rs / pap, torch.zeros_like(pap)).to(self.x.dtype)
        self.x.add_(alpha * self.p)
        self.r.sub_(alpha * ap)
        rs_new = (self.r.double() * self.r.double()).sum()
        beta = torch.where(self.rs > 0, rs_new / self.rs, torch.zeros_like(rs_new)).to(self.x.dtype)
        self.p.mul_(beta).add_(self.r)
        self.rs.copy_(rs_new)

    def solve(self, rhs: torch.Tensor) -> torch.Tensor:
        self.x.zero_()
        self.r.copy_(rhs)
        self.p.copy_(rhs)
        self.rs.copy_((rhs.double() * rhs.double()).sum())
        if not self.graph:
            for _ in range(self.iters):
                self._iteration()
            return self.x.to(torch.float32, copy=True)
        if self._g is None:
            # warm up on a side stream (as CUDA-graph capture requires), then capture one iteration
            s = torch.cuda.Stream(self.plan.device)
            s.wait_stream(torch.cuda.current_stream(self.plan.device))
            saved = [t.clone() for t in (self.x, self.r, self.p, self.rs)]
            with torch.cuda.stream(s):
                self._iteration()
            torch.cuda.current_stream(self.plan.device).wait_stream(s)
            for t, v in zip((self.x, self.r, self.p, self.rs), saved):
                t.copy_(v)
            self._g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self._g):
                self._iteration()
            for t, v in zip((self.x, self.r, self.p, self.rs), saved):   # the capture did not run it
                t.copy_(v)
        for _ in range(self.iters):
            self._g.replay()
        return self.x.to(torch.float32, copy=True)


class _CGReconstruct(torch.autograd.Function):
    @staticmethod
    def forward(fctx, b: torch.Tensor, solver: NormalCG):
        fctx.solver = solver
        b = b.detach().contiguous().float()
        rhs = solver.plan.adjoint64(b) if solver.op64 else solver.plan.adjoint(b)
        return solver.solve(rhs)

    @staticmethod
    def backward(fctx, gx: torch.Tensor):
        # x = M^-1 A^T b with M = A^T A + lam I symmetric: dL/db = A M^-1 dL/dx
        s = fctx.solver
        y = s.solve(gx.detach().contiguous().float())
        return s.plan.forward(y), None


def cg_reconstruct(projs: torch.Tensor, solver: NormalCG) -> torch.Tensor:
    """Regularised least-squares reconstruction x = (A^T A + lam I)^-1 A^T b
    from CUDA projections b [nang, ny, nx] by ``solver``'s CG iterations,
    differentiable in b: the backward is a second CG solve (implicit
    differentiation, no stored iterates)."""
    if not projs.is_cuda:
        raise ops.SpiderError(101, "cg_reconstruct needs CUDA projections (there is no CPU path)")
    return _CGReconstruct.apply(projs, solver)
