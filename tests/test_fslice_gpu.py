"""FourierSlice on the GPU (spi_fslice_*): the central-slice extraction that
is the exact adjoint of ONELINE's insertion without weights, against the FP64
oracle pair; the differentiable slice function against central finite
differences (h = 1e-3) on 64 random voxels and against the FP64 adjoint; the
graph-captured CG on the pair against an FP64 CG on the oracle pair.

Bars: relative L2 <= 1e-5 for the FP32 operators (FP32 sums of at most 64
taps per pixel, FP32 atomics in the insertion), 1e-12 for the FP64 normal
operator; <= 1e-4 for CG iterates.  The CG runs on the FP64 normal operator
by default: with FP32 sums, late directions p (||E^T E p|| << ||E^T E|| ||p||)
lose digits, and the iterate drifts from the FP64 CG by far more than 1e-4."""
import numpy as np
import pytest

from spider_b200 import synth

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _cplx(t):
    a = t.detach().cpu().numpy().astype(np.float64)
    return a[..., 0] + 1j * a[..., 1]


def _real(z):
    import torch
    return torch.tensor(np.stack([z.real, z.imag], -1), dtype=torch.float32, device="cuda").contiguous()


@pytest.mark.parametrize("nx,order", [(24, None), (33, None), (24, "cols"), (33, "lanes4")])
def test_fslice_operators_match_oracle(ctx, orc, nx, order, monkeypatch):
    """order "cols": the insertions E^T walk every slice by half columns (the
    order boxes above 192 take per slice); "lanes4": the FP64 operators with
    four lanes per pixel instead of eight.  The results are the same."""
    from spider_b200 import autograd
    if order == "cols":
        monkeypatch.setenv("SPI_INSERT_ORDER", order)
    elif order == "lanes4":
        monkeypatch.setenv("SPI_FS_LANES", "4")
    rng = np.random.default_rng(300 + nx)
    n = 2 * nx
    ang = synth.so3_angles(40, rng)
    ang[:6, 1] = 90.0                         # planes through the x = 0 line (flips and reflected taps)
    X = (rng.standard_normal((n, n, nx + 1)) + 1j * rng.standard_normal((n, n, nx + 1))).astype(np.complex64)
    T = (rng.standard_normal((40, n, nx + 1)) + 1j * rng.standard_normal((40, n, nx + 1))).astype(np.complex64)
    plan = autograd.FourierSlicePlan(nx, ang, ctx=ctx)
    try:
        ex = _cplx(plan.forward(_real(X)))
        ref_ex = orc.fslice_extract(X.astype(np.complex128), ang)
        e1 = synth.rel_l2(np.abs(ex - ref_ex), np.abs(ref_ex))
        assert np.linalg.norm(ex - ref_ex) <= TOL * np.linalg.norm(ref_ex)
        ins = _cplx(plan.adjoint(_real(T)))
        ref_ins = orc.fslice_insert(T.astype(np.complex128), ang)
        assert np.linalg.norm(ins - ref_ins) <= TOL * np.linalg.norm(ref_ins)
        # <E X, T> = <X, E^T T> with the GPU's own pair
        lhs = np.sum((np.conj(ex) * T).real)
        rhs = np.sum((np.conj(X.astype(np.complex128)) * ins).real)
        assert abs(lhs - rhs) <= TOL * abs(lhs)
        # fused normal operator = E^T E X + lam X
        lam = 0.37
        nrm = _cplx(plan.normal(_real(X), lam))
        two = orc.fslice_insert(ref_ex, ang) + lam * X.astype(np.complex128)
        assert np.linalg.norm(nrm - two) <= TOL * np.linalg.norm(two)
        # the FP64 normal operator: FP64 sums and scatter of the same taps
        x64 = _real(X).double()
        n64 = plan.normal64(x64.contiguous(), lam).cpu().numpy()
        n64 = n64[..., 0] + 1j * n64[..., 1]
        assert np.linalg.norm(n64 - two) <= 1e-12 * np.linalg.norm(two)
        a64 = plan.adjoint64(_real(T)).cpu().numpy()
        a64 = a64[..., 0] + 1j * a64[..., 1]
        assert np.linalg.norm(a64 - ref_ins) <= 1e-12 * np.linalg.norm(ref_ins)
        print(f"nx={nx}: extract {np.linalg.norm(ex - ref_ex) / np.linalg.norm(ref_ex):.2e}, "
              f"insert {np.linalg.norm(ins - ref_ins) / np.linalg.norm(ref_ins):.2e}, "
              f"normal {np.linalg.norm(nrm - two) / np.linalg.norm(two):.2e}, adjoint identity "
              f"{abs(lhs - rhs) / abs(lhs):.2e} ({e1:.1e})")
    finally:
        plan.close()


def test_fslice_stage_matches_oracle(ctx, orc):
    import torch
    from spider_b200 import autograd
    rng = np.random.default_rng(8)
    nx, nimg = 32, 37
    imgs = rng.standard_normal((nimg, nx, nx)).astype(np.float32)
    ang = synth.so3_angles(nimg, rng)
    plan = autograd.FourierSlicePlan(nx, ang, ctx=ctx)
    try:
        got = _cplx(plan.stage(torch.from_numpy(imgs).cuda()))
    finally:
        plan.close()
    ref = np.stack([np.conj(orc.stage_image(im)) for im in imgs])
    assert np.linalg.norm(got - ref) <= TOL * np.linalg.norm(ref)


def test_fourier_slice_gradient(ctx, orc):
    """backward = E^T of the upstream gradient: against the FP64 oracle
    insertion, and against central finite differences (h = 1e-3) of the FP64
    extraction on 64 random grid voxels (real and imaginary parts)."""
    import torch
    from spider_b200 import autograd
    rng = np.random.default_rng(12)
    nx, nang = 16, 14
    n = 2 * nx
    ang = synth.so3_angles(nang, rng)
    X = rng.standard_normal((n, n, nx + 1)) + 1j * rng.standard_normal((n, n, nx + 1))
    G = rng.standard_normal((nang, n, nx + 1)) + 1j * rng.standard_normal((nang, n, nx + 1))
    plan = autograd.FourierSlicePlan(nx, ang, ctx=ctx)
    try:
        xt = _real(X).requires_grad_(True)
        loss = (autograd.fourier_slice(xt, plan).double() * _real(G).double()).sum()
        loss.backward()
        grad = _cplx(xt.grad)
    finally:
        plan.close()
    exact = orc.fslice_insert(G, ang)          # gradient of Re<E X, G> = E^T G
    assert np.linalg.norm(grad - exact) <= TOL * np.linalg.norm(exact)
    touched = np.argwhere(np.abs(exact) > 0)
    picks = touched[rng.choice(len(touched), 64, replace=False)]
    h = 1e-3
    scale = np.abs(exact).max()

    def lossf(Z):
        return float(np.sum((np.conj(orc.fslice_extract(Z, ang)) * G).real))

    for k, (a, b, c) in enumerate(picks):
        comp = 1.0 if k % 2 == 0 else 1j       # real or imaginary part of the voxel
        zp, zm = X.copy(), X.copy()
        zp[a, b, c] += h * comp
        zm[a, b, c] -= h * comp
        fd = (lossf(zp) - lossf(zm)) / (2 * h)
        g = grad[a, b, c].real if k % 2 == 0 else grad[a, b, c].imag
        assert abs(g - fd) <= 1e-4 * max(abs(fd), 1e-3 * scale)


def test_fourier_cg_graph_plain_and_fp64(ctx, orc):
    """CG on (E^T E + lam I) x = E^T b from staged PJ 3Q projections: the
    graph-captured and the op-by-op iteration agree, and both follow an FP64
    CG on the oracle pair; the volume of the solution is the phantom."""
    import torch
    from spider_b200 import autograd
    rng = np.random.default_rng(33)
    nx, nang, lam, iters = 32, 400, 1e-3, 12
    vol = synth.blob_phantom(nx, 12, sigma=(1.5, 4.0), radius=0.35 * nx, rng=rng)
    ang = synth.so3_angles(nang, rng)
    imgs = synth.projection_stack(ctx, vol, ang, snr=None, seed=3)
    plan = autograd.FourierSlicePlan(nx, ang, ctx=ctx)
    try:
        b = plan.stage(imgs)
        rhs64 = plan.adjoint64(b)
        xg = autograd.NormalCG(plan, lam, iters, graph=True).solve(rhs64)
        xp = autograd.NormalCG(plan, lam, iters, graph=False).solve(rhs64)
        x32 = autograd.NormalCG(plan, lam, iters, graph=True, fp64_operator=False).solve(plan.adjoint(b))
        assert synth.rel_l2(xp.cpu().numpy(), xg.cpu().numpy()) <= 1e-4
        v = plan.volume(xg.contiguous()).cpu().numpy()
        bh = _cplx(b)
    finally:
        plan.close()
    # FP64 CG on the oracle pair, from the GPU's staged spectra
    r = orc.fslice_insert(bh, ang)
    x = np.zeros_like(r)
    p = r.copy()
    rs = np.vdot(r, r).real
    for _ in range(iters):
        ap = orc.fslice_insert(orc.fslice_extract(p, ang), ang) + lam * p
        alpha = rs / np.vdot(p, ap).real
        x += alpha * p
        r -= alpha * ap
        rs_new = np.vdot(r, r).real
        p = r + (rs_new / rs) * p
        rs = rs_new
    e = np.linalg.norm(_cplx(xg) - x) / np.linalg.norm(x)
    e32 = np.linalg.norm(_cplx(x32) - x) / np.linalg.norm(x)
    print(f"Fourier CG, {iters} iterations: FP64 operator vs FP64 oracle CG {e:.2e}; "
          f"FP32 operator {e32:.2e}")
    assert e <= 1e-4
    g = np.arange(nx) - nx // 2
    m = (g[:, None, None] ** 2 + g[None, :, None] ** 2 + g[None, None, :] ** 2) <= (0.4 * nx) ** 2
    cc = np.corrcoef(v[m], vol[m])[0, 1]
    print(f"volume of the CG solution vs phantom: correlation {cc:.4f}")
    assert cc > 0.9


def test_fslice_volume_matches_numpy(ctx, orc):
    """spi_fslice_volume against the same steps in numpy (FP64): Hermitian
    part of plane 0, phase, SPIDER's inverse sign, inverse transform, crop,
    times |WKB| inside radius nx/2."""
    import torch
    from spider_b200 import autograd
    rng = np.random.default_rng(9)
    nx = 24
    n = 2 * nx
    X = (rng.standard_normal((n, n, nx + 1)) + 1j * rng.standard_normal((n, n, nx + 1)))
    X[:, :, nx] = 0.0      # no tap reaches i = nx (IXN <= NX - 3), so a solution grid is zero there
    plan = autograd.FourierSlicePlan(nx, synth.so3_angles(3, rng), ctx=ctx)
    try:
        got = plan.volume(_real(X)).cpu().numpy()
    finally:
        plan.close()
    Z = X.copy()
    jm, km = (-np.arange(n)) % n, (-np.arange(n)) % n
    Z[:, :, 0] = 0.5 * (X[:, :, 0] + np.conj(X[km][:, jm][:, :, 0]))
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(nx + 1), indexing="ij")
    Z = np.conj(Z * np.where((i + j + k) % 2 == 1, -1.0, 1.0))   # SPIDER's inverse sign
    Z[0, 0, 0] = Z[0, 0, 0].real
    R = np.fft.irfftn(Z, s=(n, n, n), axes=(0, 1, 2))   # sum of Z e^{+2 pi i k.x} / n^3
    ip = (n - nx) // 2 + nx % 2
    crop = R[ip:ip + nx, ip:ip + nx, ip:ip + nx]
    wkb = orc.windkb_table(nx).astype(np.float64)
    c = nx // 2 + 1
    gg = np.arange(1, nx + 1) - c
    lr = gg[:, None, None] ** 2 + gg[None, :, None] ** 2 + gg[None, None, :] ** 2
    ref = np.where(lr <= (nx // 2) ** 2, crop * wkb[np.minimum(lr, len(wkb) - 1)], 0.0)
    assert synth.rel_l2(got, ref) <= TOL


def _oracle_cg(orc, rhs, ang, lam, iters):
    x = np.zeros_like(rhs)
    r = rhs.copy()
    p = r.copy()
    rs = np.vdot(r, r).real
    for _ in range(iters):
        ap = orc.fslice_insert(orc.fslice_extract(p, ang), ang) + lam * p
        alpha = rs / np.vdot(p, ap).real
        x += alpha * p
        r -= alpha * ap
        rs_new = np.vdot(r, r).real
        p = r + (rs_new / rs) * p
        rs = rs_new
    return x


def test_fourier_cg_reconstruct_gradient(ctx, orc):
    """cg_reconstruct on the FourierSlice pair: x = (E^T E + lam I)^-1 E^T b
    by CG, differentiable in the slices b through a second CG solve (implicit
    differentiation: dL/db = E (E^T E + lam I)^-1 dL/dx).  Solution and
    gradient against the same iterations in FP64 on the oracle pair, and the
    gradient against central finite differences (h = 1e-3) of the FP64
    reconstruction on 64 random slice values."""
    import torch
    from spider_b200 import autograd
    rng = np.random.default_rng(44)
    nx, nang, lam, iters = 16, 30, 5.0, 40
    n = 2 * nx
    ang = synth.so3_angles(nang, rng)
    b = rng.standard_normal((nang, n, nx + 1)) + 1j * rng.standard_normal((nang, n, nx + 1))
    w = rng.standard_normal((n, n, nx + 1)) + 1j * rng.standard_normal((n, n, nx + 1))
    plan = autograd.FourierSlicePlan(nx, ang, ctx=ctx)
    try:
        solver = autograd.NormalCG(plan, lam, iters, graph=True)
        bt = _real(b).requires_grad_(True)
        x = autograd.cg_reconstruct(bt, solver)
        loss = (x.double() * _real(w).double()).sum()
        loss.backward()
        grad = _cplx(bt.grad)
        xg = _cplx(x)
    finally:
        plan.close()
    # the extraction leaves pixels without taps at zero, so b enters only where E^T reads it
    x_ref = _oracle_cg(orc, orc.fslice_insert(b, ang), ang, lam, iters)
    assert np.linalg.norm(xg - x_ref) <= 1e-5 * np.linalg.norm(x_ref)
    g_ref = orc.fslice_extract(_oracle_cg(orc, w, ang, lam, iters), ang)
    assert np.linalg.norm(grad - g_ref) <= 1e-5 * np.linalg.norm(g_ref)
    h = 1e-3
    scale = np.abs(g_ref).max()
    wy = _oracle_cg(orc, w, ang, lam, iters)       # M^-1 w: L(b) = Re<w, M^-1 E^T b> = Re<E M^-1 w, b>
    touched = np.argwhere(np.abs(g_ref) > 0)
    for k, (a, j, i) in enumerate(touched[rng.choice(len(touched), 64, replace=False)]):
        comp = 1.0 if k % 2 == 0 else 1j
        bp, bm = b.copy(), b.copy()
        bp[a, j, i] += h * comp
        bm[a, j, i] -= h * comp
        lp = np.sum((np.conj(wy) * orc.fslice_insert(bp, ang)).real)
        lm = np.sum((np.conj(wy) * orc.fslice_insert(bm, ang)).real)
        fd = (lp - lm) / (2 * h)
        g = grad[a, j, i].real if k % 2 == 0 else grad[a, j, i].imag
        assert abs(g - fd) <= 1e-4 * max(abs(fd), 1e-3 * scale)
