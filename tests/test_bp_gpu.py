"""Parity of the CUDA BP 3F / BP 32F path with the CPU oracle (serial FP32
restatement of bp3f.f / bp32f.f / oneline.f) and the FP64 oracle.

Tolerance (stated by the task for the FP32 path): relative L2 <= 1e-5 on the
volume against the FP32 oracle and FSC >= 0.999 at Nyquist.  Every index,
table entry and interpolation weight is bit-identical between the two; they
differ only in the order of the FP32 grid accumulations (atomics on the GPU).
"""
import os

import numpy as np
import pytest

from spider_b200 import ops, synth

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _case(nx, nimg, seed, nblobs=12, noise=None):
    rng = np.random.default_rng(seed)
    import oracle
    vol = synth.blob_phantom(nx, nblobs, sigma=(1.5, 4.0), radius=0.35 * nx, rng=rng)
    ang = synth.so3_angles(nimg, rng)
    pr = oracle.pj3q(vol, ang)
    if noise:
        pr = synth.add_noise(pr, noise, rng)
    return vol, pr, ang


@pytest.mark.parametrize("nx,nimg", [(16, 60), (32, 300), (64, 400)])
def test_bp3f_matches_oracle(ctx, orc, nx, nimg):
    _, pr, ang = _case(nx, nimg, 11 + nx)
    got = ops.bp3f(pr, ang, ctx=ctx)
    ref32 = orc.bp3f(pr, ang, prec=0, nthreads=1)
    ref64 = orc.bp3f(pr, ang, prec=1, nthreads=1)
    e32 = synth.rel_l2(got, ref32)
    e64 = synth.rel_l2(got, ref64)
    print(f"BP 3F nx={nx} nimg={nimg}: rel-L2 vs FP32 oracle {e32:.3e}, vs FP64 oracle {e64:.3e}")
    assert e32 <= TOL
    assert e64 <= TOL
    f = synth.fsc(got, ref64)
    assert f[nx // 2] >= 0.999


def test_bp32f_matches_oracle(ctx, orc):
    nx, nimg = 32, 400
    _, pr, ang = _case(nx, nimg, 5, noise=0.5)
    half = synth.half_mask(nimg, np.random.default_rng(3))
    g_all, g1, g2 = ops.bp32f(pr, ang, half, ctx=ctx)
    r_all, r1, r2 = orc.bp32f(pr, ang, half, prec=0, nthreads=1)
    for name, a, b in (("all", g_all, r_all), ("first", g1, r1), ("second", g2, r2)):
        e = synth.rel_l2(a, b)
        print(f"BP 32F {name}: rel-L2 {e:.3e}")
        assert e <= TOL, name
    # the half-set volumes are different reconstructions of the same object
    assert synth.rel_l2(g1, g2) > 1e-3


def test_bp3f_partial_and_merge(ctx, orc):
    nx, nimg = 32, 240
    _, pr, ang = _case(nx, nimg, 21)
    x, w = ops.bp3f_partial(pr, ang, ctx=ctx)
    rx, rw = orc.bp3f_partial(pr, ang, prec=1, nthreads=1)
    gx = x[..., 0] + 1j * x[..., 1]
    assert np.linalg.norm(gx - rx) / np.linalg.norm(rx) <= TOL
    assert synth.rel_l2(w, rw) <= TOL
    # BP 3F M of two halves equals BP 3F of all images
    p1 = ops.bp3f_partial(pr[:100], ang[:100], ctx=ctx)
    p2 = ops.bp3f_partial(pr[100:], ang[100:], ctx=ctx)
    merged = ops.bp3f_merge([p1, p2], ctx=ctx)
    full = ops.bp3f(pr, ang, ctx=ctx)
    assert synth.rel_l2(merged, full) <= TOL


def test_bp3f_plane0_hermitian(ctx):
    nx = 24
    _, pr, ang = _case(nx, 80, 8)
    x, w = ops.bp3f_partial(pr, ang, ctx=ctx)
    n = 2 * nx
    X = x[..., 0] + 1j * x[..., 1]           # [k][j][i]
    p0 = X[:, :, 0]
    idx = (-np.arange(n)) % n
    mirror = np.conj(p0[idx][:, idx])
    assert np.allclose(p0[1:, 1:], mirror[1:, 1:], atol=1e-6 * np.abs(p0).max())
    assert np.allclose(w[:, :, 0][1:, 1:], w[:, :, 0][idx][:, idx][1:, 1:])


def test_bp_chunked_and_device_inputs(ctx, orc):
    import torch
    nx, nimg = 32, 300
    _, pr, ang = _case(nx, nimg, 31)
    ref = orc.bp3f(pr, ang, prec=0, nthreads=1)
    os.environ["SPI_BP_CHUNK"] = "64"      # several persistent launches
    try:
        ctx.bp_open(nx, 1)
        d = torch.from_numpy(pr).cuda()
        ctx.bp_insert(d[:130], ang[:130])
        ctx.bp_insert(d[130:], ang[130:])
        out = ctx.bp_finish(("all",), device=True)["all"].cpu().numpy()
        ctx.bp_close()
    finally:
        del os.environ["SPI_BP_CHUNK"]
    assert synth.rel_l2(out, ref) <= TOL


def test_bp3f_symmetry(ctx, orc):
    nx, nimg = 24, 120
    _, pr, ang = _case(nx, nimg, 41)
    sym = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 180.0], [0.0, 180.0, 0.0]], np.float32)  # D2-like
    got = ops.bp3f(pr, ang, sym, ctx=ctx)
    ref = orc.bp3f(pr, ang, sym=sym, prec=0, nthreads=1)
    assert synth.rel_l2(got, ref) <= TOL


def test_bp32f_bf16_spectra(ctx, orc):
    nx, nimg = 32, 300
    _, pr, ang = _case(nx, nimg, 51)
    half = synth.half_mask(nimg, np.random.default_rng(4))
    g_all, _, _ = ops.bp32f(pr, ang, half, ctx=ctx, bf16=True)
    r_all, _, _ = orc.bp32f(pr, ang, half, prec=1, nthreads=1)
    e = synth.rel_l2(g_all, r_all)
    f = synth.fsc(g_all, r_all)[nx // 2]
    print(f"BF16 spectra: rel-L2 vs FP64 oracle {e:.3e}, FSC at Nyquist {f:.7f}")
    # BF16 keeps 8 bits of each spectrum value: the volume moves by ~1e-4 of
    # its norm, while every Fourier shell still correlates to >= 0.999
    assert e <= 5e-4
    assert f >= 0.999


def test_bp_errors(ctx):
    with pytest.raises(ops.SpiderError) as ei:
        ops.bp3f(np.zeros((3, 16, 18), np.float32), np.zeros((3, 3), np.float32), ctx=ctx)
    assert ei.value.code == 101
    with pytest.raises(ops.SpiderError) as ei:
        ctx.bp_open(7, 1)
    assert ei.value.code == 101
    with pytest.raises(ops.SpiderError):
        ctx.bp_open(16, 3)
    # no images: the volume is all zeros
    ctx.bp_open(16, 1)
    v = ctx.bp_finish(("all",))["all"]
    ctx.bp_close()
    assert np.all(v == 0)


def test_bp3f_config1_full(ctx, orc):
    """BP 3F at 64^3 from 2,000 PJ 3Q projections of a 20-blob phantom."""
    rng = synth.rng_for(0)
    vol = synth.blob_phantom(64, 20, sigma=(2, 5), amp=(0.5, 1.0), radius=24, rng=rng)
    ang = synth.so3_angles(2000, rng)
    pr = orc.pj3q(vol, ang)
    got = ops.bp3f(pr, ang, ctx=ctx)
    ref = orc.bp3f(pr, ang, prec=0, nthreads=1)
    e = synth.rel_l2(got, ref)
    print(f"config 1: rel-L2 vs FP32 oracle {e:.3e}")
    assert e <= TOL
    assert synth.fsc(got, ref)[32] >= 0.999
    g = np.arange(64) - 32
    m = (g[:, None, None] ** 2 + g[None, :, None] ** 2 + g[None, None, :] ** 2) <= 28 ** 2
    assert np.corrcoef(got[m], vol[m])[0, 1] > 0.98


def test_insert_kernels_agree(ctx, orc):
    """The tile-privatised insertion and the direct per-tap insertion add the
    same taps; they differ only in FP32 summation order.  So do the x4
    kernel's row-by-row, column-by-column and per-slice insertion orders."""
    nx, nimg = 48, 300
    _, pr, ang = _case(nx, nimg, 61)
    # include orientations that put the x = 0 flip line inside many tiles
    ang[:40, 1] = 90.0
    out, grids = {}, {}
    for mode in ("direct", "tile", "xlane", "x4", "tilefx", "x4:rows", "x4:cols"):
        kernel, _, order = mode.partition(":")
        os.environ["SPI_INSERT"] = kernel
        if order:
            os.environ["SPI_INSERT_ORDER"] = order
        try:
            out[mode] = ops.bp3f(pr, ang, ctx=ctx)
            grids[mode] = ops.bp3f_partial(pr, ang, ctx=ctx)
        finally:
            del os.environ["SPI_INSERT"]
            os.environ.pop("SPI_INSERT_ORDER", None)
    ref = orc.bp3f(pr, ang, prec=1, nthreads=1)
    for mode, v in out.items():
        assert synth.rel_l2(v, out["direct"]) <= 2e-6, mode
        assert synth.rel_l2(v, ref) <= TOL, mode
        # the gridded X and W themselves: same taps, only the summation order differs
        for a, b in zip(grids[mode], grids["direct"]):
            assert synth.rel_l2(a, b) <= 1e-6, mode


def test_rb3f_rb32f_match_oracle(ctx, orc):
    """RB 3F / RB 32F: images shifted by up to 3 px and rotated in plane are
    aligned by RTSQ (doc registers 6-8) before insertion."""
    nx, nimg = 32, 200
    vol, pr, ang = _case(nx, nimg, 71)
    rng = np.random.default_rng(72)
    inplane = np.stack([rng.uniform(-180, 180, nimg), rng.uniform(-3, 3, nimg), rng.uniform(-3, 3, nimg)],
                       1).astype(np.float32)
    got = ops.rb3f(pr, ang, inplane, ctx=ctx)
    ref = orc.rb3f(pr, ang, inplane, prec=0, nthreads=1)
    assert synth.rel_l2(got, ref) <= TOL
    half = synth.half_mask(nimg, rng)
    g = ops.rb32f(pr, ang, inplane, half, ctx=ctx)
    r = orc.rb3f(pr, ang, inplane, half, prec=0, nthreads=1)
    for a, b in zip(g, r):
        assert synth.rel_l2(a, b) <= TOL
    # zero in-plane parameters reproduce BP 3F exactly up to summation order
    z = ops.rb3f(pr, ang, np.zeros((nimg, 3), np.float32), ctx=ctx)
    assert synth.rel_l2(z, ops.bp3f(pr, ang, ctx=ctx)) <= 2e-6


@pytest.mark.parametrize("mode", ["one_launch", "one_launch:cols", "one_launch:own", "concurrent", "in_turn"])
def test_bp32f_multiclass(orc, mode):
    """Several classes of different box sizes (one odd, two equal) reconstructed
    from one image stream: all classes in one insertion launch per round
    (spi_bp_insert_multi; also with every slice inserted column by column),
    or one context per class inserted concurrently from one host thread
    each, or in turn."""
    classes, refs = [], []
    for k, (nx, nimg) in enumerate(((24, 120), (32, 200), (41, 150), (32, 90))):
        _, pr, ang = _case(nx, nimg, 90 + k, noise=0.5)
        half = synth.half_mask(nimg, np.random.default_rng(95 + k))
        classes.append((pr, ang, half))
        refs.append(orc.bp32f(pr, ang, half, prec=0, nthreads=1))
    mode, _, opt = mode.partition(":")
    if opt == "cols":
        os.environ["SPI_INSERT_ORDER"] = opt
    elif opt == "own":   # the own R2C for the power-of-two padded box (32 -> 64), cuFFT for the others
        os.environ["SPI_FFT"] = opt
    try:
        out = ops.bp32f_multiclass(classes, one_launch=mode == "one_launch", concurrent=mode == "concurrent")
    finally:
        os.environ.pop("SPI_INSERT_ORDER", None)
        os.environ.pop("SPI_FFT", None)
    for got, ref in zip(out, refs):
        for a, b in zip(got, ref):
            assert a.shape == b.shape
            assert synth.rel_l2(a, b) <= TOL


@pytest.mark.parametrize("one_launch", [True, False])
def test_bp32f_multiclass_reused_contexts(orc, one_launch):
    """Caller contexts stay open between calls: the second call's same-size
    open zeroes the grids and reuses buffers and FFT plans, and both calls
    give the oracle's volumes."""
    classes, refs = [], []
    for k, (nx, nimg) in enumerate(((24, 90), (32, 120))):
        _, pr, ang = _case(nx, nimg, 130 + k, noise=0.5)
        half = synth.half_mask(nimg, np.random.default_rng(135 + k))
        classes.append((pr, ang, half))
        refs.append(orc.bp32f(pr, ang, half, prec=0, nthreads=1))
    ctxs = [ops.Context(0) for _ in classes]
    try:
        for _ in range(2):
            out = ops.bp32f_multiclass(classes, one_launch=one_launch, ctxs=ctxs)
            for got, ref in zip(out, refs):
                for a, b in zip(got, ref):
                    assert synth.rel_l2(a, b) <= TOL
    finally:
        for c in ctxs:
            c.close()


def test_bp_insert_multi_rounds_and_errors(ctx, orc):
    """spi_bp_insert_multi with device images and FFT sub-batches smaller
    than the image counts (several rounds, classes running out at different
    rounds): one insertion launch per round, volumes equal to the oracle's;
    invalid calls are refused with 101."""
    import torch
    os.environ["SPI_BP_SUB"] = "64"
    ctxs = [ops.Context(0) for _ in range(3)]
    try:
        data = []
        for k, (nx, nimg) in enumerate(((16, 300), (20, 70), (16, 130))):
            _, pr, ang = _case(nx, nimg, 400 + k)
            half = synth.half_mask(nimg, np.random.default_rng(410 + k))
            data.append((torch.from_numpy(pr).cuda(), ang, half))
            ctxs[k].bp_open(nx, 2)
        l0 = ctxs[0].launches
        ops.bp_insert_multi(ctxs, data)
        rounds = (300 + 63) // 64
        # per round one insertion launch plus the staging of each class that still has images
        staged = sum((n + 63) // 64 for n in (300, 70, 130))
        assert ctxs[0].launches - l0 >= rounds
        outs = []
        for c in ctxs:
            o = c.bp_finish(("all", "1", "2"))
            outs.append((o["all"], o["1"], o["2"]))
            c.bp_close()
        for (pr, ang, half), got in zip(data, outs):
            ref = orc.bp32f(pr.cpu().numpy(), ang, half, prec=0)
            for a, b in zip(got, ref):
                assert synth.rel_l2(a, b) <= TOL
        with pytest.raises(ops.SpiderError) as e:       # a closed class
            ops.bp_insert_multi(ctxs[:1], data[:1])
        assert e.value.code == 101
        assert staged > rounds
    finally:
        del os.environ["SPI_BP_SUB"]
        for c in ctxs:
            c.close()


def test_bp_autotune(ctx, orc):
    """The autotuner picks a launch, leaves the grids empty, and the
    reconstruction after it still matches the oracle; it refuses to run once
    images are in the grids; a second open of the same shape reuses the
    cached choice."""
    nx, nimg = 48, 200
    _, pr, ang = _case(nx, nimg, 77)
    half = synth.half_mask(nimg, np.random.default_rng(78))
    ctx.bp_open(nx, 2)
    try:
        cfg = ctx.bp_autotune()
        assert cfg["kernel"] in ("insert_x4_kernel", "insert_xlane_kernel")
        assert cfg["threads"] in (128, 256, 512) and cfg["blocks_per_sm"] >= 1 and cfg["tuned_ms"] > 0
        ctx.bp_insert(pr, ang, half)
        with pytest.raises(ops.SpiderError) as e:
            ctx.bp_autotune()
        assert e.value.code == 101
        o = ctx.bp_finish(("all", "1", "2"))
    finally:
        ctx.bp_close()
    ref = orc.bp32f(pr, ang, half, prec=0, nthreads=1)
    for a, b in zip((o["all"], o["1"], o["2"]), ref):
        assert synth.rel_l2(a, b) <= TOL
    ctx.bp_open(nx, 2)
    try:
        assert ctx.bp_autotune() == cfg        # cached
    finally:
        ctx.bp_close()


def test_bp3f_max_box_linearity(ctx):
    """At the largest box (nx = 512: a 1024^3 padded grid of 8.6 GB) the
    reconstruction is linear in the images for fixed angles (X is, W depends
    only on the angles, and WINDKB2A's shell mean is linear): a size-
    independent check where the oracle would take too long."""
    nx, nimg = 512, 6
    rng = np.random.default_rng(512)
    a = rng.standard_normal((nimg, nx, nx)).astype(np.float32)
    b = rng.standard_normal((nimg, nx, nx)).astype(np.float32)
    ang = synth.so3_angles(nimg, rng)
    va = ops.bp3f(a, ang, ctx=ctx)
    vb = ops.bp3f(b, ang, ctx=ctx)
    vab = ops.bp3f(a + 2.0 * b, ang, ctx=ctx)
    assert va.shape == (nx, nx, nx)
    assert np.isfinite(vab).all()
    assert synth.rel_l2(vab, va + 2.0 * vb) <= 1e-5


def test_bp_insert_zero_images_is_noop(ctx):
    ctx.bp_open(32, 2)
    try:
        ctx.bp_insert(np.zeros((0, 32, 32), np.float32), np.zeros((0, 3), np.float32), np.zeros(0, np.uint8))
        o = ctx.bp_finish(("all", "1", "2"))
    finally:
        ctx.bp_close()
    assert all(np.all(v == 0) for v in o.values())


def test_accumulation_modes_and_flush(ctx, orc):
    """Compensated accumulation (default, and with a fold every 50 images)
    and plain FP32 atomics all match the oracle; spi_bp_flush leaves the
    grids holding the complete sums (BP 3F P after a flush equals the
    oracle's partial grids); the mode cannot change while a reconstruction
    is open."""
    nx, nimg = 32, 260
    _, pr, ang = _case(nx, nimg, 501, noise=0.5)
    ref = orc.bp3f(pr, ang, prec=1)
    rx, rw = orc.bp3f_partial(pr, ang, prec=1)
    try:
        for comp, fold in ((True, 0), (True, 50), (False, 0)):
            ctx.set_accumulation(comp, fold)
            got = ops.bp3f(pr, ang, ctx=ctx)
            assert synth.rel_l2(got, ref) <= TOL, (comp, fold)
        ctx.set_accumulation(True, 50)
        ctx.bp_open(nx, 1)
        try:
            with pytest.raises(ops.SpiderError) as e:
                ctx.set_accumulation(False)
            assert e.value.code == 101
            ctx.bp_insert(pr, ang)
            ctx.bp_flush()
            x, w = ctx.bp_partial_out(0)
        finally:
            ctx.bp_close()
        gx = x[..., 0] + 1j * x[..., 1]
        assert np.linalg.norm(gx - rx) <= TOL * np.linalg.norm(rx)
        assert synth.rel_l2(w, rw) <= TOL
        with pytest.raises(ops.SpiderError) as e:
            ctx.bp_flush()                       # nothing open
        assert e.value.code == 101
    finally:
        ctx.set_accumulation(True, 0)


def test_own_r2c_matches_cufft_path(ctx, orc):
    """The library's own two-pass R2C (SPI_FFT=own: staging fused with the row
    transforms, then the column transforms; power-of-two padded sizes) gives
    the volumes of the staging + cuFFT path and of the oracle, host and
    device images, BF16 spectra too."""
    import torch
    for nx, nimg in ((32, 200), (64, 150)):
        _, pr, ang = _case(nx, nimg, 600 + nx)
        half = synth.half_mask(nimg, np.random.default_rng(601))
        ref = orc.bp32f(pr, ang, half, prec=1)
        base = ops.bp32f(pr, ang, half, ctx=ctx)
        os.environ["SPI_FFT"] = "own"
        try:
            own = ops.bp32f(pr, ang, half, ctx=ctx)
            own_dev = ops.bp32f(torch.from_numpy(pr).cuda(), ang, half, ctx=ctx)
            own16 = ops.bp32f(pr, ang, half, ctx=ctx, bf16=True)
        finally:
            del os.environ["SPI_FFT"]
        for a, b, c, d, r in zip(own, own_dev, base, own16, ref):
            assert synth.rel_l2(a, r) <= TOL
            assert synth.rel_l2(b, r) <= TOL
            assert synth.rel_l2(a, c) <= TOL
            assert synth.rel_l2(d, r) <= 5e-4


@pytest.mark.parametrize("nx,mode", [(64, "own2"), (128, "own"), (128, "own2"), (256, "own"), (256, "own:cols8"),
                                     (256, "own2")])
def test_own_r2c_sizes(ctx, nx, mode, monkeypatch):
    """The register-FFT passes (SPI_FFT=own at padded sizes 128-512; the
    default at 512, its column pass with 4 (default) or 8 columns per CTA)
    and the shared-memory radix-2 passes (own2) give the volumes of PADD2 +
    cuFFT (SPI_FFT=cufft)."""
    if mode.endswith(":cols8"):
        monkeypatch.setenv("SPI_COLFFT_COLS", "8")
        mode = "own"
    rng = np.random.default_rng(700 + nx)
    nimg = 48
    vol = synth.blob_phantom(nx, 10, sigma=(2, 6), radius=0.35 * nx, rng=rng)
    ang = synth.so3_angles(nimg, rng)
    pr = ops.pj3q(vol, ang, ctx=ctx)
    half = synth.half_mask(nimg, rng)
    os.environ["SPI_FFT"] = "cufft"
    try:
        base = ops.bp32f(pr, ang, half, ctx=ctx)
    finally:
        del os.environ["SPI_FFT"]
    os.environ["SPI_FFT"] = mode
    try:
        own = ops.bp32f(pr, ang, half, ctx=ctx)
    finally:
        del os.environ["SPI_FFT"]
    for a, c in zip(own, base):
        e = synth.rel_l2(a, c)
        print(f"own R2C ({mode}) nx={nx}: rel-L2 vs cuFFT path {e:.2e}")
        assert e <= TOL



@pytest.mark.parametrize("fft,bf16", [("own", False), ("cufft", True), ("cufft", False)])
def test_bp_host_upload_pieces(ctx, orc, fft, bf16, monkeypatch):
    """Host images uploaded in small pieces (16 images, FFT sub-batches of 64):
    a call of one chunk takes its first piece as the first sub-batch (own R2C
    or BF16 spectra; with cuFFT's FP32 batches the sub-batches stay whole),
    and slice-sorting groups of 24, which do not divide a sub-batch, stay
    inside their sub-batch.  The volumes match the FP64 oracle."""
    nx, nimg = 64, 150
    _, pr, ang = _case(nx, nimg, 810)
    half = synth.half_mask(nimg, np.random.default_rng(811))
    ref = orc.bp32f(pr, ang, half, prec=1)
    for k, v in (("SPI_BP_SUB", "64"), ("SPI_UPLOAD_IMAGES", "16"), ("SPI_SORT_GROUP", "24"), ("SPI_FFT", fft)):
        monkeypatch.setenv(k, v)
    out = ops.bp32f(pr, ang, half, ctx=ctx, bf16=bf16)
    monkeypatch.setenv("SPI_FIRST_PIECE", "0")
    whole = ops.bp32f(pr, ang, half, ctx=ctx, bf16=bf16)
    for a, w, r in zip(out, whole, ref):
        e = synth.rel_l2(a, r)
        print(f"upload pieces ({fft}, bf16={bf16}): rel-L2 vs FP64 oracle {e:.2e}")
        assert e <= (5e-4 if bf16 else TOL)
        assert synth.rel_l2(a, w) <= (1e-4 if bf16 else TOL)
