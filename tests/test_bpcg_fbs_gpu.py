"""BP CG with FBS interpolation (the 'F' answer, BPCG_3_FBS bpcg.f:1760-1822)
on the GPU against the CPU oracle.

Both sides take the FFT derivatives in FP64, walk the sample positions with
the reference's sequential float additions and evaluate the cubics in the
same operation order; the GPU sums each projection pixel over the cube lines
in the reference's order.  What remains is the FFT implementation (cuFFT
against the oracle's own transform) and the order of the FP64 dot products,
so the FP64 solution is held to 1e-6 of the FP64 oracle (the BP CG bar is
1e-4; measured: bitwise equal), the FP32-table modes to 1e-5, and the FP32
form to 1e-4 of the FP32 oracle after one iteration.
"""
import numpy as np
import pytest

from spider_b200 import ops, synth

pytestmark = pytest.mark.gpu


def _data(n, nang, seed, snr=None):
    import oracle
    rng = np.random.default_rng(seed)
    vol = synth.blob_phantom(n, 8, sigma=(1.5, 3.5), radius=0.3 * n, rng=rng)
    ang = synth.so3_angles(nang, rng)
    pr = oracle.pj3q(vol, ang)
    if snr:
        pr = synth.add_noise(pr, snr, rng)
    return vol, pr, ang


@pytest.mark.parametrize("n,mode", [(32, 1), (32, 2), (32, 3), (25, 1), (24, 2)])
def test_bpcg_fbs_matches_fp64_oracle(ctx, orc, n, mode):
    nang = 60
    _, pr, ang = _data(n, nang, 100 + n + mode, snr=1.0)
    ri = float(n // 2 - mode - 1)
    vol, log = ops.bpcg(pr, ang, ri, errm=1e-9, chim=0.0, maxit=6, mode=mode, lam=0.5, ctx=ctx, fp64=True,
                        interp="fbs")
    ref, rlog, _, _ = orc.bpcg(pr, ang, ri, errm=1e-9, chim=0.0, maxit=6, mode=mode, lam=0.5, prec=1, fbs=True)
    lin, _, _, _ = orc.bpcg(pr, ang, ri, errm=1e-9, chim=0.0, maxit=6, mode=mode, lam=0.5, prec=1)
    e = synth.rel_l2(vol, ref)
    print(f"BP CG FBS n={n} mode {mode}: rel-err vs FP64 oracle {e:.3e}; FBS vs linear {synth.rel_l2(ref, lin):.3e}")
    assert len(log) == len(rlog)
    np.testing.assert_allclose(log[:, 1:], rlog[:, 1:], rtol=1e-5, atol=0)
    assert e <= 1e-6


def test_bpcg_fbs_precision_modes(ctx, orc):
    """Modes 2 and 3 ("mixed", the default, and "fast") keep FP64 vectors and
    arithmetic with FP32 interpolation tables; mode 4 ("mixed64") keeps FP64
    tables and equals the FP64 form."""
    n, nang = 32, 60
    _, pr, ang = _data(n, nang, 5, snr=1.0)
    kw = dict(errm=1e-9, maxit=6, mode=1, lam=0.5)
    ref, _, _, _ = orc.bpcg(pr, ang, 12.0, prec=1, fbs=True, **kw)
    full, _ = ops.bpcg(pr, ang, 12.0, ctx=ctx, fp64=True, interp="fbs", **kw)
    for prec in ("mixed", "fast"):
        v, _ = ops.bpcg(pr, ang, 12.0, ctx=ctx, fp64=prec, interp="fbs", **kw)
        e = synth.rel_l2(v, ref)
        print(f"BP CG FBS {prec} (FP32 tables): rel-err vs FP64 oracle {e:.3e}")
        assert e <= 1e-5
    v, _ = ops.bpcg(pr, ang, 12.0, ctx=ctx, fp64="mixed64", interp="fbs", **kw)
    assert synth.rel_l2(v, full) <= 1e-14


def test_bpcg_fbs_fp32_matches_fp32_oracle(ctx, orc):
    n, nang = 32, 60
    _, pr, ang = _data(n, nang, 7, snr=1.0)
    vol, _ = ops.bpcg(pr, ang, 13.0, errm=1e-9, maxit=1, mode=1, lam=0.5, ctx=ctx, fp64=False, interp="fbs")
    ref, _, _, _ = orc.bpcg(pr, ang, 13.0, errm=1e-9, maxit=1, mode=1, lam=0.5, prec=0, fbs=True)
    e = synth.rel_l2(vol, ref)
    print(f"BP CG FBS FP32, one iteration: rel-err vs FP32 oracle {e:.3e}")
    assert e <= 1e-4


def test_bpcg_fbs_duplicates_and_chunks(ctx, orc, monkeypatch):
    """HIANG merges duplicate angles (LB > 1 scales the FBS projections); the
    images and merged angles go through the operators in chunks of 7."""
    n, nang = 24, 50
    _, pr, ang = _data(n, nang, 21)
    ang[30:40] = ang[0:10]
    ang[45:50, 1] = 180.0 - ang[0:5, 1]
    ang[45:50, 2] = ang[0:5, 2] + 180.0
    ref, rlog, neff, _ = orc.bpcg(pr, ang, 9.0, errm=1e-9, maxit=5, mode=1, lam=0.2, prec=1, fbs=True)
    whole, _ = ops.bpcg(pr, ang, 9.0, errm=1e-9, maxit=5, mode=1, lam=0.2, ctx=ctx, fp64=True, interp="fbs")
    monkeypatch.setenv("SPI_FBS_CHUNK", "7")
    vol, log = ops.bpcg(pr, ang, 9.0, errm=1e-9, maxit=5, mode=1, lam=0.2, ctx=ctx, fp64=True, interp="fbs")
    assert neff < nang
    assert len(log) == len(rlog)
    assert synth.rel_l2(vol, ref) <= 1e-6
    assert synth.rel_l2(vol, whole) <= 1e-12


def test_bpcg_fbs_radius_limit(ctx):
    """FBS allows RI + MODE = N/2, one more than linear interpolation (bpcg.f:269-290)."""
    n = 16
    rng = np.random.default_rng(0)
    pr = rng.standard_normal((6, n, n)).astype(np.float32)
    ang = synth.so3_angles(6, rng)
    vol, _ = ops.bpcg(pr, ang, 7.0, maxit=2, mode=1, ctx=ctx, interp="fbs")
    assert np.isfinite(vol).all()
    with pytest.raises(ops.SpiderError) as ei:
        ops.bpcg(pr, ang, 7.0, mode=1, ctx=ctx, interp="linear")
    assert ei.value.code == 102
    with pytest.raises(ops.SpiderError) as ei:
        ops.bpcg(pr, ang, 7.5, mode=1, ctx=ctx, interp="fbs")
    assert ei.value.code == 102


def test_bpcg_fbs_rejects_bad_interpolation(ctx):
    with pytest.raises(ops.SpiderError):
        ops.bpcg(np.zeros((2, 16, 16), np.float32), np.zeros((2, 3), np.float32), 5.0, ctx=ctx, interp="cubic")
