"""RB 3F / RB 32F with SPIDER's FBS mode: the in-plane rotation and shift is
RTSF (rtsf.f:109-205, FFT derivatives + bicubic FBS2) instead of RTSQ.
Against the CPU oracle on the same inputs: the rotated images differ only
through the FFT implementation of the derivative tables (both FP64), so the
volumes meet the BP 3F bar (rel-err <= 1e-5)."""
import io

import numpy as np
import pytest

from spider_b200 import operations, ops, synth
from spider_b200 import spider_io as sio

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _case(nx, nimg, seed):
    import oracle
    rng = np.random.default_rng(seed)
    vol = synth.blob_phantom(nx, 12, sigma=(1.5, 4.0), radius=0.35 * nx, rng=rng)
    ang = synth.so3_angles(nimg, rng)
    pr = oracle.pj3q(vol, ang)
    inplane = np.stack([rng.uniform(-180, 180, nimg), rng.uniform(-4, 4, nimg), rng.uniform(-4, 4, nimg)],
                       1).astype(np.float32)
    return pr, ang, inplane, rng


@pytest.mark.parametrize("nx", [32, 33])
def test_rb3f_rb32f_rtsf_match_oracle(ctx, orc, nx):
    pr, ang, inplane, rng = _case(nx, 160, 80 + nx)
    try:
        got = ops.rb3f(pr, ang, inplane, ctx=ctx, fbs=True)
        ref = orc.rb3f(pr, ang, inplane, prec=0, fbs=True, nthreads=1)
        e = synth.rel_l2(got, ref)
        print(f"RB 3F RTSF nx={nx}: rel-err vs oracle {e:.3e}, vs RTSQ oracle "
              f"{synth.rel_l2(ref, orc.rb3f(pr, ang, inplane, prec=0, nthreads=1)):.3e}")
        assert e <= TOL
        half = synth.half_mask(len(ang), rng)
        g = ops.rb32f(pr, ang, inplane, half, ctx=ctx, fbs=True)
        r = orc.rb3f(pr, ang, inplane, half, prec=0, fbs=True, nthreads=1)
        for a, b in zip(g, r):
            assert synth.rel_l2(a, b) <= TOL
        # no rotation and no shift: RTSF returns the images themselves
        z = ops.rb3f(pr, ang, np.zeros((len(ang), 3), np.float32), ctx=ctx, fbs=True)
        assert synth.rel_l2(z, ops.bp3f(pr, ang, ctx=ctx)) <= 2e-6
    finally:
        ctx.set_fbs(False)


def test_rb3f_rtsf_batches(ctx, orc):
    """At 128^2 the RTSF scratch holds fewer images than a call brings, so the
    derivative tables are made in several batches."""
    pr, ang, inplane, _ = _case(128, 420, 9)
    try:
        got = ops.rb3f(pr, ang, inplane, ctx=ctx, fbs=True)
    finally:
        ctx.set_fbs(False)
    ref = orc.rb3f(pr, ang, inplane, prec=0, fbs=True, nthreads=1)
    assert synth.rel_l2(got, ref) <= TOL


def test_md_fbs_mode_switches_rb3f(ctx, tmp_path):
    """'MD' / 'FBS ON' makes the next RB 3F use RTSF; 'FBS OFF' restores RTSQ."""
    pr, ang, inplane, _ = _case(32, 40, 3)
    t = str(tmp_path)
    for i in range(len(ang)):
        sio.write_image(tmp_path / f"img{i + 1:03d}.spi", pr[i])
    sio.write_doc(tmp_path / "ang.spi", [list(ang[i]) + [0, 0] + list(inplane[i]) for i in range(len(ang))])
    doc = sio.read_doc(tmp_path / "ang.spi")          # the registers as the document holds them
    ang = np.array([doc[k][:3] for k in range(1, len(ang) + 1)], np.float32)
    inplane = np.array([doc[k][5:8] for k in range(1, len(ang) + 1)], np.float32)
    out = io.StringIO()
    try:
        operations.run("MD", ["FBS ON"], ctx=ctx, results=out)
        operations.run("RB 3F", [f"{t}/img***", f"1-{len(ang)}", f"{t}/ang", "*", f"{t}/vf", "*"], ctx=ctx,
                       results=out)
        operations.run("MD", ["NO FBS"], ctx=ctx, results=out)
        operations.run("RB 3F", [f"{t}/img***", f"1-{len(ang)}", f"{t}/ang", "*", f"{t}/vq", "*"], ctx=ctx,
                       results=out)
    finally:
        ctx.set_fbs(False)
    assert "USING FBS INTERPOLATION" in out.getvalue()
    vf, _ = sio.read_image(tmp_path / "vf.spi")
    vq, _ = sio.read_image(tmp_path / "vq.spi")
    assert synth.rel_l2(vf, ops.rb3f(pr, ang, inplane, ctx=ctx, fbs=True)) <= 1e-6
    ctx.set_fbs(False)
    assert synth.rel_l2(vq, ops.rb3f(pr, ang, inplane, ctx=ctx)) <= 1e-6
    assert synth.rel_l2(vf, vq) > 1e-4
