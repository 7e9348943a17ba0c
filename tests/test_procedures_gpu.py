"""The reference's procedure-level tests, replayed through the file-level
operations: testbp3f.tst (BP 3F and BP 32F of twelve 75x75 'MO T' sine images)
and testbpcg.tst (BP CG, radius 35, 25 iterations, mode 1, lambda 2000).

The reference's angle document for these tests (savangbprp) is not in its
tree, so a substitute set of twelve angles is used and documented here; the
volumes are checked against the CPU oracle on the same files instead of
against the reference's printed ranges."""
import io

import numpy as np
import pytest

from spider_b200 import operations, ops, synth
from spider_b200 import spider_io as sio

pytestmark = pytest.mark.gpu

# substitute for savangbprp: 12 projection directions (psi, theta, phi)
ANGLES = np.array([[0, 0, 0], [0, 30, 0], [0, 30, 90], [0, 30, 180], [0, 30, 270], [0, 60, 45],
                   [0, 60, 135], [0, 60, 225], [0, 60, 315], [0, 90, 0], [0, 90, 60], [0, 90, 120]],
                  np.float32)


def mo_t(nx=75, ny=75):
    """MO ... T: one sine wave, NCX = NCY = 2 (model.f:239-296)."""
    twopi = np.float32(2 * np.pi)
    i = np.arange(ny, dtype=np.float32)[:, None]
    j = np.arange(nx, dtype=np.float32)[None, :]
    phase = i * twopi / np.float32(ny)
    return np.sin(j * twopi * np.float32(2) / np.float32(nx) + phase * np.float32(2)).astype(np.float32)


def _setup(tmp_path):
    img = mo_t()
    for k in range(1, 13):
        sio.write_image(tmp_path / f"jnk{k:03d}.spi", img)
    sio.write_doc(tmp_path / "savangbprp.spi", ANGLES.tolist(), comment="PSI THETA PHI (substitute set)")
    return img


def test_testbp3f_procedure(ctx, orc, tmp_path):
    img = _setup(tmp_path)
    out = io.StringIO()
    t = str(tmp_path)
    r = operations.run("BP 3F", [f"{t}/jnk***", "1-12", f"{t}/savangbprp", "*", f"{t}/jnkbp3f_out"],
                       ctx=ctx, results=out)
    vol, h = sio.read_image(tmp_path / "jnkbp3f_out.spi")
    assert vol.shape == (75, 75, 75) and h[4] == 3
    imgs = np.stack([img] * 12)
    ref = orc.bp3f(imgs, ANGLES, nthreads=1)
    assert synth.rel_l2(vol, ref) <= 1e-5
    print(f"  BP 3F     Range: {vol.min():12.5E}...{vol.max():12.5E}")
    assert "NUMBER OF IMAGES" in out.getvalue()
    r2 = operations.run("BP 32F", [f"{t}/jnk***", "1-12", f"{t}/savangbprp", "*", f"{t}/jnkbp32fb_out",
                                    f"{t}/jnkbp32f1_out", f"{t}/jnkbp32f2_out"], ctx=ctx, results=out)
    both, _ = sio.read_image(tmp_path / "jnkbp32fb_out.spi")
    # the 'both' volume uses every image, like BP 3F
    assert synth.rel_l2(both, vol) <= 1e-5
    r_all, r1, r2v = orc.bp32f(imgs, ANGLES, r2["half"], nthreads=1)
    assert synth.rel_l2(sio.read_image(tmp_path / "jnkbp32f1_out.spi")[0], r1) <= 1e-5


def test_testbpcg_procedure(ctx, orc, tmp_path):
    img = _setup(tmp_path)
    out = io.StringIO()
    t = str(tmp_path)
    operations.run("BP CG", [f"{t}/jnk***", "1-12", "35", f"{t}/savangbprp", "N", f"{t}/jnkbpcg_out",
                             "1.0E5, 0.0", "25,1", "2000"], ctx=ctx, results=out)
    vol, _ = sio.read_image(tmp_path / "jnkbpcg_out.spi")
    ref, rlog, _, _ = orc.bpcg(np.stack([img] * 12), ANGLES, 35.0, errm=1.0e5, chim=0.0, maxit=25, mode=1,
                               lam=2000.0, prec=1)
    assert synth.rel_l2(vol, ref) <= 1e-4
    lines = [ln for ln in out.getvalue().splitlines() if "ITERATION" in ln]
    assert len(lines) == len(rlog)      # error limit 1e5 stops after the first iteration
    print(f"  BP CG    Range: {vol.min():12.5E}...{vol.max():12.5E}")


def test_bpcg_fbs_procedure(ctx, orc, tmp_path):
    """testbpcg.tst with the 'F' answer: FBS interpolation (BPCG_3_FBS)."""
    img = _setup(tmp_path)
    out = io.StringIO()
    t = str(tmp_path)
    operations.run("BP CG", [f"{t}/jnk***", "1-12", "35", f"{t}/savangbprp", "F", f"{t}/jnkbpcg_fbs",
                             "1.0E5, 0.0", "25,1", "2000"], ctx=ctx, results=out)
    vol, _ = sio.read_image(tmp_path / "jnkbpcg_fbs.spi")
    ref, rlog, _, _ = orc.bpcg(np.stack([img] * 12), ANGLES, 35.0, errm=1.0e5, chim=0.0, maxit=25, mode=1,
                               lam=2000.0, prec=1, fbs=True)
    assert synth.rel_l2(vol, ref) <= 1e-4
    assert "USING FBS INTERPOLATION" in out.getvalue()
    lines = [ln for ln in out.getvalue().splitlines() if "ITERATION" in ln]
    assert len(lines) == len(rlog)
    print(f"  BP CG F  Range: {vol.min():12.5E}...{vol.max():12.5E}")


@pytest.mark.parametrize("indexed", [False, True])
def test_streamed_bp32f_and_rb32f_procedures(ctx, tmp_path, indexed):
    """BP 32F / RB 32F read their stack in chunks (next chunk read while the
    current one is inserted); the volumes equal the one-call array operation
    up to the order of the atomic sums."""
    rng = np.random.default_rng(8)
    n, nx = 150, 32
    vol = synth.blob_phantom(nx, 8, sigma=(1.5, 4.0), radius=10, rng=rng)
    ang = synth.so3_angles(n, rng)
    import oracle
    pr = oracle.pj3q(vol, ang)
    inplane = np.stack([rng.uniform(-20, 20, n), rng.uniform(-2, 2, n), rng.uniform(-2, 2, n)], 1)
    t = str(tmp_path)
    if indexed:   # numbers 200, 199, ... stored in slots 1, 2, ...
        sio.write_stack(tmp_path / "stk.spi", pr[::-1], numbers=list(range(51, 201)), maxindx=250)
        numbers = list(range(51, 201))
        keys = numbers
    else:
        sio.write_stack(tmp_path / "stk.spi", pr)
        numbers = list(range(1, n + 1))
        keys = numbers
    order = pr[::-1] if indexed else pr
    sio.write_doc(tmp_path / "ang.spi", [list(ang[i]) + [0, 0] + list(inplane[i]) for i in range(n)], keys=keys)
    doc = sio.read_doc(tmp_path / "ang.spi")
    ang_d = np.array([doc[k][:3] for k in keys], np.float32)
    ip_d = np.array([doc[k][5:8] for k in keys], np.float32)
    spec = f"{numbers[0]}-{numbers[-1]}"
    for op, extra in (("BP 32F", []), ("RB 32F", ["*"])):
        r = operations.run(op, [f"{t}/stk@***", spec, f"{t}/ang", "*", f"{t}/v", f"{t}/v1", f"{t}/v2"] + extra,
                           ctx=ctx, results=io.StringIO(), chunk=40)
        if op == "BP 32F":
            ref = ops.bp32f(order, ang_d, r["half"], ctx=ctx)
        else:
            ref = ops.rb32f(order, ang_d, ip_d, r["half"], ctx=ctx)
        for got, want in zip((r["vol"], r["vol1"], r["vol2"]), ref):
            assert synth.rel_l2(got, want) <= 1e-6, op


def test_pj3q_and_partial_merge_procedures(ctx, orc, tmp_path):
    t = str(tmp_path)
    rng = np.random.default_rng(5)
    vol = synth.blob_phantom(40, 8, sigma=(2, 4), radius=12, rng=rng)
    sio.write_image(tmp_path / "vol.spi", vol)
    ang = synth.so3_angles(30, rng)
    sio.write_doc(tmp_path / "ang.spi", ang.tolist())
    operations.run("PJ 3Q", [f"{t}/vol", "18", "1-30", f"{t}/ang", f"{t}/prj@***"], ctx=ctx, results=io.StringIO())
    prj, nums, heads = sio.read_stack(tmp_path / "prj.spi")
    doc = sio.read_doc(tmp_path / "ang.spi")          # the angles as the document holds them
    ang = np.array([doc[k][:3] for k in range(1, 31)], np.float32)
    assert synth.rel_l2(prj, orc.pj3q(vol, ang, 18.0)) <= 1e-5
    assert tuple(heads[4][100:103]) == tuple(ang[4])
    # BP 3F P on two halves, then BP 3F M == BP 3F of all
    operations.run("BP 3F P", [f"{t}/prj@***", "1-15", f"{t}/ang", "*", f"{t}/part001"], ctx=ctx,
                   results=io.StringIO())
    operations.run("BP 3F P", [f"{t}/prj@***", "16-30", f"{t}/ang", "*", f"{t}/part002"], ctx=ctx,
                   results=io.StringIO())
    operations.run("BP 3F M", [f"{t}/part***", "1-2", "*", f"{t}/merged"], ctx=ctx, results=io.StringIO())
    operations.run("BP 3F", [f"{t}/prj@***", "1-30", f"{t}/ang", "*", f"{t}/full"], ctx=ctx, results=io.StringIO())
    merged, _ = sio.read_image(tmp_path / "merged.spi")
    full, _ = sio.read_image(tmp_path / "full.spi")
    assert synth.rel_l2(merged, full) <= 1e-5


def test_bpcg3_procedures(ctx, orc, tmp_path):
    """BP CG 3 (random sample lists) and BP CG 3L (given lists): three
    independent CG solutions, each checked against the FP64 oracle."""
    t = str(tmp_path)
    rng = np.random.default_rng(9)
    vol = synth.blob_phantom(32, 6, sigma=(2, 4), radius=10, rng=rng)
    sio.write_doc(tmp_path / "cgang.spi", synth.so3_angles(24, rng).tolist())
    doc = sio.read_doc(tmp_path / "cgang.spi")
    ang = np.array([doc[k][:3] for k in range(1, 25)], np.float32)
    prj = orc.pj3q(vol, ang, 14.0)
    sio.write_stack(tmp_path / "cg.spi", prj)
    kw = dict(errm=1e-6, chim=0.0, maxit=4, mode=1, lam=0.5, prec=1)
    tail = ["1.0E-6, 0.0", "4,1", "0.5"]
    out = io.StringIO()
    r = operations.run("BP CG 3", [f"{t}/cg@***", "1-24", "14", f"{t}/cgang", "L", f"{t}/v", f"{t}/v1",
                                   f"{t}/v2"] + tail, ctx=ctx, results=out, seed=3)
    half = r["half"].astype(bool)
    assert half.sum() == 12
    for name, sel in (("v", np.ones(24, bool)), ("v1", half), ("v2", ~half)):
        got, _ = sio.read_image(tmp_path / f"{name}.spi")
        ref = orc.bpcg(prj[sel], ang[sel], 14.0, **kw)[0]
        assert synth.rel_l2(got, ref) <= 1e-4, name
    assert "Random lists" in out.getvalue()
    operations.run("BP CG 3L", [f"{t}/cg@***", "1-24", "1-10", "11-24", "14", f"{t}/cgang", "L", f"{t}/w",
                                f"{t}/w1", f"{t}/w2"] + tail, ctx=ctx, results=io.StringIO())
    for name, sel in (("w1", slice(0, 10)), ("w2", slice(10, 24))):
        got, _ = sio.read_image(tmp_path / f"{name}.spi")
        ref = orc.bpcg(prj[sel], ang[sel], 14.0, **kw)[0]
        assert synth.rel_l2(got, ref) <= 1e-4, name
