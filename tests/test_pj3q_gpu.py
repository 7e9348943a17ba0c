"""PJ 3Q (WPRO_N, wpro_n.f:44-150) on the GPU against the CPU oracle, and
the exactness of its adjoint.  Sample positions are walked in the same
sequential float order as the reference, so only the z-sum order differs."""
import numpy as np
import pytest

from spider_b200 import ops, synth

pytestmark = pytest.mark.gpu


# packed: the warp row-task kernel on the packed volume, 32-byte cells up to
# 96 MB of cells (3M voxels) and 16-byte quads above, so (200, 192, 188)
# takes quads and the others cells; plain: SPI_PJ_QUADMAX=0, one thread per
# run on the volume
@pytest.mark.parametrize("form", ["packed", "plain"])
@pytest.mark.parametrize("shape", [(32, 32, 32), (64, 64, 64), (40, 36, 33), (200, 192, 188)])
def test_pj3q_matches_oracle(ctx, orc, shape, form, monkeypatch):
    if form == "plain":
        monkeypatch.setenv("SPI_PJ_QUADMAX", "0")
    nz, ny, nx = shape
    rng = np.random.default_rng(sum(shape))
    vol = synth.blob_phantom(max(shape), 10, sigma=(1.5, 4), radius=0.3 * min(shape), rng=rng)[:nz, :ny, :nx].copy()
    ang = synth.so3_angles(50, rng)
    got = ops.pj3q(vol, ang, ctx=ctx)
    ref = orc.pj3q(vol, ang, prec=0)
    ref64 = orc.pj3q(vol, ang, prec=1)
    e = synth.rel_l2(got, ref)
    print(f"PJ 3Q {shape} {form}: rel-L2 vs FP32 oracle {e:.3e}, vs FP64 {synth.rel_l2(got, ref64):.3e}")
    assert e <= 1e-5


def test_pj3q_radius_and_outside(ctx, orc):
    rng = np.random.default_rng(2)
    vol = rng.standard_normal((32, 32, 32)).astype(np.float32)
    ang = synth.so3_angles(20, rng)
    for ri in (5.0, 14.0, 16.0):   # 16 exceeds the no-check limit: bounds-checked branch
        got = ops.pj3q(vol, ang, ri, ctx=ctx)
        ref = orc.pj3q(vol, ang, ri, prec=0)
        assert synth.rel_l2(got, ref) <= 1e-5


def test_pj3q_adjoint_exact(ctx):
    rng = np.random.default_rng(7)
    n = 32
    x = rng.standard_normal((n, n, n)).astype(np.float32)
    y = rng.standard_normal((30, n, n)).astype(np.float32)
    ang = synth.so3_angles(30, rng)
    ax = ops.pj3q(x, ang, ctx=ctx)
    aty = ops.pj3q_adjoint(y, ang, (n, n, n), ctx=ctx)
    lhs = float(np.dot(ax.ravel().astype(np.float64), y.ravel()))
    rhs = float(np.dot(x.ravel().astype(np.float64), aty.ravel()))
    assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), abs(rhs))


def test_pj3q_adjoint_run_orders(ctx, monkeypatch):
    """The adjoint's threads take the runs in (z, y) order, (y, z) order or
    per projection the one whose neighbouring walks differ more in x (the
    default): every order adds the same weights to the same voxels."""
    rng = np.random.default_rng(17)
    n = 48
    ang = synth.so3_angles(40, rng)
    y = rng.standard_normal((40, n, n)).astype(np.float32)
    x = rng.standard_normal((n, n, n)).astype(np.float32)
    out = {}
    for order in ("0", "3", "1", "2"):
        monkeypatch.setenv("SPI_PJ_ADJ_ORDER", order)
        out[order] = ops.pj3q_adjoint(y, ang, (n, n, n), ctx=ctx)
    for order, v in out.items():
        assert synth.rel_l2(v, out["0"]) <= 1e-6, order
    ax = ops.pj3q(x, ang, ctx=ctx)
    lhs = float(np.dot(ax.ravel().astype(np.float64), y.ravel()))
    rhs = float(np.dot(x.ravel().astype(np.float64), out["1"].ravel()))
    assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), abs(rhs))


def test_pj3q_device_tensors(ctx, orc):
    import torch
    rng = np.random.default_rng(9)
    vol = synth.blob_phantom(32, 6, rng=rng)
    ang = synth.so3_angles(10, rng)
    got = ops.pj3q(torch.from_numpy(vol).cuda(), ang, ctx=ctx).cpu().numpy()
    assert synth.rel_l2(got, orc.pj3q(vol, ang)) <= 1e-5


@pytest.mark.parametrize("quadmax", [None, "0"])
def test_pj3q_plan_forward_forms(ctx, orc, quadmax, monkeypatch):
    """A plan on the packed volume (the default; cells at this size) and one
    on the plain volume both reproduce the oracle, for a ragged shape with
    several row tasks per row."""
    import torch
    from spider_b200 import autograd
    if quadmax is not None:
        monkeypatch.setenv("SPI_PJ_QUADMAX", quadmax)
    rng = np.random.default_rng(11)
    shape = (72, 80, 76)
    vol = synth.blob_phantom(80, 12, sigma=(1.5, 4), radius=24, rng=rng)[:72, :80, :76].copy()
    ang = synth.so3_angles(24, rng)
    plan = autograd.PJ3QPlan(shape, ang, ctx=ctx)
    got = plan.forward(torch.from_numpy(vol).cuda()).cpu().numpy()
    plan.close()
    assert synth.rel_l2(got, orc.pj3q(vol, ang, prec=0)) <= 1e-5


def test_pj3q_adjoint_slabs(ctx, monkeypatch):
    """At 168^3 the quad accumulator (76 MB) is filled in two z slabs; the
    result equals the scalar-atomic adjoint (SPI_PJ_QUADMAX=0) up to the
    order of the float sums, and <A x, y> = <x, A^T y> holds."""
    rng = np.random.default_rng(13)
    n = 168
    ang = synth.so3_angles(12, rng)
    y = rng.standard_normal((12, n, n)).astype(np.float32)
    x = rng.standard_normal((n, n, n)).astype(np.float32)
    slabs = ops.pj3q_adjoint(y, ang, (n, n, n), ctx=ctx)
    monkeypatch.setenv("SPI_PJ_QUADMAX", "0")
    plain = ops.pj3q_adjoint(y, ang, (n, n, n), ctx=ctx)
    monkeypatch.delenv("SPI_PJ_QUADMAX")
    assert synth.rel_l2(slabs, plain) <= 1e-6
    ax = ops.pj3q(x, ang, ctx=ctx)
    lhs = float(np.dot(ax.ravel().astype(np.float64), y.ravel()))
    rhs = float(np.dot(x.ravel().astype(np.float64), slabs.ravel()))
    assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), abs(rhs))


def test_pj3q_forward_slabs(ctx, orc):
    """At 240^3 the quads (221 MB) are read in three z slabs that each stay
    in L2, with the row tasks in z order; the projections match the oracle."""
    rng = np.random.default_rng(17)
    n = 240
    vol = synth.blob_phantom(n, 12, sigma=(2, 6), radius=80, rng=rng)
    ang = synth.so3_angles(4, rng)
    got = ops.pj3q(vol, ang, ctx=ctx)
    assert synth.rel_l2(got, orc.pj3q(vol, ang, prec=0)) <= 1e-5
