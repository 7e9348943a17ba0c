"""The file-level SPIDER operations (spider_b200.operations.run) on the CPU:
prompt order, angle and in-plane registers, half sets, sample lists, output
files and the reference's error codes, with the GPU work replaced by a
recording stand-in context and stand-ins for the ops calls.  The GPU tests
(tests/test_procedures_gpu.py) run the same operations on the library."""
import io

import numpy as np
import pytest

from spider_b200 import operations, ops
from spider_b200 import spider_io as sio


class FakeCtx:
    """Records the back-projection calls; bp_finish returns volumes filled
    with 1, 2, 3 for the reconstructions asked for, in order."""

    def __init__(self):
        self.opened = []
        self.inserts = []
        self.closed = 0
        self.fbs = False

    def bp_open(self, nx, ngrids, sym=None):
        self.nx = nx
        self.opened.append((nx, ngrids, None if sym is None else np.array(sym)))

    def bp_insert(self, imgs, ang, half, inplane=None):
        self.inserts.append((np.array(imgs, copy=True), np.array(ang, copy=True),
                             None if half is None else np.array(half, copy=True),
                             None if inplane is None else np.array(inplane, copy=True)))

    def bp_finish(self, which):
        return {w: np.full((self.nx,) * 3, i + 1, np.float32) for i, w in enumerate(which)}

    def bp_partial_out(self, g):
        n = self.nx
        return (np.arange(2 * n * 2 * n * (n + 1) * 2, dtype=np.float32),
                np.ones((2 * n, 2 * n, n + 1), np.float32))

    def bp_close(self):
        self.closed += 1

    def set_fbs(self, on):
        self.fbs = bool(on)


def _images(tmp_path, n, nx=8, ny=None, start=1):
    rng = np.random.default_rng(n + nx)
    imgs = rng.standard_normal((n, ny or nx, nx)).astype(np.float32)
    for i in range(n):
        sio.write_image(str(tmp_path / f"img{start + i:03d}.spi"), imgs[i])
    return imgs


def _angle_doc(tmp_path, keys, nreg=3, name="ang"):
    rng = np.random.default_rng(len(keys) + nreg)
    rows = [list(rng.uniform(0, 180, nreg)) for _ in keys]
    path = str(tmp_path / f"{name}.spi")
    sio.write_doc(path, rows, keys=keys)
    return sio.read_doc(path)   # the registers as the document holds them


def _run(op, answers, tmp_path, ctx, **kw):
    out = io.StringIO()
    res = operations.run(op, [str(a).replace("@D/", str(tmp_path) + "/") for a in answers], ctx=ctx,
                         results=out, **kw)
    return res, out.getvalue()


def test_bp32f_prompts_half_sets_and_outputs(tmp_path):
    imgs = _images(tmp_path, 10)
    doc = _angle_doc(tmp_path, list(range(1, 11)))
    ctx = FakeCtx()
    res, text = _run("bp  32f", ["@D/img***", "1-10", "@D/ang", "*", "@D/vol", "@D/v1", "@D/v2"], tmp_path, ctx,
                     chunk=4)
    assert ctx.opened[0][:2] == (8, 2) and ctx.opened[0][2] is None
    assert [len(c[0]) for c in ctx.inserts] == [4, 4, 2]          # chunk by chunk
    np.testing.assert_array_equal(np.concatenate([c[0] for c in ctx.inserts]), imgs)
    ang = np.concatenate([c[1] for c in ctx.inserts])
    np.testing.assert_array_equal(ang, np.array([doc[k][:3] for k in range(1, 11)], np.float32))
    half = np.concatenate([c[2] for c in ctx.inserts])
    assert int(half.sum()) == 5 and set(np.unique(half)) <= {0, 1}   # NANG/2 in the first sample
    np.testing.assert_array_equal(half, res["half"])
    for name, v in (("vol", 1), ("v1", 2), ("v2", 3)):
        arr, _ = sio.read_image(str(tmp_path / f"{name}.spi"))
        assert arr.shape == (8, 8, 8) and np.all(arr == v)
    assert "NUMBER OF IMAGES:      10" in text
    assert ctx.closed == 1


def test_bp3f_symmetries_from_document(tmp_path):
    _images(tmp_path, 3)
    _angle_doc(tmp_path, [1, 2, 3])
    sym = _angle_doc(tmp_path, [1, 2], name="sym")
    ctx = FakeCtx()
    _run("BP 3F", ["@D/img***", "1-3", "@D/ang", "@D/sym", "@D/vol"], tmp_path, ctx)
    assert ctx.opened[0][1] == 1
    np.testing.assert_array_equal(ctx.opened[0][2], np.array([sym[1][:3], sym[2][:3]], np.float32))
    assert ctx.inserts[0][2] is None


def test_rb3f_in_plane_registers(tmp_path):
    _images(tmp_path, 4)
    doc = _angle_doc(tmp_path, [1, 2, 3, 4], nreg=8)
    ctx = FakeCtx()
    _run("RB 3F", ["@D/img***", "1-4", "@D/ang", "*", "@D/vol", "*"], tmp_path, ctx)
    ip = np.concatenate([c[3] for c in ctx.inserts])
    np.testing.assert_array_equal(ip, np.array([doc[k][5:8] for k in (1, 2, 3, 4)], np.float32))
    # registers 6-8 missing: the reference's error 102
    _angle_doc(tmp_path, [1, 2, 3, 4], nreg=3, name="short")
    with pytest.raises(ops.SpiderError) as e:
        _run("RB 3F", ["@D/img***", "1-4", "@D/short", "*", "@D/vol", "*"], tmp_path, FakeCtx())
    assert e.value.code == 102


def test_back_projection_errors(tmp_path):
    _images(tmp_path, 3)
    _angle_doc(tmp_path, [1, 3])   # no angles for image 2
    with pytest.raises(ops.SpiderError) as e:
        _run("BP 3F", ["@D/img***", "1-3", "@D/ang", "*", "@D/vol"], tmp_path, FakeCtx())
    assert e.value.code == 102 and "IMAGE 2" in str(e.value)
    _images(tmp_path, 2, nx=8, ny=6, start=11)
    _angle_doc(tmp_path, [11, 12], name="ang2")
    with pytest.raises(ops.SpiderError) as e:   # bp3f.f:135-138
        _run("BP 3F", ["@D/img***", "11-12", "@D/ang2", "*", "@D/vol"], tmp_path, FakeCtx())
    assert e.value.code == 101 and "SQUARE" in str(e.value)
    with pytest.raises(ops.SpiderError) as e:
        _run("BP 7Q", [], tmp_path, FakeCtx())
    assert e.value.code == 101


def test_bp3f_partial_writes_x_and_w(tmp_path):
    _images(tmp_path, 2)
    _angle_doc(tmp_path, [1, 2])
    ctx = FakeCtx()
    res, _ = _run("BP 3F P", ["@D/img***", "1-2", "@D/ang", "*", "@D/part"], tmp_path, ctx)
    x, _ = sio.read_image(str(tmp_path / "part.spi"))
    w, _ = sio.read_image(str(tmp_path / "part_W.spi"))
    assert x.shape == (16, 16, 18) and w.shape == (16, 16, 9)
    np.testing.assert_array_equal(x.ravel(), res["x"])


def test_bp3f_merge_reads_partials(tmp_path, monkeypatch):
    n = 4
    for k in (1, 2):
        sio.write_image(str(tmp_path / f"part{k}.spi"), np.full((2 * n, 2 * n, 2 * (n + 1)), k, np.float32))
        sio.write_image(str(tmp_path / f"part{k}_W.spi"), np.full((2 * n, 2 * n, n + 1), 10 * k, np.float32))
    seen = {}

    def merge(parts, sym, ctx=None):
        seen["parts"], seen["sym"] = parts, sym
        return np.zeros((n, n, n), np.float32)

    monkeypatch.setattr(ops, "bp3f_merge", merge)
    _, text = _run("BP 3F M", ["@D/part*", "1-2", "*", "@D/vol"], tmp_path, FakeCtx())
    x1, w1 = seen["parts"][0]
    assert x1.shape == (2 * n, 2 * n, n + 1, 2) and np.all(x1 == 1) and np.all(seen["parts"][1][1] == 20)
    assert seen["sym"] is None and "NUMBER OF VOLUMES:       2" in text
    assert (tmp_path / "vol.spi").exists()


@pytest.mark.parametrize("conseq", [False, True])
def test_pj3q_radius_numbering_and_headers(tmp_path, monkeypatch, conseq):
    vol = np.zeros((8, 8, 8), np.float32)
    sio.write_image(str(tmp_path / "vol.spi"), vol)
    doc = _angle_doc(tmp_path, [5, 6, 7])
    seen = {}

    def pj3q(v, ang, ri, ctx=None):
        seen["ri"], seen["ang"] = ri, ang
        return np.stack([np.full((8, 8), k, np.float32) for k in range(len(ang))])

    monkeypatch.setattr(ops, "pj3q", pj3q)
    radius = "3, Y" if conseq else "3"
    _, text = _run("PJ 3Q", ["@D/vol", radius, "5-7", "@D/ang", "@D/prj***"], tmp_path, FakeCtx())
    assert seen["ri"] == 3.0
    for i, k in enumerate((5, 6, 7)):
        num = i + 1 if conseq else k
        arr, h = sio.read_image(str(tmp_path / f"prj{num:03d}.spi"))
        assert np.all(arr == i)
        np.testing.assert_allclose(h[100:103], np.array(doc[k][:3], np.float32))   # PSI, THETA, PHI
    assert "PJ 3Q FINISHED FOR:       3" in text


def test_pj3q_default_radius_and_stack_output(tmp_path, monkeypatch):
    sio.write_image(str(tmp_path / "vol.spi"), np.zeros((8, 8, 8), np.float32))
    _angle_doc(tmp_path, [1, 2])
    seen = {}

    def pj3f(v, ang, ri, ctx=None):
        seen["ri"] = ri
        return np.ones((len(ang), 8, 8), np.float32)

    monkeypatch.setattr(ops, "pj3f", pj3f)
    _run("PJ 3F", ["@D/vol", "", "1-2", "@D/ang", "@D/stk@***"], tmp_path, FakeCtx())
    assert seen["ri"] == 2.0   # n/2 - 2, pj3q_n.f:82
    imgs, _, _ = sio.read_stack(str(tmp_path / "stk.spi"), [1, 2])
    assert imgs.shape == (2, 8, 8) and np.all(imgs == 1)


def test_bpcg_answers(tmp_path, monkeypatch):
    imgs = _images(tmp_path, 4)
    _angle_doc(tmp_path, [1, 2, 3, 4])
    seen = {}

    def bpcg(im, ang, ri, errm, chim, maxit, mode, lam, ctx=None, interp="linear"):
        seen.update(ri=ri, errm=errm, chim=chim, maxit=maxit, mode=mode, lam=lam, interp=interp, im=im)
        return np.zeros((8, 8, 8), np.float32), [(1, 0.5, 2.0), (2, 0.25, 1.0)]

    monkeypatch.setattr(ops, "bpcg", bpcg)
    _, text = _run("BP CG", ["@D/img***", "1-4", "", "@D/ang", "F", "@D/vol", "1e-5, 0.2", "7, 1", "0.001"],
                   tmp_path, FakeCtx())
    assert seen["ri"] == 2.0 and seen["interp"] == "fbs"           # radius default n/2 - 2; 'F' = FBS
    assert (seen["errm"], seen["chim"], seen["maxit"], seen["mode"], seen["lam"]) == (1e-5, 0.2, 7, 1, 0.001)
    np.testing.assert_array_equal(seen["im"], imgs)
    assert "USING FBS INTERPOLATION" in text and "ITERATION:   2" in text
    assert (tmp_path / "vol.spi").exists()


def test_bpcg3l_sample_lists(tmp_path, monkeypatch):
    imgs = _images(tmp_path, 6)
    _angle_doc(tmp_path, list(range(1, 7)))
    seen = {}

    def bpcg3(im, ang, half, ri, errm, chim, maxit, mode, lam, ctx=None, interp="linear"):
        seen.update(im=im, half=half, interp=interp)
        z = np.zeros((8, 8, 8), np.float32)
        return z, z, z, [[(1, 0.1, 1.0)], [(1, 0.2, 1.0)], [(1, 0.3, 1.0)]]

    monkeypatch.setattr(ops, "bpcg3", bpcg3)
    ans = ["@D/img***", "1-6", "1,3,5", "2,4,6", "5", "@D/ang", "L", "@D/vol", "@D/v1", "@D/v2", "0, 0", "3, 1",
           "0.5"]
    _run("BP CG 3L", ans, tmp_path, FakeCtx())
    np.testing.assert_array_equal(seen["im"], imgs[[0, 2, 4, 1, 3, 5]])
    np.testing.assert_array_equal(seen["half"], [1, 1, 1, 0, 0, 0])
    assert seen["interp"] == "linear"
    bad = list(ans)
    bad[3] = "2,4,9"   # image 9 is not in the image list
    with pytest.raises(ops.SpiderError) as e:
        _run("BP CG 3L", bad, tmp_path, FakeCtx())
    assert e.value.code == 102


def test_md_modes(tmp_path):
    ctx = FakeCtx()
    _, text = _run("MD", ["FBS ON"], tmp_path, ctx)
    assert ctx.fbs and "USING FBS" in text
    _run("MD", ["no fbs"], tmp_path, ctx)
    assert not ctx.fbs
    with pytest.raises(ops.SpiderError) as e:
        _run("MD", ["TR OFF"], tmp_path, ctx)
    assert e.value.code == 101
