"""SPIDER image/stack/doc formats and the file-number / template syntax."""
import numpy as np
import pytest

from spider_b200 import spider_io as sio


def test_header_layout(tmp_path):
    for nx in (16, 75, 256, 300):
        assert sio._labrec(nx) == -(-1024 // (4 * nx))
    img = np.arange(75 * 75, dtype=np.float32).reshape(75, 75)
    p = tmp_path / "jnk001.spi"
    sio.write_image(p, img, angles=(10.0, 20.0, 30.0))
    h, order = sio.read_header(p)
    assert order == "<"
    assert h[0] == 1 and h[1] == 75 and h[4] == 1 and h[11] == 75
    assert h[12] == 4 and h[21] == 4 * 300 and h[22] == 300          # LABREC, LABBYT, LENBYT
    assert tuple(h[100:104]) == (10.0, 20.0, 30.0, 1.0)
    assert h[6] == img.max() and h[7] == img.min()
    got, _ = sio.read_image(p)
    assert np.array_equal(got, img)
    assert p.stat().st_size == 4 * 300 + 75 * 75 * 4


def test_volume_and_byteswap(tmp_path):
    vol = np.random.default_rng(0).standard_normal((8, 9, 10)).astype(np.float32)
    p = tmp_path / "v.spi"
    sio.write_image(p, vol)
    got, h = sio.read_image(p)
    assert got.shape == (8, 9, 10) and np.array_equal(got, vol) and h[4] == 3
    # byte-swapped copy is recognised by header plausibility
    raw = np.fromfile(p, "<f4").astype(">f4")
    q = tmp_path / "v_swapped.spi"
    raw.tofile(q)
    got2, _ = sio.read_image(q)
    assert np.array_equal(got2, vol)


def test_stack_roundtrip(tmp_path):
    imgs = np.random.default_rng(1).standard_normal((5, 12, 12)).astype(np.float32)
    ang = np.arange(15, dtype=np.float32).reshape(5, 3)
    p = tmp_path / "stk.spi"
    sio.write_stack(p, imgs, angles=ang)
    h, _ = sio.read_header(p)
    assert h[23] > 0 and h[25] == 5
    got, nums, heads = sio.read_stack(p)
    assert nums == [1, 2, 3, 4, 5] and np.array_equal(got, imgs)
    assert [int(x[26]) for x in heads] == nums
    assert tuple(heads[2][100:103]) == tuple(ang[2])
    sub = sio.read_images(str(tmp_path / "stk@***"), [2, 4])
    assert np.array_equal(sub, imgs[[1, 3]])


def test_doc_files(tmp_path):
    p = tmp_path / "ang.spi"
    sio.write_doc(p, [[1.0, 2.0, 3.0], [4.5, -5.25, 6.0, 7, 8, 9, 10, 11]], comment="PSI THETA PHI")
    d = sio.read_doc(p)
    assert sorted(d) == [1, 2]
    np.testing.assert_allclose(d[2], [4.5, -5.25, 6.0, 7, 8, 9, 10, 11])
    txt = " ;tst/tst   16-JUN-1999\n    9 1  11.000\n 5556 7  5554.0 6.0 13.0 14.0 15.0 16.0 16.0\n ;-88 2 -88. -88.\n"
    q = tmp_path / "d.spi"
    q.write_text(txt)
    d = sio.read_doc(q)
    assert sorted(d) == [9, 5556] and d[5556][0] == 5554.0


def test_numbers_and_templates():
    assert sio.parse_numbers("1-12") == list(range(1, 13))
    assert sio.parse_numbers("1-3,7, 9-10") == [1, 2, 3, 7, 9, 10]
    assert sio.expand_template("jnk***", 7) == "jnk007"
    assert sio.expand_template("stk@****", 12) == "stk@0012"
    assert sio.add_extension("jnk001") == "jnk001.spi"
    assert sio.add_extension("stk@***") == "stk.spi@***"
    with pytest.raises(ValueError):
        sio.read_header(__file__)


def test_indexed_stack(tmp_path):
    """Indexed stacks (ISTACK = -MAXINDX, lunsethdr.f:505-530, 2140-2200):
    image numbers map to storage slots through the int32 index records."""
    rng = np.random.default_rng(5)
    imgs = rng.standard_normal((3, 7, 10)).astype(np.float32)
    p = tmp_path / "ix.spi"
    sio.write_stack(p, imgs, numbers=[15, 2, 9], maxindx=17)   # NX = 10: two index records
    h, _ = sio.read_header(p)
    assert int(h[23]) == -17
    got, nums, heads = sio.read_stack(p, [2, 9, 15])
    assert nums == [2, 9, 15]
    assert np.array_equal(got, imgs[[1, 2, 0]])
    assert [int(x[26]) for x in heads] == [2, 9, 15]          # IMGNUM of each stored image
    every, nums, _ = sio.read_stack(p)                         # every number in the index
    assert nums == [2, 9, 15] and np.array_equal(every, imgs[[1, 2, 0]])
    with pytest.raises(ValueError):
        sio.read_stack(p, [3])
    # the same file byte-swapped (every word is 4 bytes) reads the same
    q = tmp_path / "ix_swapped.spi"
    q.write_bytes(np.frombuffer(p.read_bytes(), "<u4").byteswap().tobytes())
    got2, _, _ = sio.read_stack(q, [9])
    assert np.array_equal(got2[0], imgs[2])
    # and through a template
    assert np.array_equal(sio.read_images(str(tmp_path / "ix@***"), [15, 2]), imgs[[0, 1]])


@pytest.mark.parametrize("kind", ["files", "stack", "indexed"])
@pytest.mark.parametrize("chunk", [1, 4, 7, 100])
def test_stream_images(tmp_path, kind, chunk):
    """stream_images yields the images in file-number order, chunk by chunk,
    from image files, a stack or an indexed stack (read ahead on a thread)."""
    rng = np.random.default_rng(11)
    imgs = rng.standard_normal((10, 6, 6)).astype(np.float32)
    if kind == "files":
        for i in range(10):
            sio.write_image(tmp_path / f"im{i + 1:03d}.spi", imgs[i])
        tmpl, numbers, want = str(tmp_path / "im***"), [3, 1, 10, 4], imgs[[2, 0, 9, 3]]
    elif kind == "stack":
        sio.write_stack(tmp_path / "st.spi", imgs)
        tmpl, numbers, want = str(tmp_path / "st@***"), list(range(10, 0, -1)), imgs[::-1]
    else:
        sio.write_stack(tmp_path / "ix.spi", imgs, numbers=[20 - i for i in range(10)], maxindx=25)
        tmpl, numbers, want = str(tmp_path / "ix@***"), [11, 20, 15], imgs[[9, 0, 5]]
    src = sio.ImageSource(tmpl, numbers)
    assert src.shape == (6, 6) and len(src) == len(numbers)
    got, starts = [], []
    for start, c in sio.stream_images(src, chunk):
        starts.append(start)
        got.append(c.copy())
    assert np.array_equal(np.concatenate(got), want)
    assert starts == list(range(0, len(numbers), min(chunk, len(numbers))))
