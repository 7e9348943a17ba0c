"""The oracle's FourierSlice pair (FP64): its insertion is ONELINE's X
insertion without the weight grid (bp3f_partial's X off the SYMPLANE0 plane,
from the staged spectra), and its extraction is the exact adjoint of that
insertion."""
import numpy as np

import oracle
from spider_b200 import synth


def test_fslice_insert_is_oneline_without_weights():
    rng = np.random.default_rng(4)
    nx = 20
    imgs = rng.standard_normal((9, nx, nx)).astype(np.float32)
    ang = synth.so3_angles(9, rng)
    T = np.stack([np.conj(oracle.stage_image(im)) for im in imgs])   # ONELINE reads BI = conj(T)
    X = oracle.fslice_insert(T, ang)
    ref, _ = oracle.bp3f_partial(imgs, ang, prec=1, nthreads=1)
    # plane i = 0 is rewritten by SYMPLANE0 in BP 3F P; every other voxel is the insertion itself
    d = np.abs(X[:, :, 1:] - ref[:, :, 1:]).max()
    assert d <= 1e-9 * np.abs(ref).max()


def test_fslice_pair_is_adjoint():
    rng = np.random.default_rng(5)
    for nx in (16, 17):
        n = 2 * nx
        ang = synth.so3_angles(11, rng)
        X = rng.standard_normal((n, n, nx + 1)) + 1j * rng.standard_normal((n, n, nx + 1))
        T = rng.standard_normal((11, n, nx + 1)) + 1j * rng.standard_normal((11, n, nx + 1))
        lhs = np.sum((np.conj(oracle.fslice_extract(X, ang)) * T).real)
        rhs = np.sum((np.conj(X) * oracle.fslice_insert(T, ang)).real)
        assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
