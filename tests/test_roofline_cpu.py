"""The algorithmic bytes the bench's roofline divides by.  ONELINE's nonzero
taps per image (spider_b200.roofline.taps_for_slice, oneline.f:38-200) over
uniform SO(3) rotations against the per-image tap counts of the reference
formulas at 64, 96 and 128 (2.98e5, 6.73e5, 1.20e6), and the bytes per
image: 24 per tap (a 12-byte read and write of X and W) plus the input."""
import numpy as np
import pytest

import oracle
from spider_b200 import roofline, synth


@pytest.mark.parametrize("nx,ref", [(64, 2.98e5), (96, 6.73e5), (128, 1.20e6)])
def test_oneline_taps_per_image(nx, ref):
    tab, fltb = roofline.kb_table(2 * nx)
    ang = synth.so3_angles(16, np.random.default_rng(nx))
    dms = np.array([np.asarray(oracle.cang(a[2], a[1], a[0]), np.float32)[:6] for a in ang])
    taps = roofline.mean_taps(nx, dms, tab, fltb)
    assert abs(taps / ref - 1.0) < 0.01, taps


def test_bytes_per_image():
    assert roofline.BYTES_PER_TAP == 24
    assert roofline.spectrum_bytes(256) == 257 * 512 * 8
    assert roofline.spectrum_bytes(256, bf16=True) == 257 * 512 * 4
