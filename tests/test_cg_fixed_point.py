"""The mixed-precision BP CG projector accumulates each projection in 32-bit
fixed point, scaled so that no pixel sum can exceed the int32 range: the
voxels that can reach one pixel (bilinear cell [p-1, p+1) x [q-1, q+1)) lie
in a 2 x 2 prism through the sphere, and their count is bounded by the
volume of that prism grown by a unit cube's half-diagonal,
pi (sqrt 2 + sqrt 3 / 2)^2 (2 RI + sqrt 3).  Checked here by counting, for
axis-aligned, diagonal and random orientations."""
import numpy as np
import pytest
from scipy.spatial.transform import Rotation


def _mcap(ri):
    return np.pi * (np.sqrt(2.0) + np.sqrt(3.0) / 2.0) ** 2 * (2.0 * ri + np.sqrt(3.0))


@pytest.mark.parametrize("ri", [9, 21])
def test_pixel_contributor_bound(ri):
    g = np.arange(-ri, ri + 1)
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    m = x ** 2 + y ** 2 + z ** 2 <= ri * ri
    pts = np.stack([x[m], y[m], z[m]], 1).astype(np.float64)
    rots = [np.eye(3), Rotation.from_euler("z", 45, degrees=True).as_matrix(),
            Rotation.from_euler("zy", [45, 35.26], degrees=True).as_matrix()]
    rots += list(Rotation.random(40, random_state=ri).as_matrix())
    worst = 0
    for r in rots:
        uv = np.floor(pts @ r.T[:, :2] + 1000.0).astype(np.int64)
        cells, counts = np.unique(uv, axis=0, return_counts=True)
        d = {tuple(c): k for c, k in zip(cells, counts)}
        for (a, b) in d:
            for p, q in ((a, b), (a + 1, b), (a, b + 1), (a + 1, b + 1)):
                s = sum(d.get((p - i, q - j), 0) for i in (0, 1) for j in (0, 1))
                worst = max(worst, s)
    assert worst <= _mcap(ri)
