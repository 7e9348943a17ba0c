"""PJ 3F (PJ 3Q with FBS interpolation: FBS3_PREP + WPRO_FBS) on the GPU
against the CPU oracle.  Sample positions, the FBS3 tables (up to the FFT
implementation) and every tricubic are the oracle's; only the order in which
the runs of one output row are summed differs (atomics), so the bar is
PJ 3Q's rel-err <= 1e-5."""
import io

import numpy as np
import pytest

from spider_b200 import operations, ops, synth
from spider_b200 import spider_io as sio

pytestmark = pytest.mark.gpu


def _vol(n, seed):
    rng = np.random.default_rng(seed)
    return synth.blob_phantom(n, 10, sigma=(1.5, 4.0), radius=0.3 * n, rng=rng), rng


@pytest.mark.parametrize("n,ri", [(32, None), (33, None), (32, 15.0), (48, 23.5)])
def test_pj3f_matches_oracle(ctx, orc, n, ri):
    """ri = None is the default radius (the sphere fits, no bounds test);
    the larger radii take WPRO_FBS's checked branch, where positions up to
    IFIX = N wrap around."""
    vol, rng = _vol(n, 10 + n)
    ang = synth.so3_angles(40, rng)
    got = ops.pj3f(vol, ang, ri, ctx=ctx)
    ref = orc.pj3f(vol, ang, ri)
    e = synth.rel_l2(got, ref)
    print(f"PJ 3F n={n} ri={ri}: rel-err vs oracle {e:.3e}, vs PJ 3Q {synth.rel_l2(got, orc.pj3q(vol, ang, ri)):.3e}")
    assert e <= 1e-5


def test_pj3f_device_tensors(ctx, orc):
    import torch
    vol, rng = _vol(32, 3)
    ang = synth.so3_angles(16, rng)
    got = ops.pj3f(torch.from_numpy(vol).cuda(), ang, ctx=ctx)
    assert synth.rel_l2(got.cpu().numpy(), orc.pj3f(vol, ang)) <= 1e-5


def test_pj3f_operation_and_errors(ctx, orc, tmp_path):
    vol, rng = _vol(32, 4)
    t = str(tmp_path)
    sio.write_image(tmp_path / "vol.spi", vol)
    ang = synth.so3_angles(12, rng)
    sio.write_doc(tmp_path / "ang.spi", ang.tolist())
    out = io.StringIO()
    operations.run("PJ 3F", [f"{t}/vol", "14", "1-12", f"{t}/ang", f"{t}/prj@***"], ctx=ctx, results=out)
    prj, _, _ = sio.read_stack(tmp_path / "prj.spi")
    doc = sio.read_doc(tmp_path / "ang.spi")
    ang = np.array([doc[k][:3] for k in range(1, 13)], np.float32)
    assert synth.rel_l2(prj, orc.pj3f(vol, ang, 14.0)) <= 1e-5
    assert "PJ 3F FINISHED" in out.getvalue()
    with pytest.raises(ops.SpiderError):
        ops.pj3f(np.zeros((16, 16, 20), np.float32), ang, ctx=ctx)
