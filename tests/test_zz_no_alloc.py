"""spi_pj3q_noalloc: the PJ 3Q entry point for callers that must not
allocate device memory (a fixed arena or caching allocator owns it, or the
pipeline cannot take cudaMalloc/cudaFree's implicit synchronisation).

It is called through the C ABI with caller-owned device buffers, twice in a
row on fresh data, and its projections are compared with spi_pj3q's (the
existing entry point, which keeps the same scratch in cudaMalloc'd context
buffers) at the PJ 3Q tolerance of the other tests.  The second call must not
change the device's free memory.  This file is collected last so that a run
stopping at the first failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

from spider_b200 import _lib, ops, synth

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_pj3q_noalloc_matches_pj3q_twice():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = _lib.load()
    ctx = ops.Context(0)
    rng = np.random.default_rng(20261203)
    shapes = [(40, 36, 33), (32, 32, 32)]          # (nz, ny, nx), a different problem per call
    free_after_first = None
    for call, (nz, ny, nx) in enumerate(shapes):
        vol = synth.blob_phantom(max(nz, ny, nx), 9, sigma=(1.5, 4.0), radius=0.3 * min(nz, ny, nx),
                                 rng=rng)[:nz, :ny, :nx].copy()
        ang = synth.so3_angles(23 + 10 * call, rng)
        ri = float(min(nx, ny, nz) // 2 - 2)
        ref = ops.pj3q(vol, ang, ri, ctx=ctx)      # existing entry point
        dvol = torch.from_numpy(vol).cuda()
        dang = torch.from_numpy(ang).cuda()
        dout = torch.full((ang.shape[0], ny, nx), 7.0, device="cuda")   # stale contents must not leak
        torch.cuda.synchronize()
        if call == 1:
            free_after_first = torch.cuda.mem_get_info()[0]
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        rc = L.spi_pj3q_noalloc(_ptr(dvol), nx, ny, nz, ri, _ptr(dang), ang.shape[0], _ptr(dout), stream)
        assert rc == 0, L.spi_last_error()
        torch.cuda.synchronize()
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free_after_first
        got = dout.cpu().numpy()
        e = synth.rel_l2(got, ref)
        print(f"call {call}: rel-L2 against spi_pj3q {e:.3e}")
        assert e <= TOL
    ctx.close()


def test_pj3q_noalloc_rejects_oversize():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = _lib.load()
    d = torch.zeros(16, device="cuda")
    rc = L.spi_pj3q_noalloc(_ptr(d), 300, 300, 300, 10.0, _ptr(d), 1, _ptr(d), None)
    assert rc == 101
    assert b"limit" in L.spi_last_error()
    rc = L.spi_pj3q_noalloc(_ptr(d), 32, 32, 32, 10.0, _ptr(d), 20000, _ptr(d), None)
    assert rc == 101
