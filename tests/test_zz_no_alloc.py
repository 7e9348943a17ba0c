"""spi_pj3q_noalloc: the PJ 3Q entry point for callers that must not
allocate device memory (a fixed arena or caching allocator owns it, or the
pipeline cannot take cudaMalloc/cudaFree's implicit synchronisation).

It is called through the C ABI with caller-owned device buffers, twice in a
row on fresh data, and its projections are compared with the CPU oracle's
PJ 3Q and with spi_pj3q's (the existing entry point, which keeps the same
scratch in cudaMalloc'd context buffers) at the PJ 3Q tolerance of the other
tests.  The second call must not change the device's free memory.  A fresh
process checks the very first call of a process that has not used the
library yet: under lazy module loading that call may load the library's
device code and its fixed array (the driver's one implicit allocation), and
nothing more.  This file is collected last so that a run stopping at the
first failure has run every other test before it.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle
from spider_b200 import _lib, ops, synth

pytestmark = pytest.mark.gpu

TOL = 1e-5
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SCRATCH_BYTES = 1114112


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_pj3q_noalloc_matches_oracle_and_pj3q_twice():
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
        orc = oracle.pj3q(vol, ang, ri)            # CPU restatement of PJ3Q_N / WPRO_N
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
        e_orc = synth.rel_l2(got, orc)
        e_ref = synth.rel_l2(got, ref)
        print(f"call {call}: rel-L2 against the oracle {e_orc:.3e}, against spi_pj3q {e_ref:.3e}")
        assert e_orc <= TOL
        assert e_ref <= TOL
    ctx.close()


_FRESH = r"""
import ctypes, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from spider_b200 import _lib, synth
torch.cuda.init()
rng = np.random.default_rng(5)
vol = torch.from_numpy(synth.blob_phantom(32, 6, sigma=(1.5, 4.0), radius=9, rng=rng)).cuda()
ang = torch.from_numpy(synth.so3_angles(17, rng)).cuda()
out = torch.empty((17, 32, 32), device="cuda")
L = _lib.load()
p = lambda t: ctypes.c_void_p(t.data_ptr())
frees = [torch.cuda.mem_get_info()[0]]
for _ in range(2):
    rc = L.spi_pj3q_noalloc(p(vol), 32, 32, 32, 14.0, p(ang), 17, p(out), None)
    assert rc == 0, L.spi_last_error()
    torch.cuda.synchronize()
    frees.append(torch.cuda.mem_get_info()[0])
print(frees[0] - frees[1], frees[1] - frees[2])
"""


def test_pj3q_noalloc_first_call_in_fresh_process():
    """In a process that has not used the library, the first call may load
    the module (code plus the fixed array, rounded up to the driver's 2 MiB
    pages); the second call allocates nothing."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    r = subprocess.run([sys.executable, "-c", _FRESH, ROOT], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    first, second = (int(v) for v in r.stdout.split()[-2:])
    print(f"free memory taken by the first call {first} bytes, by the second {second}")
    assert second == 0
    assert 0 <= first <= SCRATCH_BYTES + (8 << 20)


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
