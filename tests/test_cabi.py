"""The C ABI library loads on a machine without a GPU and exports every
entry point include/spider_b200.h declares (no compute calls here)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from spider_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "spider_b200.h")


def declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(spi_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared()
    assert "spi_bp3f" in names and "spi_bp32f" in names and "spi_pj3q" in names and "spi_bpcg" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    L = _lib.load(build_if_missing=True)
    for name in declared():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (spi_\w+)", out))
    assert set(declared()) <= exported
    # the ctypes binding covers every declared function with a signature
    assert set(declared()) == {n for n, _, _ in _lib.SIGNATURES}


def test_library_built_for_sm100a():
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", _lib.LIB_PATH], capture_output=True,
                         text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_kb_table_host_only_matches_oracle():
    import oracle
    L = _lib.load()
    tab = np.zeros(5000, np.float32)
    fl = ctypes.c_float()
    assert L.spi_kb_table(256, tab.ctypes.data_as(ctypes.c_void_p), ctypes.cast(ctypes.byref(fl), ctypes.c_void_p)) == 0
    otab, ofl, _, _ = oracle.kb_table(256)
    assert np.array_equal(tab, otab) and fl.value == ofl
    assert L.spi_kb_table(4, tab.ctypes.data_as(ctypes.c_void_p), None) == 101


def test_errors_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    L = _lib.load()
    h = ctypes.c_void_p()
    rc = L.spi_ctx_create(0, ctypes.byref(h))
    assert rc != 0
    assert L.spi_last_error()
    assert L.spi_ctx_destroy(None) == 0
    gb = ctypes.c_longlong()
    assert L.spi_bp_grid_bytes(256, ctypes.byref(gb)) == 0
    assert gb.value == 257 * 512 * 512 * 16
    assert L.spi_bp_grid_bytes(6, ctypes.byref(gb)) == 101


@pytest.mark.parametrize("n2", [16, 128, 512])
def test_kb_table_window_of_four(n2):
    """The generalised Kaiser-Bessel table is zero for every distance >= 2
    (in fact from ~1.8 on), so of the five ONELINE taps along an axis at most
    four consecutive ones are nonzero; the four-lane insertion kernel relies
    on it (and the library falls back to five lanes otherwise)."""
    from spider_b200 import roofline
    tab, fltb = roofline.kb_table(n2)
    tab = np.asarray(tab)
    assert np.all(tab[int(np.floor(2.0 * fltb)) - 1:] == 0.0)
    first_zero = int(np.argmax(tab == 0.0))
    assert 1.7 < first_zero / fltb < 1.9
