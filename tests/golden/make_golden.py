"""Writes the golden fixtures of tests/golden/ from scipy/numpy only.

kb_table_n2_128.npy : FILLBESSIL's table (fillbessi0.f:88-125) for N2 = 128,
                      evaluated in float64 with scipy.special.i1 and the
                      single-precision index arithmetic of the Fortran.
Run: python tests/golden/make_golden.py
"""
import os

import numpy as np
import scipy.special as sp

HERE = os.path.dirname(os.path.abspath(__file__))


def kb_table(n2):
    f32 = np.float32
    ltab, ln = 4999, 5
    ln2 = ln // 2
    v = f32(ln - 1) / f32(2.0) / f32(n2)
    alpha = f32(6.5)
    aaaa = f32(0.9) * v
    fltb = f32(ltab) / f32(ln2 + 1)
    i = np.arange(ltab + 1)
    s = (i.astype(f32) / fltb) / f32(n2)
    out = np.zeros(ltab + 1, np.float32)
    inside = s <= aaaa
    x = np.sqrt(1.0 - (s[inside].astype(np.float64) / float(aaaa)) ** 2)
    a = float(alpha)
    out[inside] = (np.sqrt(a * x) * sp.i1(a * x) / (np.sqrt(a) * sp.i1(a))).astype(np.float32)
    return out


if __name__ == "__main__":
    np.save(os.path.join(HERE, "kb_table_n2_128.npy"), kb_table(128))
    print("wrote kb_table_n2_128.npy")
