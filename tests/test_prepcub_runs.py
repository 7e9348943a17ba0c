"""PREPCUB run finding (prepcub.f:54-109) as the library does it, by one
interval per x line, against the reference's voxel-by-voxel test: the same
runs over shapes, radii and centres; and the row tasks of the warp forward
projections built from them, in both orders (tests/prepcub_check.cpp, built
with the host C++ compiler)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_prepcub_intervals_match_voxel_loop(tmp_path):
    exe = tmp_path / "prepcub_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe), os.path.join(HERE, "prepcub_check.cpp")], check=True)
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    print(res.stdout)
    assert res.returncode == 0, res.stdout
    assert "561 cases, 0 mismatches" in res.stdout
