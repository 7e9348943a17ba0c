"""Builds the CUDA library ``spider_b200/_lib/libspider_b200.so`` for sm_100a.

The library is compiled in-tree with nvcc (no JIT cache): every ``.cu`` and
``.cpp`` file under ``spider_b200/csrc`` goes into one shared object that
exports the C ABI declared in ``include/spider_b200.h``.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libspider_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = [os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc"), shutil.which("nvcc") or ""]
    for c in cand:
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found: the spider_b200 CUDA library cannot be built")


def _ccbin() -> list[str]:
    for c in ("/usr/bin/g++", shutil.which("g++") or ""):
        if c and os.path.exists(c):
            return ["-ccbin", c]
    return []


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(ROOT, "include", "spider_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    nvcc = _nvcc()
    cuda_home = os.path.dirname(os.path.dirname(nvcc))
    objs = []
    tmpdir = os.path.join(OUT_DIR, "obj")
    os.makedirs(tmpdir, exist_ok=True)
    common = [nvcc, *(_ccbin()), "-std=c++17", "-O3", *ARCH, "-lineinfo", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math", "-I", os.path.join(ROOT, "include")]
    for src in sources():
        obj = os.path.join(tmpdir, os.path.basename(src) + ".o")
        cmd = common + ["-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = common + ["-x", "cu", "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    link = [nvcc, *(_ccbin()), "-shared", *ARCH, "-o", LIB + ".tmp", *objs,
            "-L", os.path.join(cuda_home, "lib64"), "-lcufft", "-Xlinker", "-rpath," + os.path.join(cuda_home, "lib64")]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.run(link, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
