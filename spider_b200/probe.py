"""Small, self-contained workloads of each kernel, for profilers (ncu).

    python -m spider_b200.probe insert --nx 192 --nimg 64 [--reps 3] [--bf16]
    python -m spider_b200.probe pj3q --nx 128 --nang 64
    python -m spider_b200.probe normalcg --nx 128 --nang 512 --iters 2
    python -m spider_b200.probe bpcg --n 64 --nang 512 --iters 2 [--prec fp64|mixed|mixed64|fast|fp32]
                                 [--interp linear|fbs]

Each run launches the kernel a few times on random data so that a profiler
can skip the first launch (`-s 1`) and capture one steady-state launch.
"""
from __future__ import annotations

import argparse
import sys

import numpy as np


def main(argv=None) -> int:
    p = argparse.ArgumentParser()
    p.add_argument("what", choices=["insert", "pj3q", "bpcg", "normalcg"])
    p.add_argument("--nx", type=int, default=192)
    p.add_argument("--n", type=int, default=64)
    p.add_argument("--nimg", type=int, default=64)
    p.add_argument("--nang", type=int, default=64)
    p.add_argument("--reps", type=int, default=3)
    p.add_argument("--iters", type=int, default=2)
    p.add_argument("--bf16", action="store_true")
    p.add_argument("--prec", choices=["fp64", "mixed", "mixed64", "fast", "fp32"], default="fp64")
    p.add_argument("--interp", choices=["linear", "fbs"], default="linear")
    a = p.parse_args(argv)
    import torch

    from . import ops, synth
    ctx = ops.Context(0)
    rng = np.random.default_rng(0)
    if a.what == "insert":
        imgs = torch.randn(a.nimg, a.nx, a.nx, device="cuda")
        ctx.bp_open(a.nx, 2, bf16=a.bf16)
        for _ in range(a.reps):
            ctx.bp_insert(imgs, synth.so3_angles(a.nimg, rng), synth.half_mask(a.nimg, rng))
        ctx.bp_close()
    elif a.what == "pj3q":
        vol = torch.randn(a.nx, a.nx, a.nx, device="cuda")
        for _ in range(a.reps):
            ops.pj3q(vol, synth.so3_angles(a.nang, rng), ctx=ctx)
    elif a.what == "normalcg":
        from . import autograd
        plan = autograd.PJ3QPlan((a.nx, a.nx, a.nx), synth.so3_angles(a.nang, rng), ctx=ctx)
        b = torch.randn(a.nang, a.nx, a.nx, device="cuda")
        for _ in range(a.reps):
            autograd.NormalCG(plan, 1e-3, a.iters, graph=False).solve(plan.adjoint(b))
        plan.close()
    else:
        projs = rng.standard_normal((a.nang, a.n, a.n)).astype(np.float32)
        prec = {"fp64": True, "fp32": False}.get(a.prec, a.prec)
        ops.bpcg(projs, synth.so3_angles(a.nang, rng), a.n / 2 - 3, errm=0.0, maxit=a.iters, mode=1,
                 lam=1e-3, ctx=ctx, fp64=prec, interp=a.interp)
    torch.cuda.synchronize()
    print(f"ok {a.what}: {ctx.launches} kernel launches")
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
