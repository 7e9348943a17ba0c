#!/usr/bin/env python
"""Benchmark: SPIDER BP 32F Fourier gridding back-projection at 256^3.

Metric: images back-projected per second at 256^3 (BP 32F: two half-set
grids, FP32 spectra, FP32 vector-atomic accumulation).  A step is one
persistent insertion launch over one chunk of 4,096 images (stage + batched
2D FFT + ONELINE insertion).  Inputs are synthetic: PJ 3Q projections of a
200-blob 256^3 phantom (sigma 1.5-10 voxels) at uniform SO(3) angles with
additive noise at SNR 0.05, and a Bernoulli(1/2) half-set mask.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank inserts its own chunks into private grids
(weak scaling); the grids are summed with one NCCL all-reduce before the
volumes are finished, the exchange the reference does with MPI_ALLREDUCE.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "images backprojected/s at 256³"
UNIT = "images/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--nx", type=int, default=256)
    p.add_argument("--chunk", type=int, default=4096)
    p.add_argument("--bf16", action="store_true", help="BF16 spectra (reduced precision variant)")
    p.add_argument("--cpu-seconds", type=float, default=15.0, help="target CPU-baseline sample time")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cg", action="store_true", help="skip the BP CG s/iter measurement")
    p.add_argument("--workload", choices=["bp32f", "multiclass", "kernel"], default="bp32f",
                   help="multiclass: eight classes of box 96-256, 80,000 images (separate JSON line); "
                        "kernel: a small run of one kernel family for profilers (--kernel)")
    p.add_argument("--kernel", choices=["insert", "pj3q", "bpcg", "normalcg", "fslice"], default="insert",
                   help="--workload kernel: insert (BP 32F insertion of --nimg images at --nx, --reps launches), "
                        "pj3q (--nang projections of an --nx^3 volume), bpcg (--iters BP CG iterations at "
                        "--n^3 with --nang images, --prec, --interp), normalcg (PJ 3Q normal-equation CG), "
                        "fslice (FourierSlice normal-equation CG)")
    p.add_argument("--nimg", type=int, default=64)
    p.add_argument("--nang", type=int, default=64)
    p.add_argument("--n", type=int, default=64)
    p.add_argument("--reps", type=int, default=3)
    p.add_argument("--iters", type=int, default=2)
    p.add_argument("--prec", choices=["fp64", "mixed", "mixed64", "fast", "fp32"], default="fp64")
    p.add_argument("--interp", choices=["linear", "fbs"], default="linear")
    p.add_argument("--mc-images", type=int, default=80000)
    p.add_argument("--no-mc", action="store_true", help="skip the multi-class measurement")
    p.add_argument("--no-config5", action="store_true",
                   help="skip the BF16 / 8,192-image-step run and the 256^3 FourierSlice CG")
    p.add_argument("--cg-n", type=int, default=128)
    p.add_argument("--cg-nang", type=int, default=10000)
    p.add_argument("--cg-iters", type=int, default=6)
    p.add_argument("--check-images", type=int, default=8192,
                   help="images of the FP64-oracle check of the 256^3 volumes (0 = skip)")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_per_image(kernel):
    """DRAM bytes per image of the insert kernel and the build they were
    measured on, from the committed ncu summary (None, None if absent)."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_traffic.txt")
    val, where = None, None
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_image"):
                    val = float(line.split("=")[1].split()[0])
                elif line.startswith("measured_at"):
                    where = line.split("=", 1)[1].strip()
    except Exception:
        pass
    return val, where


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(mhz)) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}


# ------------------------------------------------------------------ data
def make_phantom_gpu(nx, nblobs, sigma, amp, rng, device):
    """Sum of isotropic Gaussian blobs as one separable contraction."""
    import torch
    radius = 0.375 * nx
    cs, ss, aa = [], [], []
    for _ in range(nblobs):
        while True:
            p = rng.uniform(-radius, radius, 3)
            if p @ p <= radius * radius:
                break
        cs.append(p)
        ss.append(rng.uniform(*sigma))
        aa.append(rng.uniform(*amp))
    g = np.arange(nx, dtype=np.float64) - nx // 2
    c = np.array(cs)
    s2 = 2.0 * np.array(ss)[:, None] ** 2
    ex = np.exp(-(g[None, :] - c[:, 0:1]) ** 2 / s2) * np.array(aa)[:, None]
    ey = np.exp(-(g[None, :] - c[:, 1:2]) ** 2 / s2)
    ez = np.exp(-(g[None, :] - c[:, 2:3]) ** 2 / s2)
    tx, ty, tz = (torch.tensor(v, dtype=torch.float32, device=device) for v in (ex, ey, ez))
    yx = (ty[:, :, None] * tx[:, None, :]).reshape(nblobs, nx * nx)
    return (tz.t() @ yx).reshape(nx, nx, nx).contiguous()


def make_chunk(ctx, vol, angles, snr, gen):
    import torch
    from spider_b200 import ops
    pr = ops.pj3q(vol, angles, ctx=ctx)                    # [n, nx, nx] on device
    v = pr.var(dim=(1, 2), keepdim=True)
    noise = torch.randn(pr.shape, device=pr.device, generator=gen) * torch.sqrt(v / snr)
    return (pr + noise).contiguous()


# ------------------------------------------------------------------ arms
def cpu_baseline(nx, seconds, imgs_host, angles, half):
    """The oracle (CPU restatement of bp32f.f / oneline.f with the reference's
    OpenMP row striping) inserting a bounded sample on all host cores."""
    import oracle
    nthreads = os.cpu_count() or 1
    sess = oracle.BpSession(nx)            # grids allocated and zeroed once, as BP32FQ does
    # calibrate on a few images, then size the sample to ~`seconds`
    t0 = time.perf_counter()
    sess.insert(imgs_host[:4], angles[:4], half[:4], nthreads=nthreads)
    per = (time.perf_counter() - t0) / 4
    want = int(max(4, seconds / max(per, 1e-6)))
    n, dt = 0, 0.0
    while n < want:            # the pool of distinct images is reused in passes
        k = min(len(imgs_host), want - n)
        t0 = time.perf_counter()
        sess.insert(imgs_host[:k], angles[:k], half[:k], nthreads=nthreads)
        dt += time.perf_counter() - t0
        n += k
    sess.close()
    return {"value": n / dt, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"{n} images at {nx}^3 (BP 32F per-image work: PADD2 + FFT + ONELINE, FP32, "
                      f"the reference's OpenMP row striping), {dt:.1f} s"}


def fp64_check(ctx, nx, chunks, angles, halves, nimg, bf16):
    """Relative L2 of the three BP 32F volumes against the FP64 oracle
    (owner-computes schedule on all host cores) on `nimg` of the bench's
    images (the two resident chunks with the angles of the first two steps),
    for the compensated accumulation the bench times and for plain FP32
    atomics."""
    import oracle
    from spider_b200 import synth
    per = [min(nimg // 2, int(c.shape[0])) for c in chunks[:2]]
    imgs = [chunks[k][:per[k]] for k in range(2)]
    ang = np.concatenate([angles[k][:per[k]] for k in range(2)])
    half = np.concatenate([halves[k][:per[k]] for k in range(2)])
    gpu = {}
    for name, comp in (("compensated", True), ("plain", False)):
        ctx.set_accumulation(comp)
        ctx.bp_open(nx, 2, bf16=bf16)
        for k in range(2):
            ctx.bp_insert(imgs[k], angles[k][:per[k]], halves[k][:per[k]])
        o = ctx.bp_finish(("all", "1", "2"))
        ctx.bp_close()
        gpu[name] = (o["all"], o["1"], o["2"])
    ctx.set_accumulation(True)
    host = np.concatenate([t.cpu().numpy() for t in imgs])
    t0 = time.perf_counter()
    ref = oracle.bp32f(host, ang, half, prec=1)
    dt = time.perf_counter() - t0
    out = {"images": int(host.shape[0]), "oracle_s": dt, "oracle_threads": os.cpu_count()}
    for name, vols in gpu.items():
        out[name] = {k: synth.rel_l2(a, b) for k, a, b in zip(("all", "first", "second"), vols, ref)}
    out["fsc_nyquist_compensated"] = float(synth.fsc(gpu["compensated"][0], ref[0])[nx // 2])
    return out, ref


def config5_measure(args, ctx, stream, chunks, angles, halves, ref, steps=12, cg_iters=30):
    """Configuration 5's reduced-precision form at 256^3: BP 32F with BF16
    spectra, 8,192-image steps (the two resident 4,096-image chunks, new
    angles every step), `steps` steps timed on the library stream (~98k
    images); its volumes for the FP64-checked images against the FP64 oracle;
    and a FourierSlice CG at 256^3 on those 8,192 images, `cg_iters`
    iterations replayed as a CUDA graph (FP64 normal operator and vectors)
    against the same iterations launched op by op."""
    import torch
    from spider_b200 import autograd, synth
    nx = int(chunks[0].shape[-1])
    imgs = torch.cat([chunks[0], chunks[1]]).contiguous()
    n8 = int(imgs.shape[0])
    rng = np.random.default_rng(5005)
    out = {"images_per_step": n8, "steps": steps, "spectra": "bf16"}
    ctx.bp_open(nx, 2, bf16=True)
    ctx.bp_autotune()
    ctx.bp_insert(imgs, synth.so3_angles(n8, rng), synth.half_mask(n8, rng))   # warm-up
    angs = [synth.so3_angles(n8, rng) for _ in range(steps)]
    hs = [synth.half_mask(n8, rng) for _ in range(steps)]
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(steps):
        ctx.bp_insert(imgs, angs[i], hs[i])
    e1.record(stream)
    e1.synchronize()
    ctx.bp_close()
    out["images_per_s"] = n8 * steps / (e0.elapsed_time(e1) / 1e3)
    if ref is not None:
        per = [min(args.check_images // 2, int(c.shape[0])) for c in chunks[:2]]
        ctx.bp_open(nx, 2, bf16=True)
        for k in range(2):
            ctx.bp_insert(chunks[k][:per[k]], angles[k][:per[k]], halves[k][:per[k]])
        o = ctx.bp_finish(("all", "1", "2"))
        ctx.bp_close()
        out["rel_l2_vs_fp64"] = {k: synth.rel_l2(a, b) for k, a, b in
                                 zip(("all", "first", "second"), (o["all"], o["1"], o["2"]), ref)}
        out["fsc_nyquist_vs_fp64"] = float(synth.fsc(o["all"], ref[0])[nx // 2])
    # FourierSlice CG at 256^3
    ang = np.concatenate([angles[0][:int(chunks[0].shape[0])], angles[1][:int(chunks[1].shape[0])]])
    plan = autograd.FourierSlicePlan(nx, ang, ctx=ctx)
    b = plan.stage(imgs)
    rhs = plan.adjoint64(b)
    del b
    cg = {"images": n8, "iterations": cg_iters, "lambda": 1e-3}
    for name, graph, iters in (("graph", True, cg_iters), ("plain", False, 3)):
        s1 = autograd.NormalCG(plan, 1e-3, 1, graph=graph)
        sk = autograd.NormalCG(plan, 1e-3, iters, graph=graph)
        t = []
        for sv in (s1, sk):
            sv.solve(rhs)                          # warm-up (and graph capture)
            e0.record()
            sv.solve(rhs)
            e1.record()
            e1.synchronize()
            t.append(e0.elapsed_time(e1) / 1e3)
        cg[f"{name}_s_per_iter"] = (t[1] - t[0]) / (iters - 1)
        cg[f"{name}_solve_s"] = t[1]
        del s1, sk
    plan.close()
    out["fourier_cg"] = cg
    return out


def cg_measure(args, ctx, stream, rank, world):
    """BP CG seconds per iteration (configuration: 128^3, 10,000 images of a
    50-blob phantom at SNR 0.3, lambda 1e-3, linear interpolation).

    Each form runs the solver twice, with 1 and with 1 + K iterations, and
    the difference of the two device-timed calls over K is the cost of one
    iteration (setup, image upload and the initial back-projection cancel).
    `value` is the library's default form, FP64 CG vectors with 47-bit
    fixed-point projections (mode 2), each iteration replayed as a CUDA graph.
    The other forms are reported beside it.  Accuracy of every form is stated
    against the FP64 oracle on a fixed ill-conditioned check case (32^3, 120
    images, 12 iterations, lambda 0.5)."""
    import torch
    from spider_b200 import ops, synth
    n, nang, K = args.cg_n, args.cg_nang, args.cg_iters
    dev = torch.device("cuda", torch.cuda.current_device())
    rng = np.random.default_rng(1003 + 7919 * rank)
    gen = torch.Generator(device=dev)
    gen.manual_seed(1003 + rank)
    vol = make_phantom_gpu(n, 50, (2.0, 8.0), (0.5, 1.0), rng, dev)
    ang = synth.so3_angles(nang, rng)
    projs = make_chunk(ctx, vol, ang, 0.3, gen).cpu().numpy()
    del vol
    ri = float(n // 2 - 3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def timed(p, a, iters, fp64, interp="linear", r=ri):
        e0.record(stream)
        v, log = ops.bpcg(p, a, r, errm=0.0, chim=0.0, maxit=iters, mode=1, lam=1e-3, ctx=ctx, fp64=fp64,
                          interp=interp)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3, v, log

    def per_iter(p, a, fp64, k, interp="linear", r=ri):
        timed(p, a, 1, fp64, interp, r)          # warm-up (plans, buffers)
        t1, _, _ = timed(p, a, 1, fp64, interp, r)
        tk, v, _ = timed(p, a, 1 + k, fp64, interp, r)
        return (tk - t1) / k, v

    out, vols = {}, {}
    for name, fp64, graph in (("mixed_graph", "mixed", True), ("fp64_graph", True, True),
                              ("fp64_plain", True, False), ("fp32_graph", False, True),
                              ("fast_graph", "fast", True), ("mixed64_graph", "mixed64", True)):
        if not graph:
            os.environ["SPI_CG_NOGRAPH"] = "1"
        try:
            out[name], vols[name] = per_iter(projs, ang, fp64, K)
        finally:
            os.environ.pop("SPI_CG_NOGRAPH", None)

    def rel(name):
        return synth.rel_l2(vols[name], vols["fp64_graph"])

    # roofline of the iteration (both operators): per image, A reads each
    # sphere voxel and read-modify-writes a projection pixel, A^T reads the
    # pixel table and read-modify-writes the voxel, 2 x (4 + 8) bytes per
    # sphere voxel, plus the 4 n^2 bytes of the image
    c = n // 2 + 1
    g = np.arange(1, n + 1) - c
    v_sphere = int(((g[:, None, None] ** 2 + g[None, :, None] ** 2 + g[None, None, :] ** 2) <= ri * ri).sum())
    bytes_iter = nang * (2 * 12 * v_sphere + 4 * n * n)
    peak, peak_kind = measured_peak()
    achieved = bytes_iter / out["mixed_graph"] / 1e9
    res = {"metric": "BP CG s/iter", "unit": "s/iter", "value": out["mixed_graph"],
           "form": "mixed_graph: FP64 vectors, 47-bit fixed-point projections, FP32 PROJT (mode 2, the default)",
           "fp64_s_per_iter": out["fp64_graph"], "plain_gpu_s_per_iter": out["fp64_plain"],
           "fp32_vectors_s_per_iter": out["fp32_graph"], "fast_s_per_iter": out["fast_graph"],
           "mixed64_s_per_iter": out["mixed64_graph"],
           "rel_err_vs_fp64_form": {k: rel(k) for k in ("mixed_graph", "fast_graph", "mixed64_graph", "fp32_graph")},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "peak_kind": peak_kind, "algorithmic_bytes_per_iter": bytes_iter,
                        "sphere_voxels": v_sphere,
                        "note": "per image 2 x (4 + 8) B per sphere voxel + 4 n^2 B; the operators' tables and "
                                "volumes stay in L2, so this is an algorithmic, not a DRAM, figure"},
           "config": {"n": n, "images": nang, "lambda": 1e-3, "mode": 1, "iterations_timed": K,
                      "phantom": "50 Gaussian blobs, sigma 2-8, SNR 0.3, uniform SO(3)"}}
    res["check_vs_fp64_oracle"] = cg_oracle_check(ctx)
    res["n256"] = cg_256_measure(args, ctx, stream, rank)
    res["differentiable_cg"] = autograd_cg_measure(ctx, projs, ang, ri, K)
    res["differentiable_cg_fourier"] = fourier_cg_measure(ctx, projs, ang, K)
    # the 'F' answer (FBS interpolation), default precision mode: informational
    res["fbs_s_per_iter"], _ = per_iter(projs, ang, "mixed", K, "fbs")
    if rank == 0 and world == 1 and not args.no_cpu:
        res["cpu_baseline"] = cg_cpu_baseline(projs, ang, ri, n)
    return res


def cg_oracle_check(ctx):
    """Relative error of each BP CG form against the FP64 oracle on a fixed
    ill-conditioned case: 32^3, 120 PJ 3Q projections of a 12-blob phantom at
    SNR 1, radius 13, lambda 0.5, 12 iterations (where the reference's REAL CG
    drifts ~4e-2 from the exact iteration)."""
    import oracle
    from spider_b200 import ops, synth
    rng = np.random.default_rng(4242)
    n, nang = 32, 120
    vol = synth.blob_phantom(n, 12, sigma=(1.5, 4.0), radius=0.35 * n, rng=rng)
    ang = synth.so3_angles(nang, rng)
    pr = synth.add_noise(oracle.pj3q(vol, ang), 1.0, rng)
    kw = dict(errm=1e-7, chim=0.0, maxit=12, mode=1, lam=0.5)
    ref, _, _, _ = oracle.bpcg(pr, ang, 13.0, prec=1, **kw)
    out = {}
    for name, fp64 in (("mixed", "mixed"), ("fast", "fast"), ("mixed64", "mixed64"), ("fp64", True),
                       ("fp32", False)):
        v, _ = ops.bpcg(pr, ang, 13.0, ctx=ctx, fp64=fp64, **kw)
        out[name] = synth.rel_l2(v, ref)
    ref32, _, _, _ = oracle.bpcg(pr, ang, 13.0, prec=0, **kw)
    out["fp32_oracle"] = synth.rel_l2(ref32, ref)
    return out


def cg_256_measure(args, ctx, stream, rank, nang=10000, k=2):
    """BP CG at 256^3 (configuration 5's box) in the default form: 10,000 PJ 3Q
    projections of a 200-blob phantom at SNR 0.05, lambda 1e-3, seconds per
    iteration from a 1- and a (1 + k)-iteration solve."""
    import torch
    from spider_b200 import ops, synth
    n = 256
    dev = torch.device("cuda", torch.cuda.current_device())
    rng = np.random.default_rng(1105 + rank)
    gen = torch.Generator(device=dev)
    gen.manual_seed(1105 + rank)
    vol = make_phantom_gpu(n, 200, (1.5, 10.0), (0.5, 1.0), rng, dev)
    ang = synth.so3_angles(nang, rng)
    projs = torch.cat([make_chunk(ctx, vol, ang[a:a + 2500], 0.05, gen) for a in range(0, nang, 2500)]).cpu().numpy()
    del vol
    ri = float(n // 2 - 3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ts = []
    for iters in (1, 1, 1 + k):
        e0.record(stream)
        ops.bpcg(projs, ang, ri, errm=0.0, chim=0.0, maxit=iters, mode=1, lam=1e-3, ctx=ctx, fp64="mixed")
        e1.record(stream)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1) / 1e3)
    return {"s_per_iter": (ts[2] - ts[1]) / k, "images": nang, "form": "mixed_graph (mode 2)",
            "solve_1_iter_s": ts[1], "iterations_timed": k}


def fourier_cg_measure(ctx, projs, ang, K, lam=1e-3, check_images=1000, check_iters=3):
    """The differentiable reconstruction on the FourierSlice pair (E = central
    slice extraction, E^T = ONELINE's insertion without weights): CG on
    (E^T E + lam I) x = E^T b from the staged image spectra, one iteration
    (the fused normal operator + FP64 dot products) replayed as a CUDA graph
    against the same iteration launched op by op.  rel_err_vs_fp64_oracle: the
    graph-captured CG after `check_iters` iterations against an FP64 CG on
    the oracle's pair, on the first `check_images` images."""
    import oracle
    import torch
    from spider_b200 import autograd
    n = projs.shape[1]
    imgs = torch.from_numpy(projs).cuda()
    plan = autograd.FourierSlicePlan(n, ang, ctx=ctx)
    b = plan.stage(imgs)
    rhs = plan.adjoint64(b)
    rhs32 = plan.adjoint(b)
    del b
    out = {}
    for name, graph, op64 in (("graph_s_per_iter", True, True), ("plain_s_per_iter", False, True),
                              ("fp32_operator_graph_s_per_iter", True, False)):
        times = []
        for iters in (1, 1 + K):
            solver = autograd.NormalCG(plan, lam, iters, graph=graph, fp64_operator=op64)
            r = rhs if op64 else rhs32
            solver.solve(r)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            solver.solve(r)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
        out[name] = (times[1] - times[0]) / K
    plan.close()
    del rhs, rhs32
    # FP64 check on a subset
    sub = autograd.FourierSlicePlan(n, ang[:check_images], ctx=ctx)
    bs = sub.stage(imgs[:check_images].contiguous())
    x = autograd.NormalCG(sub, lam, check_iters, graph=True).solve(sub.adjoint64(bs)).cpu().numpy().astype(np.float64)
    bh = bs.cpu().numpy().astype(np.float64)
    sub.close()
    bh = bh[..., 0] + 1j * bh[..., 1]
    a = ang[:check_images]
    t0 = time.perf_counter()
    r = oracle.fslice_insert(bh, a)
    xr = np.zeros_like(r)
    p = r.copy()
    rs = np.vdot(r, r).real
    for _ in range(check_iters):
        ap = oracle.fslice_insert(oracle.fslice_extract(p, a), a) + lam * p
        alpha = rs / np.vdot(p, ap).real
        xr += alpha * p
        r -= alpha * ap
        rs_new = np.vdot(r, r).real
        p = r + (rs_new / rs) * p
        rs = rs_new
    xg = x[..., 0] + 1j * x[..., 1]
    out["rel_err_vs_fp64_oracle"] = float(np.linalg.norm(xg - xr) / np.linalg.norm(xr))
    out["check"] = f"{check_images} images, {check_iters} iterations, oracle FP64 CG {time.perf_counter() - t0:.1f} s"
    out["operator"] = "FourierSlice (central-slice extraction) and ONELINE insertion without weights, fused " \
                      "E^T E + lam I with FP64 sums and scatter (FP32 table weights), FP64 CG vectors; " \
                      "fp32_operator: the same pass with FP32 sums"
    return out


def autograd_cg_measure(ctx, projs, ang, ri, K, lam=1e-3):
    """The differentiable reconstruction of configuration 3: CG on
    (A^T A + lam I) x = A^T b with A = PJ 3Q through the capturable operator
    pair (spider_b200.autograd.NormalCG), one iteration replayed as a CUDA
    graph against the same iteration launched op by op; seconds per
    iteration from the difference of a 1- and a (1+K)-iteration solve."""
    import torch
    from spider_b200 import autograd
    n = projs.shape[1]
    plan = autograd.PJ3QPlan((n, n, n), ang, ri, ctx=ctx)
    b = torch.from_numpy(projs).cuda()
    rhs = plan.adjoint(b)
    out = {}
    for name, graph in (("graph_s_per_iter", True), ("plain_s_per_iter", False)):
        times = []
        for iters in (1, 1 + K):
            solver = autograd.NormalCG(plan, lam, iters, graph=graph)
            solver.solve(rhs)                   # warm-up (and graph capture)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            solver.solve(rhs)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
        out[name] = (times[1] - times[0]) / K
    plan.close()
    out["operator"] = "PJ 3Q and its exact adjoint (trilinear), FP32, FP64 dot products"
    return out


def cg_cpu_baseline(projs, ang, ri, n, sample=500):
    """The oracle's FP32 BP CG (the reference's loop structure, OpenMP over
    voxel runs) on a 500-image subset: one iteration's cost from the difference
    of a 1- and a 2-iteration solve, extrapolated linearly to all images
    (both operators are linear in the image count)."""
    import oracle
    nthreads = os.cpu_count() or 1
    p, a = projs[:sample], ang[:sample]
    t0 = time.perf_counter()
    oracle.bpcg(p, a, ri, errm=0.0, chim=0.0, maxit=1, mode=1, lam=1e-3, prec=0, nthreads=nthreads)
    t1 = time.perf_counter() - t0
    t0 = time.perf_counter()
    oracle.bpcg(p, a, ri, errm=0.0, chim=0.0, maxit=2, mode=1, lam=1e-3, prec=0, nthreads=nthreads)
    t2 = time.perf_counter() - t0
    per = max(t2 - t1, 1e-9) * len(projs) / sample
    return {"value": per, "unit": "s/iter", "cores": nthreads, "kind": "port",
            "sample": f"{sample} of {len(projs)} images at {n}^3, 1 iteration, extrapolated linearly "
                      f"({t1:.1f} s + {t2:.1f} s of CPU solves)"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    import oracle
    nx = args.nx
    rng = np.random.default_rng(1005)
    from spider_b200 import synth
    nthreads = os.cpu_count() or 1
    pool = 256
    imgs = rng.standard_normal((pool, nx, nx)).astype(np.float32)
    ang = synth.so3_angles(pool, rng)
    half = synth.half_mask(pool, rng)
    sess = oracle.BpSession(nx)
    # calibrate: size each step to ~ 8 s of CPU work
    t0 = time.perf_counter()
    sess.insert(imgs[:4], ang[:4], half[:4], nthreads=nthreads)
    per = (time.perf_counter() - t0) / 4
    per_step = int(max(2, min(pool, 8.0 / max(per, 1e-6))))
    for _ in range(min(args.warmup, 1)):
        sess.insert(imgs[:per_step], ang[:per_step], half[:per_step], nthreads=nthreads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sess.insert(imgs[:per_step], ang[:per_step], half[:per_step], nthreads=nthreads)
    dt = time.perf_counter() - t0
    sess.close()
    value = per_step * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"BP 32F insertion at {nx}^3, {per_step} images per step (CPU sample)",
                   "nx": nx},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                         "sample": f"{per_step} images per step x {args.steps} steps; the reference is "
                                   "Fortran+FFTW and cannot be built here, its C++ restatement is timed"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    from spider_b200 import ops, roofline, synth

    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device(f"cuda:{local}")
    nx, chunk = args.nx, args.chunk
    ctx = ops.Context(local)
    L = ctx._L
    stream = torch.cuda.ExternalStream(L.spi_ctx_stream(ctx.handle), device=dev)

    # ---- synthetic data (config: 200 blobs, sigma 1.5-10, SNR 0.05)
    rng = np.random.default_rng(1005 + 7919 * rank)
    gen = torch.Generator(device=dev)
    gen.manual_seed(1005 + rank)
    vol = make_phantom_gpu(nx, 200, (1.5, 10.0), (0.5, 1.0), rng, dev)
    nsteps = args.warmup + args.steps
    angles = [synth.so3_angles(chunk, rng) for _ in range(nsteps)]
    halves = [synth.half_mask(chunk, rng) for _ in range(nsteps)]
    chunks = [make_chunk(ctx, vol, angles[i], 0.05, gen) for i in range(2)]
    del vol
    torch.cuda.synchronize()

    # ---- grids: library-owned at N=1, caller-owned (for the all-reduce) at N>1
    grids = None
    if world > 1:
        gb = ctypes.c_longlong()
        L.spi_bp_grid_bytes(nx, ctypes.byref(gb))
        # spi_bp_open zeroes attached grids on the library stream, so no fill on torch's
        grids = [torch.empty(gb.value // 4, dtype=torch.float32, device=dev) for _ in range(2)]
        ops.check(L.spi_bp_attach_grids(ctx.handle, ctypes.c_void_p(grids[0].data_ptr()),
                                        ctypes.c_void_p(grids[1].data_ptr())))
    ctx.bp_open(nx, 2, bf16=args.bf16)
    launch_cfg = ctx.bp_autotune()          # kernel variant and launch shape, timed on this GPU

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    for i in range(args.warmup):
        ctx.bp_insert(chunks[i % 2], angles[i], halves[i])
    torch.cuda.synchronize()
    L.spi_ctx_set_timing(ctx.handle, 1)
    ms = (ctypes.c_double * 9)()
    cnt = (ctypes.c_longlong * 9)()
    L.spi_ctx_timing(ctx.handle, ms, cnt)   # reset
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = ctx.launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed_steps")
    e0.record(stream)
    for i in range(args.warmup, nsteps):
        ctx.bp_insert(chunks[i % 2], angles[i], halves[i])
    e1.record(stream)
    e1.synchronize()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    launches = ctx.launches - launches0
    t_ms = e0.elapsed_time(e1)
    L.spi_ctx_timing(ctx.handle, ms, cnt)
    insert_ms = ms[2]
    n_insert = max(int(cnt[2]), 1)
    fold_ms = ms[8]
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([t_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_ms = float(t.item())
    value = world * chunk * args.steps / (t_ms / 1e3)

    # ---- exchange + finish (per reconstruction)
    torch.cuda.synchronize()
    f0 = time.perf_counter()
    if world > 1:
        import torch.distributed as dist
        ctx.bp_flush()                       # grids hold the complete sums
        for g in grids:
            dist.all_reduce(g)
        torch.cuda.synchronize()
    outs = ctx.bp_finish(("all", "1", "2"), device=True)
    torch.cuda.synchronize()
    finish_ms = (time.perf_counter() - f0) * 1e3
    L.spi_ctx_timing(ctx.handle, ms, cnt)
    finish_phase_ms = {"symplane0": ms[3], "nrmw2": ms[4], "fft3d": ms[5], "windkb2a": ms[6]}
    del outs

    # ---- roofline of the insert kernel
    tab, fltb = roofline.kb_table(2 * nx)
    dms = []
    from spider_b200._lib import load as _load  # noqa: F401
    for a in angles[args.warmup][:16]:
        dms.append(_cang_host(a))
    taps = roofline.mean_taps(nx, np.array(dms), tab, fltb)
    bytes_per_img = roofline.BYTES_PER_TAP * taps + roofline.spectrum_bytes(nx, args.bf16)
    # one insert launch per FFT sub-batch: achieved = all images' algorithmic
    # bytes over the summed launch durations (CUDA events around each launch)
    achieved = bytes_per_img * chunk * args.steps / (insert_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    tpi, tpi_at = traffic_per_image(launch_cfg["kernel"])
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": (tpi * chunk * args.steps / n_insert) if tpi else None,
            "traffic_source": f"ncu DRAM bytes per image x images per launch, {tpi_at}" if tpi else None,
            "kernel": launch_cfg["kernel"], "launch": launch_cfg, "peak_kind": peak_kind,
            "algorithmic_bytes_per_image": bytes_per_img, "taps_per_image": taps,
            "launch_ms": insert_ms / n_insert, "launches": n_insert,
            "images_per_launch": chunk * args.steps / n_insert}

    # ---- e2e through the C ABI with host buffers (pinned), H2D/D2H inside
    e2e = None
    if not args.no_e2e:
        host_chunks = [c.cpu().pin_memory() for c in chunks]
        # per-phase timing events on the library stream were measured to
        # serialise the uploads with the compute; the e2e path runs without them
        L.spi_ctx_set_timing(ctx.handle, 0)
        if world > 1:   # caller-owned grids are attached to a closed context
            ctx.bp_close()
            ops.check(L.spi_bp_attach_grids(ctx.handle, ctypes.c_void_p(grids[0].data_ptr()),
                                            ctypes.c_void_p(grids[1].data_ptr())))
        hvol = [torch.empty((nx, nx, nx), dtype=torch.float32).pin_memory() for _ in range(3)]
        # this box's pinned host-to-device bandwidth (the e2e rate depends on it)
        probe = torch.empty_like(host_chunks[0], device=dev)
        probe.copy_(host_chunks[0], non_blocking=True)
        torch.cuda.synchronize()
        h0 = torch.cuda.Event(enable_timing=True)
        h1 = torch.cuda.Event(enable_timing=True)
        h0.record()
        probe.copy_(host_chunks[0], non_blocking=True)
        h1.record()
        h1.synchronize()
        h2d_gbs = host_chunks[0].numel() * 4 / (h0.elapsed_time(h1) / 1e3) / 1e9
        del probe
        # reopening at the same size zeroes the grids and keeps every buffer
        ctx.bp_open(nx, 2, bf16=args.bf16)
        ctx.bp_autotune()                   # cached choice
        for i in range(min(args.warmup, 1)):  # first host-image call (copy-stream events)
            ops.check(L.spi_bp_insert(ctx.handle, ctypes.c_void_p(host_chunks[i % 2].data_ptr()), chunk,
                                      angles[i].ctypes.data_as(ctypes.c_void_p),
                                      halves[i].ctypes.data_as(ctypes.c_void_p), 0))

        def e2e_pass():
            ctx.bp_open(nx, 2, bf16=args.bf16)
            ctx.bp_autotune()
            barrier()
            torch.cuda.synchronize()
            th0 = time.perf_counter()
            e0.record(stream)
            for i in range(args.warmup, nsteps):
                ops.check(L.spi_bp_insert(ctx.handle, ctypes.c_void_p(host_chunks[i % 2].data_ptr()), chunk,
                                          angles[i].ctypes.data_as(ctypes.c_void_p),
                                          halves[i].ctypes.data_as(ctypes.c_void_p), 0))
            if world > 1:
                import torch.distributed as dist
                ctx.bp_flush()             # the last insertions and folds are done on the library stream
                for g in grids:
                    dist.all_reduce(g)
                torch.cuda.synchronize()
            ops.check(L.spi_bp_finish(ctx.handle, ctypes.c_void_p(hvol[0].data_ptr()),
                                      ctypes.c_void_p(hvol[1].data_ptr()), ctypes.c_void_p(hvol[2].data_ptr()), 0))
            e1.record(stream)
            e1.synchronize()
            th = (time.perf_counter() - th0) * 1e3
            te = e0.elapsed_time(e1)
            if world > 1:
                import torch.distributed as dist
                t = torch.tensor([te], device=dev)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                te = float(t.item())
            return te, th

        # The same timed pass three times (each a fresh reconstruction of
        # the same K steps): single passes of identical code on the same box
        # were seen to vary by 20% (387 against 472 ms) with the box's H2D
        # bandwidth unchanged, so the median pass is reported.
        passes = [e2e_pass() for _ in range(3)]
        te, th = sorted(passes)[1]
        e2e = {"value": world * chunk * args.steps / (te / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": chunk * nx * nx * 4 + chunk * (12 + 1),
               "d2h_bytes_per_step": 3 * nx ** 3 * 4 / args.steps,
               "h2d_gbs": h2d_gbs, "host_clock_ms": th, "event_ms": te,
               "passes_ms": [p[0] for p in passes],
               "note": "spi_bp_insert on pinned host images per step, then one spi_bp_finish "
                       "to three host volumes; device-timed on the library stream; median of three passes"}
    ctx.bp_close()

    cg = None
    if not args.no_cg and world == 1:
        cg = cg_measure(args, ctx, stream, rank, world)

    mc = None
    if rank == 0 and world == 1 and not args.no_mc:
        mc = multiclass_measure(args)

    check, ref = None, None
    if rank == 0 and world == 1 and args.check_images > 0:
        check, ref = fp64_check(ctx, nx, chunks, angles, halves, args.check_images, args.bf16)

    c5 = None
    if rank == 0 and world == 1 and not args.no_config5 and nx == 256:
        c5 = config5_measure(args, ctx, stream, chunks, angles, halves, ref)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        hc = chunks[0][:256].cpu().numpy()
        cpu = cpu_baseline(nx, args.cpu_seconds, hc, angles[0][:256], halves[0][:256])

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"BP 32F insertion at {nx}^3 (two half-set grids), "
                                   f"{chunk} images per step in one persistent launch",
                       "nx": nx, "images_per_step": chunk, "spectra": "bf16" if args.bf16 else "f32",
                       "phantom": "200 Gaussian blobs, sigma 1.5-10, SNR 0.05, uniform SO(3)",
                       "l2": "inputs larger than L2 (1.07 GB images + 2.16 GB grids per step)",
                       "accumulation": "FP32 vector atomics into a partial grid, two-sum folded into "
                                       "grid + compensation every 4,096 images",
                       "parallelism": f"dp{world}" if world > 1 else "single GPU"},
            "roofline": roof,
            "fold_ms_per_step": fold_ms / args.steps,
            "rel_l2_vs_fp64": check,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clk,
            "gpu_launches": launches,
            "finish_ms": finish_ms,
            "finish_phase_ms": finish_phase_ms,
            "bpcg": cg,
            "multiclass": mc,
            "config5": c5,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def _cang_host(a):
    """DM(1:6) of CANG(phi, theta, psi) for an angle triple (psi, theta, phi)."""
    q = float(np.float32(3.14159265358979323846)) / 180.0
    phi, theta, psi = float(a[2]), float(a[1]), float(a[0])
    cphi, sphi = np.cos(phi * q), np.sin(phi * q)
    cthe, sthe = np.cos(theta * q), np.sin(theta * q)
    cpsi, spsi = np.cos(psi * q), np.sin(psi * q)
    return np.array([cphi * cthe * cpsi - sphi * spsi, sphi * cthe * cpsi + cphi * spsi, -sthe * cpsi,
                     -cphi * cthe * spsi - sphi * cpsi, -sphi * cthe * spsi + cphi * cpsi, sthe * spsi],
                    dtype=np.float32)


def multiclass_measure(args, steps=4):
    """Uneven multi-class insertion: K = 8 classes with boxes
    {96,128,160,192,192,224,256,256}, each a 30-80-blob phantom; images
    assigned uniformly at random to the classes, SNR 0.1, uniform SO(3);
    every class is a BP 32F with its own grids, all classes inserted through
    spi_bp_insert_multi (one insertion launch per round over every class's
    slices, one stream), then finished; open + insertion + finish of all
    classes are timed, images resident on the device; the rate with one context and host thread per class (concurrent
    streams) is given beside it.  Several streams run at once in the second
    form, so both are timed by the host clock between synchronisations.
    The contexts stay open across passes (a same-size open zeroes the grids
    and keeps buffers and FFT plans); the minimum of four passes is reported."""
    import torch
    from spider_b200 import ops, synth
    _, _, local = dist_env()
    dev = torch.device(f"cuda:{local}")
    boxes = [96, 128, 160, 192, 192, 224, 256, 256]
    rng = np.random.default_rng(1004)
    gen = torch.Generator(device=dev)
    gen.manual_seed(1004)
    assign = rng.integers(0, len(boxes), args.mc_images)
    ctx = ops.Context(local)
    classes = []
    for k, nx in enumerate(boxes):
        nk = int((assign == k).sum())
        vol = make_phantom_gpu(nx, int(rng.integers(30, 81)), (1.5, 8.0), (0.5, 1.0), rng, dev)
        ang = synth.so3_angles(nk, rng)
        imgs = torch.cat([make_chunk(ctx, vol, ang[a:a + 4096], 0.1, gen) for a in range(0, nk, 4096)])
        classes.append((imgs, ang, synth.half_mask(nk, rng)))
        del vol
    ctx.close()
    torch.cuda.synchronize()

    ctxs = [ops.Context(local) for _ in classes]      # kept open across passes

    def one_pass(one_launch):
        torch.cuda.synchronize()
        t = time.perf_counter()
        ops.bp32f_multiclass(classes, device=local, device_out=True, autotune=not one_launch,
                             one_launch=one_launch, ctxs=ctxs)
        torch.cuda.synchronize()
        return time.perf_counter() - t

    res = {}
    for name, one in (("one_launch", True), ("threads", False)):
        one_pass(one)                                  # warm-up (plans, buffers)
        res[name] = min(one_pass(one) for _ in range(max(steps, 1)))
    for c in ctxs:
        c.close()
    return {"metric": "images backprojected/s, 8 classes of box 96-256 (BP 32F each)",
            "value": args.mc_images / res["one_launch"], "unit": "images/s",
            "threads_value": args.mc_images / res["threads"],
            "config": {"workload": "multi-class BP 32F, boxes 96,128,160,192,192,224,256,256",
                       "images": args.mc_images, "per_class": [int(c[0].shape[0]) for c in classes],
                       "timing": "host clock around synchronised calls (open, insertion and finish of all eight "
                                 "classes; the contexts stay open across passes, so each pass's open zeroes the "
                                 f"grids and reuses the buffers and FFT plans), min over {max(steps, 1)} passes",
                       "forms": "value: spi_bp_insert_multi (one insertion launch per round, one stream); "
                                "threads_value: one context and host thread per class"}}


def run_multiclass(args):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    import torch
    torch.cuda.set_device(local)
    m = multiclass_measure(args, args.steps)
    line = {"metric": m["metric"], "value": m["value"], "unit": "images/s", "n_gpus": 1, "steps": args.steps,
            "warmup": 1, "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": m["config"], "threads_value": m["threads_value"]}
    print(json.dumps(line), flush=True)
    return 0


def run_kernel_workload(a):
    """Small, self-contained runs of one kernel family on random data, for
    profilers (ncu): each launches its kernels a few times, so that a
    capture can skip the first launch (-s 1) and take a steady-state one.
    Prints one line, no JSON: these are not benchmark numbers."""
    import torch
    from spider_b200 import ops, synth
    ctx = ops.Context(0)
    rng = np.random.default_rng(0)
    if a.kernel == "insert":
        imgs = torch.randn(a.nimg, a.nx, a.nx, device="cuda")
        ctx.bp_open(a.nx, 2, bf16=a.bf16)
        for _ in range(a.reps):
            ctx.bp_insert(imgs, synth.so3_angles(a.nimg, rng), synth.half_mask(a.nimg, rng))
        ctx.bp_close()
    elif a.kernel == "pj3q":
        vol = torch.randn(a.nx, a.nx, a.nx, device="cuda")
        for _ in range(a.reps):
            ops.pj3q(vol, synth.so3_angles(a.nang, rng), ctx=ctx)
    elif a.kernel == "normalcg":
        from spider_b200 import autograd
        plan = autograd.PJ3QPlan((a.nx, a.nx, a.nx), synth.so3_angles(a.nang, rng), ctx=ctx)
        b = torch.randn(a.nang, a.nx, a.nx, device="cuda")
        for _ in range(a.reps):
            autograd.NormalCG(plan, 1e-3, a.iters, graph=False).solve(plan.adjoint(b))
        plan.close()
    elif a.kernel == "fslice":
        from spider_b200 import autograd
        plan = autograd.FourierSlicePlan(a.nx, synth.so3_angles(a.nang, rng), ctx=ctx)
        b = plan.stage(torch.randn(a.nang, a.nx, a.nx, device="cuda"))
        for _ in range(a.reps):   # --prec fp32: the FP32 normal operator, else the FP64 one
            autograd.NormalCG(plan, 1e-3, a.iters, graph=False,
                              fp64_operator=a.prec != "fp32").solve(plan.adjoint(b))
        plan.close()
    else:
        projs = rng.standard_normal((a.nang, a.n, a.n)).astype(np.float32)
        prec = {"fp64": True, "fp32": False}.get(a.prec, a.prec)
        ops.bpcg(projs, synth.so3_angles(a.nang, rng), a.n / 2 - 3, errm=0.0, maxit=a.iters, mode=1,
                 lam=1e-3, ctx=ctx, fp64=prec, interp=a.interp)
    torch.cuda.synchronize()
    print(f"ok {a.kernel}: {ctx.launches} kernel launches")
    ctx.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "multiclass":
        return run_multiclass(args)
    if args.workload == "kernel":
        return run_kernel_workload(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
