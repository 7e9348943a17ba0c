"""SPIDER operations at file level, answering the prompts in the reference's order.

``run(op, answers)`` executes one operation of a ``.spi`` procedure: ``answers``
are the lines that follow the operation in the procedure, in the order the
reference subroutine prompts for them.  Files use SPIDER's image, stack and
document formats (:mod:`spider_b200.spider_io`); the compute runs on the CUDA
library.  RESULTS lines the reference prints are written to ``results``.

===========  =====================================================================
operation    answers (reference prompt order)
===========  =====================================================================
``BP 3F``    image template, file numbers, angles doc, symmetries doc ('*' = none),
             reconstructed volume                              (bp3f.f:127-181)
``BP 32F``   image template, file numbers, angles doc, symmetries doc,
             reconstructed volume, first sample volume, second sample volume
                                                               (bp32f.f:101-236)
``RB 3F``    as BP 3F, then transformed-output template ('*' = none)
                                                               (bp3f.f:350-364)
``RB 32F``   as BP 32F, then transformed-output template       (bp32f.f:507-523)
``BP 3F P``  as BP 3F with the partial volume name instead of the reconstructed
             volume; writes <name> (X) and <name>_W (W)       (bp3f.f:191-225)
``BP 3F M``  partial volume template, file numbers, symmetries doc, volume
                                                               (bp3f.f:563-648)
``PJ 3Q``    input volume, 'radius[, Y]' (consecutive numbers), angle numbers,
             angles doc, output projection template            (pj3q_n.f:73-160)
``PJ 3F``    as PJ 3Q, with FBS interpolation (cubic volumes)  (vtil2.f:222-228)
``BP CG``    image template, file numbers, radius, angles doc, L/F,
             reconstructed volume, 'error limit, chi^2 limit',
             'iteration limit, mode', lambda                   (bpcg.f:120-244)
``BP CG 3``  image template, file numbers, radius, angles doc, L/F,
             reconstructed volume, first sample volume, second sample volume,
             limits, iteration limit & mode, lambda            (bpcg.f:139-244)
``BP CG 3L`` as BP CG 3, with the file numbers of the first and of the second
             sample after the image file numbers               (bpcg.f:143-152)
``MD``       the mode: 'FBS ON' / 'USE FBS' / 'FBS' makes RB 3F and RB 32F
             rotate with RTSF, 'FBS OFF' / 'NO FBS' with RTSQ  (setmode.f:399-409);
             other modes are not provided
===========  =====================================================================

The back-projection operations read their images chunk by chunk
(``sio.stream_images``): the next chunk is read from disk into a second
pinned buffer while the GPU inserts the current one, instead of one REDVOL
per image between insertions (bp3f.f:401-430).

The reference shuffles the BP 32F and BP CG 3 half sets with RANDOM_NUMBER
(bp32f.f:543-553, bpcg.f:1593-1632); here the first sample receives NANG/2
images chosen by a seeded permutation (``seed``), which keeps the half sizes
of the reference.
"""
from __future__ import annotations

import os
import sys

import numpy as np

from . import ops
from . import spider_io as sio


def _angles(doc, numbers):
    """Angle triples (psi, theta, phi) = registers 1-3 for the image numbers."""
    d = sio.read_doc(doc)
    out = np.zeros((len(numbers), 3), np.float32)
    for i, k in enumerate(numbers):
        if k not in d:
            raise ops.SpiderError(102, f"MISSING ANGLE FOR IMAGE {k}")  # bp3f.f:1283-1288
        out[i] = d[k][:3]
    return out


def _inplane(doc, numbers):
    """RTSQ parameters (angle, sx, sy) = registers 6-8 (bp3f.f:415-418)."""
    d = sio.read_doc(doc)
    out = np.zeros((len(numbers), 3), np.float32)
    for i, k in enumerate(numbers):
        r = d[k]
        if len(r) < 8:
            raise ops.SpiderError(102, f"ANGLES DOC KEY {k} HAS NO REGISTERS 6-8")
        out[i] = r[5:8]
    return out


def _symmetries(doc):
    if doc.strip() in ("*", ""):
        return None
    d = sio.read_doc(doc)
    return np.array([d[k][:3] for k in sorted(d)], np.float32)


def _name(n, ext):
    return sio.add_extension(n.strip(), ext)


def _half_sets(n, seed):
    rng = np.random.default_rng(seed)
    half = np.zeros(n, np.uint8)
    half[rng.permutation(n)[: n // 2]] = 1
    return half


def _pinned_pair(chunk, ny, nx):
    """Two float32 [chunk, ny, nx] host buffers, page-locked when CUDA is there."""
    try:
        import torch
        if torch.cuda.is_available():
            return [torch.empty((chunk, ny, nx), dtype=torch.float32, pin_memory=True).numpy() for _ in range(2)]
    except Exception:
        pass
    return None


def _stream_insert(ctx, src, ang, half, inplane, chunk):
    """Insert every image of src, chunk by chunk, reading ahead on a thread."""
    ny, nx = src.shape
    chunk = max(1, min(len(src), chunk or max(1, (256 << 20) // (4 * nx * ny))))
    for start, imgs in sio.stream_images(src, chunk, _pinned_pair(chunk, ny, nx)):
        sl = slice(start, start + len(imgs))
        ctx.bp_insert(imgs, ang[sl], None if half is None else half[sl],
                      inplane=None if inplane is None else inplane[sl])


def run(op: str, answers, *, ext: str = "spi", ctx=None, seed: int = 0, results=None, chunk=None):
    """Run one SPIDER operation; returns a dict of the arrays it wrote.
    ``chunk``: images per insertion call of the back-projection operations
    (default: about 256 MB of images)."""
    results = results or sys.stdout
    op = " ".join(op.upper().split())
    a = [str(x) for x in answers]
    ctx = ctx or ops.default_context()
    if op in ("BP 3F", "BP 32F", "RB 3F", "RB 32F", "BP 3F P"):
        numbers = sio.parse_numbers(a[1])
        src = sio.ImageSource(a[0], numbers, ext)
        ny, nx = src.shape
        if ny != nx:
            raise ops.SpiderError(101, "ONLY WORKS ON SQUARE IMAGES")   # bp3f.f:135-138
        print(f"  NUMBER OF IMAGES: {len(numbers):7d}", file=results)
        ang = _angles(_name(a[2], ext), numbers)
        sym = _symmetries(a[3] if a[3].strip() == "*" else _name(a[3], ext))
        inplane = _inplane(_name(a[2], ext), numbers) if op.startswith("RB") else None
        half = _half_sets(len(numbers), seed) if op in ("BP 32F", "RB 32F") else None
        ctx.bp_open(nx, 1 if half is None else 2, sym)
        try:
            _stream_insert(ctx, src, ang, half, inplane, chunk)
            if op == "BP 3F P":
                x, w = ctx.bp_partial_out(0)
            elif half is None:
                vol = ctx.bp_finish(("all",))["all"]
            else:
                o = ctx.bp_finish(("all", "1", "2"))
                v_all, v1, v2 = o["all"], o["1"], o["2"]
        finally:
            ctx.bp_close()
        if op == "BP 3F P":
            xv = x.reshape(2 * nx, 2 * nx, 2 * (nx + 1))
            out = _name(a[4], ext)
            sio.write_image(out, xv)
            base, e = os.path.splitext(out)
            sio.write_image(f"{base}_W{e}", w)
            return {"x": x, "w": w}
        if half is None:
            sio.write_image(_name(a[4], ext), vol)
            return {"vol": vol}
        sio.write_image(_name(a[4], ext), v_all)
        sio.write_image(_name(a[5], ext), v1)
        sio.write_image(_name(a[6], ext), v2)
        return {"vol": v_all, "vol1": v1, "vol2": v2, "half": half}
    if op == "MD":
        mode = " ".join(a[0].upper().split()) if a else ""
        if mode in ("FBS ON", "USE FBS", "FBS"):
            ctx.set_fbs(True)
            print("  USING FBS INTERPOLATION", file=results)
        elif mode in ("FBS OFF", "NO FBS"):
            ctx.set_fbs(False)
            print("  NOT USING FBS INTERPOLATION", file=results)
        else:
            raise ops.SpiderError(101, f"MD mode {mode!r} is not provided by this library")
        return {"fbs": ctx.fbs}
    if op == "BP 3F M":
        numbers = sio.parse_numbers(a[1])
        parts = []
        for k in numbers:
            xn = sio.expand_template(_name(a[0], ext), k)
            base, e = os.path.splitext(xn)
            x, _ = sio.read_image(xn)
            w, _ = sio.read_image(f"{base}_W{e}")
            nz, ny, nxx = x.shape
            parts.append((x.reshape(nz, ny, nxx // 2, 2), w))
        print(f"  NUMBER OF VOLUMES: {len(numbers):7d}", file=results)
        sym = _symmetries(a[2] if a[2].strip() == "*" else _name(a[2], ext))
        vol = ops.bp3f_merge(parts, sym, ctx=ctx)
        sio.write_image(_name(a[3], ext), vol)
        return {"vol": vol}
    if op in ("PJ 3Q", "PJ 3F"):
        vol, _ = sio.read_image(_name(a[0], ext))
        if vol.ndim == 2:
            vol = vol[None]
        nz, ny, nx = vol.shape
        if not (nx == ny == nz):
            print(" WARNING NON-CUBIC VOLUME MAY GIVE INVALID RESULTS", file=results)
        parts = a[1].replace(",", " ").split()
        ri = float(parts[0]) if parts else float(min(nx, ny, nz) // 2 - 2)
        conseq = len(parts) > 1 and "Y" in parts[1].upper()
        numbers = sio.parse_numbers(a[2])
        ang = _angles(_name(a[3], ext), numbers)
        proj = (ops.pj3f if op == "PJ 3F" else ops.pj3q)(vol, ang, ri, ctx=ctx)
        tmpl = _name(a[4], ext)
        if "@" in tmpl:
            sio.write_stack(tmpl.split("@", 1)[0], proj, angles=ang)
        else:
            for i, k in enumerate(numbers):
                sio.write_image(sio.expand_template(tmpl, i + 1 if conseq else k), proj[i], angles=ang[i])
        print(f"  {op} FINISHED FOR: {len(numbers):7d}   PROJECTIONS -----", file=results)
        return {"proj": proj}
    if op in ("BP CG", "BP CG 3", "BP CG 3L"):
        numbers = sio.parse_numbers(a[1])
        a = list(a)
        lists = None
        if op == "BP CG 3L":   # the two sample lists follow the image numbers
            lists = (sio.parse_numbers(a[2]), sio.parse_numbers(a[3]))
            del a[2:4]
        imgs = sio.read_images(a[0], numbers, ext)
        n = imgs.shape[1]
        print(f"  NUMBER OF IMAGES:{len(numbers):8d}", file=results)
        ri = float(a[2]) if a[2].strip() else float(n // 2 - 2)
        ang = _angles(_name(a[3], ext), numbers)
        fbs = a[4].strip().upper().startswith("F")   # FBS_WANTED = (ANSW(1:1) == 'F'), bpcg.f:177-180
        interp = "fbs" if fbs else "linear"
        k = 6 if op == "BP CG" else 8   # index of the 'error limit, chi^2 limit' answer
        errm, chim = (float(v) for v in a[k].replace(",", " ").split()[:2])
        maxit, mode = (int(float(v)) for v in a[k + 1].replace(",", " ").split()[:2])
        lam = float(a[k + 2])

        def _log(lg):
            print("  USING FBS INTERPOLATION" if fbs else "  USING LINEAR INTERPOLATION", file=results)
            for it, err, chi in lg:   # bpcg.f:1213-1216
                print(f"  ITERATION: {int(it):3d}  DIFFERENCE:{err:12.4E}  CHISQ:{chi:12.4E}", file=results)

        if op == "BP CG":
            vol, log = ops.bpcg(imgs, ang, ri, errm, chim, maxit, mode, lam, ctx=ctx, interp=interp)
            _log(log)
            sio.write_image(_name(a[5], ext), vol)
            return {"vol": vol, "log": log}
        if lists is None:
            half = _half_sets(len(numbers), seed)
            print(f"  Random lists: {int(half.sum())} {len(numbers) - int(half.sum())}", file=results)
        else:
            pos = {k2: i for i, k2 in enumerate(numbers)}
            missing = [k2 for k2 in lists[0] + lists[1] if k2 not in pos]
            if missing:
                raise ops.SpiderError(102, f"SAMPLE LIST IMAGE {missing[0]} NOT IN THE IMAGE LIST")
            sel = lists[0] + lists[1]
            half = np.zeros(len(sel), np.uint8)
            half[: len(lists[0])] = 1
            imgs = imgs[[pos[k2] for k2 in sel]]
            ang = ang[[pos[k2] for k2 in sel]]
        vol, v1, v2, logs = ops.bpcg3(imgs, ang, half, ri, errm, chim, maxit, mode, lam, ctx=ctx, interp=interp)
        for lg in logs:
            _log(lg)
        sio.write_image(_name(a[5], ext), vol)
        sio.write_image(_name(a[6], ext), v1)
        sio.write_image(_name(a[7], ext), v2)
        return {"vol": vol, "vol1": v1, "vol2": v2, "logs": logs, "half": half}
    raise ops.SpiderError(101, f"operation {op!r} is not provided by this library")
