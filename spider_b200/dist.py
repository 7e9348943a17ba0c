"""Image-sharded reconstruction across GPUs (one process per GPU).

The reference distributes images with SETPART (setpart.f:4-29) and sums the
per-rank Fourier grids with MPI_ALLREDUCE before normalising (bp3f.f:1171-1187,
bp32f.f:764-774).  Here each rank inserts its block of images into grids it
owns and the grids are summed with one collective of torch.distributed
(NCCL on GPUs, gloo on CPU) before SYMPLANE0/NRMW2/WINDKB2A.
"""
from __future__ import annotations


def setpart(n: int, nprocs: int):
    """SETPART: sizes and 0-based offsets of an even block partition."""
    nloc, nrem = divmod(n, nprocs)
    psize = [nloc + (1 if p < nrem else 0) for p in range(nprocs)]
    nbase = [0] * nprocs
    for p in range(1, nprocs):
        nbase[p] = nbase[p - 1] + psize[p - 1]
    return psize, nbase


def shard(n: int, rank: int, world: int):
    """(start, count) of rank's block of n images."""
    psize, nbase = setpart(n, world)
    return nbase[rank], psize[rank]


def allreduce_grids(tensors, group=None):
    """Sum grid tensors over all ranks in place (the reference's MPI_ALLREDUCE)."""
    import torch.distributed as dist
    for t in tensors:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return tensors


def sharded_bp32f(ctx, imgs, angles, half, rank: int, world: int, device=None, allreduce=None):
    """BP 32F over all ranks: each rank passes the full image set (or its own
    block), inserts its SETPART block into caller-owned grids, the grids are
    completed (spi_bp_flush) and summed over the ranks, and every rank
    finishes the three volumes.  ``allreduce`` sums a list of tensors in place
    over the ranks (default: torch.distributed, NCCL on GPUs)."""
    import ctypes

    import torch

    from . import _lib
    L = ctx._L
    nx = int(imgs.shape[-1])
    gb = ctypes.c_longlong()
    _lib.check(L.spi_bp_grid_bytes(nx, ctypes.byref(gb)))
    dev = torch.device(device) if device is not None else torch.device(f"cuda:{ctx.device}")
    # spi_bp_open zeroes attached grids on the library stream; torch.empty
    # leaves no fill pending on torch's stream that could land after it
    grids = [torch.empty(gb.value // 4, dtype=torch.float32, device=dev) for _ in range(2)]
    _lib.check(L.spi_bp_attach_grids(ctx.handle, ctypes.c_void_p(grids[0].data_ptr()),
                                     ctypes.c_void_p(grids[1].data_ptr())))
    try:
        ctx.bp_open(nx, 2)
        start, count = shard(int(imgs.shape[0]), rank, world)
        if count:
            ctx.bp_insert(imgs[start:start + count], angles[start:start + count], half[start:start + count])
        ctx.bp_flush()                  # grids hold the complete sums; the library stream is idle
        (allreduce or allreduce_grids)(grids)
        # NCCL orders the reduce on torch's current stream only; the library
        # stream (non-blocking) would not wait for it before SYMPLANE0/NRMW2
        if dev.type == "cuda":
            torch.cuda.synchronize(dev)
        out = ctx.bp_finish(("all", "1", "2"))
        return out["all"], out["1"], out["2"]
    finally:
        ctx.bp_close()
        _lib.check(L.spi_bp_attach_grids(ctx.handle, None, None))


def sharded_bpcg(ctx, projs, angles, rank: int, world: int, ri=None, errm=5e-5, chim=0.0, maxit=20, mode=1,
                 lam=2000.0, group=None, fp64="mixed", interp="linear"):
    """BP CG over all ranks (bpcg.f:522-672, 855-1080): each rank passes the
    full image set (or its own SETPART block with the same length as the
    full set's block), back-projects its block, and works on its block of
    HIANG's merged angles; CB, the image statistics and, every iteration,
    BCKE are summed with torch.distributed (NCCL on GPUs).  Every rank
    returns the same (volume, log)."""
    import torch.distributed as tdist

    from . import ops
    nang = int(angles.shape[0])
    start, count = shard(nang, rank, world)
    block = projs[start:start + count] if int(projs.shape[0]) == nang else projs

    def sum_inplace(t):
        tdist.all_reduce(t, op=tdist.ReduceOp.SUM, group=group)

    return ops.bpcg_shard(block, start, angles, ri, errm, chim, maxit, mode, lam, rank=rank, world=world,
                          sum_inplace=sum_inplace if world > 1 else None, ctx=ctx, fp64=fp64, interp=interp)
