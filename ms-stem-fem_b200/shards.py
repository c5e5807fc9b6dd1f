"""One raster sharded over ranks, one process per GPU.

The reference splits a raster's probes over MPI ranks and combines the
detector sums with MPI_Reduce / MPI_Allgatherv (adfstem.cpp:1556-1606,
2489-2782, 2822-3612).  Here:

  * each rank takes a contiguous range of probes (``probe_range``) and runs
    it with ``Context.run_partial`` -- pixel snaps are found over the whole
    raster, because the reference's search carries its position from probe
    to probe;
  * ``exchange`` is the one collective step: an all-gather of the per-probe
    rows (ring sums and ADF annulus, padded to the largest shard) and an
    all-gather of the per-pixel sums, which every rank adds in rank order,
    so the result does not depend on the collective's reduction order;
  * ``msf.finish`` turns the rows of all probes (in raster order) into the
    ADF image and the FEM statistics on the host.

``torch.distributed`` is the transport (NCCL with CUDA tensors on GPUs,
gloo with CPU tensors in the tests).
"""
from __future__ import annotations

import numpy as np

import msf


def probe_range(n_probes: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous range of probes of `rank`: sizes differ by at most one,
    lower ranks take the larger ones."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank %d outside world of %d" % (rank, world))
    base, extra = divmod(n_probes, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def run_shard(ctx: msf.Context, spec: msf.Specimen, optics: msf.Optics, raster: msf.Raster,
              detect: msf.Detect, rank: int, world: int) -> dict:
    """This rank's probes of the raster: per-probe rows and pixel sums."""
    n = raster.n_x * raster.n_y
    b, e = probe_range(n, rank, world)
    if b == e:
        n_seg = msf.segment_count(spec.grid, detect)
        return {"amp": np.zeros((0, n_seg)), "inten": np.zeros((0, n_seg)), "acc_a": None,
                "acc_i": None, "probe_slices": 0, "seconds_raster": 0.0, "n_k": n_seg - 1}
    return ctx.run_partial(spec, optics, raster, detect, b, e)


def exchange(part: dict, n_probes: int, world: int, dist, device="cpu", plane: int = 0):
    """All ranks get every probe's rows (raster order) and the pixel sums of
    all probes (added in rank order).  Every rank must call this."""
    import torch

    amp, inten = part["amp"], part["inten"]
    n_seg = amp.shape[1]
    sizes = [probe_range(n_probes, r, world) for r in range(world)]
    rows_max = max(e - b for b, e in sizes)
    block = np.zeros((2, rows_max, n_seg))
    block[0, :amp.shape[0]] = amp
    block[1, :inten.shape[0]] = inten
    mine = torch.from_numpy(block).to(device)
    got = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(got, mine)
    all_amp = np.zeros((n_probes, n_seg))
    all_int = np.zeros((n_probes, n_seg))
    for r, (b, e) in enumerate(sizes):
        g = got[r].cpu().numpy()
        all_amp[b:e] = g[0, :e - b]
        all_int[b:e] = g[1, :e - b]
    acc_a = acc_i = None
    has_pix = torch.tensor([1 if part["acc_a"] is not None else 0], device=device)
    dist.all_reduce(has_pix, op=dist.ReduceOp.MAX)
    if int(has_pix.item()):
        pix = np.zeros((2, plane))
        if part["acc_a"] is not None:
            pix[0] = part["acc_a"]
            pix[1] = part["acc_i"]
        mine = torch.from_numpy(pix).to(device)
        got = [torch.empty_like(mine) for _ in range(world)]
        dist.all_gather(got, mine)
        acc_a = np.zeros(plane)
        acc_i = np.zeros(plane)
        for r in range(world):
            g = got[r].cpu().numpy()
            acc_a += g[0]
            acc_i += g[1]
    return all_amp, all_int, acc_a, acc_i


def run_sharded(ctx: msf.Context, spec: msf.Specimen, optics: msf.Optics,
                raster: msf.Raster, detect: msf.Detect, rank: int, world: int, dist,
                device="cpu", want_means=False):
    """The whole raster over `world` ranks; every rank returns the same
    RunResult (ADF image, V(k)) and its own shard's info."""
    part = run_shard(ctx, spec, optics, raster, detect, rank, world)
    n = raster.n_x * raster.n_y
    plane = spec.grid.nx * spec.grid.ny
    amp, inten, acc_a, acc_i = exchange(part, n, world, dist, device, plane)
    res = msf.finish(spec.grid, optics, raster, detect, amp, inten, acc_a, acc_i,
                     want_means=want_means)
    return res, part
