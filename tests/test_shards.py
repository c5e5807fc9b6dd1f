"""Host side of a raster sharded over ranks (shards.py, msf_finish).

No GPU: per-probe rows are synthetic, the exchange runs over gloo with two
CPU ranks, and msf_finish is host-only code.  The finish of the exchanged
rows must equal the finish of the whole array exactly (rows travel
unchanged and pixel sums are added in rank order)."""
import os
import socket
import tempfile

import numpy as np
import pytest

import msf
import shards

N_PROBES = 23  # uneven over two ranks


def job():
    g = msf.Grid(nx=128, ny=128, voltage=200000.0, xperiod=12.5, yperiod=12.5, zperiod=10.0,
                 dupe_x=1, dupe_y=1, dupe_z=1, replicate_atoms=0, xmin=0.0, ymin=0.0,
                 zmin=0.0, min_slice=2.0)
    o = msf.Optics(corrected=0, cs3=1.3e7, cs5=0.0, defocus=300.0, alpha_max=0.010)
    d = msf.Detect(outputs=msf.OUT_ADF_IMAGE | msf.OUT_V_OMEGA | msf.OUT_VBAR_R |
                   msf.OUT_V_RE | msf.OUT_V_GT17 | msf.OUT_V_RBAR | msf.OUT_OMEGA_VIMAGE,
                   det_inner=0.04, det_outer=0.2, dr=1.0)
    xp = np.arange(N_PROBES) * (12.5 / N_PROBES)
    yp = np.array([0.0])
    r = msf.Raster(N_PROBES, 1, xp.ctypes.data_as(msf._dp), yp.ctypes.data_as(msf._dp))
    return g, o, d, r, (xp, yp)


def synthetic_rows(n_seg, plane, seed=7):
    rng = np.random.default_rng(seed)
    amp = rng.uniform(1.0, 2.0, (N_PROBES, n_seg))
    inten = amp ** 2 * rng.uniform(1.0, 1.5, (N_PROBES, n_seg))
    acc = rng.uniform(0.1, 1.0, (2, 2, plane))  # [rank][a/i][pixel]
    return amp, inten, acc


def test_probe_range_partitions():
    for n in (1, 2, 7, 4096, 4097):
        for w in (1, 2, 3, 8):
            spans = [shards.probe_range(n, r, w) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            for (b0, e0), (b1, e1) in zip(spans, spans[1:]):
                assert e0 == b1
            sizes = [e - b for b, e in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shards.probe_range(10, 2, 2)


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g, o, d, r, keep = job()
        n_seg = msf.segment_count(g, d)
        plane = g.nx * g.ny
        amp, inten, acc = synthetic_rows(n_seg, plane)
        b, e = shards.probe_range(N_PROBES, rank, world)
        part = {"amp": amp[b:e], "inten": inten[b:e], "acc_a": acc[rank, 0],
                "acc_i": acc[rank, 1]}
        A, I, aa, ai = shards.exchange(part, N_PROBES, world, dist, "cpu", plane)
        res = msf.finish(g, o, r, d, A, I, aa, ai, want_means=True)
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), adf=res.adf_image,
                 **{k: v for k, v in res.v.items()}, mean_i=res.mean_intensity)
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_exchange_and_finish_equal_single_finish():
    import torch.multiprocessing as mp
    g, o, d, r, keep = job()
    n_seg = msf.segment_count(g, d)
    plane = g.nx * g.ny
    amp, inten, acc = synthetic_rows(n_seg, plane)
    whole = msf.finish(g, o, r, d, amp, inten, acc[0, 0] + acc[1, 0], acc[0, 1] + acc[1, 1],
                       want_means=True)
    with tempfile.TemporaryDirectory() as out:
        mp.start_processes(_rank_main, args=(2, free_port(), out), nprocs=2, join=True,
                           start_method="spawn")
        for rank in range(2):
            got = dict(np.load(os.path.join(out, "rank%d.npz" % rank)))
            assert np.array_equal(got["adf"], whole.adf_image)
            assert np.array_equal(got["mean_i"], whole.mean_intensity)
            for m, v in whole.v.items():
                assert np.array_equal(got[m], v, equal_nan=True), m


def test_finish_rejects_wrong_row_count():
    g, o, d, r, keep = job()
    n_seg = msf.segment_count(g, d)
    with pytest.raises(AssertionError):
        msf.finish(g, o, r, d, np.zeros((N_PROBES - 1, n_seg)), np.zeros((N_PROBES - 1, n_seg)))


def test_segment_count_matches_ring_bins():
    import ctypes as C
    g, o, d, r, keep = job()
    bins = np.zeros(g.nx * g.ny, dtype=np.int32)
    nk = C.c_int32()
    assert msf.lib().msf_ring_bins(C.byref(g), d.dr, bins.ctypes.data_as(msf._ip),
                                   C.byref(nk)) == 0
    assert msf.segment_count(g, d) == nk.value + 1
    adf_only = msf.Detect(outputs=msf.OUT_ADF_IMAGE, det_inner=0.04, det_outer=0.2, dr=1.0)
    assert msf.segment_count(g, adf_only) == 1


def _dying_rank(rank, world, port, out_dir):
    """Rank 1 dies between steps, before the exchange; rank 0 must get an
    error from its collective within the process group's timeout."""
    import datetime
    import time

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=10))
    g, o, d, r, keep = job()
    n_seg = msf.segment_count(g, d)
    plane = g.nx * g.ny
    amp, inten, acc = synthetic_rows(n_seg, plane)
    if rank == 1:
        os._exit(3)
    b, e = shards.probe_range(N_PROBES, rank, world)
    part = {"amp": amp[b:e], "inten": inten[b:e], "acc_a": acc[rank, 0], "acc_i": acc[rank, 1]}
    t0 = time.time()
    try:
        shards.exchange(part, N_PROBES, world, dist, "cpu", plane)
        outcome = "no-error"
    except Exception as ex:
        outcome = "error:" + type(ex).__name__
    with open(os.path.join(out_dir, "rank0.txt"), "w") as f:
        f.write("%s %.1f\n" % (outcome, time.time() - t0))
    os._exit(0)


def test_rank_failure_surfaces_as_error_not_hang():
    import multiprocessing as mpp
    ctx = mpp.get_context("spawn")
    with tempfile.TemporaryDirectory() as out:
        port = free_port()
        procs = [ctx.Process(target=_dying_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        alive = [p for p in procs if p.is_alive()]
        for p in alive:
            p.kill()
        assert not alive, "a rank hung"
        assert procs[1].exitcode == 3
        outcome, seconds = open(os.path.join(out, "rank0.txt")).read().split()
        assert outcome.startswith("error:"), outcome
        assert float(seconds) < 60.0
