"""A raster run as shards (msf_run_partial + msf_finish) on one GPU equals
msf_run: per-probe rows are computed per probe, so the ADF image and the
ring statistics match exactly; the pixel sums are added shard by shard,
which changes only their FP64 rounding."""
import numpy as np
import pytest

import msf
import shards
from test_gpu_slots import JobSpec

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("world", [2, 3])
def test_shards_equal_whole_raster(precision, world):
    j = JobSpec(256, 25.0, 16.0, 500, seed=21, raster_n=7)
    ctx = msf.Context(precision=precision, batch=8)
    spec = ctx.specimen(j.grid, j.pos, j.z)
    whole = ctx.run(spec, j.optics, j.raster, j.detect)
    parts = [shards.run_shard(ctx, spec, j.optics, j.raster, j.detect, r, world)
             for r in range(world)]
    amp = np.concatenate([p["amp"] for p in parts])
    inten = np.concatenate([p["inten"] for p in parts])
    acc_a = sum(p["acc_a"] for p in parts)
    acc_i = sum(p["acc_i"] for p in parts)
    res = msf.finish(spec.grid, j.optics, j.raster, j.detect, amp, inten, acc_a, acc_i)
    assert sum(p["probe_slices"] for p in parts) == whole.probe_slices
    assert np.array_equal(res.adf_image, whole.adf_image)
    for m in ("V_omega", "Vbar_r"):
        assert np.array_equal(res.v[m], whole.v[m], equal_nan=True), m
    for m in ("V_re", "V_gt17"):
        np.testing.assert_allclose(res.v[m], whole.v[m], rtol=1e-12, atol=1e-14)


def test_partial_range_checks():
    j = JobSpec(128, 12.5, 8.0, 80, seed=22, raster_n=3)
    ctx = msf.Context(precision="fp32")
    spec = ctx.specimen(j.grid, j.pos, j.z)
    for b, e in ((0, 0), (5, 4), (0, 10), (-1, 2)):
        with pytest.raises(msf.MsfError):
            ctx.run_partial(spec, j.optics, j.raster, j.detect, b, e)


def _sharded_rank(rank, world, port, out_dir, precision):
    import os

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        j = JobSpec(256, 25.0, 16.0, 500, seed=23, raster_n=6)
        ctx = msf.Context(precision=precision, batch=8)
        spec = ctx.specimen(j.grid, j.pos, j.z)
        res, part = shards.run_sharded(ctx, spec, j.optics, j.raster, j.detect, rank, world,
                                       dist, device="cpu")
        np.savez(os.path.join(out_dir, "r%d.npz" % rank), adf=res.adf_image,
                 **res.v, ps=part["probe_slices"])
    finally:
        dist.destroy_process_group()


def test_run_sharded_two_processes_gloo(tmp_path):
    """Two ranks as processes on the one GPU: each runs its own probes (no
    kernel waits on another process); the exchange runs over gloo."""
    import torch.multiprocessing as mp
    from test_shards import free_port
    mp.start_processes(_sharded_rank, args=(2, free_port(), str(tmp_path), "fp32"), nprocs=2,
                       join=True, start_method="spawn")
    j = JobSpec(256, 25.0, 16.0, 500, seed=23, raster_n=6)
    ctx = msf.Context(precision="fp32", batch=8)
    spec = ctx.specimen(j.grid, j.pos, j.z)
    whole = ctx.run(spec, j.optics, j.raster, j.detect)
    got = [dict(np.load(tmp_path / ("r%d.npz" % r))) for r in range(2)]
    assert int(got[0]["ps"]) + int(got[1]["ps"]) == whole.probe_slices
    for g in got:
        assert np.array_equal(g["adf"], whole.adf_image)
        for m in ("V_omega", "Vbar_r"):
            assert np.array_equal(g[m], whole.v[m], equal_nan=True), m
        for m in ("V_re", "V_gt17"):
            np.testing.assert_allclose(g[m], whole.v[m], rtol=1e-12, atol=1e-14)
