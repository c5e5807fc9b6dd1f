"""Slot batches (msf_run_batch) and the request loop (msf_server_*).

Each probe in a slot batch runs the same arithmetic as in a plain batched
raster, only its launch companions differ (probes of other rasters, at other
slices), so:
  * every raster of a mixed batch matches its own msf_run within FP32
    rounding (ADF image and V(k) to 1e-6 relative, V(k) floor 1e-9);
  * a request served in a mix returns exactly what it returns alone
    (bit-identical: detection sums run in raster order either way).
"""
import time

import numpy as np
import pytest

import msf
import specimen
from conftest import assert_variance_close, rel_err

pytestmark = pytest.mark.gpu

FEM = msf.OUT_ADF_IMAGE | msf.OUT_V_OMEGA | msf.OUT_VBAR_R | msf.OUT_V_RE | msf.OUT_V_GT17
MODES = ["V_omega", "Vbar_r", "V_re", "V_gt17"]


class JobSpec:
    """A small seeded amorphous-Si raster (arrays kept alive with the structs)."""

    def __init__(self, n, box, zbox, n_atoms, seed, raster_n, outputs=FEM, defocus=400.0):
        self.pos = specimen.amorphous_positions(n_atoms, (box, box, zbox), seed=seed)
        self.z = np.full(n_atoms, 14, dtype=np.uint32)
        self.grid = msf.Grid(nx=n, ny=n, voltage=200000.0, xperiod=box, yperiod=box,
                             zperiod=zbox, dupe_x=1, dupe_y=1, dupe_z=1, replicate_atoms=0,
                             xmin=0.0, ymin=0.0, zmin=0.0, min_slice=2.0)
        self.optics = msf.Optics(corrected=0, cs3=1.3e7, cs5=0.0, defocus=defocus,
                                 alpha_max=0.010)
        self.xp = np.arange(raster_n) * (box / raster_n)
        self.raster = msf.Raster(raster_n, raster_n, self.xp.ctypes.data_as(msf._dp),
                                 self.xp.ctypes.data_as(msf._dp))
        self.detect = msf.Detect(outputs=outputs, det_inner=0.04, det_outer=0.2, dr=1.0)


def jobs_mixed():
    return [
        JobSpec(256, 25.0, 20.0, 600, seed=11, raster_n=6),
        JobSpec(128, 12.5, 14.0, 100, seed=12, raster_n=5),   # plain column pass
        JobSpec(256, 25.0, 30.0, 900, seed=13, raster_n=4, defocus=0.0),
        JobSpec(512, 50.0, 8.0, 900, seed=14, raster_n=3),
        JobSpec(256, 25.0, 10.0, 300, seed=15, raster_n=5, outputs=msf.OUT_ADF_IMAGE),
    ]


def assert_same_run(a, b, rtol, atol, what):
    err = rel_err(a.adf_image, b.adf_image)
    m = np.abs(b.adf_image) > 0
    if m.any():
        assert err[m].max() <= rtol, (what, "ADF", err[m].max())
    assert a.n_k == b.n_k, what
    for mode, v in b.v.items():
        assert_variance_close(a.v[mode], v, rtol, atol, what="%s %s" % (what, mode))


@pytest.mark.parametrize("slots", [0, 7])
def test_batch_matches_single_runs(slots):
    ctx = msf.Context(precision="fp32", batch=16)
    js = jobs_mixed()
    specs = [ctx.specimen(j.grid, j.pos, j.z) for j in js]
    singles = [ctx.run(s, j.optics, j.raster, j.detect) for s, j in zip(specs, js)]
    outs = ctx.run_batch([(s, j.optics, j.raster, j.detect) for s, j in zip(specs, js)],
                         slots=slots)
    for k, (o, r) in enumerate(zip(outs, singles)):
        assert o.probe_slices == r.probe_slices
        assert_same_run(o, r, 1e-6, 1e-9, "job %d slots %d" % (k, slots))


@pytest.mark.parametrize("slots", [4, 9])
def test_grouped_steps_match_slot_passes(slots, monkeypatch):
    """Runs of neighbouring slots holding one raster's probes at one slice
    go through the batched passes of msf_run, one launch pair per run; with
    MSF_LANE_GROUPS=0 every step runs the slot passes.  Both give the same
    bits (4 slots: the 36-probe raster fills the lane in whole groups; 9:
    groups end part-filled and rasters share steps in several runs)."""
    ctx = msf.Context(precision="fp32")
    js = jobs_mixed()
    specs = [ctx.specimen(j.grid, j.pos, j.z) for j in js]
    batch = [(s, j.optics, j.raster, j.detect) for s, j in zip(specs, js)]
    monkeypatch.setenv("MSF_LANE_GROUPS", "0")
    slot_only = ctx.run_batch(batch, slots=slots)
    monkeypatch.setenv("MSF_LANE_GROUPS", "1")
    mixed = ctx.run_batch(batch, slots=slots)
    for k, (a, b) in enumerate(zip(mixed, slot_only)):
        assert np.array_equal(a.adf_image, b.adf_image), k
        for mode in b.v:
            assert np.array_equal(a.v[mode], b.v[mode], equal_nan=True), (k, mode)


class LargeJob(JobSpec):
    """A thin seeded slab on a 1024^2 or 2048^2 grid (positions from the
    library's generator, which is fast at these atom counts)."""

    def __init__(self, n, zbox, seed, raster_n):
        box = n * 0.09766
        super().__init__(n, box, zbox, 1, seed, raster_n)
        self.pos = msf.amorphous_positions(int(0.05 * box * box * zbox), (box, box, zbox), 2.2,
                                           seed=seed)
        self.z = np.full(len(self.pos), 14, dtype=np.uint32)


def test_large_grid_lanes_match_single_runs(monkeypatch):
    """The slot passes and the batched passes of the lanes at the 1024- and
    2048-point shapes (thin slabs, 3 slices; 7 slots, so the 25- and 9-probe
    rasters leave part-filled groups and mix): each raster matches its own
    msf_run, and the grouped steps give the same bits as slot passes only."""
    js = [LargeJob(1024, 6.0, 71, 5), LargeJob(2048, 6.0, 72, 3),
          LargeJob(1024, 6.0, 73, 3), LargeJob(2048, 6.0, 74, 3)]
    ctx = msf.Context(precision="fp32", batch=8)
    specs = [ctx.specimen(j.grid, j.pos, j.z) for j in js]
    batch = [(s, j.optics, j.raster, j.detect) for s, j in zip(specs, js)]
    singles = [ctx.run(*b) for b in batch]
    outs = ctx.run_batch(batch, slots=7)
    for k, (o, r) in enumerate(zip(outs, singles)):
        assert o.probe_slices == r.probe_slices
        assert_same_run(o, r, 1e-6, 1e-9, "large job %d" % k)
    monkeypatch.setenv("MSF_LANE_GROUPS", "0")
    slot_only = ctx.run_batch(batch, slots=7)
    for k, (a, b) in enumerate(zip(outs, slot_only)):
        assert np.array_equal(a.adf_image, b.adf_image), k
        for mode in b.v:
            assert np.array_equal(a.v[mode], b.v[mode], equal_nan=True), (k, mode)


def test_batch_rejects_fp64_context():
    ctx = msf.Context(precision="fp64")
    j = jobs_mixed()[1]
    s = ctx.specimen(j.grid, j.pos, j.z)
    with pytest.raises(msf.MsfError):
        ctx.run_batch([(s, j.optics, j.raster, j.detect)])


def serve(jobs, slots, stagger_s=0.0):
    srv = msf.Server(slots=slots)
    tickets = []
    for j in jobs:
        tickets.append(srv.submit(j.grid, j.pos, j.z, j.optics, j.raster, j.detect))
        if stagger_s:
            time.sleep(stagger_s)
    outs = []
    for t in tickets:
        r = None
        deadline = time.time() + 300
        while r is None:
            assert time.time() < deadline, "request did not finish"
            r = srv.poll(t, wait_ms=200)
        outs.append(r)
    stats = srv.stats()
    srv.close()
    return outs, stats


def test_server_result_same_alone_and_in_mix():
    js = jobs_mixed()
    alone = [serve([j], slots=5)[0][0] for j in js]
    mixed, stats = serve(js, slots=5, stagger_s=0.01)
    for k, (a, b) in enumerate(zip(mixed, alone)):
        assert np.array_equal(a.adf_image, b.adf_image), k
        for mode in b.v:
            assert np.array_equal(a.v[mode], b.v[mode], equal_nan=True), (k, mode)
    assert stats["completed"] == len(js) and stats["failed"] == 0
    assert 0 < stats["p50_s"] <= stats["p99_s"] <= stats["max_s"]


def test_server_matches_plain_run():
    ctx = msf.Context(precision="fp32")
    js = jobs_mixed()[:2]
    outs, _ = serve(js, slots=3)
    for k, (o, j) in enumerate(zip(outs, js)):
        s = ctx.specimen(j.grid, j.pos, j.z)
        r = ctx.run(s, j.optics, j.raster, j.detect)
        assert_same_run(o, r, 1e-6, 1e-9, "served job %d" % k)


def test_server_reports_request_errors():
    srv = msf.Server(slots=4)
    j = jobs_mixed()[1]
    bad = msf.Grid.from_buffer_copy(j.grid)
    bad.nx = 100  # not a power of two
    t = srv.submit(bad, j.pos, j.z, j.optics, j.raster, j.detect)
    good = srv.submit(j.grid, j.pos, j.z, j.optics, j.raster, j.detect)
    with pytest.raises(msf.MsfError):
        while srv.poll(t, wait_ms=200) is None:
            pass
    r = None
    while r is None:
        r = srv.poll(good, wait_ms=200)
    assert r.probe_slices > 0
    st = srv.stats()
    assert st["failed"] == 1 and st["completed"] == 1
    srv.close()


def test_server_cancel():
    """A cancelled request polls MSF_ERR_CANCELLED whether it was still
    queued (a 1-byte budget keeps later requests waiting while one runs) or
    already admitted; the other requests are not disturbed."""
    js = jobs_mixed()
    srv = msf.Server(slots=4, hbm_budget=1)
    ta = srv.submit(js[3].grid, js[3].pos, js[3].z, js[3].optics, js[3].raster, js[3].detect)
    tb = srv.submit(js[1].grid, js[1].pos, js[1].z, js[1].optics, js[1].raster, js[1].detect)
    tc = srv.submit(js[4].grid, js[4].pos, js[4].z, js[4].optics, js[4].raster, js[4].detect)
    srv.cancel(tc)  # queued behind ta
    srv.cancel(ta)  # admitted (or about to be): runs, results discarded
    for t in (ta, tc):
        with pytest.raises(msf.MsfError) as e:
            while srv.poll(t, wait_ms=200) is None:
                pass
        assert e.value.status == 9
    r = None
    while r is None:
        r = srv.poll(tb, wait_ms=200)
    assert r.probe_slices > 0
    with pytest.raises(msf.MsfError):
        srv.cancel(tb)  # delivered
    with pytest.raises(msf.MsfError):
        srv.cancel(10 ** 6)  # unknown
    st = srv.stats()
    assert st["completed"] == 1 and st["failed"] == 2
    srv.close()


def rect_job(seed=62):
    """256^2 grid over a 25 x 20 A cell: its band limit removes other
    columns than a square cell's."""
    j = JobSpec(256, 25.0, 14.0, 300, seed=seed, raster_n=6)
    j.pos = specimen.amorphous_positions(240, (25.0, 20.0, 14.0), seed=seed)
    j.z = np.full(len(j.pos), 14, dtype=np.uint32)
    j.grid = msf.Grid(nx=256, ny=256, voltage=200000.0, xperiod=25.0, yperiod=20.0,
                      zperiod=14.0, dupe_x=1, dupe_y=1, dupe_z=1, replicate_atoms=0,
                      xmin=0.0, ymin=0.0, zmin=0.0, min_slice=2.0)
    j.yp = np.arange(6) * (20.0 / 6)
    j.raster = msf.Raster(6, 6, j.xp.ctypes.data_as(msf._dp), j.yp.ctypes.data_as(msf._dp))
    return j


def test_lane_stops_skipping_removed_columns_midflight():
    """A lane skips the columns its first raster's band limit removes; a
    raster of the same grid size with other removed columns makes it move
    every column from then on, zeroing the skipped ones in the slots in
    flight.  Both rasters give exactly what they give alone."""
    a = JobSpec(256, 25.0, 40.0, 1000, seed=63, raster_n=24)
    b = rect_job()
    alone = [serve([j], slots=4)[0][0] for j in (a, b)]
    mixed, _ = serve([a, b], slots=4, stagger_s=0.05)
    for k, (m, r) in enumerate(zip(mixed, alone)):
        assert np.array_equal(m.adf_image, r.adf_image), k
        for mode in r.v:
            assert np.array_equal(m.v[mode], r.v[mode], equal_nan=True), (k, mode)
