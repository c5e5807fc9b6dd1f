"""Slice potentials by FFT convolution (the direct per-atom sum's exact
equivalent, used for slices of 64 atoms or more) against the reference's
transmission functions and outputs, and against the direct sum."""
import os

import numpy as np
import pytest

import msf
from conftest import assert_variance_close, case_argv, case_dir, load_case, rel_err

pytestmark = pytest.mark.gpu


def context(mode, precision="fp64"):
    old = os.environ.get("MSF_POTENTIAL")
    os.environ["MSF_POTENTIAL"] = mode
    try:
        return msf.Context(precision=precision)
    finally:
        if old is None:
            del os.environ["MSF_POTENTIAL"]
        else:
            os.environ["MSF_POTENTIAL"] = old


@pytest.mark.parametrize("name", ["fem128", "sio"])
def test_fft_potential_matches_reference(name, golden_tmp):
    meta, ref = load_case(name)
    job = msf.Job(case_argv(name, case_dir(name, golden_tmp)))
    ctx = context("fft")
    q, z = job.positions()
    spec = ctx.specimen(job.grid, q, z)
    t = spec.transmission(int(ref["transmission_slice"])).ravel()
    err = np.abs(t - ref["transmission"]).max()
    print("%s transmission max abs err (FFT potential) %.3e" % (name, err))
    assert err <= 1e-12
    res = ctx.run(spec, job.optics, job.raster, job.detect)
    assert rel_err(res.adf_image, ref["adf_image"]).max() <= 1e-5
    for mode, v in res.v.items():
        assert_variance_close(v, ref[mode][:, 1], 1e-5, 1e-12, what=mode)


def test_fft_and_direct_potentials_agree():
    box = (40.0, 40.0, 12.0)
    pos = msf.amorphous_positions(1000, box, 2.2, seed=41)
    z = np.where(np.arange(len(pos)) % 3 == 0, 8, 14).astype(np.uint32)
    g = msf.Grid(nx=256, ny=256, voltage=200000.0, xperiod=box[0], yperiod=box[1],
                 zperiod=box[2], dupe_x=1, dupe_y=1, dupe_z=1, replicate_atoms=0, xmin=0.0,
                 ymin=0.0, zmin=0.0, min_slice=2.0)
    a = context("direct").specimen(g, pos, z)
    b = context("fft").specimen(g, pos, z)
    n = a.slices()["n"]
    assert n == b.slices()["n"] and n > 2
    worst = max(np.abs(a.transmission(s) - b.transmission(s)).max() for s in range(n))
    print("direct vs FFT transmission max abs diff %.3e" % worst)
    assert worst <= 1e-12
