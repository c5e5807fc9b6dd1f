"""The plain per-pass path (msf_run_plain: one probe at a time, one launch
per reference step) computes the same raster as the fused batched path;
only the FP64 rounding of its separate passes differs."""
import numpy as np
import pytest

import msf
from test_gpu_slots import FEM, JobSpec

pytestmark = pytest.mark.gpu


def test_plain_matches_fused_fp64():
    j = JobSpec(256, 25.0, 12.0, 400, seed=31, raster_n=4, outputs=FEM)
    ctx = msf.Context(precision="fp64", batch=8)
    spec = ctx.specimen(j.grid, j.pos, j.z)
    fused = ctx.run(spec, j.optics, j.raster, j.detect, want_final_psi=True)
    plain = ctx.run_plain(spec, j.optics, j.raster, j.detect, want_final_psi=True)
    assert plain.probe_slices == fused.probe_slices
    np.testing.assert_allclose(plain.adf_image, fused.adf_image, rtol=1e-11)
    for m, v in fused.v.items():
        np.testing.assert_allclose(plain.v[m], v, rtol=1e-9, atol=1e-12, err_msg=m)
    a, b = plain.final_psi, fused.final_psi
    assert np.abs(a - b).max() <= 1e-11 * np.abs(b).max()


def test_plain_rejects_fp32_context():
    j = JobSpec(128, 12.5, 8.0, 80, seed=32, raster_n=2)
    ctx = msf.Context(precision="fp32")
    spec = ctx.specimen(j.grid, j.pos, j.z)
    with pytest.raises(msf.MsfError):
        ctx.run_plain(spec, j.optics, j.raster, j.detect)


def test_plain_matches_reference_with_mtf(golden_tmp):
    """The plain path with the detector MTF against the reference's own run
    (golden case 'mtf', made through a parameter file)."""
    from conftest import assert_variance_close, case_argv, case_dir, load_case, rel_err
    meta, ref = load_case("mtf")
    job = msf.Job(case_argv("mtf", case_dir("mtf", golden_tmp)))
    assert job.detect.n_mtf > 0
    ctx = msf.Context(precision="fp64")
    q, z = job.positions()
    spec = ctx.specimen(job.grid, q, z)
    r = ctx.run_plain(spec, job.optics, job.raster, job.detect)
    assert rel_err(r.adf_image, ref["adf_image"]).max() <= 1e-5
    for mode in ("V_omega", "V_re", "Omega_vimage"):
        assert_variance_close(r.v[mode], ref[mode][:, 1], 1e-5, 1e-12, what=mode)
