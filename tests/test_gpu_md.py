"""ms-stem-fem-md on the GPU: the drop-in driver against the reference's own
MD-coupled runs (golden fixtures from ftem_lammps.cpp with its LAMMPS
replaced by a replay of the same data files), and the properties of
msf_run_md that hold exactly.  Tolerances as the plain driver's: ADF and
V(k) within 1e-5 relative (FP64) and 1e-4 (FP32); diffraction TIFFs within
one 16-bit level."""
import subprocess
import sys

import numpy as np
import pytest

import msf
import oracle
from conftest import (GOLDEN, ROOT, assert_variance_close, case_dir, golden_cases,
                      load_case, rel_err)
from test_gpu_slots import JobSpec

sys.path.insert(0, str(GOLDEN))
from tif16 import read_tif16  # noqa: E402

pytestmark = pytest.mark.gpu

CLI_MD = ROOT / "ms-stem-fem_b200" / "bin" / "ms-stem-fem-md"
TOL = {"fp64": (1e-5, 1e-5, 1e-12), "fp32": (1e-4, 1e-4, 1e-7)}
MODES = ["V_omega", "Vbar_r", "V_re", "Omega_vimage", "V_gt17", "V_rbar"]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", golden_cases(md=True))
def test_md_cli_matches_reference(name, precision, golden_tmp, tmp_path):
    meta, ref = load_case(name)
    d = case_dir(name, tmp_path)
    p = subprocess.run([str(CLI_MD)] + meta["argv"] + meta["md_argv_extra"] +
                       ["--precision", precision], cwd=d, capture_output=True, text=True)
    assert p.returncode == 0, p.stdout + p.stderr
    adf_tol, v_rtol, v_atol = TOL[precision]
    img = np.fromfile(d / (meta["prefix"] + "_stem_image_output.f64"))
    err = rel_err(img, ref["adf_image"]).max()
    print("%s %s ADF max rel err %.3e" % (name, precision, err))
    assert err <= adf_tol
    for mode in MODES:
        if mode in ref:
            t = oracle.read_variance_txt(d / (meta["prefix"] + "_fem_%s.txt" % mode))
            np.testing.assert_allclose(t[:, 0], ref[mode][:, 0], rtol=1e-9)
            assert_variance_close(t[:, 1], ref[mode][:, 1], v_rtol, v_atol,
                                  what="%s %s %s" % (name, precision, mode))
    crtol, catol = {"fp64": (1e-8, 1e-9), "fp32": (1e-4, 1e-5)}[precision]
    for key, scale in (("correlograph_avg", 1), ("correlograph_variance", 2)):
        if key in ref:
            t = np.loadtxt(d / (meta["prefix"] + "_" + key + ".txt"), ndmin=2)
            want = ref[key]
            assert t.shape == want.shape, key
            np.testing.assert_array_equal(t[0], want[0])  # phi boundaries
            err = np.abs(t[1:, 1:] - want[1:, 1:])
            assert (err <= scale * crtol * np.abs(want[1:, 1:]) + scale * 10 * catol).all(), key
    if precision == "fp64":
        keys = [k for k in ref if "_diffraction_" in k]
        assert keys
        for key in keys:
            tag, scale = key.split("_diffraction_")
            got = read_tif16(d / ("%s_%s_diffraction_scalefactor_%s.tif" %
                                  (meta["prefix"], tag, scale))).astype(int)
            assert np.abs(got - ref[key].astype(int)).max() <= 1, key


def job(seed=31, n_atoms=120):
    return JobSpec(128, 12.5, 16.0, n_atoms, seed=seed, raster_n=4,
                   outputs=msf.OUT_ADF_IMAGE | msf.OUT_V_OMEGA | msf.OUT_VBAR_R |
                   msf.OUT_V_RE | msf.OUT_V_GT17)


def jittered(j, seed):
    rng = np.random.default_rng(seed)
    pos = j.pos + rng.normal(0.0, 0.1, j.pos.shape)
    pos[:, :2] %= 12.5
    return pos


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_one_sample_equals_plain_raster(precision):
    """psi / 1 and I / 1 are exact: one sample of one snapshot is msf_run."""
    j = job()
    ctx = msf.Context(precision=precision, batch=8)
    spec = ctx.specimen(j.grid, j.pos, j.z)
    a = ctx.run(spec, j.optics, j.raster, j.detect)
    b = ctx.run_md([spec], 1, j.optics, j.raster, j.detect)
    assert np.array_equal(a.adf_image, b.adf_image)
    for m in a.v:
        assert np.array_equal(a.v[m], b.v[m], equal_nan=True), m
    assert b.probe_slices == a.probe_slices


def test_samples_cycle_through_snapshots():
    """Sample s uses snapshot s mod K: three snapshots over six samples equal
    the six-entry list that repeats them; the average differs from any
    single snapshot."""
    j = job()
    ctx = msf.Context(precision="fp32", batch=8)
    snaps = [ctx.specimen(j.grid, p, j.z) for p in (j.pos, jittered(j, 1), jittered(j, 2))]
    a = ctx.run_md(snaps, 6, j.optics, j.raster, j.detect)
    b = ctx.run_md(snaps + snaps, 6, j.optics, j.raster, j.detect)
    assert np.array_equal(a.adf_image, b.adf_image)
    for m in a.v:
        assert np.array_equal(a.v[m], b.v[m], equal_nan=True), m
    c = ctx.run(snaps[0], j.optics, j.raster, j.detect)
    assert not np.allclose(a.v["V_omega"], c.v["V_omega"], rtol=1e-6, equal_nan=True)


def test_md_batching_does_not_change_results():
    j = job()
    outs = []
    for batch in (1, 5, 16):
        ctx = msf.Context(precision="fp32", batch=batch)
        snaps = [ctx.specimen(j.grid, p, j.z) for p in (j.pos, jittered(j, 3))]
        outs.append(ctx.run_md(snaps, 2, j.optics, j.raster, j.detect))
    for o in outs[1:]:
        assert np.array_equal(o.adf_image, outs[0].adf_image)
        for m in o.v:
            np.testing.assert_allclose(o.v[m], outs[0].v[m], rtol=1e-12, equal_nan=True)


def test_md_argument_checks():
    j = job()
    ctx = msf.Context(precision="fp32")
    a = ctx.specimen(j.grid, j.pos, j.z)
    with pytest.raises(msf.MsfError):
        ctx.run_md([a, a], 3, j.optics, j.raster, j.detect)  # 3 % 2 != 0
    other = msf.Grid.from_buffer_copy(j.grid)
    other.xperiod = 13.0
    b = ctx.specimen(other, j.pos, j.z)
    with pytest.raises(msf.MsfError):
        ctx.run_md([a, b], 2, j.optics, j.raster, j.detect)
