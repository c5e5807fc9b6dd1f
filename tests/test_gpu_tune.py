"""Launch tiling autotuner (msf_tune) and its wisdom text: the tuned tiling
is one of the candidates, survives an export / import round trip on the same
device model, is ignored for another model, and changes no result (a probe's
arithmetic does not depend on its launch companions)."""
import subprocess

import numpy as np
import pytest

import msf
from conftest import ROOT, case_dir, load_case
from test_gpu_slots import JobSpec

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_tune_picks_a_candidate_and_keeps_results(precision):
    j = JobSpec(256, 25.0, 14.0, 400, seed=51, raster_n=6)
    ctx = msf.Context(precision=precision)
    spec = ctx.specimen(j.grid, j.pos, j.z)
    before = ctx.run(spec, j.optics, j.raster, j.detect)
    t = ctx.tune(spec)
    assert (t["nx"], t["ny"]) == (256, 256)
    assert t["batch"] in (8, 16, 32, 64, 128, 256)
    fp32_pipes = (0, 1, 4, 5, 8, 9, 12, 13, 16, 17, 24, 25, 32, 33, 48, 49, 80, 81, 112, 113)
    assert t["pipe"] in (fp32_pipes if precision == "fp32" else (0, 1))
    assert t["ns_per_probe_slice"] > 0
    after = ctx.run(spec, j.optics, j.raster, j.detect)
    assert np.array_equal(after.adf_image, before.adf_image)
    for m in ("V_omega", "Vbar_r"):
        assert np.array_equal(after.v[m], before.v[m], equal_nan=True), m
    for m in ("V_re", "V_gt17"):
        np.testing.assert_allclose(after.v[m], before.v[m], rtol=1e-12, equal_nan=True)


def test_wisdom_round_trip():
    j = JobSpec(128, 12.5, 10.0, 80, seed=52, raster_n=3)
    ctx = msf.Context(precision="fp32")
    spec = ctx.specimen(j.grid, j.pos, j.z)
    t = ctx.tune(spec)
    text = ctx.wisdom_export()
    lines = text.strip().splitlines()
    assert len(lines) == 1 and lines[0].startswith("msf-wisdom 1 ")
    f = lines[0].split()
    assert f[3] == "fp32" and (int(f[4]), int(f[5]), int(f[6])) == (128, 128, t["batch"])
    other = msf.Context(precision="fp32")
    assert other.wisdom_import(text) == 1
    assert other.wisdom_export().split()[:8] == f[:8]
    f2 = list(f)
    f2[2] = "not_this_gpu"
    assert msf.Context(precision="fp32").wisdom_import(" ".join(f2) + "\n") == 0
    assert msf.Context(precision="fp64").wisdom_import(text) == 0


def test_cli_writes_and_reuses_wisdom(golden_tmp, tmp_path):
    meta, _ = load_case("fem128")
    d = case_dir("fem128", tmp_path)
    cli = ROOT / "ms-stem-fem_b200" / "bin" / "ms-stem-fem"
    for _ in range(2):
        p = subprocess.run([str(cli)] + meta["argv"], cwd=d, capture_output=True, text=True)
        assert p.returncode == 0, p.stdout + p.stderr
        w = (d / "msf_wisdom_128x128_fp64").read_text()
        assert w.startswith("msf-wisdom 1 ") and " fp64 128 128 " in w


def test_run_reports_pass_times_of_its_first_batch():
    """msf_run times the passes of its first batch with CUDA events: both
    means are positive and the batch is the context's probes per launch."""
    j = JobSpec(256, 25.0, 14.0, 400, seed=53, raster_n=6)
    ctx = msf.Context(precision="fp32", batch=16)
    spec = ctx.specimen(j.grid, j.pos, j.z)
    r = ctx.run(spec, j.optics, j.raster, j.detect)
    assert spec.slices()["n"] >= 3
    assert r.pass_batch == 16
    assert r.ms_row_pass > 0 and r.ms_col_pass > 0
    assert r.ms_row_pass + r.ms_col_pass < 1e3 * r.seconds_raster


def test_kernel_attributes_are_set_on_every_device():
    """Large-shared-memory launches (FP64 2048-point passes) on a second
    device after the first: the dynamic shared-memory limit is raised per
    device, so both runs succeed and agree.  Needs two visible GPUs."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    lam, _ = msf.wavelength(300000.0)
    g = msf.Grid(nx=2048, ny=2048, voltage=300000.0, xperiod=200.0, yperiod=200.0,
                 zperiod=10.0, dupe_x=1, dupe_y=1, dupe_z=1, replicate_atoms=0, min_slice=2.0)
    o = msf.Optics(corrected=0, cs3=1.3e7, cs5=0.0, defocus=0.87 * np.sqrt(1.3e7 * lam),
                   alpha_max=0.0084)
    probes = []
    for dev in (0, 1, 0):
        ctx = msf.Context(device=dev, precision="fp64")
        spec = ctx.specimen(g, np.zeros((0, 3)), np.zeros(0, dtype=np.uint32))
        probes.append(ctx.probe(spec, o))
        spec.close()
        ctx.close()
    assert np.array_equal(probes[0], probes[1]) and np.array_equal(probes[0], probes[2])
