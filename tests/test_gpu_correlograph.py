"""FEM correlograph (--correlograph*, adfstem.cpp:2603-2685, 3617-3760)
against the reference's own text outputs (golden case 'corrgraph'): the
raster average, the squared sums written by --correlograph_variance, and
every probe's table.  Tolerance: 1e-8 relative on the FP64 path, 1e-4 on the
FP32 path, with an absolute floor for cells at the ratio's threshold."""
import subprocess

import numpy as np
import pytest

import msf
import oracle
from conftest import ROOT, case_argv, case_dir, load_case

pytestmark = pytest.mark.gpu

TOL = {"fp64": (1e-8, 1e-9), "fp32": (1e-4, 1e-5)}


def close(got, want, rtol, atol, what):
    assert got.shape == want.shape, (what, got.shape, want.shape)
    err = np.abs(got - want)
    lim = rtol * np.abs(want) + atol
    assert (err <= lim).all(), (what, float((err / lim).max()))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_cli_correlograph_outputs(precision, golden_tmp):
    meta, ref = load_case("corrgraph")
    d = case_dir("corrgraph", golden_tmp)
    cli = ROOT / "ms-stem-fem_b200" / "bin" / "ms-stem-fem"
    p = subprocess.run([str(cli)] + meta["argv"] + ["--precision", precision], cwd=d,
                       capture_output=True, text=True)
    assert p.returncode == 0, p.stdout + p.stderr
    pre = d / meta["prefix"]
    rtol, atol = TOL[precision]
    avg = np.loadtxt(str(pre) + "_correlograph_avg.txt", ndmin=2)
    np.testing.assert_array_equal(avg[0], ref["correlograph_avg"][0])  # phi boundaries
    np.testing.assert_allclose(avg[1:, 0], ref["correlograph_avg"][1:, 0], rtol=1e-10)
    close(avg[1:, 1:], ref["correlograph_avg"][1:, 1:], rtol, atol, "avg")
    sqr = np.loadtxt(str(pre) + "_correlograph_variance.txt", ndmin=2)
    close(sqr[1:, 1:], ref["correlograph_variance"][1:, 1:], 2 * rtol, 10 * atol, "sqr sums")
    n = 0
    for key in ref:
        if key.startswith("correlograph_probe_"):
            px, py = key.split("_")[-2:]
            t = np.loadtxt("%s_%s_%s.txt" % (pre, px, py), ndmin=2)
            close(t[1:, 1:], ref[key][1:, 1:], rtol, atol, key)
            assert (d / ("%s_%s_%s.tif" % (meta["prefix"], px, py))).exists()
            n += 1
    assert n == 16
    for suffix in ("_correlograph_avg.tif", "_correlograph_variance.tif",
                   "_correlograph_variance_logscale.tif"):
        assert (d / (meta["prefix"] + suffix)).read_bytes()[:4] == b"II*\x00", suffix
    t = oracle.read_variance_txt(str(pre) + "_fem_V_omega.txt")
    np.testing.assert_allclose(t[:, 1], ref["V_omega"][:, 1], rtol=1e-4 if precision == "fp32"
                               else 1e-5, atol=1e-12)


def test_api_correlograph_matches_cli_reference(golden_tmp):
    meta, ref = load_case("corrgraph")
    job = msf.Job(case_argv("corrgraph", case_dir("corrgraph", golden_tmp)))
    assert job.detect.outputs & msf.OUT_CORRELOGRAPH
    ctx = msf.Context(precision="fp32")
    q, z = job.positions()
    spec = ctx.specimen(job.grid, q, z)
    r = ctx.run(spec, job.optics, job.raster, job.detect, want_correlograph_probes=True)
    close(r.correlograph, ref["correlograph_avg"][1:, 1:], 1e-4, 1e-5, "avg")
    close(r.correlograph_probes[1 * 4 + 2], ref["correlograph_probe_1_2"][1:, 1:], 1e-4, 1e-5,
          "probe 1 2")
    # the text holds 10 significant digits
    np.testing.assert_allclose(r.phi_lower[:-1], ref["correlograph_avg"][0, 1:], rtol=1e-9)
