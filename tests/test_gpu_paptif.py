"""--paptif (slice.cpp:1660-1690, func.cpp:2024-2362): the drop-in CLI's
per-slice 16-bit images of the projected potential before the exponential,
against the reference's own TIFFs from the golden run.  Magnitude and real
part, linear and log-scaled, must agree pixel by pixel within one 16-bit
level (FP64 rounding of the potential sum or its FFT-convolution form can
move a pixel across a rounding boundary).  The reference's imaginary-part
images scale by an uninitialised min / max and are not defined; here they
are checked against the stated convention (min / max over the slice, both
files log-scaled) applied to the potential the library returns."""
import subprocess
import sys

import numpy as np
import pytest

import msf
from conftest import GOLDEN, ROOT, case_argv, case_dir, load_case

sys.path.insert(0, str(GOLDEN))
from tif16 import read_tif16  # noqa: E402

pytestmark = pytest.mark.gpu


def log16(a, mn, mx):
    # a constant slice (mx == mn, e.g. an imaginary part that is zero
    # everywhere) gives 0 / 0 here and maps to level 0, as the writer does
    with np.errstate(invalid="ignore", divide="ignore"):
        v = np.log(a - mn + 1.0) / np.log(mx - mn + 1.0)
    return np.where(v > 0, np.floor(v * 65535.0 + 0.5), 0).astype(np.int64)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_paptif_images_match_reference(precision, golden_tmp):
    meta, ref = load_case("paptif")
    d = case_dir("paptif", golden_tmp)
    cli = ROOT / "ms-stem-fem_b200" / "bin" / "ms-stem-fem"
    p = subprocess.run([str(cli)] + meta["argv"] + ["--precision", precision], cwd=d,
                       capture_output=True, text=True)
    assert p.returncode == 0, p.stdout + p.stderr
    keys = sorted(k for k in ref if k.startswith("pap_"))
    n_slices = len(ref["slice_lower"])
    assert len(keys) == 4 * n_slices, keys
    for k in keys:
        got = read_tif16(d / ("paptif_" + k + ".tif")).astype(int)
        want = ref[k].astype(int)
        assert got.shape == want.shape, k
        diff = np.abs(got - want)
        assert diff.max() <= 1, (k, int(diff.max()), int((diff > 1).sum()))
    # imaginary part: the convention, from the library's potential
    job = msf.Job(case_argv("paptif", d))
    q, z = job.positions()
    ctx = msf.Context(precision=precision)
    ctx.keep_potentials()
    spec = ctx.specimen(job.grid, q, z)
    for s in range(n_slices):
        im = spec.potential(s)[..., 1]
        want = log16(im, im.min(), im.max())[::-1]  # the file stores rows bottom-up
        for tail in ("im", "im_logscale"):
            got = read_tif16(d / ("paptif_pap_slice%d_1_complex_fftw_operand_%s.tif"
                                  % (s + 1, tail))).astype(np.int64)
            assert np.abs(got - want).max() <= 1, (s, tail)
