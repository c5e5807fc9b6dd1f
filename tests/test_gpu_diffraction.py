"""Diffraction patterns the drop-in CLI writes with --images (write_tif.cpp
output_diffraction): the first probe's exit wave at five scale factors, the
last probe's (after the detector MTF when one is given) and, with FEM pixel
modes, the raster means of |psi(k)| and |psi(k)|^2 and the 2-D variance,
compared pixel by pixel with the reference's own TIFFs from the golden runs.
log(1 + s x^2) is min/max scaled to 16 bits, so FP64 rounding moves a pixel
by at most one level."""
import subprocess
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, case_dir, load_case

sys.path.insert(0, str(GOLDEN))
from tif16 import read_tif16  # noqa: E402

pytestmark = pytest.mark.gpu


def run_cli(name, golden_tmp):
    meta, ref = load_case(name)
    d = case_dir(name, golden_tmp)
    cli = ROOT / "ms-stem-fem_b200" / "bin" / "ms-stem-fem"
    p = subprocess.run([str(cli)] + meta["argv"] + ["--precision", "fp64"], cwd=d,
                       capture_output=True, text=True)
    assert p.returncode == 0, p.stdout + p.stderr
    return meta, ref, d


def compare(meta, ref, d, keys):
    for key in keys:
        tag, scale = key.split("_diffraction_")
        f = d / ("%s_%s_diffraction_scalefactor_%s.tif" % (meta["prefix"], tag, scale))
        got = read_tif16(f).astype(int)
        want = ref[key].astype(int)
        assert got.shape == want.shape, key
        diff = np.abs(got - want)
        assert diff.max() <= 1, (key, int(diff.max()), int((diff > 1).sum()))


@pytest.mark.parametrize("name", ["c1", "fem128", "mtf", "xyz"])
def test_cli_diffraction_images_match_reference(name, golden_tmp):
    meta, ref, d = run_cli(name, golden_tmp)
    keys = [k for k in ref if k.startswith(("first_diffraction_", "final_diffraction_"))]
    assert len(keys) == 6, keys
    compare(meta, ref, d, keys)


@pytest.mark.parametrize("name", ["fem128", "mtf"])
def test_cli_fem_average_diffraction_match_reference(name, golden_tmp):
    meta, ref, d = run_cli(name, golden_tmp)
    keys = [k for k in ref if k.startswith(("diffracted_wave_", "variance_2-D_"))]
    assert len(keys) == 4, keys
    compare(meta, ref, d, keys)
