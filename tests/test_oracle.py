"""The CPU oracle against the golden fixtures made by the reference's own
code (tests/golden/make_golden.py).  Pins the oracle before it is used to
check the CUDA path.  CPU only."""
import numpy as np
import pytest

import oracle
from conftest import assert_variance_close, case_dir, load_case, rel_err

SMALL = ["fem128", "corr", "rect", "sio", "dupe", "c1", "xyz"]


@pytest.mark.parametrize("name", SMALL)
def test_oracle_matches_reference(name, golden_tmp):
    meta, ref = load_case(name)
    d = case_dir(name, golden_tmp)
    job, q, z = oracle.job_from_argv(meta["argv"], d)
    out = oracle.run(job, q, z)
    # slicing is bit-exact (slice.cpp:469-980)
    sl = oracle.slice_atoms(q, job["min_slice"])
    assert np.array_equal(sl["lower"], ref["slice_lower"])
    assert np.array_equal(sl["thickness"], ref["slice_thickness"])
    assert np.array_equal(np.diff(sl["start"]), ref["slice_count"].astype(int))
    if "adf_image" in ref:
        assert rel_err(out["adf_image"].ravel(), ref["adf_image"]).max() <= 1e-12
    for mode in oracle.MODE_BITS:
        if mode in ref:
            np.testing.assert_allclose(out["k_lower"], ref[mode][:, 0], rtol=1e-10, atol=0)
            # the reference's text has 10 significant digits
            assert_variance_close(out[mode], ref[mode][:, 1], rtol=2e-10, atol=1e-14,
                                  what=name + " " + mode)
    if "transmission" in ref:
        s = int(ref["transmission_slice"])
        t = oracle.transmission(job, q, z, s).ravel()
        assert np.abs(t - ref["transmission"]).max() <= 1e-13


def test_oracle_constants():
    lam, gam = oracle.C.c_double(), oracle.C.c_double()
    oracle.lib().or_constants(200000.0, oracle.C.byref(lam), oracle.C.byref(gam))
    assert abs(lam.value - 0.0250798) < 1e-7 and abs(gam.value - 1.39141) < 1e-5
    oracle.lib().or_constants(300000.0, oracle.C.byref(lam), oracle.C.byref(gam))
    assert abs(lam.value - 0.0196878) < 1e-7


def test_oracle_snap_quirks():
    grid = np.arange(8, dtype=float)  # pixel centres 0..7, spacing 1
    g = grid.ctypes.data_as(oracle._dp)
    snap = oracle.lib().or_snap
    assert snap(g, 8, 2.4, 0.5, 0) == 2     # nearest pixel
    assert snap(g, 8, 2.5, 0.5, 0) == 2     # half rounds down: 3-2.5 >= 0.5
    assert snap(g, 8, 7.6, 0.5, 5) == 5     # no pixel matches: fallback kept
    assert snap(g, 8, -0.6, 0.5, 0) == -1   # size_t wrap in the reference
