"""Host-side logic of the product, CPU only: the C ABI loads and exports every
declared symbol; the drop-in parser, defaults and quirks; bit-exact slicing,
probe snaps and ring bins against the oracle and the reference fixtures."""
import re
from pathlib import Path

import numpy as np
import pytest

import msf
import oracle
from conftest import ROOT, case_argv, case_dir, golden_cases, load_case


def declared_functions():
    text = (ROOT / "include" / "msf.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(msf_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = msf.lib()
    declared = declared_functions()
    assert len(declared) >= 25
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(msf.EXPORTED)
    header = (ROOT / "include" / "msf.h").read_text()
    abi = int(re.search(r"#define MSF_ABI_VERSION (\d+)", header).group(1))
    assert lib.msf_abi_version() == abi == msf.ABI_VERSION


@pytest.mark.parametrize("name", golden_cases())
def test_parse_matches_oracle_derivation(name, golden_tmp):
    meta, ref = load_case(name)
    d = case_dir(name, golden_tmp)
    argv = case_argv(name, d)
    job = msf.Job(argv)
    ojob, q_or, z_or = oracle.job_from_argv(meta["argv"], d)
    assert job.grid.nx == ojob["nx"] and job.grid.ny == ojob["ny"]
    mj = job.oracle_job()
    for k in ("voltage", "xperiod", "yperiod", "xperiod_duped", "yperiod_duped", "min_slice",
              "cs3", "cs5", "defocus", "alpha_max", "det_inner", "det_outer", "dr"):
        assert mj[k] == ojob[k], k  # bit-exact
    np.testing.assert_array_equal(mj["x_p"], ojob["x_p"])
    np.testing.assert_array_equal(mj["y_p"], ojob["y_p"])
    assert sorted(mj["fem_modes"]) == sorted(ojob["fem_modes"])
    assert mj["images"] == ojob["images"]
    assert job.prefix == meta["prefix"]


@pytest.mark.parametrize("name", golden_cases())
def test_slicing_bit_exact(name, golden_tmp):
    meta, ref = load_case(name)
    d = case_dir(name, golden_tmp)
    ojob, q, z = oracle.job_from_argv(meta["argv"], d)
    sl = msf.slice_atoms(q, ojob["min_slice"])
    assert np.array_equal(sl["lower"], ref["slice_lower"])
    assert np.array_equal(sl["thickness"], ref["slice_thickness"])
    assert np.array_equal(sl["counts"], ref["slice_count"].astype(np.int64))


@pytest.mark.parametrize("name", ["fem128", "rect", "c1", "dupe"])
def test_probe_shifts_and_ring_bins_bit_exact(name, golden_tmp):
    meta, _ = load_case(name)
    d = case_dir(name, golden_tmp)
    argv = case_argv(name, d)
    job = msf.Job(argv)
    oj = job.oracle_job()
    sh = np.zeros(2 * job.n_probes, dtype=np.int64)
    msf._check(msf.lib().msf_probe_shifts(msf.C.byref(job.grid), msf.C.byref(job.raster),
                                          sh.ctypes.data_as(msf._lp)))
    # oracle: the reference's search with the shift carried between probes
    nx, ny = oj["nx"], oj["ny"]
    xx = np.array([0.0 + (i * (oj["xperiod_duped"] / nx)) for i in range(nx)])
    yy = np.array([0.0 + (i * (oj["yperiod_duped"] / ny)) for i in range(ny)])
    snap = oracle.lib().or_snap
    sx = sy = 0
    k = 0
    for xp in oj["x_p"]:
        for yp in oj["y_p"]:
            sx = snap(xx.ctypes.data_as(oracle._dp), nx, xp, 0.5 * (xx[1] - xx[0]), sx)
            sy = snap(yy.ctypes.data_as(oracle._dp), ny, yp, 0.5 * (yy[1] - yy[0]), sy)
            assert (sh[2 * k], sh[2 * k + 1]) == (sx, sy)
            k += 1
    bins = np.zeros(nx * ny, dtype=np.int32)
    nk = msf.C.c_int32()
    msf._check(msf.lib().msf_ring_bins(msf.C.byref(job.grid), job.detect.dr,
                                       bins.ctypes.data_as(msf._ip), msf.C.byref(nk)))
    ob = oracle.ring_bins(oj)
    assert nk.value == ob["n_k"]
    assert np.array_equal(bins, ob["bins"])


def _run_parse(argv):
    try:
        msf.Job(argv)
        return None
    except msf.MsfError as e:
        return str(e)


def test_parser_quirks_and_failures(golden_tmp):
    d = case_dir("fem128", golden_tmp)
    spec = str(d / "fem128.data")
    base = ["-a", spec, "--output_prefix", str(d / "x"), "-m", "128", "128", "200000",
            "--cs3", "1.3e7", "--scherzer_defocus", "--alphamax", "0.01"]
    assert _run_parse(base + ["--adfstemuncorr"]) is None
    # no simulation mode
    assert "no simulation mode" in _run_parse(base)
    # --detectorangles reads its first number twice and consumes one argument,
    # so the second number is an unexpected argument (tem_io.cpp:5529-5545)
    err = _run_parse(base + ["--adfstemuncorr", "--detectorangles", "0.04", "0.2"])
    assert "unexpected argument : 0.2" in err
    # one number followed by another option: inner == outer == that number
    j = msf.Job(base + ["--detectorangles", "0.03", "--adfstemuncorr"])
    assert j.detect.det_inner == 0.03 and j.detect.det_outer == 0.03
    # an inner angle beyond the band limit is rejected (tem.cpp:714-725)
    assert "beyond bandwidth" in _run_parse(base + ["--detectorangles", "0.05", "--adfstemuncorr"])
    # uncorrected without --cs3
    err = _run_parse(["-a", spec, "--output_prefix", "x", "-m", "128", "128", "200000",
                      "--adfstemuncorr", "--scherzer_defocus", "--alphamax", "0.01"])
    assert "lacking required parameters" in err
    # corrected needs --cs5
    err = _run_parse(base + ["--adfstemcorr"])
    assert "lacking required parameters" in err
    # both modes
    assert "either aberration corrected or uncorrected" in _run_parse(
        base + ["--adfstemcorr", "--adfstemuncorr", "--cs5", "1e7"])
    # unknown option
    assert "unexpected argument : --bogus" in _run_parse(base + ["--adfstemuncorr", "--bogus"])
    # missing specimen file
    err = _run_parse(["-a", str(d / "missing.data")] + base[2:] + ["--adfstemuncorr"])
    assert "Error opening position file" in err
    # defaults: detector 40-200 mrad at 200 kV, raster 1.5 A (STEM) / 10 A (FEM)
    j = msf.Job(base + ["--adfstemuncorr"])
    assert (j.detect.det_inner, j.detect.det_outer) == (0.040, 0.200)
    assert j.raster.n_x == int(np.floor(25.0 / 1.5))
    j = msf.Job(base + ["--adfstemuncorrfem"])
    assert j.raster.n_x == int(np.floor(25.0 / 10))
    assert j.fem_modes() == ["V_omega"]  # default FEM mode
    # at 100 kV the default detector is 45-200 mrad
    j = msf.Job(["-a", spec, "--output_prefix", "x", "-m", "128", "128", "100000",
                 "--cs3", "1.3e7", "--scherzer_defocus", "--alphamax", "0.01", "--adfstemuncorr"])
    assert (j.detect.det_inner, j.detect.det_outer) == (0.045, 0.200)


def test_parameter_file(golden_tmp):
    d = case_dir("fem128", golden_tmp)
    pf = d / "params.txt"
    pf.write_text("\n".join([
        "output_prefix " + str(d / "pf"), "model_file " + str(d / "fem128.data"),
        "samples_x 128", "samples_y 128", "microscope_voltage 200000",
        "cs3 1.3e7", "scherzer_defocus", "alphamax 0.010", "raster_spacing 6.25",
        "minslice 2.0", "adfstemuncorrfem", "V_re", "detectorangles 0.2 0.03", "", "images"]) + "\n")
    j = msf.Job(["--parameter_file", str(pf), "-a", str(d / "fem128.data")])
    assert j.grid.nx == 128 and j.raster.n_x == 4
    assert j.fem_modes() == ["V_re"]
    assert (j.detect.det_inner, j.detect.det_outer) == (0.03, 0.2)  # swapped
    assert j.detect.outputs & msf.OUT_ADF_IMAGE
    # the -m flag is re-derived from the file: without samples_* it fails
    pf2 = d / "params2.txt"
    pf2.write_text("cs3 1.3e7\n")
    err = _run_parse(["-a", str(d / "fem128.data"), "--output_prefix", "x", "-m", "128", "128",
                      "200000", "--parameter_file", str(pf2), "--adfstemuncorr",
                      "--scherzer_defocus", "--alphamax", "0.01"])
    assert "lacking required parameters" in err


def test_mtf_file(golden_tmp, tmp_path):
    """mtf_file / mtf_sampling_rate (tem_io.cpp:4214-4262, 5371-5440, 5722-5857;
    tem.cpp:276-285): domain on line 1, MTF on line 2, domain rescaled to
    (0.5 res d)^2; the CLI option reads the file without consuming its name."""
    d = case_dir("fem128", golden_tmp)
    spec = str(d / "fem128.data")
    (tmp_path / "m.csv").write_text("0, 0.5, 1.0\n1.0, 0.6, 0.2\n")
    (tmp_path / "m.param").write_text("mtf_file %s\nmtf_sampling_rate 20\n" % (tmp_path / "m.csv"))
    base = ["-a", spec, "--output_prefix", str(d / "x"), "--parameter_file",
            str(tmp_path / "m.param"), "-m", "128", "128", "200000", "--cs3", "1.3e7",
            "--scherzer_defocus", "--alphamax", "0.01", "--adfstemuncorrfem"]
    j = msf.Job(base)
    det = j.detect
    assert det.n_mtf == 3 and det.mtf_resolution == 20
    assert [det.mtf[k] for k in range(3)] == [1.0, 0.6, 0.2]
    assert [det.mtf_domain_sqr[k] for k in range(3)] == [(0.5 * 20 * v) ** 2
                                                        for v in (0.0, 0.5, 1.0)]
    # without a sampling rate the MTF is off and the run is refused (flags differ)
    (tmp_path / "m2.param").write_text("mtf_file %s\n" % (tmp_path / "m.csv"))
    base2 = list(base)
    base2[base2.index(str(tmp_path / "m.param"))] = str(tmp_path / "m2.param")
    assert "lacking required parameters" in _run_parse(base2)
    # CLI: the file name is left behind as an unexpected argument
    err = _run_parse(["-a", spec, "--output_prefix", "x", "-m", "128", "128", "200000",
                      "--cs3", "1.3e7", "--scherzer_defocus", "--alphamax", "0.01",
                      "--adfstemuncorrfem", "--mtf_file", str(tmp_path / "m.csv"),
                      "--mtf_sampling_rate", "20"])
    assert "unexpected argument : " + str(tmp_path / "m.csv") in err
    # unequal lines, a missing second newline, a missing file
    for text in ("0, 0.5\n1.0\n", "0, 0.5\n1.0, 0.5"):
        (tmp_path / "bad.csv").write_text(text)
        (tmp_path / "bad.param").write_text("mtf_file %s\nmtf_sampling_rate 20\n"
                                            % (tmp_path / "bad.csv"))
        b = list(base)
        b[b.index(str(tmp_path / "m.param"))] = str(tmp_path / "bad.param")
        assert "could not read MTF file" in _run_parse(b)
    (tmp_path / "none.param").write_text("mtf_file %s\n" % (tmp_path / "none.csv"))
    b = list(base)
    b[b.index(str(tmp_path / "m.param"))] = str(tmp_path / "none.param")
    assert "Error opening MTF file" in _run_parse(b)


def test_lammps_reader_errors(tmp_path):
    good = ["# c", "", "2 atoms", "1 atom types", "", "0 10 xlo xhi", "0 10 ylo yhi",
            "0 10 zlo zhi", "", "Masses", "", "1 28.0855", "", "Atoms", "",
            "1 1 1.0 2.0 3.0", "2 1 4.0 5.0 6.0"]
    p = tmp_path / "g.data"
    p.write_text("\n".join(good) + "\n")
    h = msf.C.c_void_p()
    assert msf.lib().msf_read_specimen(str(p).encode(), msf.C.byref(h)) == 0
    msf.lib().msf_job_destroy(h)
    bad_cases = {
        "outside box": good[:15] + ["1 1 11.0 2.0 3.0", good[16]],
        "unknown mass": good[:11] + ["1 3.3"] + good[12:],
        "missing atoms": good[:16],
        "bad header": good[:2] + ["2 atomz"] + good[3:],
    }
    for what, lines in bad_cases.items():
        p.write_text("\n".join(lines) + "\n")
        rc = msf.lib().msf_read_specimen(str(p).encode(), msf.C.byref(h))
        assert rc != 0, what


def test_guess_z_table_matches_reference_rules(tmp_path):
    # a handful of the reference's mass rules (tem_io.cpp:1030-1258),
    # including its quirks: Ar accepts exactly 36.0, Tm's range is empty
    cases = {28.0855: 14, 15.999: 8, 1.008: 1, 196.97: 79, 36.0: 18, 39.95: 18,
             168.93: 0, 138.0: 69}
    for mass, zexp in cases.items():
        lines = ["# c", "1 atoms", "1 atom types", "0 1 xlo xhi", "0 1 ylo yhi",
                 "0 1 zlo zhi", "Masses", "1 %r" % mass, "Atoms", "1 1 0.5 0.5 0.5"]
        p = tmp_path / "m.data"
        p.write_text("\n".join(lines) + "\n")
        h = msf.C.c_void_p()
        rc = msf.lib().msf_read_specimen(str(p).encode(), msf.C.byref(h))
        if zexp == 0:
            assert rc != 0, mass
            continue
        assert rc == 0, mass
        atoms = msf.Atoms()
        msf.lib().msf_job_describe(h, None, msf.C.byref(atoms), None, None, None)
        assert atoms.z[0] == zexp, mass
        msf.lib().msf_job_destroy(h)
