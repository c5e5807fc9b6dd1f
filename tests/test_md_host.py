"""ms-stem-fem-md (the MD-coupled FEM driver) on the CPU: the golden runs of
the reference's own ftem_lammps.cpp (its LAMMPS replaced by a replay of data
files) against the oracle, and the drop-in driver's argument handling up to
the point where it needs a GPU.

With --lammps_TEM_steps 0 nothing runs between samples, so every sample sees
the initial configuration: psi / 2 + psi / 2 and I / 2 + I / 2 are exact in
FP64, and the MD driver's outputs equal the plain raster of that
configuration (computed here by the C oracle)."""
import subprocess

import numpy as np
import pytest

import oracle
from conftest import (ROOT, assert_variance_close, case_dir, golden_cases, load_case,
                      rel_err)

CLI_MD = ROOT / "ms-stem-fem_b200" / "bin" / "ms-stem-fem-md"
CLI = ROOT / "ms-stem-fem_b200" / "bin" / "ms-stem-fem"


def test_md_cases_present():
    assert golden_cases(md=True) == ["md", "md_mtf", "md_static"]


def plain_argv(meta):
    """The case's argv for ms-stem-fem: the LAMMPS options dropped."""
    out, skip = [], 0
    for a in meta["argv"]:
        if skip:
            skip -= 1
            continue
        if a in ("--lammps_preTEM_file_name", "--lammps_TEM_steps", "--lammps_TEM_samples"):
            skip = 1
            continue
        out.append(a)
    return out


def test_static_md_equals_plain_raster_oracle(golden_tmp):
    meta, ref = load_case("md_static")
    d = case_dir("md_static", golden_tmp)
    ojob, q, z = oracle.job_from_argv(plain_argv(meta), d)
    out = oracle.run(ojob, q, z)
    assert rel_err(out["adf_image"].ravel(), ref["adf_image"]).max() <= 1e-10
    for mode in ("V_omega", "Vbar_r"):
        np.testing.assert_allclose(out["k_lower"], ref[mode][:, 0], rtol=1e-12)
        assert_variance_close(out[mode], ref[mode][:, 1], 1e-9, 1e-12, what=mode)


def test_md_samples_change_the_result():
    """The jittered configurations make the coherent average differ from any
    single one: V(k) of the MD case is finite and not all zero."""
    meta, ref = load_case("md")
    assert meta["snapshots"] == 3 and "--lammps_TEM_samples" in meta["argv"]
    v = ref["V_omega"][:, 1]
    assert np.isfinite(v).all() and (v != 0).any()


def run_cli(cli, args, cwd):
    return subprocess.run([str(cli)] + args, cwd=cwd, capture_output=True, text=True,
                          timeout=120)


def test_md_driver_needs_replay_list(golden_tmp):
    meta, _ = load_case("md")
    d = case_dir("md", golden_tmp)
    p = run_cli(CLI_MD, meta["argv"], d)
    assert p.returncode == 1
    assert "--md_replay" in p.stdout + p.stderr


def test_md_driver_samples_multiple_of_snapshots(golden_tmp):
    meta, _ = load_case("md")
    d = case_dir("md", golden_tmp)
    argv = list(meta["argv"])
    argv[argv.index("--lammps_TEM_samples") + 1] = "4"  # 3 snapshots
    p = run_cli(CLI_MD, argv + meta["md_argv_extra"], d)
    assert p.returncode == 1
    assert "multiple" in p.stdout + p.stderr


def test_md_driver_needs_lammps_options(golden_tmp):
    meta, _ = load_case("md_static")
    d = case_dir("md_static", golden_tmp)
    p = run_cli(CLI_MD, plain_argv(meta), d)
    assert p.returncode == 1
    assert "lammps_preTEM_file_name" in p.stdout + p.stderr


def test_plain_driver_rejects_lammps_options(golden_tmp):
    meta, _ = load_case("md_static")
    d = case_dir("md_static", golden_tmp)
    p = run_cli(CLI, meta["argv"], d)
    assert p.returncode == 1
    assert "ms-stem-fem-md" in p.stdout + p.stderr


@pytest.mark.parametrize("bad,needle", [
    ("pair_style lj/cut 2.5\npair_coeff * * 1.0 1.0\n", "only tersoff"),
    ("pair_style sw\npair_coeff * * Si.sw Xx\n", "unknown element"),
    ("pair_style sw\n", "no pair_coeff"),
])
def test_md_driver_pre_tem_errors(golden_tmp, tmp_path, bad, needle):
    meta, _ = load_case("md_static")
    d = case_dir("md_static", golden_tmp)
    pre = tmp_path / "bad.in"
    pre.write_text("read_data %s\n" % (d / "md_static_0.data") + bad)
    argv = list(meta["argv"])
    argv[argv.index("--lammps_preTEM_file_name") + 1] = str(pre)
    argv[argv.index("-a") + 1] = str(d / "md_static_0.data")
    p = run_cli(CLI_MD, argv, tmp_path)
    assert p.returncode == 1
    assert needle in p.stdout + p.stderr
