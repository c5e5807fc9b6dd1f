"""One raster over several ranks in the C++ library (msf_run_sharded) and the
drop-in CLI (one process per rank, as `mpirun -np K ms-stem-fem.x` runs the
reference).

* One rank through NCCL: the exchange runs on device buffers and the
  result equals msf_run bit for bit.
* Two ranks sharing this GPU through the host transport (NCCL refuses two
  ranks on one device; the pool gives one GPU per call): rows travel
  unchanged, so the ADF image and the ring-sum modes equal msf_run bit for
  bit, and the pixel-sum modes, whose per-rank sums are added in rank
  order, agree to 1e-12.
* The CLI under a torchrun-style environment (WORLD_SIZE, RANK,
  LOCAL_RANK, MASTER_ADDR, MASTER_PORT): rank 0 writes the reference's
  files with the values of a single-process run; rank 1 writes none."""
import multiprocessing as mpp
import os
import socket
import subprocess
import sys
import tempfile

import numpy as np
import pytest

import msf
import oracle
from conftest import ROOT, case_argv, case_dir, load_case

pytestmark = pytest.mark.gpu

ROW_MODES = ("V_omega", "Vbar_r")
PIX_MODES = ("V_re", "Omega_vimage", "V_gt17", "V_rbar")


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _job(name, tmp):
    d = case_dir(name, tmp)
    job = msf.Job(case_argv(name, d))
    return job


def test_single_rank_nccl_equals_msf_run(golden_tmp):
    job = _job("fem128", golden_tmp)
    q, z = job.positions()
    ctx = msf.Context(precision="fp32", batch=5)
    spec = ctx.specimen(job.grid, q, z)
    whole = ctx.run(spec, job.optics, job.raster, job.detect)
    comm = msf.Comm(0, 1, "", msf.COMM_NCCL, device=0)
    got = ctx.run_sharded(spec, job.optics, job.raster, job.detect, comm)
    comm.close()
    assert np.array_equal(got.adf_image, whole.adf_image)
    for m, v in whole.v.items():
        assert np.array_equal(got.v[m], v, equal_nan=True), m
    assert got.shard["p_begin"] == 0 and got.shard["p_end"] == job.n_probes


def _host_rank(rank, world, port, argv, out_dir):
    job = msf.Job(argv)
    q, z = job.positions()
    ctx = msf.Context(precision="fp32", batch=3)
    spec = ctx.specimen(job.grid, q, z)
    comm = msf.Comm(rank, world, "127.0.0.1:%d" % port, msf.COMM_HOST, timeout_s=120)
    got = ctx.run_sharded(spec, job.optics, job.raster, job.detect, comm)
    np.savez(os.path.join(out_dir, "rank%d.npz" % rank), adf=got.adf_image,
             b=got.shard["p_begin"], e=got.shard["p_end"], **got.v)
    comm.close()


def test_two_ranks_host_transport_equal_msf_run(golden_tmp):
    d = case_dir("fem128", golden_tmp)
    argv = case_argv("fem128", d)
    job = msf.Job(argv)
    q, z = job.positions()
    ctx = msf.Context(precision="fp32", batch=3)
    whole = ctx.run(ctx.specimen(job.grid, q, z), job.optics, job.raster, job.detect)
    spawn = mpp.get_context("spawn")
    with tempfile.TemporaryDirectory() as out:
        port = free_port()
        procs = [spawn.Process(target=_host_rank, args=(r, 2, port, argv, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
        alive = [p for p in procs if p.is_alive()]
        for p in alive:
            p.kill()
        assert not alive and all(p.exitcode == 0 for p in procs)
        spans = []
        for r in range(2):
            g = dict(np.load(os.path.join(out, "rank%d.npz" % r)))
            spans.append((int(g["b"]), int(g["e"])))
            assert np.array_equal(g["adf"], whole.adf_image)
            for m in ROW_MODES:
                assert np.array_equal(g[m], whole.v[m], equal_nan=True), m
            for m in PIX_MODES:
                np.testing.assert_allclose(g[m], whole.v[m], rtol=1e-12, atol=1e-15,
                                           equal_nan=True, err_msg=m)
        assert spans[0][0] == 0 and spans[0][1] == spans[1][0] and spans[1][1] == job.n_probes


def test_cli_over_two_ranks_writes_single_run_outputs(tmp_path):
    meta, ref = load_case("fem128")
    single = case_dir("fem128", tmp_path / "single")
    multi = case_dir("fem128", tmp_path / "multi")
    cli = str(ROOT / "ms-stem-fem_b200" / "bin" / "ms-stem-fem")
    # a fixed launch tiling in both runs (no per-run tuning)
    fixed = ["--precision", "fp32", "--batch", "8"]
    p = subprocess.run([cli] + meta["argv"] + fixed, cwd=single,
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    port = free_port()
    procs = []
    for r in range(2):
        # the CLI's rendezvous is the port after MASTER_PORT (torchrun's own
        # store listens on MASTER_PORT)
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(r), LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port - 1), MSF_COMM="host",
                   MSF_COMM_TIMEOUT="120")
        wd = multi if r == 0 else tmp_path / "rank1"
        wd.mkdir(exist_ok=True)
        argv = [a if a != meta["argv"][1] else str(multi / a) for a in meta["argv"]]
        procs.append(subprocess.Popen([cli] + argv + fixed, cwd=wd, env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True))
    outs = [pr.communicate(timeout=300) for pr in procs]
    assert all(pr.returncode == 0 for pr in procs), outs
    assert not list((tmp_path / "rank1").glob("*_adfstem_*")), "rank 1 wrote outputs"
    for mode in ROW_MODES + PIX_MODES:
        a = oracle.read_variance_txt(single / (meta["prefix"] + "_fem_%s.txt" % mode))
        b = oracle.read_variance_txt(multi / (meta["prefix"] + "_fem_%s.txt" % mode))
        np.testing.assert_allclose(b, a, rtol=1e-9, atol=1e-15, equal_nan=True, err_msg=mode)
    ia = np.fromfile(single / (meta["prefix"] + "_stem_image_output.f64"))
    ib = np.fromfile(multi / (meta["prefix"] + "_stem_image_output.f64"))
    assert np.array_equal(ia, ib)
    # the first and last exit waves' diffraction patterns (--images)
    for f in sorted(single.glob(meta["prefix"] + "_*_diffraction_*.tif")):
        assert (multi / f.name).read_bytes() == f.read_bytes(), f.name


def test_nccl_communicator_leaves_torch_importable():
    """The communicator loads the NCCL the environment's torch links against
    (or one already loaded), so torch still imports afterwards in the same
    process; a second NCCL under the same soname would break its symbols."""
    code = ("import sys; sys.path.insert(0, %r)\n"
            "import msf\n"
            "c = msf.Comm(0, 1, '', msf.COMM_NCCL, device=0)\n"
            "c.close()\n"
            "import torch\n"
            "assert torch.cuda.is_available()\n"
            "print('ok')\n" % str(ROOT / "ms-stem-fem_b200"))
    env = {k: v for k, v in os.environ.items() if k != "MSF_NCCL_LIBRARY"}
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       timeout=300, env=env)
    assert p.returncode == 0 and "ok" in p.stdout, p.stdout + p.stderr
