#!/usr/bin/env python3
"""Benchmark of the multislice raster: probe*slice propagations per second.

Workload (the configuration the headline metric is quoted on): FEM variance
of one amorphous-Si specimen, ~50,000 atoms at seeded random positions with
a 2.2 A minimum separation in a 100 A cube, 1024x1024 grid, 2 A minimum slice
thickness (~50 slices), 200 kV, 1.5 mrad probe aperture, 64x64 probe raster,
V_omega and V_re over 200 k bins (--dr 1.2065).  Synthetic, seeded inputs
stand in for real specimens.

One step = one whole raster (4,096 probes through every slice, detection and
FEM statistics) on a device-resident specimen; `value` is whole-job
throughput over all ranks.  `e2e` is the same metric through the C ABI from
host buffers: each step uploads the atoms, builds the specimen on the device
(LUTs, slicing, transmission functions), runs the raster and copies the
results back.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun (N ranks, one per GPU) the raster grows to (64 N) x 64 probes
(x spacing / N) and is sharded: each rank runs its contiguous 4,096 probes,
then the one exchange step all-gathers the per-probe detector rows and the
per-pixel sums over NCCL and every rank finishes the FEM statistics.  Work
per GPU is fixed, so scaling is weak; a step is timed with CUDA events around
shard + exchange + finish, max over ranks; rank 0 prints one JSON line.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "ms-stem-fem_b200"))

METRIC = "probe*slice props/s @1024^2 (FEM V(k), batched FP32 wavefields)"
UNIT = "probe*slices/s"
WORKLOAD = dict(n_atoms=50000, box=(100.0, 100.0, 100.0), seed=2,
                argv=("-m 1024 1024 200000 --adfstemuncorrfem --V_omega --V_re --cs3 1.3e7 "
                      "--defocus 0 --alphamax 0.0015 --rasterspacing 1.5625 --minslice 2.0 "
                      "--dr 1.2065"))


def make_specimen(path):
    import specimen
    specimen.make_specimen(path, WORKLOAD["n_atoms"], WORKLOAD["box"], seed=WORKLOAD["seed"])


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def ncu_traffic(which, name="row_col_pass_1024_fp32.md"):
    """DRAM bytes per launch of the row or column pass ("row" / "col") from
    the committed ncu summary (profiles/), or None before one was captured."""
    p = ROOT / "profiles" / name
    if not p.exists():
        return None
    key = "traffic_bytes_per_launch_%s:" % which
    for line in p.read_text().splitlines():
        if line.startswith(key):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def plain_and_precision(msf, job, q, z, device, argv_sample, res32):
    """The two comparisons the headline metric is quoted with.

    plain: probe*slices/s of the plain GPU path - FP64 wavefields, one probe
    per launch, no CUDA graph, same specimen - on an 8x8 raster sample.
    v_err: per FEM mode, the largest relative deviation over the k bins of
    the FP32 run's V(k) from an FP64 GPU run of the full workload (bins with
    |V| <= 1e-6 excluded)."""
    jp = msf.Job(argv_sample)
    cp = msf.Context(device=device, precision="fp64", batch=1, graphs=False)
    sp = cp.specimen(jp.grid, q, z)
    cp.run(sp, jp.optics, jp.raster, jp.detect)
    rp = cp.run(sp, jp.optics, jp.raster, jp.detect)
    plain = rp.probe_slices / rp.seconds_raster
    sp.close()
    cp.close()
    c64 = msf.Context(device=device, precision="fp64")
    s64 = c64.specimen(job.grid, q, z)
    r64 = c64.run(s64, job.optics, job.raster, job.detect)
    errs = {}
    for m, v64 in r64.v.items():
        v32 = res32.v[m]
        ok = np.isfinite(v64) & (np.abs(v64) > 1e-6)
        errs[m] = float(np.max(np.abs(v32[ok] - v64[ok]) / np.abs(v64[ok]))) if ok.any() else None
    fp64_rate = r64.probe_slices / r64.seconds_raster
    s64.close()
    c64.close()
    return plain, errs, fp64_rate


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = Path(tempfile.mkstemp(prefix="msf_clocks", suffix=".csv")[1])

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


def reference_sample(n_procs, cap_seconds=240):
    """The reference's own CPU code (oracle/_ref, FFTW replaced by the oracle
    shim's FP64 FFT) on a bounded sample of the workload: the same 1024^2
    grid, optics and 1.5625 A raster spacing on a 100x100x6 A slab of the
    specimen (3 slices) and 4 probes, one process per host core.  Returns
    aggregate probe*slices/s over the cores and the sample description."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    import specimen
    if not oracle.ref_available():
        return None
    work = Path(tempfile.mkdtemp(prefix="msf_refbench"))
    rng_pos = specimen.amorphous_positions(3000, (100.0, 100.0, 6.0), seed=21)
    rng_pos = np.round(rng_pos, 6)
    specimen.write_lammps_data(work / "slab.data", rng_pos, (100.0, 100.0, 6.0))
    argv = ["-a", "slab.data", "--output_prefix", "s"] + WORKLOAD["argv"].split()
    argv[argv.index("--rasterspacing") + 1] = "50"
    procs = []
    t0 = time.time()
    for k in range(n_procs):
        d = work / ("p%d" % k)
        d.mkdir()
        os.link(work / "slab.data", d / "slab.data")
        procs.append(subprocess.Popen([str(oracle.REF_BIN)] + argv, cwd=d,
                                      stdout=subprocess.DEVNULL, stderr=subprocess.PIPE,
                                      text=True))
    total_ps, worst = 0, 0.0
    for p in procs:
        try:
            _, err = p.communicate(timeout=cap_seconds)
        except subprocess.TimeoutExpired:
            p.kill()
            continue
        for line in err.splitlines():
            if "adfstem_seconds=" in line:
                kv = dict(x.split("=") for x in line.split()[1:])
                total_ps += int(kv["probes"]) * int(kv["slices"])
                worst = max(worst, float(kv["adfstem_seconds"]))
    wall = time.time() - t0
    if not worst:
        return None
    return {"value": total_ps / worst, "cores": n_procs,
            "sample": "%d processes x (4 probes x 3 slices at 1024^2, 100x100x6 A slab, "
                      "3000 Si); raster time only; FFT = oracle shim FP64 radix-2 (FFTW "
                      "absent)" % n_procs, "wall_s": round(wall, 1)}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cores = os.cpu_count() or 1
    vals = []
    sample = None
    for _ in range(max(1, args.steps)):  # no warm-up: nothing to compile or cache
        s = reference_sample(cores, cap_seconds=300)
        if s is None:
            print(json.dumps({"impl": "reference", "unavailable":
                              "oracle/_ref/ms-stem-fem-ref was not built (needs the "
                              "reference sources at build time)"}))
            return 0
        vals.append(s["value"])
        sample = s
        if len(vals) >= max(1, args.steps):
            break
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
            "n_gpus": args.gpus, "steps": len(vals), "warmup": 0,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "FEM 1024^2 amorphous Si (bounded CPU sample)",
                       "grid": 1024, "raster": "2x2", "slices": 3},
            "cpu_baseline": {"kind": "reference", "cores": sample["cores"],
                             "sample": sample["sample"], "value": v, "unit": UNIT},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="msf", choices=["msf", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--no-graphs", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the plain-path and FP64 comparison runs")
    ap.add_argument("--raster", type=int, default=0,
                    help="probes per raster side (default 64, the workload's); smaller "
                         "values make a short case for profiling")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

    import msf
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    work = Path(tempfile.mkdtemp(prefix="msf_bench_r%d_" % rank))
    spec_path = work / "c2.data"
    make_specimen(spec_path)
    argv = ["-a", str(spec_path), "--output_prefix", str(work / "c2")] + WORKLOAD["argv"].split()
    if args.raster:
        argv[argv.index("--rasterspacing") + 1] = repr(WORKLOAD["box"][0] / args.raster)
    job = msf.Job(argv)
    q, z = job.positions()
    ctx = msf.Context(device=local, precision=args.precision, batch=args.batch,
                      graphs=not args.no_graphs)
    t0 = time.time()
    spec = ctx.specimen(job.grid, q, z)
    setup_s = time.time() - t0
    n_slices = spec.slices()["n"]

    def barrier():
        if dist is not None:
            dist.barrier()

    if world > 1:
        # weak scaling: one raster of (64 N) x 64 probes (x spacing / N); each
        # rank runs its contiguous 4,096 probes, then the per-probe rows and
        # pixel sums are exchanged and every rank finishes the FEM statistics
        import shards
        import torch
        n_x = job.raster.n_x * world
        xp_w = np.arange(n_x) * (job.grid.xperiod / n_x)
        yp_w = np.array(job.raster.y_p[:job.raster.n_y])
        raster_w = msf.Raster(n_x, job.raster.n_y, xp_w.ctypes.data_as(msf._dp),
                              yp_w.ctypes.data_as(msf._dp))

        def step():
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record()
            res, part = shards.run_sharded(ctx, spec, job.optics, raster_w, job.detect, rank,
                                           world, dist, device="cuda")
            ev1.record()
            torch.cuda.synchronize()
            return res, part, 1e-3 * ev0.elapsed_time(ev1)
    for _ in range(args.warmup):
        if world > 1:
            step()
        else:
            ctx.run(spec, job.optics, job.raster, job.detect)
    barrier()
    dev_times, launches, ps = [], 0, 0
    with ClockSampler(local) as clocks:
        wall0 = time.time()
        for _ in range(args.steps):
            if world > 1:
                r, part, t_step = step()
                dev_times.append(t_step)
                launches += part.get("kernel_launches", 0)
                ps += part["probe_slices"]
            else:
                r = ctx.run(spec, job.optics, job.raster, job.detect)
                dev_times.append(r.seconds_raster)
                launches += r.kernel_launches
                ps += r.probe_slices
            last = r
        wall = time.time() - wall0
    barrier()
    total_dev = sum(dev_times)
    if dist is not None:
        import torch
        t = torch.tensor([total_dev], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_dev = float(t.item())
    value = ps * world / total_dev  # ps: this rank's probe*slices (equal shards)
    ms_per_step = 1e3 * total_dev / args.steps

    # roofline of the dominant kernel (fused row / column slice pass)
    nb = max(1, min(32, job.n_probes))
    ms_row, ms_col = ctx.time_passes(spec, nb, reps=20)
    n = job.grid.nx
    cbytes = 8 if args.precision == "fp32" else 16
    alg = 2.0 * n * n * cbytes * nb  # read + write of nb wavefields per pass
    dom = "col" if ms_col >= ms_row else "row"
    t_dom = max(ms_row, ms_col) * 1e-3
    peak, peak_kind = measured_peaks()
    achieved = alg / t_dom / 1e9
    # the ncu capture is at 1024^2 FP32 with 32 probes per launch
    traffic = ncu_traffic(dom) if (n == 1024 and args.precision == "fp32" and nb == 32) else None
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "kernel": "%s pass (fused FFT + %s), %d probes/launch" %
                          (dom, "transmission" if dom == "row" else "propagator", nb),
                "peak_source": peak_kind, "ms_row": round(ms_row, 4), "ms_col": round(ms_col, 4),
                "algorithmic_bytes_per_launch": alg}

    # end to end through the C ABI from host buffers
    e2e = None
    if not args.no_e2e:
        ctx.transfer_bytes(reset=True)
        t0 = time.time()
        e2e_steps = max(1, min(2, args.steps))
        e2e_ps = 0
        for _ in range(e2e_steps):
            s2 = ctx.specimen(job.grid, q, z)
            if world > 1:
                _, p2 = shards.run_sharded(ctx, s2, job.optics, raster_w, job.detect, rank,
                                           world, dist, device="cuda")
                e2e_ps += p2["probe_slices"]
            else:
                r2 = ctx.run(s2, job.optics, job.raster, job.detect)
                e2e_ps += r2.probe_slices
            s2.close()
        e2e_t = time.time() - t0
        h2d, d2h = ctx.transfer_bytes(reset=True)
        h2d += q.nbytes + z.nbytes  # atoms staged into the specimen build
        e2e = {"value": e2e_ps * world / e2e_t if world == 1 else None, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d / e2e_steps),
               "d2h_bytes_per_step": int(d2h / e2e_steps),
               "includes": "atom upload, LUT/slicing/transmission build, raster, result copy"}
        if dist is not None:
            import torch
            t = torch.tensor([e2e_t], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e["value"] = e2e_ps * world / float(t.item())

    # plain one-probe-at-a-time GPU path and the FP32 outputs' error
    versus = None
    if world == 1 and not args.no_plain and args.precision == "fp32":
        sample = list(argv)
        sample[sample.index("--rasterspacing") + 1] = repr(WORKLOAD["box"][0] / 8)
        plain, v_err, fp64_rate = plain_and_precision(msf, job, q, z, local, sample, last)
        versus = {"plain_gpu": {"value": round(plain, 1), "unit": UNIT,
                                "path": "FP64 wavefields, 1 probe per launch, no CUDA graph",
                                "sample": "8x8 raster of the same specimen"},
                  "batched_vs_plain": round(value / plain, 2),
                  "fp64_batched": {"value": round(fp64_rate, 1), "unit": UNIT},
                  "v_err_vs_fp64": v_err, "v_err_bound": 1e-4}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        s = reference_sample(os.cpu_count() or 1)
        if s is not None:
            cpu = {"value": s["value"], "unit": UNIT, "cores": s["cores"], "kind": "reference",
                   "sample": s["sample"]}

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 2),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32" if args.precision == "fp32" else "f64", "data": "synthetic",
                "config": {"workload": "FEM V(k) single specimen: 50k Si, 100 A cube, 1024^2, "
                                       "64x64 raster, %d slices" % n_slices,
                           "probes": job.n_probes, "slices": n_slices,
                           "probe_slices_per_step": ps // args.steps,
                           "parallelism": ("one raster of %dx64 probes sharded over %d GPUs, "
                                           "per-probe rows all-gathered for the FEM finish"
                                           % (64 * world, world)) if world > 1 else
                                          "1 GPU",
                           "l2": "inputs exceed L2: %.0f MB of transmission functions" %
                                 (spec.device_bytes() / 1e6),
                           "graphs": not args.no_graphs, "batch": args.batch or "auto",
                           "specimen_setup_s": round(setup_s, 3)},
                "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "versus": versus,
                "clocks": clocks.summary(), "gpu_launches": int(launches),
                "wall_s_timed": round(wall, 3)}
        print(json.dumps(line))
    spec.close()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
