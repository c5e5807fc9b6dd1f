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
(x spacing / N) and is sharded through the library (msf_run_sharded): each
rank runs its contiguous 4,096 probes, then the one exchange step
all-gathers the per-probe detector rows and the per-pixel sums over NCCL on
device buffers and every rank finishes the FEM statistics.  The ranks join
at MASTER_ADDR and the port after MASTER_PORT (MSF_COMM=host exchanges
through that bootstrap instead, for ranks sharing a GPU).  Work per GPU is
fixed, so scaling is weak; a step is timed as the rank's raster device time
(CUDA events) + exchange + host finish, max over ranks; rank 0 prints one
JSON line.
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


def fp32_peak_tflops(device, sm_max_mhz):
    """FP32 CUDA-core peak of the device: SMs x 128 FP32 lanes x 2 flops
    (FMA) x the maximum SM clock (computed from the part's description)."""
    try:
        import torch
        sms = torch.cuda.get_device_properties(device).multi_processor_count
    except Exception:
        sms = 148
    return sms * 128 * 2 * sm_max_mhz * 1e6 / 1e12


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def ncu_l2_bytes(which, nb, pipe):
    """L2 bytes (lts__t_bytes) per launch of the row or column pass captured
    at nb probes per launch with the slice-pass variants `pipe`, from the
    committed ncu summaries; (bytes, file) or (None, None)."""
    key = "l2_bytes_per_launch_%s_b%d_pipe%s:" % (which, nb, pipe)
    for p in sorted((ROOT / "profiles").glob("*.md")):
        for line in p.read_text().splitlines():
            if line.startswith(key):
                try:
                    return float(line.split(":", 1)[1].split()[0]), p.name
                except ValueError:
                    pass
    return None, None


def ncu_traffic(which, nb, pipe=None):
    """DRAM bytes per launch of the row or column pass ("row" / "col") at nb
    probes per launch, from the committed ncu summaries (profiles/*.md): a
    figure captured at nb with the same slice-pass variants (`pipe`, the
    tuner's mask) when one exists, else one captured at nb, else the
    32-probe capture scaled by nb / 32 (DRAM bytes grow in proportion to the
    probes a launch carries).  Returns (bytes, how) or (None, None)."""
    same = "traffic_bytes_per_launch_%s_b%d_pipe%s:" % (which, nb, pipe)
    exact = "traffic_bytes_per_launch_%s_b%d:" % (which, nb)
    base = "traffic_bytes_per_launch_%s:" % which
    found = {}
    for p in sorted((ROOT / "profiles").glob("*.md")):
        for line in p.read_text().splitlines():
            for key in (same, exact, base):
                if line.startswith(key) and key not in found:
                    try:
                        found[key] = (float(line.split(":", 1)[1].split()[0]), p.name)
                    except ValueError:
                        pass
    if pipe is not None and same in found:
        return found[same][0], ("ncu capture at %d probes per launch, slice-pass variants %s "
                                "(%s)" % (nb, pipe, found[same][1]))
    if exact in found:
        return found[exact][0], "ncu capture at %d probes per launch (%s)" % (nb, found[exact][1])
    if base in found:
        return (found[base][0] * nb / 32.0,
                "ncu capture at 32 probes per launch scaled by %d/32 (%s)" % (nb, found[base][1]))
    return None, None

def plain_and_precision(msf, job, q, z, device, argv_sample, res32):
    """The two comparisons the headline metric is quoted with.

    plain: probe*slices/s of the plain GPU path (msf_run_plain: FP64
    wavefields, one probe at a time, one launch per step of the reference's
    slice loop, no CUDA graph) on an 8x8 raster sample of the same specimen;
    fused_1: the fused FP64 passes with one probe per launch, same sample.
    v_err: per FEM mode, the largest relative deviation over the k bins of
    the FP32 run's V(k) from an FP64 GPU run of the full workload (bins with
    |V| <= 1e-6 excluded)."""
    jp = msf.Job(argv_sample)
    cp = msf.Context(device=device, precision="fp64", batch=1, graphs=False)
    sp = cp.specimen(jp.grid, q, z)
    cp.run_plain(sp, jp.optics, jp.raster, jp.detect)
    rp = cp.run_plain(sp, jp.optics, jp.raster, jp.detect)
    plain = rp.probe_slices / rp.seconds_raster
    rf = cp.run(sp, jp.optics, jp.raster, jp.detect)
    fused_1 = rf.probe_slices / rf.seconds_raster
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
    return plain, fused_1, errs, fp64_rate


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
    for _ in range(max(0, args.warmup)):  # page cache, process start-up, CPU clocks
        reference_sample(cores, cap_seconds=300)
    for _ in range(max(1, args.steps)):
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
            "n_gpus": args.gpus, "steps": len(vals), "warmup": max(0, args.warmup),
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


# ---------------------------------------------------------------- configs
def _grid(msf, n, box, zbox, voltage=200000.0):
    return msf.Grid(nx=n, ny=n, voltage=voltage, xperiod=box, yperiod=box, zperiod=zbox,
                    dupe_x=1, dupe_y=1, dupe_z=1, replicate_atoms=0, xmin=0.0, ymin=0.0,
                    zmin=0.0, min_slice=2.0)


class Raster:
    """n x n probes at i * box / n (func.cpp:108-127), arrays kept alive."""

    def __init__(self, msf, n, box):
        self.xp = np.arange(n) * (box / n)
        self.r = msf.Raster(n, n, self.xp.ctypes.data_as(msf._dp),
                            self.xp.ctypes.data_as(msf._dp))


def fem_optics(msf):
    return msf.Optics(corrected=0, cs3=1.3e7, cs5=0.0, defocus=0.0, alpha_max=0.0015)


def adf_optics(msf, voltage=200000.0):
    lam = msf.wavelength(voltage)[0]
    return msf.Optics(corrected=0, cs3=1.3e7, cs5=0.0,
                      defocus=msf.lib().msf_scherzer(0, lam, 1.3e7), alpha_max=0.010)


def batch_specimens(msf):
    """Eight seeded amorphous-Si cubes, edges 50..200 A, grids 512^2..2048^2
    at ~0.1 A sampling, 50 atoms/nm^3, 32x32 rasters."""
    grids = [512, 512, 1024, 1024, 1024, 2048, 2048, 2048]
    out = []
    for s, n in enumerate(grids):
        edge = 50.0 + 150.0 * s / 7
        q = msf.amorphous_positions(int(round(0.05 * edge ** 3)), (edge, edge, edge), 2.2,
                                    seed=31 + s)
        out.append((n, edge, q))
    return out


def workload_batch(args, msf, local):
    """8 uneven specimens in slot lanes (one per grid size) against the same
    rasters run one after another with msf_run."""
    ctx = msf.Context(device=local, precision="fp32")
    det = msf.Detect(outputs=msf.OUT_ADF_IMAGE | msf.OUT_V_OMEGA, det_inner=0.04,
                     det_outer=0.2, dr=1.2065)
    jobs, keep = [], []
    t0 = time.time()
    for n, edge, q in batch_specimens(msf):
        spec = ctx.specimen(_grid(msf, n, edge, edge), q, np.full(len(q), 14, np.uint32))
        r = Raster(msf, 32, edge)
        keep.append(r)
        jobs.append((spec, fem_optics(msf), r.r, det))
    setup = time.time() - t0
    for _ in range(max(1, args.warmup)):
        ctx.run_batch(jobs, slots=args.batch)
    times, ps = [], 0
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            outs = ctx.run_batch(jobs, slots=args.batch)
            times.append(max(o.seconds_raster for o in outs))
            ps = sum(o.probe_slices for o in outs)
            launches = max(o.kernel_launches for o in outs)
    seq = 0.0
    for spec, o, r, d in jobs:
        seq += ctx.run(spec, o, r, d).seconds_raster
    t = statistics.median(times)
    line = {"metric": "probe*slice props/s, 8 uneven specimens 512^2-2048^2 in slot lanes",
            "value": round(ps / t, 1), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * t, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "8 amorphous-Si cubes 50..200 A, grids 512,512,1024x3,"
                                   "2048x3, 32x32 rasters, 2 A slices, V_omega + ADF",
                       "probe_slices_per_step": ps,
                       "slots_per_lane": args.batch or "auto: ~2 GiB of wavefields per lane",
                       "specimen_setup_s": round(setup, 2)},
            "sequential_msf_run": {"value": round(ps / seq, 1), "unit": UNIT},
            "clocks": clocks.summary(), "gpu_launches": int(launches)}
    print(json.dumps(line))
    return 0


def stress_specimen(msf, path):
    """The precision-stress specimen as the reference reads it: 600k Si at
    seeded positions (msf_amorphous_positions, seed 4) in 200x200x300 A,
    written with 6 decimals and parsed back by the drop-in reader."""
    import specimen
    box = np.array([200.0, 200.0, 300.0])
    pos = np.minimum(np.round(msf.amorphous_positions(600000, box, 2.2, seed=4), 6),
                     np.round(box, 6))
    specimen.write_lammps_data(path, pos, box)
    return msf.Job(["-a", str(path), "--output_prefix", "stress", "-m", "2048", "2048",
                    "300000", "--adfstemuncorrfem", "--V_omega", "--images", "--cs3", "1.3e7",
                    "--scherzer_defocus", "--scherzer_alphamax", "--rasterspacing", "50",
                    "--minslice", "2.0"])


def workload_stress(args, msf, local):
    """600k atoms, 200x200x300 A, 2048^2, 300 kV, 150 slices, 16x16 raster:
    FP32 split-wave against FP64 wavefields, per-output error; and both
    precisions on a 4x4 raster against the reference's own FP64 result for
    the same specimen (the committed fixture tests/golden/c4_r4.npz)."""
    box = (200.0, 200.0, 300.0)
    work = Path(tempfile.mkdtemp(prefix="msf_stress_"))
    job4 = stress_specimen(msf, work / "c4.data")
    q, z = job4.positions()
    lam = msf.wavelength(300000.0)[0]
    optics = msf.Optics(corrected=0, cs3=1.3e7, cs5=0.0,
                        defocus=msf.lib().msf_scherzer(0, lam, 1.3e7),
                        alpha_max=msf.lib().msf_scherzer(1, lam, 1.3e7))
    det = msf.Detect(outputs=msf.OUT_ADF_IMAGE | msf.OUT_V_OMEGA, det_inner=0.04,
                     det_outer=0.2, dr=1.0)
    r = Raster(msf, 16, box[0])
    out, vs_ref = {}, {}
    golden = ROOT / "tests" / "golden" / "c4_r4.npz"
    ref = dict(np.load(golden)) if golden.exists() else None
    for prec in ("fp32", "fp64"):
        ctx = msf.Context(device=local, precision=prec)
        t0 = time.time()
        spec = ctx.specimen(job4.grid, q, z)
        setup = time.time() - t0
        # launch tiling and slice-pass variants measured once for the grid
        # before timing, as the headline workload does
        tuning = None if args.no_tune else ctx.tune(spec)
        ctx.run(spec, optics, r.r, det)
        res = ctx.run(spec, optics, r.r, det)
        out[prec] = (res, setup, spec.slices()["n"], tuning)
        if ref is not None:  # the reference's 4x4 raster of the same specimen
            r4 = ctx.run(spec, job4.optics, job4.raster, job4.detect)
            want = ref["V_omega"][:, 1]
            m = np.isfinite(want) & (np.abs(want) > 1e-6)
            vs_ref[prec] = {
                "adf_image_max_rel": float(np.max(np.abs(r4.adf_image - ref["adf_image"]) /
                                                  np.abs(ref["adf_image"]))),
                "v_omega_max_rel": float(np.max(np.abs(r4.v["V_omega"][m] - want[m]) /
                                                np.abs(want[m]))),
                "v_omega_bins": int(m.sum())}
        spec.close()
        ctx.close()
    r32, r64 = out["fp32"][0], out["fp64"][0]
    adf_err = float(np.max(np.abs(r32.adf_image - r64.adf_image) / np.abs(r64.adf_image)))
    v64 = r64.v["V_omega"]
    ok = np.isfinite(v64) & (np.abs(v64) > 1e-6)
    v_err = float(np.max(np.abs(r32.v["V_omega"][ok] - v64[ok]) / np.abs(v64[ok])))
    line = {"metric": "probe*slice props/s @2048^2, 150 slices, 300 kV (FP32 split-wave)",
            "value": round(r32.probe_slices / r32.seconds_raster, 1), "unit": UNIT,
            "n_gpus": 1, "steps": 1, "warmup": 1,
            "ms_per_step": round(1e3 * r32.seconds_raster, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "600k Si atoms 200x200x300 A, 2048^2, 300 kV, Scherzer, "
                                   "16x16 raster", "slices": out["fp32"][2],
                       "specimen_setup_s": round(out["fp32"][1], 2), "tuning": out["fp32"][3]},
            "fp64": {"value": round(r64.probe_slices / r64.seconds_raster, 1), "unit": UNIT,
                     "specimen_setup_s": round(out["fp64"][1], 2), "tuning": out["fp64"][3]},
            "error_fp32_vs_fp64": {"adf_image_max_rel": adf_err, "v_omega_max_rel": v_err},
            "error_vs_reference": dict(vs_ref, raster="4x4 (rasterspacing 50 A)",
                                       bins="V_omega bins above 1e-6",
                                       reference="the reference's own sources, FP64, FFTW "
                                                 "replaced by an FP64 radix-2 shim") if vs_ref
                                  else "tests/golden/c4_r4.npz absent",
            "gpu_launches": int(r32.kernel_launches)}
    print(json.dumps(line))
    return 0


def serving_requests(msf, n_jobs, seed=5):
    """Seeded request stream: grid from {256,512,1024,2048}^2 at 0.09766 A
    sampling, raster 8..64 per side, thickness 50..300 A, ADF or FEM V(k)
    with probability 1/2, 50 atoms/nm^3 per request."""
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(n_jobs):
        n = int(rng.choice([256, 512, 1024, 2048]))
        edge = n * 0.09766
        n_r = int(rng.integers(8, 65))
        thick = float(rng.uniform(50.0, 300.0))
        fem = bool(rng.random() < 0.5)
        q = msf.amorphous_positions(int(round(0.05 * edge * edge * thick)), (edge, edge, thick),
                                    2.2, seed=5000 + k)
        det = (msf.Detect(outputs=msf.OUT_V_OMEGA, det_inner=0.04, det_outer=0.2, dr=1.0)
               if fem else
               msf.Detect(outputs=msf.OUT_ADF_IMAGE, det_inner=0.04, det_outer=0.2, dr=1.0))
        reqs.append({"grid": _grid(msf, n, edge, thick), "q": q,
                     "z": np.full(len(q), 14, np.uint32),
                     "optics": fem_optics(msf) if fem else adf_optics(msf),
                     "raster": Raster(msf, n_r, edge), "detect": det, "n": n, "fem": fem})
    return reqs


def run_serving(msf, local, n_jobs, rate, slots, seed=5):
    """Poisson arrivals at `rate` jobs/s into msf_server; returns the summary."""
    reqs = serving_requests(msf, n_jobs, seed)
    gaps = np.random.default_rng(seed + 1).exponential(1.0 / rate, n_jobs)
    srv = msf.Server(device=local, slots=slots)
    # warm-up: one small request per grid size (lanes, graphs, module load)
    warm = []
    for n in (256, 512, 1024, 2048):
        edge = n * 0.09766
        q = msf.amorphous_positions(int(0.05 * edge * edge * 6), (edge, edge, 6.0), 2.2, seed=n)
        r = Raster(msf, 2, edge)
        warm.append((srv.submit(_grid(msf, n, edge, 6.0), q, np.full(len(q), 14, np.uint32),
                                fem_optics(msf), r.r,
                                msf.Detect(outputs=msf.OUT_V_OMEGA, det_inner=0.04,
                                           det_outer=0.2, dr=1.0)), r))
    for t, _ in warm:
        while srv.poll(t, wait_ms=100) is None:
            pass
    srv.close()
    srv = msf.Server(device=local, slots=slots)
    tickets = []
    t_start = time.time()
    t_next = t_start
    for req, gap in zip(reqs, gaps):
        t_next += gap
        dt = t_next - time.time()
        if dt > 0:
            time.sleep(dt)
        tickets.append(srv.submit(req["grid"], req["q"], req["z"], req["optics"],
                                  req["raster"].r, req["detect"]))
    for t in tickets:
        while srv.poll(t, wait_ms=200) is None:
            pass
    st = srv.stats()
    by_grid = srv.grid_stats()
    wall = time.time() - t_start
    srv.close()
    return {"jobs": n_jobs, "arrival_rate_per_s": rate, "slots_per_lane": slots,
            "p50_s": round(st["p50_s"], 3), "p99_s": round(st["p99_s"], 3),
            "max_s": round(st["max_s"], 3), "completed": st["completed"],
            "failed": st["failed"], "probe_slices": st["probe_slices"],
            "throughput": round(st["probe_slices"] / wall, 1), "unit": UNIT,
            "offered": round(st["probe_slices"] / max(float(gaps.sum()), 1e-9), 1),
            "wall_s": round(wall, 2),
            "by_grid": {"%dx%d" % (g["nx"], g["ny"]): {
                "completed": g["completed"], "p50_s": round(g["p50_s"], 3),
                "p99_s": round(g["p99_s"], 3), "max_s": round(g["max_s"], 3)}
                for g in by_grid},
            "mix": {str(n): sum(1 for r in reqs if r["n"] == n) for n in (256, 512, 1024, 2048)}}


def workload_serving(args, msf, local):
    s = run_serving(msf, local, args.jobs, args.rate, args.batch)
    # the same stream at a rate one GPU sustains (offered load below
    # capacity): latency is then service time plus a short queue
    sustained = (run_serving(msf, local, args.sustained_jobs, args.sustained_rate, args.batch,
                             seed=7) if args.sustained_jobs > 0 else None)
    line = {"metric": "serving p99 latency, Poisson arrivals, mixed 256^2-2048^2 requests",
            "value": s["p99_s"], "unit": "s", "n_gpus": 1, "steps": 1, "warmup": 1,
            "ms_per_step": None, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "request stream: grids 256..2048^2, rasters 8..64^2, "
                                   "5..30 nm thick, ADF or FEM, 50 atoms/nm^3"},
            "serving": s, "sustained": sustained}
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
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the launch tiling autotuner (batch from free memory)")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the plain-path and FP64 comparison runs")
    ap.add_argument("--raster", type=int, default=0,
                    help="probes per raster side (default 64, the workload's); smaller "
                         "values make a short case for profiling")
    ap.add_argument("--workload", default="fem",
                    choices=["fem", "batch", "stress", "serving"],
                    help="fem: the headline FEM raster (default); batch: 8 uneven specimens "
                         "in slot lanes; stress: 2048^2, 150 slices, FP32 vs FP64; serving: "
                         "Poisson request stream through msf_server")
    ap.add_argument("--jobs", type=int, default=24, help="requests of --workload serving")
    ap.add_argument("--rate", type=float, default=20.0, help="request arrivals per second")
    ap.add_argument("--sustained-jobs", type=int, default=12,
                    help="requests of the second --workload serving run, at --sustained-rate")
    ap.add_argument("--sustained-rate", type=float, default=0.2,
                    help="arrivals per second one GPU sustains for the mixed stream")
    ap.add_argument("--serving-jobs", type=int, default=50,
                    help="requests of the serving sample in the headline line (0: none)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

    import msf
    if args.workload != "fem":
        local = int(os.environ.get("LOCAL_RANK", "0"))
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        return {"batch": workload_batch, "stress": workload_stress,
                "serving": workload_serving}[args.workload](args, msf, local)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    comm = None
    if world > 1:
        import torch
        local = local % max(1, torch.cuda.device_count())
        # the library's communicator: NCCL on device buffers by default;
        # MSF_COMM=host exchanges through the bootstrap (ranks may then
        # share a GPU).  Every wait is bounded, so a rank that stops ends
        # the others' next exchange with an error instead of a hang.
        transport = msf.COMM_HOST if os.environ.get("MSF_COMM") == "host" else msf.COMM_NCCL
        rdv = "%s:%d" % (os.environ.get("MASTER_ADDR", "127.0.0.1"),
                         int(os.environ.get("MASTER_PORT", "29500")) + 1)
        comm = msf.Comm(rank, world, rdv, transport, device=local, timeout_s=180)

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
    # launch tiling measured once per grid before timing (the analogue of
    # the reference's FFTW planning); later runs on this grid use it
    tuning = None
    if not args.batch and not args.no_tune:
        t0 = time.time()
        tuning = ctx.tune(spec)
        tuning["seconds"] = round(time.time() - t0, 3)

    def barrier():
        if comm is not None:
            comm.allgather(np.zeros(1))

    def max_over_ranks(x):
        return float(comm.allgather(np.array([x])).max()) if comm is not None else x

    if world > 1:
        # weak scaling: one raster of (64 N) x 64 probes (x spacing / N); each
        # rank runs its contiguous 4,096 probes, then the per-probe rows and
        # pixel sums are exchanged and every rank finishes the FEM statistics
        n_x = job.raster.n_x * world
        xp_w = np.arange(n_x) * (job.grid.xperiod / n_x)
        yp_w = np.array(job.raster.y_p[:job.raster.n_y])
        raster_w = msf.Raster(n_x, job.raster.n_y, xp_w.ctypes.data_as(msf._dp),
                              yp_w.ctypes.data_as(msf._dp))

        def step():
            # device time of this rank's probes (msf's own events on its
            # stream) + the exchange + the host finish (wall clock)
            res = ctx.run_sharded(spec, job.optics, raster_w, job.detect, comm)
            sh = res.shard
            return res, res.seconds_raster + sh["seconds_exchange"] + sh["seconds_finish"]
    for _ in range(args.warmup):
        if world > 1:
            step()
        else:
            ctx.run(spec, job.optics, job.raster, job.detect)
    barrier()
    dev_times, launches, ps, step_results = [], 0, 0, []
    with ClockSampler(local) as clocks:
        wall0 = time.time()
        for _ in range(args.steps):
            if world > 1:
                r, t_step = step()
                dev_times.append(t_step)
                launches += r.kernel_launches
                ps += r.probe_slices
            else:
                r = ctx.run(spec, job.optics, job.raster, job.detect)
                dev_times.append(r.seconds_raster)
                launches += r.kernel_launches
                ps += r.probe_slices
                step_results.append(r)
            last = r
        wall = time.time() - wall0
    barrier()
    total_dev = max_over_ranks(sum(dev_times))
    value = ps * world / total_dev  # ps: this rank's probe*slices (equal shards)
    ms_per_step = 1e3 * total_dev / args.steps

    # roofline of the dominant kernel (fused row / column slice pass)
    # (at the tuned probes per launch; the ncu capture is of 32-probe
    # launches, its DRAM bytes scale with the probes a launch carries)
    # Measured live: msf_run times the passes of its first batch with CUDA
    # events on the launching stream; the timed steps' means are used.
    # (Sharded runs return no pass times: the passes are then timed alone.)
    live = [(r.ms_row_pass, r.ms_col_pass, r.pass_batch) for r in step_results
            if getattr(r, "pass_batch", 0) > 0]
    if live:
        nb = live[0][2]
        ms_row = statistics.mean(x[0] for x in live)
        ms_col = statistics.mean(x[1] for x in live)
        timing = "CUDA events around each pass of the first batch of every timed step"
    else:
        nb = max(1, min(tuning["batch"] if tuning else 32, job.n_probes))
        ms_row, ms_col = ctx.time_passes(spec, nb, reps=20)
        timing = "msf_time_passes after the timed region"
    n = job.grid.nx
    cbytes = 8 if args.precision == "fp32" else 16
    # read + write of nb wavefields per pass, less the columns the band limit
    # removes entirely (zero between the passes: neither pass moves them)
    live = spec.live_columns() / float(job.grid.ny)
    alg = 2.0 * n * n * cbytes * nb * live
    dom = "col" if ms_col >= ms_row else "row"
    t_dom = max(ms_row, ms_col) * 1e-3
    peak, peak_kind = measured_peaks()
    achieved = alg / t_dom / 1e9
    pipe_used = tuning["pipe"] if tuning else int(os.environ.get("MSF_PIPE", "17"))
    traffic, traffic_src = (ncu_traffic(dom, nb, pipe_used)
                            if (n == 1024 and args.precision == "fp32") else (None, None))
    # the flop ceiling beside the HBM one: two complex 2-D FFTs at
    # 5 n log2 n plus the point-wise work, per probe*slice, against the
    # FP32 CUDA-core peak (SMs x 128 lanes x 2 flops x max SM clock;
    # computed, not measured -- the FFT does not run on tensor cores)
    flops_ps = 10.0 * n * n * math.log2(float(n * n)) + 20.0 * n * n
    sm_max = clocks.summary().get("sm_max_mhz") or 1965.0
    fp32_peak = fp32_peak_tflops(local, sm_max)
    flop_rate = value / world * flops_ps / 1e12
    # L2 bytes of the same launch (ncu lts__t_bytes at this tiling): the
    # L2 rate it implies beside the DRAM one (no measured L2 peak exists
    # for this part, so no fraction is given)
    l2_bytes, l2_src = (ncu_l2_bytes(dom, nb, pipe_used)
                        if (n == 1024 and args.precision == "fp32") else (None, None))
    l2 = ({"bytes_per_launch": l2_bytes, "achieved_gbs": round(l2_bytes / t_dom / 1e9, 1),
           "peak": None, "source": l2_src} if l2_bytes else None)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "flops_per_probe_slice": flops_ps,
                "flop_achieved_tflops_per_gpu": round(flop_rate, 2),
                "fp32_peak_tflops": round(fp32_peak, 1),
                "flop_frac": round(flop_rate / fp32_peak, 4),
                "kernel": "%s pass (fused FFT + %s), %d probes/launch" %
                          (dom, "transmission" if dom == "row" else "propagator", nb),
                "peak_source": peak_kind, "ms_row": round(ms_row, 4), "ms_col": round(ms_col, 4),
                "algorithmic_bytes_per_launch": alg, "live_column_fraction": round(live, 4),
                "traffic_source": traffic_src, "l2": l2,
                "timing": timing}

    # end to end through the C ABI from host buffers
    e2e = None
    if not args.no_e2e:
        ctx.transfer_bytes(reset=True)
        t0 = time.time()
        e2e_steps = max(1, args.steps)  # as many as the timed region
        e2e_ps = 0
        for _ in range(e2e_steps):
            s2 = ctx.specimen(job.grid, q, z)
            if world > 1:
                r2 = ctx.run_sharded(s2, job.optics, raster_w, job.detect, comm)
                e2e_ps += r2.probe_slices
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
        if comm is not None:
            e2e["value"] = e2e_ps * world / max_over_ranks(e2e_t)

    # plain one-probe-at-a-time GPU path and the FP32 outputs' error
    versus = None
    if world == 1 and not args.no_plain and args.precision == "fp32":
        sample = list(argv)
        sample[sample.index("--rasterspacing") + 1] = repr(WORKLOAD["box"][0] / 8)
        plain, fused_1, v_err, fp64_rate = plain_and_precision(msf, job, q, z, local, sample,
                                                               last)
        need = 50.0 * plain * flops_ps / 1e12
        versus = {"target_50x_plain": {
                      "value": round(50.0 * plain, 1), "unit": UNIT,
                      "flops_needed_tflops": round(need, 1),
                      "fp32_peak_tflops": round(fp32_peak, 1),
                      "reachable": need <= fp32_peak,
                      "why": "50x the plain path needs %.0f TFLOP/s of FFT arithmetic, "
                             "%.1fx the FP32 CUDA-core peak; the FFT is not a dense "
                             "contraction and runs without tensor cores" %
                             (need, need / fp32_peak)},
                  "plain_gpu": {"value": round(plain, 1), "unit": UNIT,
                                "path": "msf_run_plain: FP64, one probe at a time, one launch "
                                        "per reference step, no CUDA graph",
                                "sample": "8x8 raster of the same specimen"},
                  "batched_vs_plain": round(value / plain, 2),
                  "fused_fp64_one_probe": {"value": round(fused_1, 1), "unit": UNIT},
                  "batched_vs_fused_one_probe": round(value / fused_1, 2),
                  "fp64_batched": {"value": round(fp64_rate, 1), "unit": UNIT},
                  "v_err_vs_fp64": v_err, "v_err_bound": 1e-4}

    serving = None
    if world == 1 and args.serving_jobs > 0:
        serving = run_serving(msf, local, args.serving_jobs, args.rate, 0)

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
                           "graphs": not args.no_graphs,
                           "batch": args.batch or (tuning["batch"] if tuning else "auto"),
                           "tuning": tuning,
                           "specimen_setup_s": round(setup_s, 3)},
                "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "versus": versus,
                "serving": serving,
                "clocks": clocks.summary(), "gpu_launches": int(launches),
                "wall_s_timed": round(wall, 3)}
        print(json.dumps(line))
    spec.close()
    ctx.close()
    if comm is not None:
        comm.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
