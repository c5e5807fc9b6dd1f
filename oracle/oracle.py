"""ctypes binding of the CPU oracle (oracle/msf_oracle.c) and runners for the
reference's own binaries (oracle/_ref/ms-stem-fem-ref and, for the
MD-coupled driver with LAMMPS replaced by a data-file replay,
oracle/_ref/ms-stem-fem-md-ref).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use this module as the checker; the product never does.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import re
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_BIN = HERE / "_ref" / "ms-stem-fem-ref"
REF_MD_BIN = HERE / "_ref" / "ms-stem-fem-md-ref"

OR_ADF, OR_D1, OR_D2, OR_D3, OR_D4, OR_GT17, OR_RVA = 1, 2, 4, 8, 16, 32, 64
MODE_BITS = {"V_omega": OR_D1, "Vbar_r": OR_D2, "V_re": OR_D3,
             "Omega_vimage": OR_D4, "V_gt17": OR_GT17, "V_rbar": OR_RVA}

_dp = C.POINTER(C.c_double)


class OrJob(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("voltage", C.c_double),
                ("xperiod", C.c_double), ("yperiod", C.c_double),
                ("xperiod_duped", C.c_double), ("yperiod_duped", C.c_double),
                ("xmin", C.c_double), ("ymin", C.c_double),
                ("min_slice", C.c_double), ("corrected", C.c_int32),
                ("cs3", C.c_double), ("cs5", C.c_double),
                ("defocus", C.c_double), ("alpha_max", C.c_double),
                ("det_inner", C.c_double), ("det_outer", C.c_double),
                ("dr", C.c_double), ("n_rx", C.c_int32), ("n_ry", C.c_int32),
                ("x_p", _dp), ("y_p", _dp), ("flags", C.c_uint32)]


class OrAtoms(C.Structure):
    _fields_ = [("n_atoms", C.c_int64), ("q", _dp),
                ("z", C.POINTER(C.c_uint32))]


class OrResult(C.Structure):
    _fields_ = [("adf_image", _dp), ("cap_k", C.c_int32), ("n_k", C.c_int32),
                ("k_lower", _dp), ("v_omega", _dp), ("vbar_r", _dp),
                ("v_re", _dp), ("omega_vimage", _dp), ("v_gt17", _dp),
                ("v_rbar", _dp), ("bin_counts", C.POINTER(C.c_int32)),
                ("last_psi", _dp), ("n_slices", C.c_int32)]


def build_lib() -> Path:
    """Compile the oracle into oracle/liboracle.so (gcc, FP64, no contraction)."""
    src = HERE / "msf_oracle.c"
    if LIB_PATH.exists() and LIB_PATH.stat().st_mtime >= src.stat().st_mtime:
        return LIB_PATH
    subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared",
                           "-o", str(LIB_PATH), str(src), "-lm"])
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(str(build_lib()))
        _lib.or_run.argtypes = [C.POINTER(OrJob), C.POINTER(OrAtoms), C.POINTER(OrResult)]
        _lib.or_transmission.argtypes = [C.POINTER(OrJob), C.POINTER(OrAtoms),
                                         C.c_int32, _dp]
        _lib.or_probe.argtypes = [C.POINTER(OrJob), _dp]
        _lib.or_constants.argtypes = [C.c_double, _dp, _dp]
        _lib.or_slice_atoms.argtypes = [C.c_int64, _dp, C.c_double, C.c_double,
                                        C.c_double, C.POINTER(C.c_int64),
                                        C.POINTER(C.c_int64), _dp, _dp]
        _lib.or_slice_atoms.restype = C.c_int64
        _lib.or_snap.argtypes = [_dp, C.c_int64, C.c_double, C.c_double, C.c_int64]
        _lib.or_snap.restype = C.c_int64
        _lib.or_ring_bins.argtypes = [C.POINTER(OrJob), C.POINTER(C.c_int32),
                                      C.POINTER(C.c_int32), _dp, C.c_int32]
        _lib.or_ring_bins.restype = C.c_int32
    return _lib


def _p(a):
    return a.ctypes.data_as(_dp)


def make_job(job: dict):
    """Build an OrJob from a plain dict (the same keys the product's job uses);
    returns (OrJob, keep-alive list)."""
    x_p = np.ascontiguousarray(job["x_p"], dtype=np.float64)
    y_p = np.ascontiguousarray(job["y_p"], dtype=np.float64)
    flags = OR_ADF if job.get("images") else 0
    for m in job.get("fem_modes", []):
        flags |= MODE_BITS[m]
    j = OrJob(job["nx"], job["ny"], job["voltage"], job["xperiod"], job["yperiod"],
              job.get("xperiod_duped", job["xperiod"]),
              job.get("yperiod_duped", job["yperiod"]),
              job.get("xmin", 0.0), job.get("ymin", 0.0), job["min_slice"],
              int(job.get("corrected", 0)), job.get("cs3", 0.0), job.get("cs5", 0.0),
              job["defocus"], job["alpha_max"], job["det_inner"], job["det_outer"],
              job.get("dr", 0.70710678118654746), len(x_p), len(y_p),
              _p(x_p), _p(y_p), flags)
    return j, [x_p, y_p]


def make_atoms(q: np.ndarray, z: np.ndarray):
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1)
    z = np.ascontiguousarray(z, dtype=np.uint32)
    return OrAtoms(len(z), _p(q), z.ctypes.data_as(C.POINTER(C.c_uint32))), [q, z]


def run(job: dict, q: np.ndarray, z: np.ndarray, cap_k: int = 4096,
        want_last_psi: bool = False) -> dict:
    """Run the whole raster job on the CPU oracle."""
    j, keep = make_job(job)
    a, keep2 = make_atoms(q, z)
    n_r = j.n_rx * j.n_ry
    img = np.zeros(n_r)
    arrs = {k: np.full(cap_k, np.nan) for k in
            ("k_lower", "V_omega", "Vbar_r", "V_re", "Omega_vimage", "V_gt17", "V_rbar")}
    counts = np.zeros(cap_k, dtype=np.int32)
    last = np.zeros(2 * job["nx"] * job["ny"]) if want_last_psi else None
    r = OrResult(_p(img), cap_k, 0, _p(arrs["k_lower"]), _p(arrs["V_omega"]),
                 _p(arrs["Vbar_r"]), _p(arrs["V_re"]), _p(arrs["Omega_vimage"]),
                 _p(arrs["V_gt17"]), _p(arrs["V_rbar"]),
                 counts.ctypes.data_as(C.POINTER(C.c_int32)),
                 _p(last) if last is not None else None, 0)
    rc = lib().or_run(C.byref(j), C.byref(a), C.byref(r))
    if rc != 0:
        raise RuntimeError("oracle or_run failed with code %d" % rc)
    nk = r.n_k
    out = {"adf_image": img.reshape(j.n_rx, j.n_ry), "n_slices": r.n_slices,
           "n_k": nk, "k_lower": arrs["k_lower"][:nk], "bin_counts": counts[:nk]}
    for m in MODE_BITS:
        if m in job.get("fem_modes", []):
            out[m] = arrs[m][:nk]
    if last is not None:
        out["last_psi"] = last.reshape(job["nx"], job["ny"], 2)
    return out


def transmission(job: dict, q, z, slice_index: int) -> np.ndarray:
    j, keep = make_job(job)
    a, keep2 = make_atoms(q, z)
    t = np.zeros(2 * job["nx"] * job["ny"])
    rc = lib().or_transmission(C.byref(j), C.byref(a), slice_index, _p(t))
    if rc != 0:
        raise RuntimeError("oracle or_transmission failed with code %d" % rc)
    return t.reshape(job["nx"], job["ny"], 2)


def probe(job: dict) -> np.ndarray:
    j, keep = make_job(job)
    pr = np.zeros(2 * job["nx"] * job["ny"])
    lib().or_probe(C.byref(j), _p(pr))
    return pr.reshape(job["nx"], job["ny"], 2)


def ring_bins(job: dict):
    j, keep = make_job(job)
    bins = np.zeros(job["nx"] * job["ny"], dtype=np.int32)
    counts = np.zeros(8192, dtype=np.int32)
    bounds = np.zeros(8192)
    nk = lib().or_ring_bins(C.byref(j), bins.ctypes.data_as(C.POINTER(C.c_int32)),
                            counts.ctypes.data_as(C.POINTER(C.c_int32)), _p(bounds), 8192)
    return {"n_k": nk, "bins": bins, "counts": counts[:nk], "k_lower": bounds[:nk]}


def replicate(q, z, dupe, periods):
    """--dupe atom replication in tem.cpp:1051-1143 order."""
    q = np.asarray(q).reshape(-1, 3)
    out_q, out_z = [], []
    for ii in range(dupe[0]):
        for jj in range(dupe[1]):
            for kk in range(dupe[2]):
                out_q.append(q + np.array([ii * periods[0], jj * periods[1], kk * periods[2]]))
                out_z.append(np.asarray(z))
    return np.concatenate(out_q), np.concatenate(out_z).astype(np.uint32)


def slice_atoms(q: np.ndarray, min_thickness: float):
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1)
    n = q.size // 3
    order = np.zeros(n + 1, dtype=np.int64)
    start = np.zeros(n + 2, dtype=np.int64)
    lower = np.zeros(n + 1)
    thick = np.zeros(n + 1)
    ns = lib().or_slice_atoms(n, _p(q), 0.0, 0.0, min_thickness,
                              order.ctypes.data_as(C.POINTER(C.c_int64)),
                              start.ctypes.data_as(C.POINTER(C.c_int64)),
                              _p(lower), _p(thick))
    return {"n": ns, "order": order[:n], "start": start[:ns + 1],
            "lower": lower[:ns], "thickness": thick[:ns]}


# ----------------------------------------------------- reference binary ----
def ref_available() -> bool:
    return REF_BIN.exists()


def run_reference(args, cwd, env_extra=None, timeout=None, md=False) -> dict:
    """Run oracle/_ref/ms-stem-fem-ref (md: ms-stem-fem-md-ref, whose LAMMPS
    "run" loads the next file of the list MSF_MD_REPLAY names) with argv
    ``args`` in ``cwd``; returns stdout, stderr and the adfstem wall time
    the link-time hook printed."""
    env = dict(os.environ)
    if env_extra:
        env.update(env_extra)
    p = subprocess.run([str(REF_MD_BIN if md else REF_BIN)] + list(args), cwd=str(cwd), env=env,
                       capture_output=True, text=True, timeout=timeout)
    m = re.search(r"adfstem_seconds=([0-9.eE+-]+) probes=(\d+) slices=(\d+)", p.stderr)
    return {"returncode": p.returncode, "stdout": p.stdout, "stderr": p.stderr,
            "adfstem_seconds": float(m.group(1)) if m else None,
            "probes": int(m.group(2)) if m else None,
            "slices": int(m.group(3)) if m else None}


def read_variance_txt(path) -> np.ndarray:
    """Read a ``k_lower value`` text file written by output_variance_to_txt."""
    rows = [l.split() for l in Path(path).read_text().splitlines() if l.strip()]
    return np.array([[float(a), float(b)] for a, b in rows])


# ------------------------------------------------------ job from argv -----
def read_lammps(path):
    """Minimal reader of the LAMMPS data grammar (tem_io.cpp:36-1028) for the
    oracle: returns positions shifted by the box origin, Z, periods."""
    lines = [l for l in Path(path).read_text().splitlines()]
    it = iter([l for l in lines[1:] if l.strip()])
    n = int(next(it).split()[0])
    nt = int(next(it).split()[0])
    lo, hi = [], []
    for _ in range(3):
        a, b = next(it).split()[:2]
        lo.append(float(a))
        hi.append(float(b))
    assert next(it).split()[0].lower() == "masses"
    zmap = {}
    for _ in range(nt):
        t, m = next(it).split()[:2]
        m = float(m)
        zmap[int(t)] = 14 if 28.0 <= m <= 28.1 else 8 if 15.9 <= m <= 16.0 else 0
    assert next(it).split()[0].lower() == "atoms"
    q, z = [], []
    for _ in range(n):
        p = next(it).split()
        q.append([float(p[2]) - lo[0], float(p[3]) - lo[1], float(p[4]) - lo[2]])
        z.append(zmap[int(p[1])])
    return np.array(q), np.array(z, dtype=np.uint32), [h - l for h, l in zip(hi, lo)]


def read_xyz(path):
    """Minimal reader of the xyz grammar (tem_io.cpp:4627-4958) for the
    oracle: count, periods, then element and position per line (symbols of
    the golden cases: Si in any case, or 14); positions shifted by their
    minimum taken from 0."""
    lines = Path(path).read_text().splitlines()
    n = int(lines[0].split()[0])
    per = [float(v) for v in lines[1].split()[:3]]
    q, z = [], []
    for line in lines[2:2 + n]:
        p = line.split()
        assert p[0].lower() in ("si", "14")
        q.append([float(v) for v in p[1:4]])
        z.append(14)
    q = np.array(q)
    q = q - np.minimum(q.min(axis=0), 0.0)
    return q, np.array(z, dtype=np.uint32), per


def job_from_argv(argv, cwd):
    """The oracle's own derivation of tem.cpp:405-1378 for an argv (the option
    subset the golden cases use).  Returns (job dict, q, z)."""
    a = list(argv)
    opt = {}
    flags = set()
    i = 0
    while i < len(a):
        k = a[i]
        if k in ("-a", "--output_prefix", "--cs3", "--cs5", "--defocus", "--alphamax",
                 "--rasterspacing", "--minslice", "--dr"):
            opt[k] = a[i + 1]
            i += 2
        elif k == "-m":
            opt[k] = a[i + 1:i + 4]
            i += 4
        elif k == "--dupe":
            opt[k] = a[i + 1:i + 4]
            i += 4
        else:
            flags.add(k)
            i += 1
    spec = Path(cwd) / opt["-a"]
    q, z, per = read_xyz(spec) if spec.suffix == ".xyz" else read_lammps(spec)
    nx, ny, vv = int(opt["-m"][0]), int(opt["-m"][1]), float(opt["-m"][2])
    lam = C.c_double()
    gam = C.c_double()
    lib().or_constants(vv, C.byref(lam), C.byref(gam))
    lam = lam.value
    fem = bool(flags & {"--adfstemuncorrfem", "--adfstemcorrfem"})
    corrected = bool(flags & {"--adfstemcorr", "--adfstemcorrfem"})
    cs3 = float(opt.get("--cs3", 0.0))
    cs5 = float(opt.get("--cs5", 0.0))
    defocus = float(opt.get("--defocus", 0.0))
    alpha = float(opt.get("--alphamax", 0.0))
    if not corrected:
        if "--scherzer_defocus" in flags:
            defocus = 0.87 * math.sqrt(cs3 * lam)
        if "--scherzer_alphamax" in flags:
            alpha = 1.34 * math.pow(lam / cs3, 0.25)
    else:
        if "--scherzer_defocus" in flags:
            defocus = -0.983 * math.pow(math.pow(lam, 2) * cs5, 1.0 / 3.0)
        if "--scherzer_alphamax" in flags:
            alpha = 1.513 * math.pow(lam / cs5, 1.0 / 6.0)
        if "--scherzer_cs3" in flags:
            cs3 = -2.289 * math.pow(lam * math.pow(cs5, 2), 1.0 / 3.0)
    spacing = float(opt.get("--rasterspacing", 10 if fem else 1.5))
    nrx = int(math.floor(per[0] / spacing))
    nry = int(math.floor(per[1] / spacing))
    xp = [0.0 + (i * (per[0] / nrx)) for i in range(nrx)]
    yp = [0.0 + (i * (per[1] / nry)) for i in range(nry)]
    dupe = [int(v) for v in opt.get("--dupe", [1, 1, 1])]
    if fem and "--dupe" in opt and max(dupe) > 1:
        q, z = replicate(q, z, dupe, per)
    modes = [m for m in MODE_BITS if "--" + m in flags] if fem else []
    if fem and not modes:
        modes = ["V_omega"]
    job = dict(nx=nx, ny=ny, voltage=vv, xperiod=per[0], yperiod=per[1],
               xperiod_duped=per[0] * dupe[0], yperiod_duped=per[1] * dupe[1],
               min_slice=float(opt.get("--minslice", 1.0)), corrected=int(corrected),
               cs3=cs3, cs5=cs5, defocus=defocus, alpha_max=alpha,
               det_inner=0.040 if vv >= 200000 else 0.045, det_outer=0.200,
               dr=float(opt.get("--dr", 0.70710678118654746)), x_p=xp, y_p=yp,
               images="--images" in flags, fem_modes=modes)
    return job, q, z
