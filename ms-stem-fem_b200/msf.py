"""Python binding of libmsf.so (the C ABI in include/msf.h).

This is the host-side mirror of the reference's interface for the
multislice path: ``parse_cmdline`` takes the reference's argv, ``Specimen``
does what tem.cpp:944-1276 does (LUTs, slicing, propagators, transmission
functions) and ``Context.run`` is ``adfstem()``.  All compute runs in the
CUDA library; there is no CPU fallback -- if libmsf.so is missing or no GPU
is present the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libmsf.so"
CLI_PATH = HERE / "bin" / "ms-stem-fem"
ABI_VERSION = 4  # MSF_ABI_VERSION of the include/msf.h these structs mirror

MSF_FP64, MSF_FP32 = 0, 1
OUT_ADF_IMAGE = 1 << 0
OUT_V_OMEGA, OUT_VBAR_R, OUT_V_RE = 1 << 1, 1 << 2, 1 << 3
OUT_OMEGA_VIMAGE, OUT_V_GT17, OUT_V_RBAR = 1 << 4, 1 << 5, 1 << 6
OUT_CORRELOGRAPH, OUT_CORRELOGRAPH_VAR = 1 << 7, 1 << 8
FEM_MODES = {"V_omega": OUT_V_OMEGA, "Vbar_r": OUT_VBAR_R, "V_re": OUT_V_RE,
             "Omega_vimage": OUT_OMEGA_VIMAGE, "V_gt17": OUT_V_GT17,
             "V_rbar": OUT_V_RBAR}
_FIELD = {"V_omega": "v_omega", "Vbar_r": "vbar_r", "V_re": "v_re",
          "Omega_vimage": "omega_vimage", "V_gt17": "v_gt17", "V_rbar": "v_rbar"}

# every symbol include/msf.h declares
EXPORTED = [
    "msf_abi_version", "msf_last_error", "msf_status_string",
    "msf_context_create", "msf_context_destroy", "msf_context_synchronize",
    "msf_specimen_create", "msf_specimen_destroy", "msf_specimen_slices",
    "msf_specimen_transmission", "msf_specimen_device_bytes", "msf_run",
    "msf_probe", "msf_wavelength", "msf_scherzer", "msf_raster_points",
    "msf_probe_shifts", "msf_ring_bins", "msf_parse_cmdline",
    "msf_job_destroy", "msf_job_describe", "msf_job_output_prefix",
    "msf_read_specimen", "msf_write_outputs", "msf_main", "msf_slice_atoms",
    "msf_time_passes", "msf_context_transfer_bytes", "msf_probe_noalloc",
    "msf_run_batch", "msf_server_create", "msf_server_submit", "msf_server_poll",
    "msf_server_stats_get", "msf_server_destroy", "msf_segment_count", "msf_run_partial",
    "msf_finish", "msf_run_plain", "msf_amorphous_positions", "msf_run_md", "msf_md_main",
    "msf_tune", "msf_wisdom_export", "msf_wisdom_import", "msf_server_cancel",
    "msf_specimen_live_columns", "msf_comm_create", "msf_comm_destroy",
    "msf_comm_allgather_host", "msf_run_sharded", "msf_server_grid_stats_get",
    "msf_context_keep_potentials", "msf_specimen_potential",
]
COMM_NCCL, COMM_HOST = 1, 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)


class Tuning(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("batch", C.c_int32),
                ("pipe", C.c_int32), ("ns_per_probe_slice", C.c_double)]


class Options(C.Structure):
    _fields_ = [("device", C.c_int32), ("precision", C.c_int32), ("batch", C.c_int32),
                ("use_graphs", C.c_int32), ("hbm_budget", C.c_int64)]


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("voltage", C.c_double),
                ("xperiod", C.c_double), ("yperiod", C.c_double), ("zperiod", C.c_double),
                ("dupe_x", C.c_int32), ("dupe_y", C.c_int32), ("dupe_z", C.c_int32),
                ("replicate_atoms", C.c_int32),
                ("xmin", C.c_double), ("ymin", C.c_double), ("zmin", C.c_double),
                ("min_slice", C.c_double)]


class Atoms(C.Structure):
    _fields_ = [("n_atoms", C.c_int64), ("q", _dp), ("z", C.POINTER(C.c_uint32))]


class Optics(C.Structure):
    _fields_ = [("corrected", C.c_int32), ("cs3", C.c_double), ("cs5", C.c_double),
                ("defocus", C.c_double), ("alpha_max", C.c_double)]


class Raster(C.Structure):
    _fields_ = [("n_x", C.c_int32), ("n_y", C.c_int32), ("x_p", _dp), ("y_p", _dp)]


class Detect(C.Structure):
    _fields_ = [("outputs", C.c_uint32), ("det_inner", C.c_double),
                ("det_outer", C.c_double), ("dr", C.c_double), ("n_mtf", C.c_int32),
                ("mtf", _dp), ("mtf_domain_sqr", _dp), ("mtf_resolution", C.c_double)]


class Results(C.Structure):
    _fields_ = [("adf_image", _dp), ("cap_k", C.c_int32), ("n_k", C.c_int32),
                ("k_lower", _dp), ("bin_counts", _ip), ("v_omega", _dp), ("vbar_r", _dp),
                ("v_re", _dp), ("omega_vimage", _dp), ("v_gt17", _dp), ("v_rbar", _dp),
                ("final_psi", _dp), ("mean_amplitude", _dp), ("mean_intensity", _dp),
                ("ring_amplitude", _dp), ("ring_intensity", _dp),
                ("probe_slices", C.c_int64), ("kernel_launches", C.c_int64),
                ("seconds_setup", C.c_double),
                ("seconds_raster", C.c_double),
                ("cap_phi", C.c_int32), ("n_phi", C.c_int32), ("phi_lower", _dp),
                ("correlograph", _dp), ("correlograph_sqr", _dp),
                ("correlograph_probes", _dp), ("first_psi", _dp),
                ("ms_row_pass", C.c_double), ("ms_col_pass", C.c_double),
                ("pass_batch", C.c_int32)]


class GridStats(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("completed", C.c_int64),
                ("p50_s", C.c_double), ("p99_s", C.c_double), ("max_s", C.c_double)]


class ShardInfo(C.Structure):
    _fields_ = [("p_begin", C.c_int64), ("p_end", C.c_int64), ("seconds_shard", C.c_double),
                ("seconds_exchange", C.c_double), ("seconds_finish", C.c_double)]


class Request(C.Structure):
    _fields_ = [("grid", Grid), ("atoms", Atoms), ("optics", Optics), ("raster", Raster),
                ("detect", Detect)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64),
                ("running", C.c_int64), ("waiting", C.c_int64), ("p50_s", C.c_double),
                ("p99_s", C.c_double), ("max_s", C.c_double),
                ("probe_slices_per_s", C.c_double), ("probe_slices", C.c_int64),
                ("device_bytes", C.c_int64)]


class MsfError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("msf status %d: %s" % (status, message))
        self.status = status


_lib = None


def lib() -> C.CDLL:
    """Load libmsf.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError("libmsf.so not built: run `make -C ms-stem-fem_b200` "
                               "(or __graft_entry__.build())")
        L = C.CDLL(str(LIB_PATH))
        L.msf_last_error.restype = C.c_char_p
        L.msf_status_string.restype = C.c_char_p
        L.msf_context_create.argtypes = [C.POINTER(Options), C.POINTER(C.c_void_p)]
        L.msf_context_destroy.argtypes = [C.c_void_p]
        L.msf_context_synchronize.argtypes = [C.c_void_p]
        L.msf_specimen_create.argtypes = [C.c_void_p, C.POINTER(Grid), C.POINTER(Atoms),
                                          C.POINTER(C.c_void_p)]
        L.msf_specimen_destroy.argtypes = [C.c_void_p]
        L.msf_specimen_slices.argtypes = [C.c_void_p, _ip, _dp, _dp, _lp, C.c_int32]
        L.msf_specimen_transmission.argtypes = [C.c_void_p, C.c_int32, _dp]
        L.msf_specimen_device_bytes.argtypes = [C.c_void_p]
        L.msf_specimen_device_bytes.restype = C.c_int64
        L.msf_specimen_live_columns.argtypes = [C.c_void_p]
        L.msf_specimen_live_columns.restype = C.c_int32
        L.msf_run.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(Optics), C.POINTER(Raster),
                              C.POINTER(Detect), C.POINTER(Results)]
        L.msf_probe.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(Optics), _dp]
        L.msf_amorphous_positions.argtypes = [C.c_int64, _dp, C.c_double, C.c_uint64,
                                              C.c_int64, _dp]
        L.msf_run_plain.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(Optics),
                                    C.POINTER(Raster), C.POINTER(Detect), C.POINTER(Results)]
        L.msf_wavelength.argtypes = [C.c_double, _dp, _dp]
        L.msf_wavelength.restype = None
        L.msf_scherzer.argtypes = [C.c_int32, C.c_double, C.c_double]
        L.msf_scherzer.restype = C.c_double
        L.msf_raster_points.argtypes = [C.c_double, C.c_double, C.c_double, _dp, C.c_int32]
        L.msf_probe_shifts.argtypes = [C.POINTER(Grid), C.POINTER(Raster), _lp]
        L.msf_ring_bins.argtypes = [C.POINTER(Grid), C.c_double, _ip, _ip]
        L.msf_parse_cmdline.argtypes = [C.c_int32, C.POINTER(C.c_char_p), C.POINTER(C.c_void_p)]
        L.msf_job_destroy.argtypes = [C.c_void_p]
        L.msf_job_describe.argtypes = [C.c_void_p, C.POINTER(Grid), C.POINTER(Atoms),
                                       C.POINTER(Optics), C.POINTER(Raster), C.POINTER(Detect)]
        L.msf_job_output_prefix.argtypes = [C.c_void_p]
        L.msf_job_output_prefix.restype = C.c_char_p
        L.msf_read_specimen.argtypes = [C.c_char_p, C.POINTER(C.c_void_p)]
        L.msf_write_outputs.argtypes = [C.c_void_p, C.POINTER(Results)]
        L.msf_main.argtypes = [C.c_int32, C.POINTER(C.c_char_p), C.POINTER(Options)]
        L.msf_md_main.argtypes = [C.c_int32, C.POINTER(C.c_char_p), C.POINTER(Options)]
        L.msf_tune.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(Tuning)]
        L.msf_wisdom_export.argtypes = [C.c_void_p, C.c_char_p, C.c_int64]
        L.msf_wisdom_export.restype = C.c_int64
        L.msf_wisdom_import.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_int32)]
        L.msf_run_md.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p), C.c_int32,
                                 C.POINTER(Optics), C.POINTER(Raster), C.POINTER(Detect),
                                 C.POINTER(Results)]
        L.msf_run_batch.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p),
                                    C.POINTER(Optics), C.POINTER(Raster), C.POINTER(Detect),
                                    C.POINTER(Results), C.c_int32]
        L.msf_server_create.argtypes = [C.POINTER(Options), C.c_int32, C.POINTER(C.c_void_p)]
        L.msf_server_submit.argtypes = [C.c_void_p, C.POINTER(Request), C.POINTER(C.c_uint64)]
        L.msf_server_poll.argtypes = [C.c_void_p, C.c_uint64, C.c_int32, C.POINTER(Results)]
        L.msf_server_cancel.argtypes = [C.c_void_p, C.c_uint64]
        L.msf_server_stats_get.argtypes = [C.c_void_p, C.POINTER(ServerStats)]
        L.msf_server_destroy.argtypes = [C.c_void_p]
        L.msf_segment_count.argtypes = [C.POINTER(Grid), C.POINTER(Detect)]
        L.msf_segment_count.restype = C.c_int32
        L.msf_run_partial.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(Optics),
                                      C.POINTER(Raster), C.POINTER(Detect), C.c_int64,
                                      C.c_int64, _dp, _dp, _dp, _dp, C.POINTER(Results)]
        L.msf_finish.argtypes = [C.POINTER(Grid), C.POINTER(Optics), C.POINTER(Detect),
                                 C.c_int64, _dp, _dp, _dp, _dp, C.POINTER(Results)]
        L.msf_slice_atoms.argtypes = [C.c_int64, _dp, C.c_double, C.c_double, C.c_double,
                                      _ip, _dp, _dp, _lp, _lp, C.c_int32]
        L.msf_context_transfer_bytes.argtypes = [C.c_void_p, _lp, _lp, C.c_int32]
        L.msf_probe_noalloc.argtypes = [C.POINTER(Grid), C.POINTER(Optics), C.c_void_p,
                                        C.c_void_p]
        L.msf_time_passes.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, _dp, _dp]
        L.msf_context_keep_potentials.argtypes = [C.c_void_p, C.c_int32]
        L.msf_specimen_potential.argtypes = [C.c_void_p, C.c_int32, _dp]
        L.msf_server_grid_stats_get.argtypes = [C.c_void_p, C.POINTER(GridStats), C.c_int32]
        L.msf_comm_create.argtypes = [C.c_int32, C.c_int32, C.c_char_p, C.c_int32, C.c_int32,
                                      C.c_double, C.POINTER(C.c_void_p)]
        L.msf_comm_destroy.argtypes = [C.c_void_p]
        L.msf_comm_destroy.restype = None
        L.msf_comm_allgather_host.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
        L.msf_run_sharded.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(Optics),
                                      C.POINTER(Raster), C.POINTER(Detect), C.c_void_p,
                                      C.POINTER(Results), C.POINTER(ShardInfo)]
        if L.msf_abi_version() != ABI_VERSION:
            raise RuntimeError("libmsf.so has ABI version %d, these bindings expect %d: "
                               "rebuild it" % (L.msf_abi_version(), ABI_VERSION))
        _lib = L
    return _lib


def _check(status):
    if status != 0:
        raise MsfError(status, lib().msf_last_error().decode(errors="replace"))


def _p(a):
    return a.ctypes.data_as(_dp)


def slice_atoms(q: np.ndarray, min_slice: float, zmin: float = 0.0, zperiod: float = 0.0):
    """Host-only slicing (slice.cpp:469-980): boundaries, counts, atom order."""
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1)
    n = q.size // 3
    cap = max(1, n)
    lower, thick = np.zeros(cap), np.zeros(cap)
    counts, order = np.zeros(cap, dtype=np.int64), np.zeros(cap, dtype=np.int64)
    ns = C.c_int32()
    _check(lib().msf_slice_atoms(n, _p(q), zmin, zperiod, min_slice, C.byref(ns), _p(lower),
                                 _p(thick), counts.ctypes.data_as(_lp),
                                 order.ctypes.data_as(_lp), cap))
    k = ns.value
    return {"n": k, "lower": lower[:k], "thickness": thick[:k], "counts": counts[:k],
            "order": order[:n]}


def wavelength(voltage: float):
    lam, gam = C.c_double(), C.c_double()
    lib().msf_wavelength(voltage, C.byref(lam), C.byref(gam))
    return lam.value, gam.value


class Job:
    """A parsed reference command line plus its specimen (tem.cpp:81-1378)."""

    def __init__(self, argv):
        argv = [str(a) for a in argv]
        if not argv or not argv[0].endswith("ms-stem-fem"):
            argv = ["ms-stem-fem"] + argv
        arr = (C.c_char_p * len(argv))(*[a.encode() for a in argv])
        h = C.c_void_p()
        _check(lib().msf_parse_cmdline(len(argv), arr, C.byref(h)))
        self._h = h
        self.grid, self.atoms = Grid(), Atoms()
        self.optics, self.raster, self.detect = Optics(), Raster(), Detect()
        _check(lib().msf_job_describe(h, C.byref(self.grid), C.byref(self.atoms),
                                      C.byref(self.optics), C.byref(self.raster),
                                      C.byref(self.detect)))
        self.prefix = lib().msf_job_output_prefix(h).decode()

    @property
    def n_probes(self):
        return self.raster.n_x * self.raster.n_y

    def positions(self):
        n = self.atoms.n_atoms
        q = np.ctypeslib.as_array(self.atoms.q, shape=(3 * n,)).copy().reshape(n, 3)
        z = np.ctypeslib.as_array(self.atoms.z, shape=(n,)).copy()
        return q, z

    def raster_points(self):
        r = self.raster
        return (np.ctypeslib.as_array(r.x_p, shape=(r.n_x,)).copy(),
                np.ctypeslib.as_array(r.y_p, shape=(r.n_y,)).copy())

    def fem_modes(self):
        return [m for m, b in FEM_MODES.items() if self.detect.outputs & b]

    def oracle_job(self) -> dict:
        """The same job as a plain dict (the CPU oracle's input format)."""
        xp, yp = self.raster_points()
        g, o, d = self.grid, self.optics, self.detect
        return dict(nx=g.nx, ny=g.ny, voltage=g.voltage, xperiod=g.xperiod,
                    yperiod=g.yperiod, xperiod_duped=g.xperiod * max(1, g.dupe_x),
                    yperiod_duped=g.yperiod * max(1, g.dupe_y), xmin=g.xmin, ymin=g.ymin,
                    min_slice=g.min_slice, corrected=o.corrected, cs3=o.cs3, cs5=o.cs5,
                    defocus=o.defocus, alpha_max=o.alpha_max, det_inner=d.det_inner,
                    det_outer=d.det_outer, dr=d.dr, x_p=xp, y_p=yp,
                    images=bool(d.outputs & OUT_ADF_IMAGE), fem_modes=self.fem_modes())

    def write_outputs(self, res: "RunResult"):
        _check(lib().msf_write_outputs(self._h, C.byref(res._struct)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.msf_job_destroy(h)
            self._h = None


class Context:
    """One CUDA device, one stream, one wavefield precision."""

    def __init__(self, device=0, precision="fp64", batch=0, graphs=True, hbm_budget=0):
        opt = Options(device, MSF_FP32 if precision == "fp32" else MSF_FP64, batch,
                      1 if graphs else 0, hbm_budget)
        h = C.c_void_p()
        _check(lib().msf_context_create(C.byref(opt), C.byref(h)))
        self._h = h
        self.precision = precision

    def keep_potentials(self, on=True):
        """Specimens built from now on keep their slices' projected
        potentials (msf_context_keep_potentials; --paptif)."""
        _check(lib().msf_context_keep_potentials(self._h, 1 if on else 0))

    def close(self):
        if getattr(self, "_h", None) is not None:
            lib().msf_context_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def transfer_bytes(self, reset=False):
        """(host->device, device->host) bytes copied since the last reset."""
        h, d = C.c_int64(), C.c_int64()
        _check(lib().msf_context_transfer_bytes(self._h, C.byref(h), C.byref(d), int(reset)))
        return h.value, d.value

    def synchronize(self):
        _check(lib().msf_context_synchronize(self._h))

    def specimen(self, grid: Grid, q: np.ndarray, z: np.ndarray) -> "Specimen":
        return Specimen(self, grid, q, z)

    def tune(self, spec: "Specimen") -> dict:
        """Measure the launch tiling for the specimen's grid (msf_tune); the
        context uses the winner for that grid from then on."""
        t = Tuning()
        _check(lib().msf_tune(self._h, spec._h, C.byref(t)))
        return {"nx": t.nx, "ny": t.ny, "batch": t.batch, "pipe": t.pipe,
                "ns_per_probe_slice": t.ns_per_probe_slice}

    def wisdom_export(self) -> str:
        n = lib().msf_wisdom_export(self._h, None, 0)
        buf = C.create_string_buffer(n + 1)
        lib().msf_wisdom_export(self._h, buf, n + 1)
        return buf.value.decode()

    def wisdom_import(self, text: str) -> int:
        n = C.c_int32()
        _check(lib().msf_wisdom_import(self._h, text.encode(), C.byref(n)))
        return n.value

    def run(self, spec: "Specimen", optics: Optics, raster: Raster, detect: Detect,
            want_final_psi=False, want_means=False, want_rings=False,
            cap_k=8192, want_correlograph_probes=False) -> "RunResult":
        nx, ny = spec.grid.nx, spec.grid.ny
        n_r = raster.n_x * raster.n_y
        if want_rings:
            cap_k = min(cap_k, 1024)
        out = RunResult(n_r, cap_k, nx, ny, want_final_psi, want_means, want_rings)
        if detect.outputs & OUT_CORRELOGRAPH:
            out.add_correlograph(spec.grid, detect, n_r, want_correlograph_probes)
        _check(lib().msf_run(self._h, spec._h, C.byref(optics), C.byref(raster),
                             C.byref(detect), C.byref(out._struct)))
        out.finish(raster, detect)
        return out

    def run_md(self, snapshots, samples: int, optics: Optics, raster: Raster, detect: Detect,
               want_final_psi=False, want_means=False, want_rings=False,
               cap_k=8192) -> "RunResult":
        """MD-coupled FEM (msf_run_md): each probe through `samples`
        configurations, sample s through snapshots[s % len(snapshots)], exit
        waves averaged coherently before the FEM statistics."""
        g = snapshots[0].grid
        n_r = raster.n_x * raster.n_y
        if want_rings:
            cap_k = min(cap_k, 1024)
        out = RunResult(n_r, cap_k, g.nx, g.ny, want_final_psi, want_means, want_rings)
        if detect.outputs & OUT_CORRELOGRAPH:
            out.add_correlograph(g, detect, n_r, False)
        hs = (C.c_void_p * len(snapshots))(*[sp._h.value for sp in snapshots])
        _check(lib().msf_run_md(self._h, len(snapshots), hs, int(samples), C.byref(optics),
                                C.byref(raster), C.byref(detect), C.byref(out._struct)))
        out.finish(raster, detect)
        return out

    def run_plain(self, spec: "Specimen", optics: Optics, raster: Raster, detect: Detect,
                  want_final_psi=False, cap_k=8192) -> "RunResult":
        """The raster one probe at a time, one launch per reference step
        (msf_run_plain; FP64 contexts)."""
        out = RunResult(raster.n_x * raster.n_y, cap_k, spec.grid.nx, spec.grid.ny,
                        want_final_psi, False)
        _check(lib().msf_run_plain(self._h, spec._h, C.byref(optics), C.byref(raster),
                                   C.byref(detect), C.byref(out._struct)))
        out.finish(raster, detect)
        return out

    def run_batch(self, jobs, slots=0, want_means=False, want_rings=False, cap_k=8192):
        """Several rasters through slot lanes (msf_run_batch).

        jobs: sequence of (Specimen, Optics, Raster, Detect); returns one
        RunResult per job, as ``run`` would (without the final wave)."""
        n = len(jobs)
        specs = (C.c_void_p * n)(*[j[0]._h.value for j in jobs])
        optics = (Optics * n)(*[j[1] for j in jobs])
        rasters = (Raster * n)(*[j[2] for j in jobs])
        detects = (Detect * n)(*[j[3] for j in jobs])
        outs = []
        for spec, _, raster, _ in jobs:
            ck = min(cap_k, 1024) if want_rings else cap_k
            outs.append(RunResult(raster.n_x * raster.n_y, ck, spec.grid.nx, spec.grid.ny,
                                  False, want_means, want_rings))
        structs = (Results * n)(*[o._struct for o in outs])
        _check(lib().msf_run_batch(self._h, n, specs, optics, rasters, detects, structs,
                                   slots))
        for k, (o, j) in enumerate(zip(outs, jobs)):
            o._struct = structs[k]
            o.finish(j[2], j[3])
        return outs

    def run_partial(self, spec: "Specimen", optics: Optics, raster: Raster, detect: Detect,
                    p_begin: int, p_end: int) -> dict:
        """Per-probe sums of probes [p_begin, p_end) (msf_run_partial)."""
        n_seg = segment_count(spec.grid, detect)
        rows = max(p_end - p_begin, 0)  # the library rejects empty or reversed ranges
        amp = np.zeros((rows, n_seg))
        inten = np.zeros((rows, n_seg))
        plane = spec.grid.nx * spec.grid.ny
        pix = bool(detect.outputs & (OUT_V_RE | OUT_OMEGA_VIMAGE | OUT_V_GT17 | OUT_V_RBAR))
        acc_a = np.zeros(plane) if pix else None
        acc_i = np.zeros(plane) if pix else None
        info = Results()
        _check(lib().msf_run_partial(self._h, spec._h, C.byref(optics), C.byref(raster),
                                     C.byref(detect), p_begin, p_end, _p(amp), _p(inten),
                                     _p(acc_a) if pix else None, _p(acc_i) if pix else None,
                                     C.byref(info)))
        return {"amp": amp, "inten": inten, "acc_a": acc_a, "acc_i": acc_i,
                "probe_slices": info.probe_slices, "kernel_launches": info.kernel_launches,
                "seconds_raster": info.seconds_raster, "n_k": info.n_k}

    def run_sharded(self, spec: "Specimen", optics: Optics, raster: Raster, detect: Detect,
                    comm: "Comm", want_means=False, cap_k=8192) -> "RunResult":
        """msf_run over the communicator's ranks (msf_run_sharded): every rank
        returns the whole raster's ADF image and FEM statistics; `shard` on
        the result holds this rank's probe range and timings."""
        nx, ny = spec.grid.nx, spec.grid.ny
        out = RunResult(raster.n_x * raster.n_y, cap_k, nx, ny, False, want_means)
        info = ShardInfo()
        _check(lib().msf_run_sharded(self._h, spec._h, C.byref(optics), C.byref(raster),
                                     C.byref(detect), comm._h, C.byref(out._struct),
                                     C.byref(info)))
        out.finish(raster, detect)
        out.shard = {f: getattr(info, f) for f, _ in ShardInfo._fields_}
        return out

    def time_passes(self, spec: "Specimen", nb: int, reps: int = 10):
        """Mean ms per launch of the fused row and column slice passes."""
        r, c = C.c_double(), C.c_double()
        _check(lib().msf_time_passes(self._h, spec._h, nb, reps, C.byref(r), C.byref(c)))
        return r.value, c.value

    def probe(self, spec: "Specimen", optics: Optics) -> np.ndarray:
        out = np.zeros(2 * spec.grid.nx * spec.grid.ny)
        _check(lib().msf_probe(self._h, spec._h, C.byref(optics), _p(out)))
        return out.reshape(spec.grid.nx, spec.grid.ny, 2)


def amorphous_positions(n_atoms: int, box, min_sep: float = 2.2, seed: int = 0,
                        max_proposals: int = 0) -> np.ndarray:
    """Seeded random-sequential-addition positions ((n_atoms, 3), host C++;
    msf_amorphous_positions)."""
    q = np.zeros((n_atoms, 3))
    b = np.ascontiguousarray(box, dtype=np.float64)
    _check(lib().msf_amorphous_positions(n_atoms, _p(b), min_sep, seed, max_proposals, _p(q)))
    return q


def segment_count(grid: Grid, detect: Detect) -> int:
    """Detector segments per probe: FEM ring bins, then the ADF annulus."""
    return lib().msf_segment_count(C.byref(grid), C.byref(detect))


def finish(grid: Grid, optics: Optics, raster: Raster, detect: Detect, amp, inten,
           acc_a=None, acc_i=None, want_means=False, cap_k=8192) -> "RunResult":
    """ADF image and FEM statistics from the per-probe rows of a whole raster
    (msf_finish; host only, no GPU)."""
    amp = np.ascontiguousarray(amp, dtype=np.float64)
    inten = np.ascontiguousarray(inten, dtype=np.float64)
    n = raster.n_x * raster.n_y
    assert amp.shape[0] == n and inten.shape[0] == n
    out = RunResult(n, cap_k, grid.nx, grid.ny, False, want_means)
    a_a = None if acc_a is None else np.ascontiguousarray(acc_a, dtype=np.float64)
    a_i = None if acc_i is None else np.ascontiguousarray(acc_i, dtype=np.float64)
    _check(lib().msf_finish(C.byref(grid), C.byref(optics), C.byref(detect), n, _p(amp),
                            _p(inten), None if a_a is None else _p(a_a),
                            None if a_i is None else _p(a_i), C.byref(out._struct)))
    out.finish(raster, detect)
    return out


def _prefer_framework_nccl():
    """Point the library at the NCCL of the Python environment's `nvidia-nccl`
    wheel (the one torch links against) unless MSF_NCCL_LIBRARY is set, so
    that a later `import torch` in this process finds the NCCL it expects."""
    if os.environ.get("MSF_NCCL_LIBRARY"):
        return
    import importlib.util
    try:
        spec = importlib.util.find_spec("nvidia.nccl")
    except (ImportError, ValueError):
        spec = None
    for base in (spec.submodule_search_locations if spec else None) or []:
        path = os.path.join(base, "lib", "libnccl.so.2")
        if os.path.exists(path):
            os.environ["MSF_NCCL_LIBRARY"] = path
            return


class Comm:
    """A communicator of `world` ranks (msf_comm_create): rank 0 listens at
    `rendezvous` ("host:port"), the others connect; transport COMM_NCCL
    (device buffers, one GPU per rank) or COMM_HOST (through the bootstrap
    connections).  Collective: every rank creates one."""

    def __init__(self, rank: int, world: int, rendezvous: str = "", transport: int = COMM_HOST,
                 device: int = -1, timeout_s: float = 60.0):
        if transport == COMM_NCCL:
            _prefer_framework_nccl()
        h = C.c_void_p()
        _check(lib().msf_comm_create(rank, world, rendezvous.encode(), transport, device,
                                     timeout_s, C.byref(h)))
        self._h = h
        self.rank, self.world = rank, world

    def allgather(self, a: np.ndarray) -> np.ndarray:
        """Every rank's `a` (same shape and dtype on all ranks), stacked in
        rank order."""
        a = np.ascontiguousarray(a)
        out = np.empty((self.world,) + a.shape, dtype=a.dtype)
        _check(lib().msf_comm_allgather_host(self._h, a.ctypes.data, a.nbytes,
                                             out.ctypes.data))
        return out

    def close(self):
        if self._h:
            lib().msf_comm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Request loop with continuous batching (msf_server_*), FP32 wavefields."""

    def __init__(self, device=0, slots=0, hbm_budget=0, graphs=True):
        opt = Options(device, MSF_FP32, 0, 1 if graphs else 0, hbm_budget)
        h = C.c_void_p()
        _check(lib().msf_server_create(C.byref(opt), slots, C.byref(h)))
        self._h = h
        self._pending = {}

    def submit(self, grid: Grid, q, z, optics: Optics, raster: Raster, detect: Detect) -> int:
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1)
        z = np.ascontiguousarray(z, dtype=np.uint32)
        req = Request(grid, Atoms(len(z), _p(q), z.ctypes.data_as(C.POINTER(C.c_uint32))),
                      optics, raster, detect)
        t = C.c_uint64()
        _check(lib().msf_server_submit(self._h, C.byref(req), C.byref(t)))
        self._pending[t.value] = (grid.nx, grid.ny, raster, detect)
        return t.value

    def poll(self, ticket: int, wait_ms=0, want_means=False, want_rings=False, cap_k=8192):
        """RunResult when finished, None while queued or running."""
        nx, ny, raster, detect = self._pending[ticket]
        ck = min(cap_k, 1024) if want_rings else cap_k
        out = RunResult(raster.n_x * raster.n_y, ck, nx, ny, False, want_means, want_rings)
        st = lib().msf_server_poll(self._h, ticket, int(wait_ms), C.byref(out._struct))
        if st == 8:  # MSF_ERR_BUSY
            return None
        del self._pending[ticket]
        _check(st)
        out.finish(raster, detect)
        return out

    def cancel(self, ticket: int):
        """Cancel a request (msf_server_cancel): its poll then raises
        MsfError with status MSF_ERR_CANCELLED (9)."""
        _check(lib().msf_server_cancel(self._h, C.c_uint64(ticket)))

    def stats(self) -> dict:
        s = ServerStats()
        _check(lib().msf_server_stats_get(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in ServerStats._fields_}

    def grid_stats(self) -> list:
        """Latency per grid size of the completed requests
        (msf_server_grid_stats_get), in order of grid size."""
        n = lib().msf_server_grid_stats_get(self._h, None, 0)
        arr = (GridStats * max(n, 1))()
        n = lib().msf_server_grid_stats_get(self._h, arr, n)
        return [{f: getattr(arr[k], f) for f, _ in GridStats._fields_} for k in range(n)]

    def close(self):
        if getattr(self, "_h", None) is not None:
            lib().msf_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class Specimen:
    """Device-resident LUTs, slices, propagators and transmission functions."""

    def __init__(self, ctx: Context, grid: Grid, q: np.ndarray, z: np.ndarray):
        self.ctx = ctx
        self.grid = grid
        self._q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1)
        self._z = np.ascontiguousarray(z, dtype=np.uint32)
        atoms = Atoms(len(self._z), _p(self._q), self._z.ctypes.data_as(C.POINTER(C.c_uint32)))
        h = C.c_void_p()
        _check(lib().msf_specimen_create(ctx._h, C.byref(grid), C.byref(atoms), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None:
            lib().msf_specimen_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def slices(self):
        n = C.c_int32()
        lib().msf_specimen_slices(self._h, C.byref(n), None, None, None, 0)
        k = n.value
        lower, thick = np.zeros(k), np.zeros(k)
        counts = np.zeros(k, dtype=np.int64)
        _check(lib().msf_specimen_slices(self._h, C.byref(n), _p(lower), _p(thick),
                                         counts.ctypes.data_as(_lp), k))
        return {"n": k, "lower": lower, "thickness": thick, "counts": counts}

    def transmission(self, s: int) -> np.ndarray:
        out = np.zeros(2 * self.grid.nx * self.grid.ny)
        _check(lib().msf_specimen_transmission(self._h, s, _p(out)))
        return out.reshape(self.grid.nx, self.grid.ny, 2)

    def potential(self, s: int) -> np.ndarray:
        """Slice s's projected potential before the exponential
        (msf_specimen_potential; the context must keep potentials)."""
        out = np.zeros(2 * self.grid.nx * self.grid.ny)
        _check(lib().msf_specimen_potential(self._h, s, _p(out)))
        return out.reshape(self.grid.nx, self.grid.ny, 2)

    def device_bytes(self) -> int:
        return lib().msf_specimen_device_bytes(self._h)

    def live_columns(self) -> int:
        """Columns in which the band limit keeps any kx."""
        return lib().msf_specimen_live_columns(self._h)


class RunResult:
    def __init__(self, n_r, cap_k, nx, ny, want_psi, want_means, want_rings=False):
        self.adf_image = np.zeros(n_r)
        self.k_lower = np.zeros(cap_k)
        self.bin_counts = np.zeros(cap_k, dtype=np.int32)
        self._v = {m: np.full(cap_k, np.nan) for m in FEM_MODES}
        self.final_psi = np.zeros(2 * nx * ny) if want_psi else None
        self.first_psi = np.zeros(2 * nx * ny) if want_psi else None
        self.mean_amplitude = np.zeros(nx * ny) if want_means else None
        self.mean_intensity = np.zeros(nx * ny) if want_means else None
        s = Results()
        s.adf_image = _p(self.adf_image)
        s.cap_k = cap_k
        s.k_lower = _p(self.k_lower)
        s.bin_counts = self.bin_counts.ctypes.data_as(_ip)
        for m, f in _FIELD.items():
            setattr(s, f, _p(self._v[m]))
        if want_psi:
            s.final_psi = _p(self.final_psi)
            s.first_psi = _p(self.first_psi)
        if want_means:
            s.mean_amplitude = _p(self.mean_amplitude)
            s.mean_intensity = _p(self.mean_intensity)
        self.ring_amp = np.zeros(n_r * cap_k) if want_rings else None
        self.ring_int = np.zeros(n_r * cap_k) if want_rings else None
        if want_rings:
            s.ring_amplitude = _p(self.ring_amp)
            s.ring_intensity = _p(self.ring_int)
        self._cap_k = cap_k
        self._n_r = n_r
        self._struct = s
        self._shape = (nx, ny)

    def add_correlograph(self, grid, detect, n_r, per_probe):
        """Buffers for the FEM correlograph, sized from the segment counts."""
        plain = Detect.from_buffer_copy(detect)
        plain.outputs = (detect.outputs & ~(OUT_CORRELOGRAPH | OUT_CORRELOGRAPH_VAR)) | OUT_V_OMEGA
        n_k = segment_count(grid, plain) - 1
        n_phi = (segment_count(grid, detect) - 1 - n_k) // max(n_k, 1)
        nc = max(1, n_k * n_phi)
        self.phi_lower = np.zeros(n_phi + 1)
        self._corr = np.zeros(nc)
        self._corr_sqr = np.zeros(nc)
        self._corr_probes = np.zeros(nc * n_r) if per_probe else None
        s = self._struct
        s.cap_phi = n_phi
        s.phi_lower = _p(self.phi_lower)
        s.correlograph = _p(self._corr)
        s.correlograph_sqr = _p(self._corr_sqr)
        if per_probe:
            s.correlograph_probes = _p(self._corr_probes)
        self._corr_shape = (n_k, n_phi)

    def finish(self, raster, detect):
        s = self._struct
        self.n_k = s.n_k
        self.probe_slices = s.probe_slices
        self.kernel_launches = s.kernel_launches
        self.seconds_raster = s.seconds_raster
        self.ms_row_pass, self.ms_col_pass = s.ms_row_pass, s.ms_col_pass
        self.pass_batch = s.pass_batch
        self.adf_image_2d = self.adf_image.reshape(raster.n_x, raster.n_y)
        self.v = {m: self._v[m][:self.n_k] for m in FEM_MODES if detect.outputs & FEM_MODES[m]}
        self.k = self.k_lower[:self.n_k]
        self.counts = self.bin_counts[:self.n_k]
        if getattr(self, "_corr_shape", None):
            n_k, n_phi = self._corr_shape
            # [jj * n_k + ii] -> array [ii (k), jj (phi)]
            self.correlograph = self._corr[:n_k * n_phi].reshape(n_phi, n_k).T
            self.correlograph_sqr = self._corr_sqr[:n_k * n_phi].reshape(n_phi, n_k).T
            if self._corr_probes is not None:
                self.correlograph_probes = self._corr_probes.reshape(
                    -1, n_phi, n_k).transpose(0, 2, 1)
        if self.ring_amp is not None:
            self.rings_amp = self.ring_amp.reshape(self._n_r, self._cap_k)[:, :self.n_k]
            self.rings_int = self.ring_int.reshape(self._n_r, self._cap_k)[:, :self.n_k]
        if self.final_psi is not None:
            self.final_psi_2d = self.final_psi.reshape(*self._shape, 2)


def run_job(argv, precision="fp64", device=0, batch=0, graphs=True, write=False,
            want_final_psi=False):
    """Parse a reference command line and run it end to end on the GPU."""
    job = Job(argv)
    ctx = Context(device=device, precision=precision, batch=batch, graphs=graphs)
    q, z = job.positions()
    spec = ctx.specimen(job.grid, q, z)
    res = ctx.run(spec, job.optics, job.raster, job.detect, want_final_psi=want_final_psi)
    if write:
        job.write_outputs(res)
    return job, spec, res, ctx


def main(argv, precision="fp64", device=0, batch=0, md=False) -> int:
    """The whole drop-in program (msf_main, or msf_md_main for the
    MD-coupled driver); returns the exit status."""
    argv = [str(a) for a in argv]
    arr = (C.c_char_p * len(argv))(*[a.encode() for a in argv])
    opt = Options(device, MSF_FP32 if precision == "fp32" else MSF_FP64, batch, 1, 0)
    return (lib().msf_md_main if md else lib().msf_main)(len(argv), arr, C.byref(opt))
