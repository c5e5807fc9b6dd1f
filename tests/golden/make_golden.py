#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ by running the reference's
own sources (built by oracle/Makefile into oracle/_ref/ms-stem-fem-ref) on
seeded specimens.

    make -C oracle && python tests/golden/make_golden.py [case ...]

Each case writes ``<case>.npz`` (outputs of the reference run: raw FP64 ADF
image, every FEM V(k) text file, slice boundaries, optionally one slice's
transmission function) and ``<case>.json`` (argv, specimen recipe, sha256 of
the specimen file).  Small specimens are committed as ``<case>.data``; large
ones are regenerated from their seed by the tests and checked against the
recorded sha256.  Needs the reference sources; the GPU box only reads the
committed fixtures.
"""
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "ms-stem-fem_b200"))
sys.path.insert(0, str(ROOT / "oracle"))
import specimen  # noqa: E402
import oracle  # noqa: E402
from tif16 import read_tif16  # noqa: E402

FEM_ALL = ["--V_omega", "--Vbar_r", "--V_re", "--Omega_vimage", "--V_gt17", "--V_rbar"]

# name -> (specimen recipe, argv after "-a <file> --output_prefix <name>",
#          commit the specimen file?, dump transmission of this slice or None)
CASES = {
    # configuration 1: plain ADF-STEM, 780 Si in 25 A, 256^2, 16x16 probes
    "c1": (dict(n=780, box=(25, 25, 25), seed=1),
           "-m 256 256 200000 --adfstemuncorr --cs3 1.3e7 --scherzer_defocus "
           "--alphamax 0.010 --rasterspacing 1.5625 --minslice 2.0 --images", True, None),
    # every FEM mode on a small grid; alpha_max zeroes the first bins
    "fem128": (dict(n=780, box=(25, 25, 25), seed=1),
               "-m 128 128 200000 --adfstemuncorrfem " + " ".join(FEM_ALL) +
               " --cs3 1.3e7 --scherzer_defocus --alphamax 0.010 --rasterspacing 6.25 "
               "--minslice 2.0 --images", True, 2),
    # aberration-corrected probe with Scherzer Cs3/defocus/aperture
    "corr": (dict(n=780, box=(25, 25, 25), seed=1),
             "-m 128 128 200000 --adfstemcorrfem --V_omega --V_re --cs5 5e7 --scherzer_cs3 "
             "--scherzer_defocus --scherzer_alphamax --rasterspacing 6.25 --minslice 2.0 "
             "--images", True, None),
    # non-square grid (sqrt(NxNy) scaling, different k steps along x and y)
    "rect": (dict(n=780, box=(25, 25, 25), seed=1),
             "-m 128 64 200000 --adfstemuncorrfem --V_omega --Vbar_r --cs3 1.3e7 --defocus 300 "
             "--alphamax 0.012 --rasterspacing 5 --minslice 2.0 --images --dr 1.0", True, None),
    # two species (Si + O) and 300 kV
    "sio": (dict(n=400, box=(20, 20, 20), seed=7, two_species=True),
            "-m 128 128 300000 --adfstemuncorrfem --V_omega --V_gt17 --cs3 1.3e7 "
            "--scherzer_defocus --scherzer_alphamax --rasterspacing 5 --minslice 2.0 --images",
            True, 0),
    # --dupe 2 1 1 in an FEM run replicates the atoms; raster uses one cell
    "dupe": (dict(n=390, box=(25, 25, 12.5), seed=11),
             "-m 128 64 200000 --adfstemuncorrfem --V_omega --dupe 2 1 1 --cs3 1.3e7 "
             "--scherzer_defocus --alphamax 0.010 --rasterspacing 6.25 --minslice 2.0 --images",
             True, None),
    # configuration 2's specimen and grid on a 2x2 raster (the full 64x64
    # raster would take hours on one CPU core)
    "c2_small": (dict(n=50000, box=(100, 100, 100), seed=2),
                 "-m 1024 1024 200000 --adfstemuncorrfem --V_omega --V_re --cs3 1.3e7 "
                 "--defocus 0 --alphamax 0.0015 --rasterspacing 50 --minslice 2.0 --dr 1.2065",
                 False, None),
    # configuration 2 on a 16x16 raster: enough probes that the V(k) bins sit
    # well above the cancellation floor of n*sum(A^2)/sum(A)^2 - 1
    "c2_r16": (dict(n=50000, box=(100, 100, 100), seed=2),
               "-m 1024 1024 200000 --adfstemuncorrfem --V_omega --V_re --cs3 1.3e7 "
               "--defocus 0 --alphamax 0.0015 --rasterspacing 6.25 --minslice 2.0 "
               "--dr 1.2065", False, None),
    # 512^2 grid (the smallest grid of the uneven batch), thin slab, 200 kV
    "g512": (dict(n=1250, box=(50, 50, 10), seed=51, gen="msf"),
             "-m 512 512 200000 --adfstemuncorrfem --V_omega --V_re --cs3 1.3e7 "
             "--scherzer_defocus --alphamax 0.010 --rasterspacing 16.5 --minslice 2.0 "
             "--images", False, None),
    # 2048^2 grid with the precision-stress optics (300 kV, Scherzer defocus
    # and aperture), thin slab
    "g2048": (dict(n=20000, box=(200, 200, 10), seed=52, gen="msf"),
              "-m 2048 2048 300000 --adfstemuncorrfem --V_omega --V_re --cs3 1.3e7 "
              "--scherzer_defocus --scherzer_alphamax --rasterspacing 66 --minslice 2.0 "
              "--images", False, None),
    # the largest grid the library supports, 4096^2 (a dilute 4 A slab keeps
    # the reference's atom-by-pixel potential sum short), 300 kV Scherzer
    "g4096": (dict(n=60, box=(400, 400, 4), seed=81, gen="msf"),
              "-m 4096 4096 300000 --adfstemuncorrfem --V_omega --cs3 1.3e7 "
              "--scherzer_defocus --scherzer_alphamax --rasterspacing 200 --minslice 2.0 "
              "--images", False, None),
    # the precision-stress specimen itself (600k Si, 200x200x300 A, 2048^2,
    # 300 kV, ~150 slices) on a 4x4 raster
    "c4_r4": (dict(n=600000, box=(200, 200, 300), seed=4, gen="msf"),
              "-m 2048 2048 300000 --adfstemuncorrfem --V_omega --images --cs3 1.3e7 "
              "--scherzer_defocus --scherzer_alphamax --rasterspacing 50 --minslice 2.0",
              False, None),
    # --paptif: per slice, 16-bit images of the projected potential before
    # the exponential (magnitude, real and imaginary parts, linear and log)
    "paptif": (dict(n=390, box=(25, 25, 12.5), seed=11),
               "-m 128 128 200000 --adfstemuncorr --paptif --cs3 1.3e7 --scherzer_defocus "
               "--alphamax 0.010 --rasterspacing 12.5 --minslice 2.0", True, None),
    # detector MTF: only the parameter-file route works in the reference (its
    # --mtf_file option does not consume its argument); FEM pixel modes too
    "mtf": (dict(n=780, box=(25, 25, 25), seed=1),
            "--parameter_file mtf.param -m 128 128 200000 --adfstemuncorrfem --V_omega --V_re "
            "--Omega_vimage --cs3 1.3e7 --scherzer_defocus --alphamax 0.010 "
            "--rasterspacing 6.25 --minslice 2.0 --images", True, None),
    # xyz specimen file (element symbols in any case, or the atomic number)
    "xyz": (dict(n=780, box=(25, 25, 25), seed=3, xyz=True),
            "-m 128 128 200000 --adfstemuncorrfem --V_omega --cs3 1.3e7 --scherzer_defocus "
            "--alphamax 0.010 --rasterspacing 6.25 --minslice 2.0 --images", True, None),
    # FEM correlograph: average, variance (squared sums) and every probe's text
    "corrgraph": (dict(n=780, box=(25, 25, 25), seed=1),
                  "-m 128 128 200000 --adfstemuncorrfem --V_omega --correlograph "
                  "--correlograph_variance --correlograph_everytxt --correlograph_everyimage "
                  "--cs3 1.3e7 --scherzer_defocus --alphamax 0.010 --rasterspacing 6.25 "
                  "--minslice 2.0 --dr 1.0", True, None),
}

# cases whose --images diffraction TIFFs are not kept in the fixture (large
# grids: only the ADF image and V(k) are compared)
NO_DIFFRACTION = {"g512", "g2048", "g4096", "c4_r4"}

# extra input files of a case, written beside the specimen (name -> text)
FILES = {
    "mtf": {"mtf.param": "mtf_file mtf.csv\nmtf_sampling_rate 20\n",
            "mtf.csv": "0, 0.25, 0.5, 0.75, 1.0, 1.5\n1.0, 0.8, 0.55, 0.35, 0.2, 0.1\n"},
}
FILES["md_mtf"] = FILES["mtf"]


def write_xyz(path, pos, box):
    """xyz specimen (tem_io.cpp:4627-4958): count, periods, then element and
    position per line; element names in mixed case and as a number."""
    names = ["Si", "si", "SI", "14"]
    lines = ["%d" % len(pos), "%.6f %.6f %.6f" % tuple(box)]
    for k, p in enumerate(pos):
        lines.append("%s %.6f %.6f %.6f" % (names[k % 4], p[0], p[1], p[2]))
    Path(path).write_text("\n".join(lines) + "\n")


def make_specimen_file(recipe, path):
    if recipe.get("xyz"):
        pos = specimen.amorphous_positions(recipe["n"], recipe["box"], seed=recipe["seed"])
        pos = np.minimum(np.round(pos, 6), np.round(np.asarray(recipe["box"], float), 6))
        write_xyz(path, pos, recipe["box"])
        return pos
    if recipe.get("gen") == "msf":
        # the library's C++ generator (msf_amorphous_positions): fast enough
        # for the 600k-atom specimen; host-only, no GPU needed
        import msf
        box = np.asarray(recipe["box"], dtype=np.float64)
        pos = msf.amorphous_positions(recipe["n"], box, 2.2, seed=recipe["seed"])
        pos = np.minimum(np.round(pos, 6), np.round(box, 6))
        specimen.write_lammps_data(path, pos, box)
        return pos
    pos = specimen.make_specimen(path, recipe["n"], recipe["box"], seed=recipe["seed"])
    if recipe.get("two_species"):
        # every third atom becomes oxygen (mass 15.999 -> Z = 8)
        text = Path(path).read_text().splitlines()
        out, in_atoms, k = [], False, 0
        for line in text:
            if line.strip() == "1 atom types":
                line = "2 atom types"
            if line.strip() == "1 28.0855":
                line = "1 28.0855\n2 15.999"
            if in_atoms and line.strip():
                parts = line.split()
                if k % 3 == 2:
                    parts[1] = "2"
                line = " ".join(parts)
                k += 1
            if line.strip() == "Atoms":
                in_atoms = True
            out.append(line)
        Path(path).write_text("\n".join(out) + "\n")
    return pos


def sha256(path):
    return hashlib.sha256(Path(path).read_bytes()).hexdigest()


def run_case(name):
    recipe, args, commit, tslice = CASES[name]
    work = Path(tempfile.mkdtemp(prefix="golden_" + name))
    spec = work / (name + (".xyz" if recipe.get("xyz") else ".data"))
    make_specimen_file(recipe, spec)
    for fname, text in FILES.get(name, {}).items():
        (work / fname).write_text(text)
    argv = ["-a", spec.name, "--output_prefix", name] + args.split()
    env = {"MSF_REF_DUMP_SLICES": str(work / "slices.txt")}
    if tslice is not None:
        env["MSF_REF_DUMP_T"] = str(work / "t_")
    r = oracle.run_reference(argv, cwd=work, env_extra=env)
    if r["returncode"] != 0:
        raise RuntimeError("reference failed for %s:\n%s\n%s" % (name, r["stdout"], r["stderr"]))
    out = {}
    corr = any(a in ("--adfstemcorr", "--adfstemcorrfem") for a in args.split())
    prefix = work / (name + ("_adfstem_corr" if corr else "_adfstem_uncorr"))
    for f in work.iterdir():
        if f.name.endswith("_stem_image_output.f64"):
            out["adf_image"] = np.fromfile(f)
            prefix = Path(str(f)[: -len("_stem_image_output.f64")])
    for f in sorted(work.glob("*_fem_*.txt")):
        mode = f.stem.split("_fem_")[1]
        out[mode] = oracle.read_variance_txt(f)
    # correlograph tables: first row "0 phi...", then "k values..."
    for f in sorted(work.glob("*_correlograph_*.txt")):
        out["correlograph_" + f.stem.split("_correlograph_")[1]] = np.loadtxt(f, ndmin=2)
    for f in sorted(work.glob(name + "_adfstem_*corr_[0-9]*_[0-9]*.txt")):
        px, py = f.stem.split("_")[-2:]
        out["correlograph_probe_%s_%s" % (px, py)] = np.loadtxt(f, ndmin=2)
    # diffraction patterns written with --images: first and last probe, and
    # with FEM pixel modes the raster averages and the 2-D variance
    for tag in ("first", "final", "diffracted_wave_avg", "diffracted_wave_sqr_avg",
                "variance_2-D"):
        if name in NO_DIFFRACTION:
            break
        for f in work.glob("*_adfstem_*corr_%s_diffraction_scalefactor_*.tif" % tag):
            out["%s_diffraction_%s" % (tag, f.stem.split("_scalefactor_")[1])] = read_tif16(f)
    # --paptif images: magnitude and real part (the imaginary part's min/max
    # are uninitialised in the reference, func.cpp:2063-2065, so its images
    # are not defined and not kept)
    for f in sorted(work.glob(name + "_pap_slice*_complex_fftw_operand_*.tif")):
        if "_operand_im" not in f.name:
            out["pap_" + f.stem.split("_pap_")[1]] = read_tif16(f)
    sl = np.loadtxt(work / "slices.txt", ndmin=2)
    out["slice_lower"], out["slice_thickness"], out["slice_count"] = sl[:, 0], sl[:, 1], sl[:, 2]
    if tslice is not None:
        t = np.fromfile(work / ("t_%d.c128" % (tslice + 1)))
        out["transmission_slice"] = np.array(tslice)
        out["transmission"] = t
    np.savez_compressed(HERE / (name + ".npz"), **out)
    meta = dict(case=name, argv=argv, recipe=recipe, specimen_sha256=sha256(spec),
                committed_specimen=commit, prefix=prefix.name, files=FILES.get(name, {}),
                adfstem_seconds=r["adfstem_seconds"], probes=r["probes"], slices=r["slices"])
    (HERE / (name + ".json")).write_text(json.dumps(meta, indent=1) + "\n")
    if commit:
        shutil.copy(spec, HERE / spec.name)
    shutil.rmtree(work)
    print(name, "ok", r["adfstem_seconds"], "s", sorted(out))


# MD-coupled cases (the reference's ms-stem-fem-md with LAMMPS replaced by
# the data-file replay of oracle/shims/lammps): an initial configuration in a
# box with a non-zero origin, `snapshots` jittered copies of it (positions
# left unwrapped, so the driver's periodic wrap is exercised) and the argv.
# name -> (recipe, box origin, snapshots, jitter [A], seed, argv, steps, samples)
MD_CASES = {
    # three configurations, each seen twice per probe; every FEM mode
    "md": (dict(n=780, box=(25, 25, 25), seed=1), (-12.5, -5.0, -3.0), 3, 0.15, 41,
           "-m 128 128 200000 --adfstemuncorrfem " + " ".join(FEM_ALL) +
           " --cs3 1.3e7 --scherzer_defocus --alphamax 0.010 --rasterspacing 6.25 "
           "--minslice 2.0 --images", 10, 6),
    # detector MTF (parameter file) and the correlograph on the averaged wave
    "md_mtf": (dict(n=780, box=(25, 25, 25), seed=1), (0.0, 0.0, 0.0), 2, 0.2, 43,
               "--parameter_file mtf.param -m 128 128 200000 --adfstemuncorrfem --V_omega "
               "--V_re --Omega_vimage --correlograph --correlograph_variance --cs3 1.3e7 "
               "--scherzer_defocus --alphamax 0.010 --rasterspacing 8.333 --minslice 2.0 "
               "--dr 1.0 --images", 5, 4),
    # no MD steps: every sample sees the initial configuration
    "md_static": (dict(n=390, box=(25, 25, 12.5), seed=11), (0.0, 0.0, 0.0), 0, 0.0, 0,
                  "-m 128 64 200000 --adfstemuncorrfem --V_omega --Vbar_r --cs3 1.3e7 "
                  "--defocus 300 --alphamax 0.012 --rasterspacing 5 --minslice 2.0 --images",
                  0, 2),
}

PRE_TEM = ("units metal\natom_style atomic\nboundary p p p\nread_data {initial}\n"
           "pair_style sw\npair_coeff * * Si.sw Si\nvelocity all create 300.0 4928459\n"
           "fix 1 all nve\ntimestep 0.001\n")


def write_frame(path, header, pos):
    rows = ["%d 1 %.6f %.6f %.6f" % (k + 1, p[0], p[1], p[2]) for k, p in enumerate(pos)]
    Path(path).write_text("\n".join(header + rows) + "\n")


def run_md_case(name):
    recipe, origin, n_snap, jitter, seed, args, steps, samples = MD_CASES[name]
    work = Path(tempfile.mkdtemp(prefix="golden_" + name))
    base = work / "base.data"
    pos = specimen.make_specimen(base, recipe["n"], recipe["box"], seed=recipe["seed"])
    pos = np.asarray(pos, float) + np.asarray(origin)
    lo, hi = np.asarray(origin), np.asarray(origin) + np.asarray(recipe["box"], float)
    header = ["# " + name, "", "%d atoms" % len(pos), "1 atom types", ""]
    header += ["%.6f %.6f %s %s" % (lo[d], hi[d], a, b)
               for d, (a, b) in enumerate((("xlo", "xhi"), ("ylo", "yhi"), ("zlo", "zhi")))]
    header += ["", "Masses", "", "1 28.0855", "", "Atoms", ""]
    files = {}
    initial = name + "_0.data"
    write_frame(work / initial, header, pos)
    files[initial] = (work / initial).read_text()
    rng = np.random.default_rng(seed)
    replay = []
    for k in range(1, n_snap + 1):
        f = "%s_%d.data" % (name, k)
        write_frame(work / f, header, pos + rng.normal(0.0, jitter, pos.shape))
        files[f] = (work / f).read_text()
        replay.append(f)
    files[name + ".in"] = PRE_TEM.format(initial=initial)
    files.update(FILES.get(name, {}))
    if replay:
        files[name + "_replay.txt"] = "\n".join(replay) + "\n"
    for f, text in files.items():
        (work / f).write_text(text)
    argv = (["-a", initial, "--output_prefix", name] + args.split() +
            ["--lammps_preTEM_file_name", name + ".in", "--lammps_TEM_steps", str(steps),
             "--lammps_TEM_samples", str(samples)])
    env = {"MSF_MD_REPLAY": str(work / (name + "_replay.txt"))} if replay else {}
    r = oracle.run_reference(argv, cwd=work, env_extra=env, md=True)
    if r["returncode"] != 0:
        raise RuntimeError("reference failed for %s:\n%s\n%s" % (name, r["stdout"], r["stderr"]))
    out = {}
    out["adf_image"] = np.fromfile(work / (name + "_stem_image_output.f64"))
    for f in sorted(work.glob(name + "_fem_*.txt")):
        out[f.stem.split("_fem_")[1]] = oracle.read_variance_txt(f)
    for tag in ("final", "diffracted_wave_avg", "diffracted_wave_sqr_avg", "variance_2-D"):
        for f in work.glob("%s_%s_diffraction_scalefactor_*.tif" % (name, tag)):
            out["%s_diffraction_%s" % (tag, f.stem.split("_scalefactor_")[1])] = read_tif16(f)
    for f in sorted(work.glob(name + "_correlograph_*.txt")):
        out["correlograph_" + f.stem.split("_correlograph_")[1]] = np.loadtxt(f, ndmin=2)
    np.savez_compressed(HERE / (name + ".npz"), **out)
    extra = ["--md_replay", name + "_replay.txt"] if replay else []
    meta = dict(case=name, argv=argv, md_argv_extra=extra, recipe=recipe, origin=origin,
                snapshots=n_snap, jitter=jitter, seed=seed, prefix=name,
                committed_specimen=False, specimen_sha256=None,
                files={f: "" for f in files}, md=True)
    (HERE / (name + ".json")).write_text(json.dumps(meta, indent=1) + "\n")
    mddir = HERE / name
    mddir.mkdir(exist_ok=True)
    for f, text in files.items():
        (mddir / f).write_text(text)
    shutil.rmtree(work)
    print(name, "ok", sorted(out))


def main():
    names = sys.argv[1:] or list(CASES) + list(MD_CASES)
    for n in names:
        if n in MD_CASES:
            run_md_case(n)
        else:
            run_case(n)


if __name__ == "__main__":
    main()
