// Drop-in front end: the reference's command line, parameter file, specimen
// readers and output writers, on top of the C ABI.
//
//   parse_args         read_cmdline_options   (tem_io.cpp:5277-5720)
//   parse_param_file   read_parameter_file    (tem_io.cpp:4063-4626)
//   check_flags        check_runtime_flags    (tem_io.cpp:5858-6169)
//   read_lammps        read_position_lammps_data_file (tem_io.cpp:36-1028)
//   finish_job         tem.cpp:405-1378 (lambda, cut-offs, defaults, raster,
//                      Scherzer conditions, output prefix)
//   write_outputs      output_variance_to_txt (io_txt.cpp:30-94) and
//                      output_stem_image (write_tif.cpp:1552-1605,
//                      write_tif.hpp:143-335)
// Quirks of the reference's parser are kept where they change what a
// command line means (--detectorangles reads its first number twice,
// --mtf_file does not consume its argument, the parameter file resets the
// -m flag); they are marked where they occur.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "engine.hpp"
#include "msf.h"
#include "setup.hpp"

namespace msf {
const char* last_error();
}

struct Flags {
  unsigned m = 0, pf = 0, o = 0, a = 0, defocus = 0, spread = 0, adfstem_corrected = 0,
           adfstem_uncorrected = 0, bfctem_corrected = 0, bfctem_uncorrected = 0, fem = 0,
           gt17 = 0, d1 = 0, d2 = 0, d3 = 0, d4 = 0, rva = 0, scherzer_defocus = 0,
           scherzer_alphamax = 0, scherzer_cs3 = 0, cs3 = 0, cs5 = 0, alpha_max = 0,
           adfstem_detector_angles = 0, raster_spacing = 0, mtf_file = 0, mtf_resolution = 0,
           pap_tif = 0, dupe = 0, image_output = 0, diffraction_output = 0, netcdf_images = 0,
           netcdf_variance = 0, nx = 0, ny = 0, microscope_voltage = 0, debug = 0,
           correlograph = 0, correlograph_variance = 0, correlograph_everyimage = 0,
           correlograph_everytxt = 0, lammps_preTEM_file = 0, lammps_TEM_steps = 0,
           lammps_TEM_samples = 0, fail = 0;
};

struct msf_job {
  Flags flags;
  std::string program = "ms-stem-fem";
  std::string model_file, output_prefix, full_prefix;
  int nx = 0, ny = 0;
  double VV = 0, defocus = 0, alpha_max = 0, defocus_spread = 1.0, cond_angle = 0, Cs3 = 0,
         Cs5 = 0, det_inner = 0, det_outer = 0, raster_spacing = 0, mtf_resolution = 0;
  double dr = 0.70710678118654746;  // tem.cpp:186
  double min_slice = 1.0;           // tem.cpp:188
  unsigned dupe_x = 1, dupe_y = 1, dupe_z = 1;
  std::string lammps_pre;
  unsigned lammps_steps = 0, lammps_samples = 0;
  bool md = false;  // parsed for ms-stem-fem-md (the LAMMPS-coupled driver)
  std::vector<double> mtf, mtf_domain;  // mtf_file: MTF values and domain
  // specimen
  std::vector<double> q;
  std::vector<uint32_t> z;
  double xperiod = 0, yperiod = 0, zperiod = 0, xmin = 0, ymin = 0, zmin = 0;
  // derived
  double lambda = 0, gamma = 0;
  std::vector<double> x_p, y_p;
  bool corrected = false;
  double cs3_used = 0;
  std::string messages;  // what the reference would print on failure
};

namespace {

std::string lower(std::string s) {
  std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return std::tolower(c); });
  return s;
}

template <typename T>
void parse_into(const std::string& s, T& v) {
  std::istringstream is(s);
  is >> v;  // failed extraction leaves 0 (C++11), as the reference's istringstream
}

bool blank(const std::string& l) { return l.find_first_not_of(" \t") == std::string::npos; }

// read_mtf_file (tem_io.cpp:5722-5857): first line the domain, second line
// the MTF, commas read as spaces; each line is read by extracting until the
// stream reports eof (a trailing blank adds one more value, as there), and a
// line counts only if the stream is still good after reading it.
bool read_mtf(const std::string& name, msf_job* j) {
  std::ifstream in(name.c_str());
  if (!in.is_open()) {
    j->messages += "Error opening MTF file: " + name + "\n";
    return false;
  }
  auto values = [](std::string line, std::vector<double>* out) {
    for (size_t at = line.find(','); at != std::string::npos; at = line.find(','))
      line.replace(at, 1, " ");
    std::istringstream ls(line);
    double v;
    while (!ls.eof()) {
      ls >> v;
      out->push_back(v);
    }
  };
  std::string line;
  if (std::getline(in, line) && in.good()) values(line, &j->mtf_domain);
  if (std::getline(in, line) && in.good()) values(line, &j->mtf);
  if (j->mtf_domain.size() != j->mtf.size()) {
    j->messages += "Error reading MTF file: " + name + "\n MTF (1st line) and MTF domain (2nd "
                   "line) do not have the same number of elements.\n";
    return false;
  }
  return true;
}

// getline that skips whitespace-only lines, as the reference's readers do
bool next_line(std::istream& in, std::string& line) {
  if (!(std::getline(in, line) && in.good())) return false;
  while (blank(line)) {
    if (!std::getline(in, line)) return false;
  }
  return true;
}

bool parse_param_file(const std::string& path, msf_job* j) {
  Flags& f = j->flags;
  std::ifstream in(path.c_str());
  if (!in.is_open()) return false;
  std::string line;
  while (std::getline(in, line) && in.good()) {
    while (blank(line)) {
      if (!std::getline(in, line)) break;
    }
    if (blank(line)) break;
    std::istringstream ls(line);
    std::string key;
    ls >> key;
    key = lower(key);
    if (key == "debug") f.debug = 1;
    else if (key == "output_prefix") { ls >> j->output_prefix; f.o = 1; }
    else if (key == "samples_x") { int v = 0; ls >> v; j->nx = v; f.nx = 1; }
    else if (key == "samples_y") { int v = 0; ls >> v; j->ny = v; f.ny = 1; }
    else if (key == "model_file") { ls >> j->model_file; f.a = 1; }
    else if (key == "microscope_voltage") { ls >> j->VV; f.microscope_voltage = 1; }
    else if (key == "scherzer_defocus") f.scherzer_defocus = 1;
    else if (key == "scherzer_alphamax") f.scherzer_alphamax = 1;
    else if (key == "scherzer_cs3") f.scherzer_cs3 = 1;
    else if (key == "defocus") { ls >> j->defocus; f.defocus = 1; }
    else if (key == "alphamax") { ls >> j->alpha_max; f.alpha_max = 1; }
    else if (key == "spread") { ls >> j->defocus_spread >> j->cond_angle; f.spread = 1; }
    else if (key == "cs3") { ls >> j->Cs3; f.cs3 = 1; }
    else if (key == "cs5") { ls >> j->Cs5; f.cs5 = 1; }
    else if (key == "detectorangles") {
      ls >> j->det_inner >> j->det_outer;
      if (j->det_inner > j->det_outer) std::swap(j->det_inner, j->det_outer);
      f.adfstem_detector_angles = 1;
    } else if (key == "mtf_file") {
      std::string name;
      ls >> name;
      if (!read_mtf(name, j)) {
        j->messages += "Error, could not read MTF file : " + name + "\n";
        f.fail = 1;
      } else {
        f.mtf_file = 1;
      }
    } else if (key == "mtf_sampling_rate") {
      j->mtf_resolution = 0;
      if (!ls.eof()) ls >> j->mtf_resolution;
      f.mtf_resolution = j->mtf_resolution == 0 ? 0 : 1;
    } else if (key == "raster_spacing") { ls >> j->raster_spacing; f.raster_spacing = 1; }
    else if (key == "adfstemuncorrfem") { f.adfstem_uncorrected = 1; f.fem = 1; }
    else if (key == "adfstemcorrfem") { f.adfstem_corrected = 1; f.fem = 1; }
    else if (key == "v_gt17") f.gt17 = 1;
    else if (key == "v_omega") f.d1 = 1;
    else if (key == "vbar_r") f.d2 = 1;
    else if (key == "v_re") f.d3 = 1;
    else if (key == "omega_vimage") f.d4 = 1;
    else if (key == "v_rbar") f.rva = 1;
    else if (key == "adfstemcorr") f.adfstem_corrected = 1;
    else if (key == "adfstemuncorr") f.adfstem_uncorrected = 1;
    else if (key == "bfctemcorr") f.bfctem_corrected = 1;
    else if (key == "bfctemuncorr") f.bfctem_uncorrected = 1;
    else if (key == "paptif") f.pap_tif = 1;
    else if (key == "dupe") f.dupe = 1;
    else if (key == "dr") ls >> j->dr;
    else if (key == "minslice") ls >> j->min_slice;
    else if (key == "images") f.image_output = 1;
    else if (key == "diffractionimages") f.diffraction_output = 1;
    else if (key == "netcdfimages") f.netcdf_images = 1;
    else if (key == "netcdfvariance") f.netcdf_variance = 1;
    else if (key == "correlograph") f.correlograph = 1;
    else if (key == "correlograph_variance") { f.correlograph_variance = 1; f.correlograph = 1; }
    else if (key == "correlograph_everyimage") { f.correlograph_everyimage = 1; f.correlograph = 1; }
    else if (key == "correlograph_everytxt") { f.correlograph_everytxt = 1; f.correlograph = 1; }
    else if (key == "lammps_pretem_file_name") { ls >> j->lammps_pre; f.lammps_preTEM_file = 1; }
    else if (key == "lammps_tem_steps") { ls >> j->lammps_steps; f.lammps_TEM_steps = 1; }
    else if (key == "lammps_tem_samples") { ls >> j->lammps_samples; f.lammps_TEM_samples = 1; }
    else {
      j->messages += "Error, unexpected keyword in parameter file : " + key + "\n";
      return false;
    }
  }
  if (f.fem && !(f.d1 || f.d2 || f.d3 || f.d4 || f.gt17 || f.rva || f.correlograph)) f.d1 = 1;
  return f.fail == 0;
}

void parse_args(const std::vector<std::string>& args, msf_job* j) {
  Flags& f = j->flags;
  for (size_t idx = 1; idx < args.size(); ++idx) {
    const std::string& a = args[idx];
    auto has = [&](size_t k) { return idx + k < args.size(); };
    if (a == "--parameter_file") {
      std::string name;
      if (has(1)) name = args[idx + 1];
      if (!parse_param_file(name, j)) {
        j->messages += "Error, could not read parameter file : " + name + "\n";
        f.fail = 1;
      }
      // quirk kept: -m given earlier is re-derived from the file's keys
      f.m = (f.microscope_voltage && f.nx && f.ny) ? 1 : 0;
      f.pf = 1;
      idx += 1;
    } else if (a == "--mtf_file") {
      // the reference reads the file but does not consume the argument, so
      // the file name is then rejected as an unexpected argument
      const std::string name = has(1) ? args[idx + 1] : std::string();
      if (!read_mtf(name, j)) {
        j->messages += "Error, could not read MTF file : " + name + "\n";
        f.fail = 1;
      } else {
        f.mtf_file = 1;
      }
    } else if (a == "--mtf_sampling_rate") {
      j->mtf_resolution = 0;
      if (has(1)) { parse_into(args[idx + 1], j->mtf_resolution); idx += 1; }
      f.mtf_resolution = j->mtf_resolution <= 0 ? 0 : 1;
    } else if (a == "--debug") f.debug = 1;
    else if (a == "--output_prefix") {
      if (has(1)) { j->output_prefix = args[idx + 1]; f.o = 1; }
      idx += 1;
    } else if (a == "-m") {
      int nx = 0, ny = 0;
      if (has(1)) parse_into(args[idx + 1], nx);
      if (has(2)) parse_into(args[idx + 2], ny);
      if (has(3)) parse_into(args[idx + 3], j->VV);
      j->nx = nx;
      j->ny = ny;
      f.m = 1;
      idx += 3;
    } else if (a == "-a") {
      if (has(1)) j->model_file = args[idx + 1];
      f.a = 1;
      idx += 1;
    } else if (a == "--scherzer_defocus") f.scherzer_defocus = 1;
    else if (a == "--scherzer_alphamax") f.scherzer_alphamax = 1;
    else if (a == "--scherzer_cs3") f.scherzer_cs3 = 1;
    else if (a == "--defocus") { if (has(1)) parse_into(args[idx + 1], j->defocus); f.defocus = 1; idx += 1; }
    else if (a == "--alphamax") { if (has(1)) parse_into(args[idx + 1], j->alpha_max); f.alpha_max = 1; idx += 1; }
    else if (a == "--spread") {
      if (has(1)) parse_into(args[idx + 1], j->defocus_spread);
      if (has(2)) parse_into(args[idx + 2], j->cond_angle);
      f.spread = 1;
      idx += 2;
    } else if (a == "--cs3") { if (has(1)) parse_into(args[idx + 1], j->Cs3); f.cs3 = 1; idx += 1; }
    else if (a == "--cs5") { if (has(1)) parse_into(args[idx + 1], j->Cs5); f.cs5 = 1; idx += 1; }
    else if (a == "--detectorangles") {
      // quirk kept (tem_io.cpp:5529-5545): both angles read from args[idx+1]
      // and only one argument consumed
      if (has(1)) parse_into(args[idx + 1], j->det_inner);
      if (has(2)) parse_into(args[idx + 1], j->det_outer);
      if (j->det_inner > j->det_outer) std::swap(j->det_inner, j->det_outer);
      f.adfstem_detector_angles = 1;
      idx += 1;
    } else if (a == "--rasterspacing") {
      if (has(1)) parse_into(args[idx + 1], j->raster_spacing);
      f.raster_spacing = 1;
      idx += 1;
    } else if (a == "--adfstemuncorrfem") { f.adfstem_uncorrected = 1; f.fem = 1; }
    else if (a == "--adfstemcorrfem") { f.adfstem_corrected = 1; f.fem = 1; }
    else if (a == "--V_gt17") f.gt17 = 1;
    else if (a == "--V_omega") f.d1 = 1;
    else if (a == "--Vbar_r") f.d2 = 1;
    else if (a == "--V_re") f.d3 = 1;
    else if (a == "--Omega_vimage") f.d4 = 1;
    else if (a == "--V_rbar") f.rva = 1;
    else if (a == "--adfstemcorr") f.adfstem_corrected = 1;
    else if (a == "--adfstemuncorr") f.adfstem_uncorrected = 1;
    else if (a == "--bfctemcorr") f.bfctem_corrected = 1;
    else if (a == "--bfctemuncorr") f.bfctem_uncorrected = 1;
    else if (a == "--paptif") f.pap_tif = 1;
    else if (a == "--dupe") {
      if (has(3)) parse_into(args[idx + 1], j->dupe_x);
      if (idx + 2 < args.size()) parse_into(args[idx + 2], j->dupe_y);
      if (idx + 3 < args.size()) parse_into(args[idx + 3], j->dupe_z);
      f.dupe = 1;
      idx += 3;
    } else if (a == "--dr") { if (has(1)) parse_into(args[idx + 1], j->dr); idx += 1; }
    else if (a == "--minslice") { if (has(1)) parse_into(args[idx + 1], j->min_slice); idx += 1; }
    else if (a == "--images") f.image_output = 1;
    else if (a == "--netcdfimages") f.netcdf_images = 1;
    else if (a == "--netcdfvariance") f.netcdf_variance = 1;
    else if (a == "--correlograph") f.correlograph = 1;
    else if (a == "--correlograph_variance") { f.correlograph_variance = 1; f.correlograph = 1; }
    else if (a == "--correlograph_everyimage") { f.correlograph_everyimage = 1; f.correlograph = 1; }
    else if (a == "--correlograph_everytxt") { f.correlograph_everytxt = 1; f.correlograph = 1; }
    else if (a == "--lammps_preTEM_file_name") {
      if (has(1)) { j->lammps_pre = args[idx + 1]; f.lammps_preTEM_file = 1; }
      idx += 1;
    } else if (a == "--lammps_TEM_steps") {
      if (has(1)) { parse_into(args[idx + 1], j->lammps_steps); f.lammps_TEM_steps = 1; }
      idx += 1;
    } else if (a == "--lammps_TEM_samples") {
      if (has(1)) { parse_into(args[idx + 1], j->lammps_samples); f.lammps_TEM_samples = 1; }
      idx += 1;
    } else {
      j->messages += "Error, unexpected argument : " + a + "\n";
      f.fail = 1;
    }
  }
  if (!f.gt17 && !f.d1 && !f.d2 && !f.d3 && !f.d4 && !f.rva && !f.correlograph) f.d1 = 1;
}

// check_runtime_flags (tem_io.cpp:5858-6169)
void check_flags(msf_job* j) {
  Flags& f = j->flags;
  const bool ok =
      f.o && f.m && !((f.adfstem_corrected || f.bfctem_corrected) && !(f.cs5 && (f.scherzer_cs3 || f.cs3))) &&
      !((f.adfstem_uncorrected || f.bfctem_uncorrected) && !f.cs3) &&
      !(f.mtf_file != f.mtf_resolution) && (f.scherzer_defocus || f.defocus) &&
      (f.scherzer_alphamax || f.alpha_max) &&
      !((f.lammps_preTEM_file != f.lammps_TEM_steps) || (f.lammps_preTEM_file != f.lammps_TEM_samples));
  if (!ok) {
    j->messages += j->program + " : lacking required parameters\n";
    if (!(f.scherzer_defocus || f.defocus))
      j->messages += "You must specify either --defocus <value [angstrom]> or --scherzer_defocus\n";
    if (!(f.scherzer_alphamax || f.alpha_max))
      j->messages += "You must specify either --alphamax <value [radians]> or --scherzer_alphamax\n";
    if ((f.adfstem_uncorrected || f.bfctem_uncorrected) && !f.cs3)
      j->messages += "You must specify --cs3 when not using aberration correction\n";
    if ((f.adfstem_corrected || f.bfctem_corrected) && !((f.cs3 || f.scherzer_cs3) && f.cs5))
      j->messages += "Aberration correction requires --cs5 and either --cs3 or --scherzer_cs3\n";
    f.fail = 1;
  }
  if (f.fail == 0 && !f.adfstem_uncorrected && !f.adfstem_corrected) {
    j->messages += "Error: no simulation mode given (--adfstemuncorr, --adfstemcorr, "
                   "--adfstemuncorrfem or --adfstemcorrfem)\n";
    f.fail = 1;
  }
  if (f.adfstem_uncorrected && f.adfstem_corrected) {
    j->messages += "Error: choose either aberration corrected or uncorrected modes\n";
    f.fail = 1;
  }
  if (f.lammps_preTEM_file && !j->md) {
    j->messages += "Error, the LAMMPS-coupled FEM mode runs in ms-stem-fem-md\n";
    f.fail = 1;
  }
  if (j->md && !(f.lammps_preTEM_file && f.lammps_TEM_steps && f.lammps_TEM_samples)) {
    j->messages += j->program + " needs --lammps_preTEM_file_name, --lammps_TEM_steps and "
                   "--lammps_TEM_samples\n";
    f.fail = 1;
  }
  if (j->md && f.lammps_TEM_samples && j->lammps_samples == 0) {
    j->messages += "Error: lammps_TEM_samples must be at least 1\n";
    f.fail = 1;
  }
}

}  // namespace

// read_position_lammps_data_file (tem_io.cpp:36-1028)
msf_status read_lammps(const std::string& path, msf_job* j) {
  std::ifstream in(path.c_str(), std::ifstream::in);
  if (!in.is_open()) { j->messages += "Error opening position file\n"; return MSF_ERR_IO; }
  auto fail = [&](const std::string& m) { j->messages += "Error reading position data file; " + m + "\n"; return MSF_ERR_PARSE; };
  std::string line;
  std::getline(in, line);  // first line is a comment
  size_t declared = 0;
  if (!next_line(in, line)) return fail("expected '<N> atoms'");
  {
    std::istringstream ls(line);
    std::string d;
    ls >> declared >> d;
    if (!declared || lower(d) != "atoms") return fail("expected '<N> atoms'");
  }
  unsigned n_species = 0;
  if (!next_line(in, line)) return fail("expected '<T> atom types'");
  {
    std::istringstream ls(line);
    std::string d1, d2;
    ls >> n_species >> d1 >> d2;
    if (!n_species || lower(d1) != "atom" || lower(d2) != "types") return fail("expected '<T> atom types'");
  }
  double lo[3], hi[3];
  const char* names[3][2] = {{"xlo", "xhi"}, {"ylo", "yhi"}, {"zlo", "zhi"}};
  for (int d = 0; d < 3; ++d) {
    if (!next_line(in, line)) return fail("expected box bounds");
    std::istringstream ls(line);
    std::string d1, d2;
    ls >> lo[d] >> hi[d] >> d1 >> d2;
    if (lower(d1) != names[d][0] || lower(d2) != names[d][1])
      return fail(std::string("expected '<lo> <hi> ") + names[d][0] + " " + names[d][1] + "'");
  }
  for (int d = 0; d < 3; ++d)
    if (hi[d] <= lo[d]) return fail("upper bound <= lower bound");
  j->xperiod = hi[0] - lo[0];
  j->yperiod = hi[1] - lo[1];
  j->zperiod = hi[2] - lo[2];
  if (!next_line(in, line)) return fail("expected 'Masses'");
  {
    std::istringstream ls(line);
    std::string sec;
    ls >> sec;
    if (lower(sec) != "masses") return fail("expected 'Masses'");
  }
  std::vector<size_t> species_id(n_species, 0);
  std::vector<double> masses(n_species, 0.0);
  std::vector<unsigned> zs(n_species, 0);
  for (unsigned k = 0; k < n_species && in.good(); ++k) {
    if (next_line(in, line)) {
      std::istringstream ls(line);
      ls >> species_id[k] >> masses[k];
    }
  }
  for (unsigned k = 0; k < n_species; ++k) {
    zs[k] = msf::guess_z(masses[k]);
    if (!zs[k]) {
      j->messages += "Error: could not guess element having mass " + std::to_string(masses[k]) + "\n";
      return MSF_ERR_PARSE;
    }
  }
  if (!next_line(in, line)) return fail("expected 'Atoms'");
  {
    std::istringstream ls(line);
    std::string sec;
    ls >> sec;
    if (lower(sec) != "atoms") return fail("expected 'Atoms'");
  }
  j->q.clear();
  j->z.clear();
  std::vector<size_t> types;
  for (size_t read = 0; read < declared; ++read) {
    if (!next_line(in, line)) return fail("fewer atoms than declared");
    std::istringstream ls(line);
    size_t id = 0, type = 0;
    double p[3] = {0, 0, 0};
    ls >> id >> type >> p[0] >> p[1] >> p[2];
    size_t k = 0;
    for (; k < n_species; ++k)
      if (type == species_id[k]) break;
    if (k >= n_species) return fail("atom type not declared in Masses");
    if (id > declared || p[0] > hi[0] || p[0] < lo[0] || p[1] > hi[1] || p[1] < lo[1] ||
        p[2] > hi[2] || p[2] < lo[2])
      return fail("atom id or position outside the declared box");
    for (int d = 0; d < 3; ++d) j->q.push_back(p[d]);
    j->z.push_back(zs[k]);
    types.push_back(type);
  }
  std::vector<size_t> uniq(types);
  std::sort(uniq.begin(), uniq.end());
  uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
  if (uniq.size() != n_species) return fail("number of atom types used differs from declared");
  for (size_t a = 0; a < j->z.size(); ++a) {  // tem_io.cpp:907-916
    j->q[3 * a] = j->q[3 * a] - lo[0];
    j->q[3 * a + 1] = j->q[3 * a + 1] - lo[1];
    j->q[3 * a + 2] = j->q[3 * a + 2] - lo[2];
  }
  j->xmin = j->ymin = j->zmin = 0.0;
  return MSF_OK;
}

namespace {

// Atomic number of an element symbol (lower case) or of its number written
// out, 1..103; 0 otherwise (tem_io.cpp:6171-6380).
unsigned element_z(const std::string& name) {
  static const char* const symbols[103] = {
      "h",  "he", "li", "be", "b",  "c",  "n",  "o",  "f",  "ne", "na", "mg", "al", "si", "p",
      "s",  "cl", "ar", "k",  "ca", "sc", "ti", "v",  "cr", "mn", "fe", "co", "ni", "cu", "zn",
      "ga", "ge", "as", "se", "br", "kr", "rb", "sr", "y",  "zr", "nb", "mo", "tc", "ru", "rh",
      "pd", "ag", "cd", "in", "sn", "sb", "te", "i",  "xe", "cs", "ba", "la", "ce", "pr", "nd",
      "pm", "sm", "eu", "gd", "tb", "dy", "ho", "er", "tm", "yb", "lu", "hf", "ta", "w",  "re",
      "os", "ir", "pt", "au", "hg", "tl", "pb", "bi", "po", "at", "rn", "fr", "ra", "ac", "th",
      "pa", "u",  "np", "pu", "am", "cm", "bk", "cf", "es", "fm", "md", "no", "lr"};
  for (unsigned z = 1; z <= 103; ++z)
    if (name == symbols[z - 1] || name == std::to_string(z)) return z;
  return 0;
}

}  // namespace

// read_position_xyz_file (tem_io.cpp:4627-4958): atom count, then the three
// periods, then one "element x y z" line per atom (each line followed by a
// newline).  Coordinates are shifted by the smallest value of each axis,
// which starts at 0 (so only negative coordinates move); a spread larger
// than the period is an error.
msf_status read_xyz(const std::string& path, msf_job* j) {
  std::ifstream in(path.c_str());
  if (!in.is_open()) {
    j->messages += "Error opening position file: " + path + "\n";
    return MSF_ERR_IO;
  }
  auto fail = [&](const std::string& m) {
    j->messages += "Error reading position data file; " + m + "\n";
    return MSF_ERR_PARSE;
  };
  std::string line;
  size_t declared = 0;
  if (!(std::getline(in, line) && in.good())) return fail("data_line : " + line);
  {
    std::istringstream ls(line);
    ls >> declared;
    if (!declared) return fail("declared_population : 0");
  }
  if (!(std::getline(in, line) && in.good())) return fail("data_line : " + line);
  {
    std::istringstream ls(line);
    double px = 0, py = 0, pz = 0;
    ls >> px >> py >> pz;
    if (!(px > 0.0 && py > 0.0 && pz > 0.0))
      return fail("second line should begin with <xperiod> <yperiod> <zperiod>");
    j->xperiod = px;
    j->yperiod = py;
    j->zperiod = pz;
  }
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  j->q.clear();
  j->z.clear();
  for (size_t n = 0; n < declared; ++n) {
    if (!(std::getline(in, line) && in.good()))
      return fail("atoms read : " + std::to_string(n) + ", declared population : " +
                  std::to_string(declared));
    std::istringstream ls(line);
    std::string element;
    ls >> element;
    element = lower(element);
    const unsigned zz = element_z(element);
    if (zz < 1 || zz > 103)
      return fail("atom " + std::to_string(n) + ", element " + element + " invalid");
    double q[3] = {0, 0, 0};
    ls >> q[0] >> q[1] >> q[2];
    for (int d = 0; d < 3; ++d) {
      if (q[d] < lo[d]) lo[d] = q[d];
      if (q[d] > hi[d]) hi[d] = q[d];
      j->q.push_back(q[d]);
    }
    j->z.push_back(zz);
  }
  if (hi[0] - lo[0] > j->xperiod || hi[1] - lo[1] > j->yperiod || hi[2] - lo[2] > j->zperiod)
    return fail("positions exceed period");
  for (size_t a = 0; a < j->z.size(); ++a)
    for (int d = 0; d < 3; ++d) j->q[3 * a + d] = j->q[3 * a + d] - lo[d];
  j->xmin = j->ymin = j->zmin = 0.0;
  return MSF_OK;
}

namespace {

// tem.cpp:405-1378 after the inputs are read
msf_status finish_job(msf_job* j) {
  Flags& f = j->flags;
  if (f.mtf_file && f.mtf_resolution)  // tem.cpp:276-285: domain in Nyquist units, squared
    for (double& d : j->mtf_domain) d = std::pow((0.5 * j->mtf_resolution * d), 2);
  msf::wavelength(j->VV, &j->lambda, &j->gamma);
  const double xpd = j->xperiod * j->dupe_x, ypd = j->yperiod * j->dupe_y;
  double bw_pap = (j->nx / (2 * xpd) < j->ny / (2 * ypd)) ? j->nx / (2 * xpd) : j->ny / (2 * ypd);
  double bw_t = (2.0 / 3.0) * bw_pap;
  if ((f.adfstem_corrected || f.adfstem_uncorrected) && f.adfstem_detector_angles) {
    if (j->det_inner < 0.0) { j->messages += "Error: detector_inner_angle < 0\n"; f.fail = 1; }
    if (j->det_outer < 0.0) { j->messages += "Error: detector_outer_angle < 0\n"; f.fail = 1; }
    if (j->det_inner > bw_t * j->lambda) {
      j->messages += "Error: detector inner angle falls beyond bandwidth limits\n";
      f.fail = 1;
    }
  }
  if (f.fail) return MSF_ERR_ARG;
  if (!f.adfstem_detector_angles) {  // tem.cpp:1320-1337
    if (j->VV >= 200000) { j->det_inner = 0.040; j->det_outer = 0.200; }
    else { j->det_inner = 0.045; j->det_outer = 0.200; }
  }
  if (!f.raster_spacing) j->raster_spacing = f.fem ? 10 : 1.5;  // tem.cpp:1342-1348
  j->x_p = msf::raster_points(j->xperiod, j->xmin, j->raster_spacing);
  j->y_p = msf::raster_points(j->yperiod, j->ymin, j->raster_spacing);
  if (f.adfstem_uncorrected) {  // tem.cpp:1526-1558
    if (f.scherzer_defocus) j->defocus = msf::scherzer(0, j->lambda, j->Cs3);
    if (f.scherzer_alphamax) j->alpha_max = msf::scherzer(1, j->lambda, j->Cs3);
    j->corrected = false;
    j->cs3_used = j->Cs3;
    j->full_prefix = j->output_prefix + "_adfstem_uncorr";
  } else {  // tem.cpp:1565-1639
    if (f.scherzer_defocus) j->defocus = msf::scherzer(2, j->lambda, j->Cs5);
    if (f.scherzer_alphamax) j->alpha_max = msf::scherzer(3, j->lambda, j->Cs5);
    j->cs3_used = f.scherzer_cs3 ? msf::scherzer(4, j->lambda, j->Cs5) : j->Cs3;
    j->corrected = true;
    j->full_prefix = j->output_prefix + "_adfstem_corr";
  }
  return MSF_OK;
}

// write_tif_grayscale<uint16_t> (write_tif.hpp:143-335): min/max scaled or
// log-scaled 16-bit samples, rows written bottom-up, baseline tags.
bool write_tif16(const std::string& name, const double* data, size_t height, size_t width,
                 double mn, double mx, bool logscale, double xres, double yres,
                 unsigned short res_unit) {
  std::vector<uint16_t> img(width * height);
  const double digits = std::pow(2, 16) - 1;
  if (logscale) {
    const double dl = std::log(mx - mn + 1);
    for (size_t i = 0; i < height; ++i)
      for (size_t k = 0; k < width; ++k) {
        const double v = std::log(data[k + width * i] - mn + 1) / dl;
        img[k + width * i] = v > 0.0 ? (uint16_t)(v * digits + 0.5) : (uint16_t)0;
      }
  } else {
    const double sc = digits / (mx - mn);
    for (size_t i = 0; i < height; ++i)
      for (size_t k = 0; k < width; ++k)
        img[k + width * i] = (uint16_t)((data[k + width * i] - mn) * sc + 0.5);
  }
  std::vector<unsigned char> out;
  auto p16 = [&](unsigned v) { out.push_back(v & 0xff); out.push_back((v >> 8) & 0xff); };
  auto p32 = [&](unsigned v) { for (int b = 0; b < 4; ++b) out.push_back((v >> (8 * b)) & 0xff); };
  out.push_back('I'); out.push_back('I'); p16(42); p32(0);
  const uint32_t rps = (uint32_t)width;  // TIFFDefaultStripSize(width) = width
  const size_t line = width * 2;
  std::vector<uint32_t> offs, counts;
  for (size_t r0 = 0; r0 < height; r0 += rps) {
    const size_t r1 = std::min(height, r0 + rps);
    offs.push_back((uint32_t)out.size());
    counts.push_back((uint32_t)((r1 - r0) * line));
    for (size_t r = r0; r < r1; ++r) {
      const uint16_t* src = &img[(height - r - 1) * width];
      for (size_t k = 0; k < width; ++k) p16(src[k]);
    }
  }
  if (out.size() & 1) out.push_back(0);
  const uint32_t den = 10000;
  const uint32_t xoff = (uint32_t)out.size();
  p32((uint32_t)std::llround(xres * den)); p32(den);
  const uint32_t yoff = (uint32_t)out.size();
  p32((uint32_t)std::llround(yres * den)); p32(den);
  uint32_t soff = 0, coff = 0;
  if (offs.size() > 1) {
    soff = (uint32_t)out.size();
    for (uint32_t v : offs) p32(v);
    coff = (uint32_t)out.size();
    for (uint32_t v : counts) p32(v);
  }
  struct E { unsigned tag, type, count, value; };
  const unsigned ns = (unsigned)offs.size();
  std::vector<E> es = {{256, 4, 1, (unsigned)width},  {257, 4, 1, (unsigned)height},
                       {258, 3, 1, 16},               {259, 3, 1, 1},
                       {262, 3, 1, 1},                {273, 4, ns, ns > 1 ? soff : offs[0]},
                       {274, 3, 1, 1},                {277, 3, 1, 1},
                       {278, 4, 1, rps},              {279, 4, ns, ns > 1 ? coff : counts[0]},
                       {282, 5, 1, xoff},             {283, 5, 1, yoff},
                       {284, 3, 1, 1},                {296, 3, 1, res_unit}};
  const uint32_t ifd = (uint32_t)out.size();
  for (int b = 0; b < 4; ++b) out[4 + b] = (ifd >> (8 * b)) & 0xff;
  p16((unsigned)es.size());
  for (const E& e : es) {
    p16(e.tag); p16(e.type); p32(e.count);
    if (e.type == 3 && e.count == 1) { p16(e.value); p16(0); } else p32(e.value);
  }
  p32(0);
  FILE* fp = std::fopen(name.c_str(), "wb");
  if (!fp) return false;
  const bool ok = std::fwrite(out.data(), 1, out.size(), fp) == out.size();
  std::fclose(fp);
  return ok;
}

// output_correlograph_to_txt (io_txt.cpp:96-170): "0 " and the phi lower
// boundaries on the first line, then per k bin its lower boundary and the
// values [ii + jj*n_k], each followed by a space.
bool write_correlograph_txt(const std::string& prefix, const double* data,
                            const double* phi_lower, int n_phi, const double* k_lower,
                            int n_k) {
  FILE* fp = std::fopen((prefix + ".txt").c_str(), "w");
  if (!fp) return false;
  std::fprintf(fp, "0 ");
  for (int jj = 0; jj < n_phi; ++jj) std::fprintf(fp, "%.10e ", phi_lower[jj]);
  std::fprintf(fp, "\n");
  for (int ii = 0; ii < n_k; ++ii) {
    std::fprintf(fp, "%.10e ", k_lower[ii]);
    for (int jj = 0; jj < n_phi; ++jj) std::fprintf(fp, "%.10e ", data[ii + (size_t)jj * n_k]);
    std::fprintf(fp, "\n");
  }
  std::fclose(fp);
  return true;
}

bool write_variance(const std::string& prefix, const double* k_lower, const double* v, int n) {
  FILE* fp = std::fopen((prefix + ".txt").c_str(), "w");
  if (!fp) return false;
  for (int i = 0; i < n; ++i) std::fprintf(fp, "%.10e %.10e\n", k_lower[i], v[i]);
  std::fclose(fp);
  return true;
}

}  // namespace

// ---------------------------------------------- MD-coupled driver ------
// ms-stem-fem-md (ftem_lammps.cpp) takes its specimen from LAMMPS: the
// commands of the pre-TEM file set the system up (read_data, pair_style,
// pair_coeff ...) and, before every sample of every probe, "run <steps>"
// advances the MD.  Without LAMMPS the trajectory is a replay of LAMMPS data
// files: "read_data" in the pre-TEM file gives the initial configuration and
// the i-th run loads entry (i - 1) mod K of the replay list.
namespace {

struct MdFrame {
  std::vector<int> type;     // by atom id - 1
  std::vector<double> x;     // [id - 1][3], as in the file
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
};

// A LAMMPS data file of atom style atomic: the "N atoms" and box lines of
// the header, then the "Atoms" section of "id type x y z" lines.
bool read_md_frame(const std::string& path, MdFrame* fr, std::string* err) {
  std::ifstream in(path.c_str());
  if (!in.is_open()) {
    *err = "Error opening LAMMPS data file " + path + "\n";
    return false;
  }
  std::string line;
  long long n = -1, seen = 0;
  bool atoms = false;
  while (std::getline(in, line)) {
    const size_t hash = line.find('#');
    std::istringstream ls(hash == std::string::npos ? line : line.substr(0, hash));
    if (!atoms) {
      std::vector<std::string> tok;
      std::string t;
      while (ls >> t) tok.push_back(t);
      if (tok.empty()) continue;
      if (tok.size() >= 2 && tok[1] == "atoms") n = std::atoll(tok[0].c_str());
      static const char* los[3] = {"xlo", "ylo", "zlo"};
      for (int d = 0; d < 3; ++d)
        if (tok.size() >= 4 && tok[2] == los[d]) {
          fr->lo[d] = std::atof(tok[0].c_str());
          fr->hi[d] = std::atof(tok[1].c_str());
        }
      if (tok[0] == "Atoms") {
        if (n < 0) break;
        fr->type.assign(n, 0);
        fr->x.assign(3 * n, 0.0);
        atoms = true;
      }
      continue;
    }
    long long id = 0;
    int ty = 0;
    double p[3];
    if (!(ls >> id >> ty >> p[0] >> p[1] >> p[2])) continue;
    if (id < 1 || id > n || fr->type[id - 1] != 0) {
      *err = "Error: atom id " + std::to_string(id) + " out of range or repeated in " + path + "\n";
      return false;
    }
    fr->type[id - 1] = ty;
    for (int d = 0; d < 3; ++d) fr->x[3 * (id - 1) + d] = p[d];
    if (++seen == n) break;
  }
  if (n < 0 || seen != n) {
    *err = "Error: " + path + " holds " + std::to_string(seen) + " of " +
           std::to_string(std::max<long long>(n, 0)) + " atoms\n";
    return false;
  }
  return true;
}

struct MdSetup {
  std::vector<std::string> elements;  // pair_coeff element names, by type
  std::string initial;                // read_data file
};

// The pre-TEM commands (ftem_lammps.cpp:400-590): the element names of a
// tersoff / sw / eam pair_coeff line map LAMMPS types to Z; read_data names
// the initial configuration.
bool read_pre_tem(const std::string& path, MdSetup* md, std::string* err) {
  std::ifstream in(path.c_str());
  if (!in.is_open()) {
    *err = "Error opening lammps_preTEM_file_name " + path + "\n";
    return false;
  }
  bool style_ok = false;
  std::string line;
  while (std::getline(in, line) && in.good()) {
    if (line.find("pair_style") != std::string::npos &&
        (line.find("sw") != std::string::npos || line.find("tersoff") != std::string::npos ||
         line.find("eam") != std::string::npos))
      style_ok = true;
    const size_t at = line.find("pair_coeff");
    if (at != std::string::npos) {
      if (!style_ok) {
        *err = "Error in reading lammps_preTEM_file_name : only tersoff, stillinger-weber, "
               "and eam pair_coeff commands currently allowed\n";
        return false;
      }
      // "pair_coeff * * <file> <element> ...": as the reference reads it,
      // until the stream is no longer good (a trailing blank repeats the
      // last name, which changes nothing)
      std::istringstream pc(line.substr(at));
      std::string tmp;
      pc >> tmp >> tmp >> tmp;
      pc >> tmp;
      md->elements.clear();
      while (pc.good()) {
        pc >> tmp;
        md->elements.push_back(tmp);
      }
    }
    std::istringstream ls(line);
    std::string word;
    if ((ls >> word) && word == "read_data") ls >> md->initial;
  }
  if (md->initial.empty()) {
    *err = "Error: the lammps_preTEM_file_name commands have no read_data\n";
    return false;
  }
  if (md->elements.empty()) {
    *err = "Error: the lammps_preTEM_file_name commands have no pair_coeff element names\n";
    return false;
  }
  return true;
}

// One configuration as the reference gathers it from LAMMPS (ftem_lammps.
// cpp:1640-1740): atoms by id, x and y wrapped into (min, max] of the
// initial box, Z from the type's element name.
bool md_positions(const MdFrame& fr, const MdFrame& init, const MdSetup& md,
                  std::vector<double>* q, std::vector<uint32_t>* z, std::string* err) {
  const size_t n = fr.type.size();
  q->assign(3 * n, 0.0);
  z->assign(n, 0);
  const double xmin = init.lo[0], xmax = init.hi[0], ymin = init.lo[1], ymax = init.hi[1];
  const double xperiod = fr.hi[0] - fr.lo[0], yperiod = fr.hi[1] - fr.lo[1];
  for (size_t a = 0; a < n; ++a) {
    const int t = fr.type[a];
    if (t < 1 || (size_t)t > md.elements.size()) {
      *err = "Error: atom type " + std::to_string(t) + " has no pair_coeff element name\n";
      return false;
    }
    const unsigned zz = element_z(lower(md.elements[t - 1]));
    if (zz < 1 || zz > 103) {
      *err = "Error: unknown element " + md.elements[t - 1] + "\n";
      return false;
    }
    (*z)[a] = zz;
    double x = fr.x[3 * a], y = fr.x[3 * a + 1];
    while (x <= xmin) x += xperiod;
    while (x > xmax) x -= xperiod;
    while (y <= ymin) y += yperiod;
    while (y > ymax) y -= yperiod;
    (*q)[3 * a] = x;
    (*q)[3 * a + 1] = y;
    (*q)[3 * a + 2] = fr.x[3 * a + 2];
  }
  return true;
}

// Parse argv (tem.cpp:81-403, or ftem_lammps.cpp:95-1420 when `md`): the
// options, --parameter_file, the specimen file, the flag checks and the
// defaults.  The MD driver also reads the pre-TEM commands and the initial
// configuration, whose box sets the cell (ftem_lammps.cpp:1122-1148), and
// writes its outputs under the plain output prefix.
msf_status parse_job(int32_t argc, const char* const* argv, bool md, msf_job** out,
                     MdSetup* setup, MdFrame* init) {
  if (!out || argc < 1 || !argv) return MSF_ERR_ARG;
  msf_job* j = new msf_job;
  std::vector<std::string> args(argv, argv + argc);
  j->program = args[0];
  j->md = md;
  parse_args(args, j);
  // tem.cpp:240-330: the specimen is read before the flag checks
  msf_status st = MSF_OK;
  const bool xyz = j->model_file.substr(j->model_file.find_last_of('.') + 1) == "xyz";
  if ((xyz ? read_xyz(j->model_file, j) : read_lammps(j->model_file, j)) != MSF_OK) {
    j->messages += "Error, file could not be read : " + j->model_file + "\n";
    j->flags.fail = 1;
    st = MSF_ERR_IO;
  }
  check_flags(j);
  if (!j->flags.fail && md) {
    std::string err;
    if (!read_pre_tem(j->lammps_pre, setup, &err) ||
        !read_md_frame(setup->initial, init, &err)) {
      j->messages += err;
      j->flags.fail = 1;
      st = MSF_ERR_IO;
    } else {
      j->xmin = init->lo[0];
      j->ymin = init->lo[1];
      j->zmin = init->lo[2];
      j->xperiod = init->hi[0] - init->lo[0];
      j->yperiod = init->hi[1] - init->lo[1];
      j->zperiod = init->hi[2] - init->lo[2];
    }
  }
  if (j->flags.fail) {
    msf::set_error(j->messages + "Exiting ms-stem-fem due to failure.\n");
    delete j;
    return st != MSF_OK ? st : MSF_ERR_PARSE;
  }
  st = finish_job(j);
  if (st != MSF_OK) {
    msf::set_error(j->messages);
    delete j;
    return st;
  }
  if (md) j->full_prefix = j->output_prefix;
  *out = j;
  return MSF_OK;
}

// Host result buffers for a drop-in run: every V(k) mode, the ADF image,
// correlograph tables, and the diffraction planes --images writes.
struct RunBuffers {
  std::vector<double> img, kl, v[6], phi, corr, corr_sqr, corr_probes, final_psi, first_psi,
      mean_a, mean_i;
  msf_results r{};
  void setup(const msf_job* j, const msf_grid& grid, const msf_raster& raster,
             const msf_detect& det, bool want_first) {
    const size_t nr = raster.n_x * (size_t)raster.n_y;
    const size_t plane = (size_t)grid.nx * grid.ny;
    img.assign(nr, 0.0);
    kl.assign(8192, 0.0);
    for (auto& a : v) a.assign(8192, 0.0);
    r = msf_results{};
    r.adf_image = img.data();
    r.cap_k = 8192;
    r.k_lower = kl.data();
    r.v_omega = v[0].data();
    r.vbar_r = v[1].data();
    r.v_re = v[2].data();
    r.omega_vimage = v[3].data();
    r.v_gt17 = v[4].data();
    r.v_rbar = v[5].data();
    // correlograph: bins from the segment counts with and without the cells
    if (det.outputs & MSF_OUT_CORRELOGRAPH) {
      msf_detect rings = det;
      rings.outputs &= ~(uint32_t)(MSF_OUT_CORRELOGRAPH | MSF_OUT_CORRELOGRAPH_VAR);
      rings.outputs |= MSF_OUT_V_OMEGA;
      const int32_t n_k = msf_segment_count(&grid, &rings) - 1;
      const int32_t cells = msf_segment_count(&grid, &det) - 1 - n_k;
      const int32_t n_phi = n_k > 0 ? cells / n_k : 0;
      const size_t nc = std::max<size_t>(1, (size_t)n_k * n_phi);
      phi.assign(n_phi + 1, 0.0);
      corr.assign(nc, 0.0);
      corr_sqr.assign(nc, 0.0);
      r.cap_phi = n_phi;
      r.phi_lower = phi.data();
      r.correlograph = corr.data();
      r.correlograph_sqr = corr_sqr.data();
      if (j->flags.correlograph_everyimage || j->flags.correlograph_everytxt) {
        corr_probes.assign(nc * nr, 0.0);
        r.correlograph_probes = corr_probes.data();
      }
    }
    if (j->flags.image_output) {  // the first and last exit waves' diffraction
      final_psi.assign(2 * plane, 0.0);
      r.final_psi = final_psi.data();
      if (want_first) {
        first_psi.assign(2 * plane, 0.0);
        r.first_psi = first_psi.data();
      }
    }
    if (j->flags.image_output &&  // the FEM pixel modes' diffraction averages
        (det.outputs & (MSF_OUT_V_RE | MSF_OUT_OMEGA_VIMAGE | MSF_OUT_V_GT17 | MSF_OUT_V_RBAR))) {
      mean_a.assign(plane, 0.0);
      mean_i.assign(plane, 0.0);
      r.mean_amplitude = mean_a.data();
      r.mean_intensity = mean_i.data();
    }
  }
};

// The analogue of the reference's FFTW wisdom file (tem.cpp:583-616,
// 1748-1765): msf_wisdom_<Nx>x<Ny>_<fp32|fp64> in the working directory is
// imported when it exists and holds a line for this grid and device model;
// otherwise the launch tiling is measured (msf_tune) and the file written.
// Skipped when --batch fixes the tiling.
void apply_wisdom(const msf_grid& grid, msf_context* ctx, const msf_specimen* spec,
                  const msf_options& o, bool write_file = true) {
  if (o.batch > 0) return;
  const std::string name = "msf_wisdom_" + std::to_string(grid.nx) + "x" +
                           std::to_string(grid.ny) + (o.precision == MSF_FP32 ? "_fp32" : "_fp64");
  std::ifstream in(name.c_str());
  if (in.is_open()) {
    std::stringstream text;
    text << in.rdbuf();
    int32_t n = 0;
    if (msf_wisdom_import(ctx, text.str().c_str(), &n) == MSF_OK && n > 0) return;
  }
  msf_tuning t;
  if (msf_tune(ctx, spec, &t) != MSF_OK) return;  // the untuned defaults still run
  const int64_t len = msf_wisdom_export(ctx, nullptr, 0);
  std::vector<char> buf((size_t)len + 1);
  msf_wisdom_export(ctx, buf.data(), len + 1);
  if (!write_file) return;
  std::ofstream out(name.c_str());
  out << buf.data();
}

}  // namespace

// ------------------------------------------------------------- C ABI ------
extern "C" {

msf_status msf_read_specimen(const char* path, msf_job** out) {
  if (!path || !out) return MSF_ERR_ARG;
  msf_job* j = new msf_job;
  const std::string p(path);
  msf_status st;
  if (p.substr(p.find_last_of('.') + 1) == "xyz")  // tem.cpp:288-330
    st = read_xyz(p, j);
  else
    st = read_lammps(p, j);
  if (st != MSF_OK) {
    msf::set_error(j->messages);
    delete j;
    return st;
  }
  *out = j;
  return MSF_OK;
}

msf_status msf_parse_cmdline(int32_t argc, const char* const* argv, msf_job** out) {
  return parse_job(argc, argv, false, out, nullptr, nullptr);
}

msf_status msf_job_destroy(msf_job* job) {
  delete job;
  return MSF_OK;
}

msf_status msf_job_describe(const msf_job* j, msf_grid* grid, msf_atoms* atoms,
                            msf_optics* optics, msf_raster* raster, msf_detect* det) {
  if (!j) return MSF_ERR_ARG;
  const Flags& f = j->flags;
  if (grid) {
    *grid = msf_grid{};
    grid->nx = j->nx;
    grid->ny = j->ny;
    grid->voltage = j->VV;
    grid->xperiod = j->xperiod;
    grid->yperiod = j->yperiod;
    grid->zperiod = j->zperiod;
    grid->dupe_x = (int32_t)j->dupe_x;
    grid->dupe_y = (int32_t)j->dupe_y;
    grid->dupe_z = (int32_t)j->dupe_z;
    // tem.cpp:1051-1058
    grid->replicate_atoms = (f.dupe && f.fem && (j->dupe_x > 1 || j->dupe_y > 1 || j->dupe_z > 1) &&
                             (j->dupe_x > 0 && j->dupe_y > 0 && j->dupe_z > 0)) ? 1 : 0;
    grid->xmin = j->xmin;
    grid->ymin = j->ymin;
    grid->zmin = j->zmin;
    grid->min_slice = j->min_slice;
  }
  if (atoms) {
    atoms->n_atoms = (int64_t)j->z.size();
    atoms->q = j->q.data();
    atoms->z = j->z.data();
  }
  if (optics) {
    optics->corrected = j->corrected ? 1 : 0;
    optics->cs3 = j->cs3_used;
    optics->cs5 = j->Cs5;
    optics->defocus = j->defocus;
    optics->alpha_max = j->alpha_max;
  }
  if (raster) {
    raster->n_x = (int32_t)j->x_p.size();
    raster->n_y = (int32_t)j->y_p.size();
    raster->x_p = j->x_p.data();
    raster->y_p = j->y_p.data();
  }
  if (det) {
    det->outputs = 0;
    if (f.image_output) det->outputs |= MSF_OUT_ADF_IMAGE;
    if (f.fem) {
      if (f.d1) det->outputs |= MSF_OUT_V_OMEGA;
      if (f.d2) det->outputs |= MSF_OUT_VBAR_R;
      if (f.d3) det->outputs |= MSF_OUT_V_RE;
      if (f.d4) det->outputs |= MSF_OUT_OMEGA_VIMAGE;
      if (f.gt17) det->outputs |= MSF_OUT_V_GT17;
      if (f.rva) det->outputs |= MSF_OUT_V_RBAR;
      if (f.correlograph) det->outputs |= MSF_OUT_CORRELOGRAPH;
      if (f.correlograph_variance) det->outputs |= MSF_OUT_CORRELOGRAPH_VAR;
    }
    det->det_inner = j->det_inner;
    det->det_outer = j->det_outer;
    det->dr = j->dr;
    det->n_mtf = 0;
    det->mtf = det->mtf_domain_sqr = nullptr;
    det->mtf_resolution = 0;
    if (f.mtf_file && f.mtf_resolution) {
      det->n_mtf = (int32_t)j->mtf.size();
      det->mtf = j->mtf.data();
      det->mtf_domain_sqr = j->mtf_domain.data();
      det->mtf_resolution = j->mtf_resolution;
    }
  }
  return MSF_OK;
}

const char* msf_job_output_prefix(const msf_job* j) { return j ? j->full_prefix.c_str() : ""; }

msf_status msf_write_outputs(const msf_job* j, const msf_results* r) {
  if (!j || !r) return MSF_ERR_ARG;
  const Flags& f = j->flags;
  const std::string& pre = j->full_prefix;
  if (f.fem && r->k_lower) {
    struct M { unsigned on; const double* v; const char* name; };
    const M modes[] = {{f.d1, r->v_omega, "_fem_V_omega"},   {f.d2, r->vbar_r, "_fem_Vbar_r"},
                       {f.gt17, r->v_gt17, "_fem_V_gt17"},   {f.d3, r->v_re, "_fem_V_re"},
                       {f.rva, r->v_rbar, "_fem_V_rbar"},    {f.d4, r->omega_vimage, "_fem_Omega_vimage"}};
    for (const M& m : modes)
      if (m.on && m.v && !write_variance(pre + m.name, r->k_lower, m.v, r->n_k)) {
        msf::set_error("Unable to write variance to file: " + pre + m.name + ".txt");
        return MSF_ERR_IO;
      }
  }
  if (f.fem && f.correlograph && r->correlograph && r->phi_lower && r->k_lower) {
    // adfstem.cpp:2652-2685, 3617-3760
    const int n_k = r->n_k, n_phi = r->n_phi;
    const size_t nc = (size_t)n_k * n_phi;
    const double k_res = (n_k / (1.0 - 0.2)) * 1.0e8;
    const double phi_res = (double)((unsigned)n_phi / 360);  // integer division, as there
    auto image = [&](const std::string& name, const double* d, size_t h, size_t w, bool logscale) {
      if (h * w == 0) return true;
      double mn = d[0], mx = d[0];
      for (size_t k = 0; k < h * w; ++k) { mx = std::max(mx, d[k]); mn = std::min(mn, d[k]); }
      return write_tif16(name + (logscale ? "_logscale.tif" : ".tif"), d, h, w, mn, mx, logscale,
                         phi_res, k_res, 3);
    };
    bool ok = true;
    if (r->correlograph_probes && (f.correlograph_everyimage || f.correlograph_everytxt)) {
      const size_t ny = j->y_p.size();
      for (size_t p = 0; p < j->x_p.size() * ny && ok; ++p) {
        const std::string name = pre + "_" + std::to_string(p / ny) + "_" + std::to_string(p % ny);
        const double* c = r->correlograph_probes + p * nc;
        if (f.correlograph_everyimage) ok = ok && image(name, c, n_phi, n_k, false);
        if (f.correlograph_everytxt)
          ok = ok && write_correlograph_txt(name, c, r->phi_lower, n_phi, r->k_lower, n_k);
      }
    }
    ok = ok && write_correlograph_txt(pre + "_correlograph_avg", r->correlograph, r->phi_lower,
                                      n_phi, r->k_lower, n_k) &&
         image(pre + "_correlograph_avg", r->correlograph, n_phi, n_k, false);
    if (ok && f.correlograph_variance && r->correlograph_sqr) {
      // k bins of [0.2, 1.0]; boundary ii is ii * delta_k (adfstem.cpp:1020-1026)
      auto bound = [&](int ii) { return ii < n_k ? r->k_lower[ii] : ii * r->k_lower[1]; };
      size_t start = 0, end = n_k > 0 ? n_k - 1 : 0;
      for (int ii = 0; ii < n_k; ++ii) {
        if (bound(ii) <= 0.2 && bound(ii + 1) > 0.2) start = ii;
        if (bound(ii) <= 1.0 && bound(ii + 1) > 1.0) end = ii;
      }
      const size_t n_red = end >= start ? end - start : 0;
      const double n_r = (double)(j->x_p.size() * j->y_p.size());
      std::vector<double> var(n_red * n_phi, 0.0);
      for (size_t ii = start; ii < end; ++ii)
        for (int jj = 0; jj < n_phi; ++jj) {
          const size_t c = ii + (size_t)jj * n_k, d = (ii - start) + (size_t)jj * n_red;
          const double sq = r->correlograph_sqr[c], av = r->correlograph[c];
          const double t = sq / (n_r * av * av);
          var[d] = (sq != 0 && n_r != 0 && av != 0 && t >= 1) ? t - 1 : 0;
        }
      ok = write_correlograph_txt(pre + "_correlograph_variance", r->correlograph_sqr,
                                  r->phi_lower, n_phi, r->k_lower, n_k) &&
           image(pre + "_correlograph_variance", var.data(), n_phi, n_red, true) &&
           image(pre + "_correlograph_variance", var.data(), n_phi, n_red, false);
    }
    if (!ok) {
      msf::set_error("could not write the correlograph outputs of " + pre);
      return MSF_ERR_IO;
    }
  }
  if (f.image_output) {
    // output_diffraction (write_tif.cpp:817-1098): log(1 + s |psi|^2),
    // quadrants swapped, min/max scaled, rows bottom-up; resolution
    // xperiod_duped * 1e-8, unit none; the scale factor in the file name is
    // printed by an ostringstream.  The first probe at five scales
    // (adfstem.cpp:2139-2221), the last one at scale 1 (:3778-3799).
    const size_t nx = (size_t)j->nx, ny = (size_t)j->ny;
    const double xres = j->xperiod * j->dupe_x * 1.0e-8, yres = j->yperiod * j->dupe_y * 1.0e-8;
    auto diffraction = [&](const double* psi, double scale, const std::string& tag) {
      std::vector<double> m(nx * ny);
      for (size_t k = 0; k < nx * ny; ++k) {
        const double re = psi[2 * k], im = psi[2 * k + 1];
        m[k] = std::log(1.0 + (scale * (re * re + im * im)));
      }
      double mn = m[0], mx = m[0];
      for (size_t k = 1; k < nx * ny; ++k) { mx = std::max(mx, m[k]); mn = std::min(mn, m[k]); }
      for (size_t i = 0; i < nx / 2; ++i) {
        for (size_t k = 0; k < ny / 2; ++k)
          std::swap(m[k + i * ny], m[(k + ny / 2) + (i + nx / 2) * ny]);
        for (size_t k = ny / 2; k < ny; ++k)
          std::swap(m[k + i * ny], m[(k - ny / 2) + (i + nx / 2) * ny]);
      }
      std::ostringstream sf;
      sf << scale;
      const std::string name = pre + tag + "_diffraction_scalefactor_" + sf.str() + ".tif";
      if (!write_tif16(name, m.data(), nx, ny, mn, mx, false, xres, yres, 1)) {
        msf::set_error("could not write " + name);
        return false;
      }
      return true;
    };
    if (r->first_psi)
      for (double scale : {1.0e-5, 1.0e-1, 1.0e0, 1.0e10, 1.0e+20})
        if (!diffraction(r->first_psi, scale, "_first")) return MSF_ERR_IO;
    if (r->final_psi && !diffraction(r->final_psi, 1.0e+0, "_final")) return MSF_ERR_IO;
    // FEM pixel modes (adfstem.cpp:3062-3097, 3468-3530): the raster means
    // of |psi(k)| and |psi(k)|^2 through the real-array output_diffraction
    // (write_tif.cpp:1413-1551, log(1 + s x^2)), and with --Omega_vimage the
    // 2-D variance <I>/<|psi|>^2 - 1 with the aperture disc zeroed.
    const bool pix = f.fem && (f.gt17 || f.d3 || f.d4 || f.rva);
    if (pix && r->mean_amplitude) {
      std::vector<double> c(2 * nx * ny, 0.0);
      auto real_diffraction = [&](const double* x, double scale, const std::string& tag) {
        for (size_t k = 0; k < nx * ny; ++k) c[2 * k] = x[k];
        return diffraction(c.data(), scale, tag);
      };
      if (!real_diffraction(r->mean_amplitude, 1.0e13, "_diffracted_wave_avg"))
        return MSF_ERR_IO;
      if ((f.gt17 || f.d3 || f.d4) && r->mean_intensity &&
          !real_diffraction(r->mean_intensity, 1.0e13, "_diffracted_wave_sqr_avg"))
        return MSF_ERR_IO;
      if (f.d4 && r->mean_intensity) {
        const msf::Grid g = msf::make_grid(
            j->nx, j->ny, j->VV, j->xperiod * j->dupe_x, j->yperiod * j->dupe_y,
            j->zperiod * j->dupe_z, j->xmin, j->ymin, j->zmin, j->xperiod, j->yperiod, j->zperiod);
        const double lambda_sqr = g.lambda * g.lambda, alpha_max_sqr = j->alpha_max * j->alpha_max;
        std::vector<double> var(nx * ny);
        for (size_t k = 0; k < nx * ny; ++k)
          var[k] = (r->mean_intensity[k] / (r->mean_amplitude[k] * r->mean_amplitude[k])) - 1.0;
        for (size_t i = 0; i < nx; ++i)
          for (size_t k = 0; k < ny; ++k) {
            const double ksqr = std::pow(g.kx[i], 2) + std::pow(g.ky[k], 2);
            if (lambda_sqr * ksqr <= alpha_max_sqr) var[k + ny * i] = 0.0;
          }
        if (!real_diffraction(var.data(), 1.0e0, "_variance_2-D") ||
            !real_diffraction(var.data(), 1.0e-10, "_variance_2-D"))
          return MSF_ERR_IO;
      }
    }
  }
  if (f.image_output && r->adf_image) {
    const size_t nx = j->x_p.size(), ny = j->y_p.size();
    const double* img = r->adf_image;
    double mn = img[0], mx = img[0];
    for (size_t k = 0; k < nx * ny; ++k) { mx = std::max(mx, img[k]); mn = std::min(mn, img[k]); }
    const double xres = (nx / j->xperiod) * 1.0e8, yres = (ny / j->yperiod) * 1.0e8;
    const std::string base = pre + "_stem_image_output";
    if (!write_tif16(base + ".tif", img, nx, ny, mn, mx, false, xres, yres, 3) ||
        !write_tif16(base + "_logscale.tif", img, nx, ny, mn, mx, true, xres, yres, 3)) {
      msf::set_error("could not write " + base + ".tif");
      return MSF_ERR_IO;
    }
    FILE* fp = std::fopen((base + ".f64").c_str(), "wb");
    if (fp) { std::fwrite(img, sizeof(double), nx * ny, fp); std::fclose(fp); }
  }
  return MSF_OK;
}

namespace {

// --paptif (slice.cpp:1660-1690 through func.cpp:2024-2362): per slice
// n = 1, 2, ..., 16-bit images of the projected potential before the
// exponential: magnitude (linear and log), real part (linear and log) and
// imaginary part, named <prefix>_pap_slice<n>_1_complex_fftw_operand_*.
// Each image is min/max scaled over the slice.  The reference starts the
// imaginary part's running min / max from uninitialised values (its
// initialisation lines set the real part's twice), so its imaginary images
// are not defined; here they start from the first sample like the others.
// As in the reference both imaginary images use the log scaling.
msf_status write_paptif(const msf_job* j, const msf_specimen* spec) {
  const size_t nx = j->nx, ny = j->ny, plane = nx * ny;
  const double xres = nx / (j->xperiod * j->dupe_x * 1e-8);
  const double yres = ny / (j->yperiod * j->dupe_y * 1e-8);
  std::vector<double> v(2 * plane), mag(plane), re(plane), im(plane);
  for (int32_t sl = 0; sl < spec->n_slices; ++sl) {
    msf_status st = msf_specimen_potential(spec, sl, v.data());
    if (st != MSF_OK) return st;
    for (size_t k = 0; k < plane; ++k) {
      re[k] = v[2 * k];
      im[k] = v[2 * k + 1];
      mag[k] = std::sqrt(std::pow(re[k], 2) + std::pow(im[k], 2));
    }
    auto range = [&](const std::vector<double>& a, double* mn, double* mx) {
      *mn = *mx = a[0];
      for (double x : a) { if (x > *mx) *mx = x; if (x < *mn) *mn = x; }
    };
    const std::string base = j->output_prefix + "_pap_slice" + std::to_string(sl + 1) +
                             "_1_complex_fftw_operand_";
    double mn, mx;
    bool ok = true;
    range(mag, &mn, &mx);
    ok = ok && write_tif16(base + "mag_output.tif", mag.data(), nx, ny, mn, mx, false, xres, yres, 3);
    ok = ok && write_tif16(base + "mag_output_logscale.tif", mag.data(), nx, ny, mn, mx, true,
                           xres, yres, 3);
    range(re, &mn, &mx);
    ok = ok && write_tif16(base + "re.tif", re.data(), nx, ny, mn, mx, false, xres, yres, 3);
    ok = ok && write_tif16(base + "re_logscale.tif", re.data(), nx, ny, mn, mx, true, xres, yres, 3);
    range(im, &mn, &mx);
    ok = ok && write_tif16(base + "im.tif", im.data(), nx, ny, mn, mx, true, xres, yres, 3);
    ok = ok && write_tif16(base + "im_logscale.tif", im.data(), nx, ny, mn, mx, true, xres, yres, 3);
    if (!ok) {
      msf::set_error("could not write " + base + "*.tif");
      return MSF_ERR_IO;
    }
  }
  return MSF_OK;
}

// One raster over `world` processes (one per GPU): every rank builds the
// specimen, runs its share of the probes and joins the exchange; rank 0
// alone writes the output files, as the reference's root rank does.  The
// rendezvous is MSF_RENDEZVOUS (host:port), else MASTER_ADDR with the port
// after MASTER_PORT (torchrun's own store listens on MASTER_PORT); the
// transport MSF_COMM = nccl (default; one GPU per rank) or host (ranks may
// share a GPU); the device is the local rank modulo the GPUs present.
int32_t sharded_main(msf_job* j, msf_options o, int rank, int world, int local) {
  std::string rdv;
  if (const char* r = std::getenv("MSF_RENDEZVOUS")) rdv = r;
  const char* ma = std::getenv("MASTER_ADDR");
  const char* mp = std::getenv("MASTER_PORT");
  if (rdv.empty() && ma && mp) rdv = std::string(ma) + ":" + std::to_string(std::atoi(mp) + 1);
  const char* tr = std::getenv("MSF_COMM");
  const int transport = (tr && std::string(tr) == "host") ? MSF_COMM_HOST : MSF_COMM_NCCL;
  double timeout_s = 300.0;
  if (const char* t = std::getenv("MSF_COMM_TIMEOUT")) timeout_s = std::atof(t);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) ndev = 1;
  o.device = local % ndev;
  msf_comm* comm = nullptr;
  msf_context* ctx = nullptr;
  msf_specimen* spec = nullptr;
  msf_grid grid;
  msf_atoms atoms;
  msf_optics optics;
  msf_raster raster;
  msf_detect det;
  msf_job_describe(j, &grid, &atoms, &optics, &raster, &det);
  int rc = 1;
  msf_status st = MSF_OK;
  if (rdv.empty()) {
    msf::set_error("a run over " + std::to_string(world) + " ranks needs MSF_RENDEZVOUS=host:port "
                   "or MASTER_ADDR and MASTER_PORT");
    st = MSF_ERR_ARG;
  } else if ((st = msf_context_create(&o, &ctx)) == MSF_OK &&
             (st = msf_context_keep_potentials(ctx, rank == 0 && j->flags.pap_tif)) == MSF_OK &&
             (st = msf_comm_create(rank, world, rdv.c_str(), transport, o.device, timeout_s,
                                   &comm)) == MSF_OK &&
             (st = msf_specimen_create(ctx, &grid, &atoms, &spec)) == MSF_OK &&
             (rank != 0 || !j->flags.pap_tif || (st = write_paptif(j, spec)) == MSF_OK)) {
    apply_wisdom(grid, ctx, spec, o, rank == 0);  // one writer of the wisdom file
    RunBuffers b;
    b.setup(j, grid, raster, det, true);
    if ((st = msf_run_sharded(ctx, spec, &optics, &raster, &det, comm, &b.r, nullptr)) ==
            MSF_OK &&
        (rank != 0 || (st = msf_write_outputs(j, &b.r)) == MSF_OK))
      rc = 0;
  }
  if (rc != 0) std::cerr << "ms-stem-fem (rank " << rank << "): " << msf::last_error() << std::endl;
  msf_comm_destroy(comm);
  msf_specimen_destroy(spec);
  msf_context_destroy(ctx);
  msf_job_destroy(j);
  return rc;
}

// Ranks of a multi-process launch, as `mpirun -np K` gives the reference
// (tem.cpp:90): torchrun's RANK / WORLD_SIZE / LOCAL_RANK, Open MPI's
// OMPI_COMM_WORLD_*, MPICH's PMI_RANK / PMI_SIZE, or Slurm's SLURM_PROCID /
// SLURM_NTASKS / SLURM_LOCALID.  world 1 when none is set.
struct Launch {
  int rank = 0, world = 1, local = 0;
};
Launch launch_from_env() {
  auto num = [](const char* name, int* out) {
    const char* v = std::getenv(name);
    if (!v || !*v) return false;
    *out = std::atoi(v);
    return true;
  };
  Launch l;
  const char* sets[][3] = {{"WORLD_SIZE", "RANK", "LOCAL_RANK"},
                           {"OMPI_COMM_WORLD_SIZE", "OMPI_COMM_WORLD_RANK",
                            "OMPI_COMM_WORLD_LOCAL_RANK"},
                           {"PMI_SIZE", "PMI_RANK", "MPI_LOCALRANKID"},
                           {"SLURM_NTASKS", "SLURM_PROCID", "SLURM_LOCALID"}};
  for (auto& s : sets) {
    int w = 0, r = 0;
    if (num(s[0], &w) && w > 1 && num(s[1], &r)) {
      l.world = w;
      l.rank = r;
      if (!num(s[2], &l.local)) l.local = r;
      break;
    }
  }
  return l;
}

}  // namespace

int32_t msf_main(int32_t argc, const char* const* argv, const msf_options* opt) {
  msf_job* j = nullptr;
  msf_status st = msf_parse_cmdline(argc, argv, &j);
  if (st != MSF_OK) {
    std::cout << msf::last_error();
    return 1;
  }
  msf_options o{};
  o.precision = MSF_FP64;
  o.use_graphs = 1;
  if (opt) o = *opt;
  const Launch launch = launch_from_env();
  if (launch.world > 1) return sharded_main(j, o, launch.rank, launch.world, launch.local);
  msf_context* ctx = nullptr;
  msf_specimen* spec = nullptr;
  msf_grid grid;
  msf_atoms atoms;
  msf_optics optics;
  msf_raster raster;
  msf_detect det;
  msf_job_describe(j, &grid, &atoms, &optics, &raster, &det);
  int rc = 1;
  if ((st = msf_context_create(&o, &ctx)) == MSF_OK &&
      (st = msf_context_keep_potentials(ctx, j->flags.pap_tif)) == MSF_OK &&
      (st = msf_specimen_create(ctx, &grid, &atoms, &spec)) == MSF_OK &&
      (!j->flags.pap_tif || (st = write_paptif(j, spec)) == MSF_OK)) {
    apply_wisdom(grid, ctx, spec, o);
    RunBuffers b;
    b.setup(j, grid, raster, det, true);
    if ((st = msf_run(ctx, spec, &optics, &raster, &det, &b.r)) == MSF_OK &&
        (st = msf_write_outputs(j, &b.r)) == MSF_OK)
      rc = 0;
  }
  if (rc != 0) std::cerr << "ms-stem-fem: " << msf::last_error() << std::endl;
  msf_specimen_destroy(spec);
  msf_context_destroy(ctx);
  msf_job_destroy(j);
  return rc;
}

int32_t msf_md_main(int32_t argc, const char* const* argv, const msf_options* opt) {
  std::vector<const char*> args;
  std::string replay_list;
  for (int32_t i = 0; i < argc; ++i) {
    if (i > 0 && std::string(argv[i]) == "--md_replay" && i + 1 < argc)
      replay_list = argv[++i];
    else
      args.push_back(argv[i]);
  }
  msf_job* j = nullptr;
  MdSetup md;
  MdFrame init;
  std::string err;
  msf_status st = parse_job((int32_t)args.size(), args.data(), true, &j, &md, &init);
  if (st != MSF_OK) {
    std::cout << msf::last_error();
    return 1;
  }
  // the configurations the samples see: the initial one when LAMMPS runs
  // no steps, else the replay list, sample s taking entry s mod K (every
  // probe's run count p * samples + s then maps to the same entry)
  std::vector<MdFrame> frames;
  bool ok = true;
  if (j->lammps_steps == 0) {
    frames.push_back(init);
  } else {
    std::vector<std::string> files;
    std::ifstream in(replay_list.c_str());
    std::string line;
    while (std::getline(in, line)) {
      std::istringstream ls(line);
      std::string path;
      if (ls >> path) files.push_back(path);
    }
    if (files.empty()) {
      err = "LAMMPS is not available here; give --md_replay <file> listing the "
            "LAMMPS data files its runs would produce, one per line\n";
      ok = false;
    } else if (j->lammps_samples % files.size() != 0) {
      err = "Error: lammps_TEM_samples (" + std::to_string(j->lammps_samples) +
            ") must be a multiple of the " + std::to_string(files.size()) + " replayed "
            "configurations\n";
      ok = false;
    }
    for (size_t k = 0; ok && k < files.size(); ++k) {
      frames.emplace_back();
      ok = read_md_frame(files[k], &frames.back(), &err);
    }
  }
  // every configuration's atoms, checked before any device work
  std::vector<std::vector<double>> qs(frames.size());
  std::vector<std::vector<uint32_t>> zs(frames.size());
  for (size_t k = 0; ok && k < frames.size(); ++k) {
    const MdFrame& fr = frames[k];
    if (fr.hi[0] - fr.lo[0] != j->xperiod || fr.hi[1] - fr.lo[1] != j->yperiod) {
      err = "Error: replayed configuration " + std::to_string(k) + " changes the x or y "
            "period of the box, which this driver does not support\n";
      ok = false;
    } else {
      ok = md_positions(fr, init, md, &qs[k], &zs[k], &err);
    }
  }
  msf_options o{};
  o.precision = MSF_FP64;
  o.use_graphs = 1;
  if (opt) o = *opt;
  msf_context* ctx = nullptr;
  std::vector<msf_specimen*> specs(frames.size(), nullptr);
  msf_grid grid;
  msf_optics optics;
  msf_raster raster;
  msf_detect det;
  msf_job_describe(j, &grid, nullptr, &optics, &raster, &det);
  int rc = 1;
  if (ok && (st = msf_context_create(&o, &ctx)) == MSF_OK) {
    for (size_t k = 0; ok && k < frames.size(); ++k) {
      msf_grid gk = grid;
      gk.zperiod = frames[k].hi[2] - frames[k].lo[2];  // follows the box (ftem_lammps.cpp:1611)
      msf_atoms a{(int64_t)zs[k].size(), qs[k].data(), zs[k].data()};
      if ((st = msf_specimen_create(ctx, &gk, &a, &specs[k])) != MSF_OK) ok = false;
    }
    if (ok) {
      apply_wisdom(grid, ctx, specs[0], o);
      RunBuffers b;
      b.setup(j, grid, raster, det, false);
      if ((st = msf_run_md(ctx, (int32_t)specs.size(), specs.data(),
                           (int32_t)j->lammps_samples, &optics, &raster, &det, &b.r)) == MSF_OK &&
          (st = msf_write_outputs(j, &b.r)) == MSF_OK)
        rc = 0;
    }
  }
  if (rc != 0) std::cerr << j->program << ": " << (err.empty() ? msf::last_error() : err.c_str())
                         << std::endl;
  for (msf_specimen* sp : specs) msf_specimen_destroy(sp);
  msf_context_destroy(ctx);
  msf_job_destroy(j);
  return rc;
}

}  // extern "C"
