// ms-stem-fem: drop-in replacement for the reference executable's ADF-STEM /
// FEM path (tem.cpp:81-1771); built with MSF_MD_DRIVER it is ms-stem-fem-md,
// the replacement of the LAMMPS-coupled driver (ftem_lammps.cpp), which also
// takes --md_replay <file> (msf_md_main in msf.h).  Accepts the reference's
// options and parameter files unchanged; three options of this build are
// taken out before the reference's parser sees the rest, and none changes a
// default:
//   --precision fp64|fp32   wavefield/FFT precision (default fp64, as the
//                           reference)
//   --batch <n>             probes per launch (default: from free memory)
//   --device <n>            CUDA device ordinal (default 0)
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "msf.h"

int main(int argc, char** argv) {
  msf_options opt{};
  opt.precision = MSF_FP64;
  opt.use_graphs = 1;
  std::vector<const char*> rest;
  rest.push_back(argv[0]);
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--precision" && i + 1 < argc) {
      const std::string v = argv[++i];
      if (v == "fp32") opt.precision = MSF_FP32;
      else if (v == "fp64") opt.precision = MSF_FP64;
      else { std::cerr << "--precision must be fp32 or fp64" << std::endl; return 1; }
    } else if (a == "--batch" && i + 1 < argc) {
      opt.batch = std::atoi(argv[++i]);
    } else if (a == "--device" && i + 1 < argc) {
      opt.device = std::atoi(argv[++i]);
    } else {
      rest.push_back(argv[i]);
    }
  }
#ifdef MSF_MD_DRIVER
  return msf_md_main((int32_t)rest.size(), rest.data(), &opt);
#else
  return msf_main((int32_t)rest.size(), rest.data(), &opt);
#endif
}
