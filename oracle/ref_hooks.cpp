// Link-time hooks around four of the reference's own functions (GNU ld
// --wrap), compiled into the oracle binary oracle/_ref/ms-stem-fem-ref only.
// Test infrastructure: each hook calls the reference's real function
// unchanged and then records what the oracle tests need.
//
//  * TEM_NS::adfstem (adfstem.cpp:37) -- wall-clock time of the whole raster
//    (probe build, every probe through every slice, detection, FEM), printed
//    to stderr as "msf-ref: adfstem_seconds=..." so a timed CPU baseline can
//    exclude the specimen set-up that tem.cpp does before it.
//  * TEM_NS::output_stem_image (write_tif.cpp:1552) -- also writes the raw
//    FP64 ADF image to <prefix>_stem_image_output.f64 (the TIFF is 16-bit
//    quantised, too coarse for a 1e-5 parity check).
//  * TEM_NS::assign_atoms_to_slices_z_auto (slice.cpp:469) -- when
//    MSF_REF_DUMP_SLICES names a file, writes "lower_bound thickness count"
//    per slice with 17 significant digits.
//  * TEM_NS::slice::update_transmission_function (slice.cpp:1451) -- when
//    MSF_REF_DUMP_T names a path prefix, writes each slice's transmission
//    function as raw complex128 to <prefix><slice number>.c128.
#include "adfstem.hpp"
#include "slice.hpp"
#include "write_tif.hpp"

#include <cstdio>
#include <cstdlib>
#include <list>
#include <string>
#include <sys/time.h>
#include <vector>

using namespace TEM_NS;

static double now_seconds() {
  struct timeval tv;
  gettimeofday(&tv, 0);
  return (double)tv.tv_sec + 1e-6 * (double)tv.tv_usec;
}

#define ADFSTEM_SYM _ZN6TEM_NS7adfstemERKNS_11input_flagsERNSt7__cxx114listIPNS_5sliceESaIS6_EEERKdSB_SB_SB_SB_RKNS4_IdSaIdEEESF_SB_SB_SB_SB_PSA_SG_SG_SG_SG_RKlSI_SG_SI_SB_SB_SB_SB_SB_SB_SB_RKSt6vectorIdSC_ESM_SB_SB_RKNS3_12basic_stringIcSt11char_traitsIcESaIcEEESI_SI_PKiSV_SV_SV_RSU_SW_SW_i
#define STEMIMG_SYM _ZN6TEM_NS17output_stem_imageEPKdRKlS3_RKmRS0_S6_RKNSt7__cxx1112basic_stringIcSt11char_traitsIcESaIcEEE
#define SLICER_SYM _ZN6TEM_NS29assign_atoms_to_slices_z_autoERKSt6vectorINS_9scattererESaIS1_EERKdS7_S7_S7_S7_S7_S7_RNSt7__cxx114listIPNS_5sliceESaISB_EEERKjRKiSI_i
#define TRANS_SYM _ZN6TEM_NS5slice28update_transmission_functionERKdS2_S2_S2_PS1_RKlS3_S3_S5_S3_S3_S5_S2_RKjRKNSt7__cxx1112basic_stringIcSt11char_traitsIcESaIcEEERKmS5_S5_PKiSJ_RSI_SK_i

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define REAL(s) CAT(__real_, s)
#define WRAP(s) CAT(__wrap_, s)

#define ADFSTEM_PARAMS                                                       \
  const input_flags &flags, std::list<slice *> &slices,                      \
      const double &bwcutoff_pap, const double &bwcutoff_t,                  \
      const double &binfac, const double &xmin, const double &ymin,          \
      const std::list<double> &x_p, const std::list<double> &y_p,            \
      const double &xperiod, const double &yperiod, const double &xpd,       \
      const double &ypd, const double *const xx_local,                       \
      const double *const xx_joined, const double *const yy,                 \
      const double *const kx_local, const double *const kx_joined,           \
      const ptrdiff_t &Nx, const ptrdiff_t &Nx_local, const double *const ky, \
      const ptrdiff_t &Ny, const double &Cs3, const double &Cs5,             \
      const double &defocus, const double &defocus_spread,                   \
      const double &alpha_max, const double &det_in, const double &det_out,  \
      const std::vector<double> &mtf, const std::vector<double> &mtf_dom,    \
      const double &mtf_res, const double &lambda, const string &prefix,     \
      const ptrdiff_t &las, const ptrdiff_t &l0s, const int *const nxs,      \
      const int *const nxd, const int *const pms, const int *const pmd,      \
      const int &mynode, const int &rootnode, const int &totalnodes,         \
      MPI_Comm comm
#define ADFSTEM_ARGS                                                          \
  flags, slices, bwcutoff_pap, bwcutoff_t, binfac, xmin, ymin, x_p, y_p,      \
      xperiod, yperiod, xpd, ypd, xx_local, xx_joined, yy, kx_local,          \
      kx_joined, Nx, Nx_local, ky, Ny, Cs3, Cs5, defocus, defocus_spread,     \
      alpha_max, det_in, det_out, mtf, mtf_dom, mtf_res, lambda, prefix, las, \
      l0s, nxs, nxd, pms, pmd, mynode, rootnode, totalnodes, comm

extern "C" int REAL(ADFSTEM_SYM)(ADFSTEM_PARAMS);
extern "C" int WRAP(ADFSTEM_SYM)(ADFSTEM_PARAMS) {
  double t0 = now_seconds();
  int rc = REAL(ADFSTEM_SYM)(ADFSTEM_ARGS);
  double t1 = now_seconds();
  std::fprintf(stderr,
               "msf-ref: adfstem_seconds=%.6f probes=%zu slices=%zu nx=%ld "
               "ny=%ld\n",
               t1 - t0, x_p.size() * y_p.size(), slices.size(), (long)Nx,
               (long)Ny);
  return rc;
}

extern "C" void REAL(STEMIMG_SYM)(const double *const img, const ptrdiff_t &nx,
                                  const ptrdiff_t &ny, const size_t &ru,
                                  const double &xr, const double &yr,
                                  const string &prefix);
extern "C" void WRAP(STEMIMG_SYM)(const double *const img, const ptrdiff_t &nx,
                                  const ptrdiff_t &ny, const size_t &ru,
                                  const double &xr, const double &yr,
                                  const string &prefix) {
  std::string name = prefix + "_stem_image_output.f64";
  FILE *f = std::fopen(name.c_str(), "wb");
  if (f) {
    std::fwrite(img, sizeof(double), (size_t)(nx * ny), f);
    std::fclose(f);
  }
  REAL(STEMIMG_SYM)(img, nx, ny, ru, xr, yr, prefix);
}

#define SLICER_PARAMS                                                       \
  const std::vector<scatterer> &all, const double &xmin, const double &ymin, \
      const double &zmin, const double &xperiod, const double &yperiod,      \
      const double &zperiod, const double &min_thickness,                    \
      std::list<slice *> &slice_list, const unsigned int &dbg,               \
      const int &mynode, const int &rootnode, MPI_Comm comm

extern "C" int REAL(SLICER_SYM)(SLICER_PARAMS);
extern "C" int WRAP(SLICER_SYM)(SLICER_PARAMS) {
  int rc = REAL(SLICER_SYM)(all, xmin, ymin, zmin, xperiod, yperiod, zperiod,
                            min_thickness, slice_list, dbg, mynode, rootnode,
                            comm);
  const char *path = std::getenv("MSF_REF_DUMP_SLICES");
  if (path && *path) {
    FILE *f = std::fopen(path, "w");
    if (f) {
      for (std::list<slice *>::const_iterator it = slice_list.begin();
           it != slice_list.end(); ++it)
        std::fprintf(f, "%.17g %.17g %zu\n", (*it)->lower_bound,
                     (*it)->thickness, (*it)->scatterers->size());
      std::fclose(f);
    }
  }
  return rc;
}

#define TRANS_PARAMS                                                          \
  slice *self, const double &lambda, const double &gamma,                     \
      const double &ab_inv, const double &bwcutoff_t,                         \
      const double *const kx_local, const ptrdiff_t &Nx_local,                \
      const double *const kx_joined, const double *const xx_joined,           \
      const ptrdiff_t &Nx_joined, const double *const ky,                     \
      const double *const yy, const ptrdiff_t &Ny, const double &NxNy,        \
      const unsigned int &paptif, const string &outname,                      \
      const size_t &slice_number, const ptrdiff_t &las, const ptrdiff_t &l0s, \
      const int *const pms, const int *const pmd, const int &mynode,          \
      const int &rootnode, MPI_Comm comm

extern "C" int REAL(TRANS_SYM)(TRANS_PARAMS);
extern "C" int WRAP(TRANS_SYM)(TRANS_PARAMS) {
  int rc = REAL(TRANS_SYM)(self, lambda, gamma, ab_inv, bwcutoff_t, kx_local,
                           Nx_local, kx_joined, xx_joined, Nx_joined, ky, yy,
                           Ny, NxNy, paptif, outname, slice_number, las, l0s,
                           pms, pmd, mynode, rootnode, comm);
  const char *prefix = std::getenv("MSF_REF_DUMP_T");
  if (prefix && *prefix) {
    char name[4096];
    std::snprintf(name, sizeof(name), "%s%zu.c128", prefix, slice_number);
    FILE *f = std::fopen(name, "wb");
    if (f) {
      std::fwrite(self->exp_i_sigma_v, sizeof(fftw_complex),
                  (size_t)(Nx_local * Ny), f);
      std::fclose(f);
    }
  }
  return rc;
}
