// Host-side set-up of the multislice path: every scalar, domain, slice
// boundary, pixel snap, mask and bin index the device kernels consume.
// These must equal the reference's values bit for bit, so they are computed
// on the host in FP64 with the reference's operation order (this file is
// compiled with -ffp-contract=off).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace msf {

constexpr double kPi = 3.14159265369;  // the reference's PI (adfstem.hpp:55)

struct Grid {
  int nx = 0, ny = 0;
  double voltage = 0;
  double xperiod = 0, yperiod = 0, zperiod = 0;        // specimen (raster)
  double xpd = 0, ypd = 0, zpd = 0;                    // duped cell
  double xmin = 0, ymin = 0, zmin = 0;
  double lambda = 0, gamma = 0;
  double bw_pap = 0, bw_t = 0;
  double s = 1;      // sqrtNxNy (tem.cpp:407-408, adfstem.cpp:196-198)
  double nxny = 1;   // NxNy as double
  std::vector<double> xx, yy, kx, ky;
};

// lambda, gamma (tem.cpp:424-438)
void wavelength(double voltage, double* lambda, double* gamma);
// Domains, cut-offs and constants for a cell (tem.cpp:683-788).
Grid make_grid(int nx, int ny, double voltage, double xpd, double ypd, double zpd,
               double xmin, double ymin, double zmin, double xperiod, double yperiod,
               double zperiod);

struct Slicing {
  std::vector<int64_t> order;   // atom indices in slice order
  std::vector<int64_t> start;   // n_slices + 1 offsets into order
  std::vector<double> lower, thickness;
  int64_t n() const { return (int64_t)lower.size(); }
};
// assign_atoms_to_slices_z_auto (slice.cpp:469-980)
Slicing slice_atoms(int64_t n, const double* q, double zmin, double zperiod,
                    double min_thickness);

// (first i with grid[i] - q >= half) - 1; `fallback` when no i matches; -1
// where the reference's size_t index would wrap (slice.cpp:1556-1572,
// adfstem.cpp:1590-1606).
int64_t snap(const std::vector<double>& grid, double q, double half, int64_t fallback);

// Per-probe pixel shifts in raster order (x outer, y inner) with the shift
// carried over from the previous probe when no pixel matches.
bool probe_shifts(const Grid& g, const std::vector<double>& x_p,
                  const std::vector<double>& y_p, std::vector<int32_t>* shifts);

// Band-limit mask kx^2+ky^2 < bw_t^2 as, per column j, "keep i < lo[j] or
// i >= hi[j]" (bw_limit.cpp:30-47 and slice.cpp:1385-1419 use the same set).
bool bandlimit_mask(const Grid& g, double cutoff, std::vector<int32_t>* lo,
                    std::vector<int32_t>* hi);

// Propagator tables (slice.cpp:1293-1363), interleaved re/im.
void propagator(const Grid& g, double thickness, std::vector<double>* px,
                std::vector<double>* py);

// FEM ring bins (adfstem.cpp:947-1062, variance.cpp:64-300).
struct Rings {
  int32_t n_k = 0;
  double delta_k = 0;
  std::vector<double> bounds;      // n_k + 1
  std::vector<int32_t> bin;        // per pixel, -1 outside
  std::vector<int32_t> counts;     // per bin
  std::vector<int32_t> pix;        // pixels grouped by bin, ascending k^2
  std::vector<int32_t> start;      // n_k + 1 offsets into pix
  std::vector<uint8_t> inside;     // lambda*b_{k+1} <= alpha_max
};
Rings make_rings(const Grid& g, double dr);

// Azimuthal cells of the FEM correlograph (adfstem.cpp:956-1062,
// variance.cpp:227-251): n_phi = (ring boundaries in [0.2, 1.0]) - 1 bins of
// 2 PI / n_phi (PI as the reference's), phi = PI + atan2(ky, kx) per pixel,
// bin chosen by the reference's loop; pixel lists per (k bin, phi bin) cell
// [ii * n_phi + jj], each in ring order.
struct Cells {
  int32_t n_phi = 0;
  std::vector<double> phi_bounds;  // n_phi + 1
  std::vector<int32_t> pix;
  std::vector<int32_t> start;      // n_k * n_phi + 1 offsets into pix
};
Cells make_cells(const Grid& g, const Rings& r);

// Two-dimensional detector MTF before its band limiting (adfstem.cpp:298-384):
// interleaved complex [nx][ny], real part interpolated from (mtf,
// domain_sqr) at r^2 = (xpd^2 kx/Nx)^2 + (ypd^2 ky/Ny)^2 and multiplied by
// sinc(xpd^2 kx/Nx / res) sinc(ypd^2 ky/Ny / res) where r^2 lies in the table;
// 0 elsewhere.  Every table interval is tested (the last match wins).
std::vector<double> mtf_2d(const Grid& g, const double* mtf, const double* domain_sqr, int n,
                           double resolution);

// ADF detector pixels k1 < kx*kx+ky*ky <= k2 (func.cpp:2593-2640).
std::vector<int32_t> detector_pixels(const Grid& g, double k1, double k2);

// Raster positions (func.cpp:108-127, tem.cpp:1358-1378).
std::vector<double> raster_points(double period, double origin, double spacing);

// Scherzer conditions (scherzer.cpp:61-168).
double scherzer(int which, double lambda, double aberration);

// mass -> Z (tem_io.cpp:1030-1258); 0 when no rule matches.
unsigned guess_z(double mass);
// Kirkland parameters as the reference stores them, {a0..a2,b0..b2,c0..c2,
// d0..d2}, for Z = 1..103.
const double* kirkland_params(unsigned z);

}  // namespace msf
