// Bit-exact host set-up (see setup.hpp).  Compile with -ffp-contract=off.
#include "setup.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace msf {

namespace {
const double kKirkland[103][12] = {
#include "kirkland_table.inc"
};
struct MassRule { double exact, lo, hi; int hi_inclusive; unsigned z; };
const MassRule kMassRules[] = {
#include "mass_table.inc"
};
}  // namespace

void wavelength(double VV, double* lambda, double* gamma) {
  const double m_e0 = 9.109e-31, cc = 299792458, ee = 1.60217662e-19;
  const double hh = 6.62607004e-34;
  *lambda = hh * cc * std::pow(10, 10) / std::sqrt(ee * VV * (2.0 * m_e0 * cc * cc + ee * VV));
  *gamma = (hh * std::pow(10, 10) / *lambda) * (hh * std::pow(10, 10) / *lambda) *
           (m_e0 * cc * cc + ee * VV) / ((2 * m_e0 * cc * cc + ee * VV) * ee * VV * m_e0);
}

Grid make_grid(int nx, int ny, double voltage, double xpd, double ypd, double zpd,
               double xmin, double ymin, double zmin, double xperiod, double yperiod,
               double zperiod) {
  Grid g;
  g.nx = nx; g.ny = ny; g.voltage = voltage;
  g.xpd = xpd; g.ypd = ypd; g.zpd = zpd;
  g.xperiod = xperiod; g.yperiod = yperiod; g.zperiod = zperiod;
  g.xmin = xmin; g.ymin = ymin; g.zmin = zmin;
  const long Nx = nx, Ny = ny;
  g.xx.resize(nx); g.yy.resize(ny); g.kx.resize(nx); g.ky.resize(ny);
  // tem.cpp:756-788, func.cpp:92-106 and 147-167
  const double dx = xpd / Nx, dy = ypd / Ny, dkx = 1.0 / xpd, dky = 1.0 / ypd;
  const double kxp = Nx / xpd, kyp = Ny / ypd;
  for (int i = 0; i < Nx; ++i) g.xx[i] = xmin + (i * dx);
  for (int i = 0; i < Ny; ++i) g.yy[i] = ymin + (i * dy);
  for (int i = 0; i < Nx / 2; ++i) g.kx[i] = i * dkx;
  for (int i = Nx / 2; i < Nx; ++i) g.kx[i] = i * dkx - kxp;
  for (int i = 0; i < Ny / 2; ++i) g.ky[i] = i * dky;
  for (int i = Ny / 2; i < Ny; ++i) g.ky[i] = i * dky - kyp;
  // tem.cpp:683-695
  if (Nx / (2 * xpd) < Ny / (2 * ypd)) g.bw_pap = Nx / (2 * xpd);
  else g.bw_pap = Ny / (2 * ypd);
  g.bw_t = (2.0 / 3.0) * g.bw_pap;
  wavelength(voltage, &g.lambda, &g.gamma);
  g.nxny = (double)(Nx * Ny);
  g.s = (Nx == Ny) ? (double)Nx : std::sqrt(g.nxny);
  return g;
}

Slicing slice_atoms(int64_t n, const double* q, double zmin, double zperiod,
                    double min_thickness) {
  Slicing sl;
  if (n == 0) {  // slice.cpp:632-639
    sl.start = {0, 0};
    sl.lower = {zmin};
    sl.thickness = {zperiod};
    return sl;
  }
  // scatterer_sorting_lt_z (scatterer.hpp:192); ties share a slice and a
  // mean, so their order is immaterial -- keep index order.  Sorting
  // contiguous (z, index) pairs lexicographically gives exactly that order
  // (a stable sort by z) without chasing q through an indirect comparator.
  std::vector<std::pair<double, int64_t>> keys((size_t)n);
  for (int64_t k = 0; k < n; ++k) keys[(size_t)k] = {q[3 * k + 2], k};
  std::sort(keys.begin(), keys.end());
  sl.order.resize(n);
  for (int64_t k = 0; k < n; ++k) sl.order[(size_t)k] = keys[(size_t)k].second;
  sl.start.push_back(0);
  sl.lower.push_back(0.0);
  double first = q[3 * sl.order[0] + 2];
  for (int64_t k = 0; k < n; ++k) {
    const double z = q[3 * sl.order[k] + 2];
    if (z - first <= min_thickness) {
      sl.lower.back() += z;
    } else {
      sl.start.push_back(k);
      sl.lower.push_back(z);
      first = z;
    }
  }
  sl.start.push_back(n);
  const int64_t ns = (int64_t)sl.lower.size();
  for (int64_t s = 0; s < ns; ++s)
    sl.lower[s] = sl.lower[s] / (double)(size_t)(sl.start[s + 1] - sl.start[s]);
  sl.thickness.resize(ns);
  for (int64_t s = 0; s < ns; ++s) {
    if (s + 1 == ns)
      sl.thickness[s] = q[3 * sl.order[sl.start[s + 1] - 1] + 2] + min_thickness - sl.lower[s];
    else
      sl.thickness[s] = sl.lower[s + 1] - sl.lower[s];
  }
  return sl;
}

int64_t snap(const std::vector<double>& grid, double q, double half, int64_t fallback) {
  // The reference scans for the first i with grid[i] - q >= half.  grid is
  // increasing and rounded subtraction is monotone, so that predicate is
  // false then true along i: a binary search over the same predicate finds
  // the same first index (O(log n) instead of O(n) per atom).
  size_t lo = 0, hi = grid.size();
  while (lo < hi) {
    const size_t mid = lo + (hi - lo) / 2;
    if (grid[mid] - q >= half) hi = mid;
    else lo = mid + 1;
  }
  return lo < grid.size() ? (int64_t)lo - 1 : fallback;
}

bool probe_shifts(const Grid& g, const std::vector<double>& x_p,
                  const std::vector<double>& y_p, std::vector<int32_t>* shifts) {
  const double hx = 0.5 * (g.xx[1] - g.xx[0]);
  const double hy = 0.5 * (g.yy[1] - g.yy[0]);
  shifts->assign(2 * x_p.size() * y_p.size(), 0);
  int64_t sx = 0, sy = 0;  // adfstem.cpp:1525-1528, never reset per probe
  size_t k = 0;
  for (double xp : x_p) {
    for (double yp : y_p) {
      sx = snap(g.xx, xp, hx, sx);
      sy = snap(g.yy, yp, hy, sy);
      if (sx < 0 || sy < 0) return false;
      (*shifts)[2 * k] = (int32_t)sx;
      (*shifts)[2 * k + 1] = (int32_t)sy;
      ++k;
    }
  }
  return true;
}

bool bandlimit_mask(const Grid& g, double cutoff, std::vector<int32_t>* lo,
                    std::vector<int32_t>* hi) {
  const double csq = std::pow(cutoff, 2);
  lo->assign(g.ny, 0);
  hi->assign(g.ny, g.nx);
  for (int j = 0; j < g.ny; ++j) {
    std::vector<uint8_t> keep(g.nx);
    for (int i = 0; i < g.nx; ++i)
      keep[i] = (std::pow(g.kx[i], 2) + std::pow(g.ky[j], 2)) < csq;
    int a = 0;
    while (a < g.nx && keep[a]) ++a;
    int b = g.nx;
    while (b > a && keep[b - 1]) --b;
    for (int i = a; i < b; ++i)
      if (keep[i]) return false;  // not of the form [0,a) U [b,n)
    (*lo)[j] = a;
    (*hi)[j] = b;
  }
  return true;
}

void propagator(const Grid& g, double thickness, std::vector<double>* px,
                std::vector<double>* py) {
  px->assign(2 * g.nx, 0.0);
  py->assign(2 * g.ny, 0.0);
  for (int i = 0; i < g.nx; ++i)
    if (g.kx[i] < g.bw_t && g.kx[i] > -1.0 * g.bw_t) {
      const double a = kPi * g.lambda * thickness * std::pow(g.kx[i], 2);
      (*px)[2 * i] = std::cos(a);
      (*px)[2 * i + 1] = -std::sin(a);
    }
  for (int j = 0; j < g.ny; ++j)
    if (g.ky[j] < g.bw_t && g.ky[j] > -1.0 * g.bw_t) {
      const double a = kPi * g.lambda * thickness * std::pow(g.ky[j], 2);
      (*py)[2 * j] = std::cos(a);
      (*py)[2 * j + 1] = -std::sin(a);
    }
}

Rings make_rings(const Grid& g, double dr) {
  Rings r;
  r.delta_k = dr * std::sqrt((g.kx[1] - g.kx[0]) * (g.kx[1] - g.kx[0]) +
                             (g.ky[1] - g.ky[0]) * (g.ky[1] - g.ky[0]));
  const unsigned nk = (unsigned)(g.bw_t / r.delta_k);
  r.n_k = (int32_t)nk;
  for (unsigned ii = 0; ii < nk + 1; ++ii) r.bounds.push_back(ii * r.delta_k);
  const int64_t np = (int64_t)g.nx * g.ny;
  r.bin.assign(np, -1);
  r.counts.assign(nk, 0);
  std::vector<double> ub2(nk);
  for (unsigned ii = 0; ii < nk; ++ii) ub2[ii] = r.bounds[ii + 1] * r.bounds[ii + 1];
  std::vector<std::pair<double, int32_t>> sorted;
  sorted.reserve(np);
  for (int i = 0; i < g.nx; ++i)
    for (int j = 0; j < g.ny; ++j) {
      const double ksq = g.kx[i] * g.kx[i] + g.ky[j] * g.ky[j];
      // smallest ii with ksq <= ub2[ii] (ub2 ascending)
      const auto it = std::lower_bound(ub2.begin(), ub2.end(), ksq);
      const int32_t b = (it == ub2.end()) ? -1 : (int32_t)(it - ub2.begin());
      r.bin[j + (int64_t)i * g.ny] = b;
      if (b >= 0) {
        r.counts[b] += 1;
        sorted.emplace_back(ksq, (int32_t)(j + (int64_t)i * g.ny));
      }
    }
  std::stable_sort(sorted.begin(), sorted.end(),
                   [](const std::pair<double, int32_t>& a, const std::pair<double, int32_t>& b) {
                     return a.first < b.first;
                   });
  r.start.assign(nk + 1, 0);
  for (unsigned ii = 0; ii < nk; ++ii) r.start[ii + 1] = r.start[ii] + r.counts[ii];
  r.pix.resize(sorted.size());
  for (size_t k = 0; k < sorted.size(); ++k) r.pix[k] = sorted[k].second;
  r.inside.assign(nk, 0);
  return r;
}

Cells make_cells(const Grid& g, const Rings& r) {
  Cells c;
  unsigned count = 0;
  for (double b : r.bounds)
    if (b >= 0.2 && b <= 1.0) ++count;
  c.n_phi = count > 0 ? (int32_t)(count - 1) : 0;
  const size_t n_cells = (size_t)r.n_k * c.n_phi;
  c.start.assign(n_cells + 1, 0);
  if (c.n_phi == 0) {
    c.phi_bounds.assign(1, 0.0);
    return c;
  }
  const double delta_phi = 2 * kPi / c.n_phi;
  for (int32_t ii = 0; ii < c.n_phi + 1; ++ii) c.phi_bounds.push_back(ii * delta_phi);
  // cell of every ring pixel, in ring order
  std::vector<int32_t> cell_of(r.pix.size(), -1);
  std::vector<int32_t> counts(n_cells, 0);
  for (int32_t ii = 0; ii < r.n_k; ++ii)
    for (int32_t q = r.start[ii]; q < r.start[ii + 1]; ++q) {
      const int32_t p = r.pix[q];
      const int i = p / g.ny, j = p % g.ny;
      const double phi = kPi + std::atan2(g.ky[j], g.kx[i]);
      double lower = c.phi_bounds[0];
      for (int32_t jj = 0; jj < c.n_phi; ++jj) {
        if (phi > lower && phi <= c.phi_bounds[jj + 1]) {
          cell_of[q] = ii * c.n_phi + jj;
          ++counts[(size_t)ii * c.n_phi + jj];
          break;
        }
        lower = c.phi_bounds[jj];  // lags one boundary behind, as there
      }
    }
  for (size_t k = 0; k < n_cells; ++k) c.start[k + 1] = c.start[k] + counts[k];
  c.pix.assign(c.start[n_cells], 0);
  std::vector<int32_t> fill(c.start.begin(), c.start.end() - 1);
  for (size_t q = 0; q < r.pix.size(); ++q)
    if (cell_of[q] >= 0) c.pix[fill[cell_of[q]]++] = r.pix[q];
  return c;
}

std::vector<int32_t> detector_pixels(const Grid& g, double k1, double k2) {
  std::vector<int32_t> out;
  for (int i = 0; i < g.nx; ++i)
    for (int j = 0; j < g.ny; ++j) {
      const double ksq = g.kx[i] * g.kx[i] + g.ky[j] * g.ky[j];
      if (ksq > k1 && ksq <= k2) out.push_back((int32_t)(j + (int64_t)i * g.ny));
    }
  return out;
}

std::vector<double> raster_points(double period, double origin, double spacing) {
  const size_t n = (size_t)std::floor(period / spacing);
  std::vector<double> out;
  const double d = period / (int)n;
  for (int i = 0; i < (int)n; ++i) out.push_back(origin + (i * d));
  return out;
}

double scherzer(int which, double lambda, double a) {
  switch (which) {
    case 0: return 0.87 * std::sqrt(a * lambda);
    case 1: return 1.34 * std::pow(lambda / a, 0.25);
    case 2: return -0.983 * std::pow(std::pow(lambda, 2) * a, 1.0 / 3.0);
    case 3: return 1.513 * std::pow(lambda / a, 1.0 / 6.0);
    case 4: return -2.289 * std::pow(lambda * std::pow(a, 2), 1.0 / 3.0);
  }
  return 0.0;
}

unsigned guess_z(double mass) {
  for (const MassRule& r : kMassRules) {
    if (r.exact >= 0.0 && mass == r.exact) return r.z;
    const bool below_hi = r.hi_inclusive ? (mass <= r.hi) : (mass < r.hi);
    if (mass >= r.lo && below_hi) return r.z;
  }
  return 0;
}

const double* kirkland_params(unsigned z) {
  if (z < 1 || z > 103) return nullptr;
  return kKirkland[z - 1];
}

}  // namespace msf

namespace msf {

std::vector<double> mtf_2d(const Grid& g, const double* mtf, const double* domain_sqr, int n,
                           double resolution) {
  std::vector<double> out(2 * (size_t)g.nx * g.ny, 0.0);
  const double nx = (double)g.nx, ny = (double)g.ny;
  for (int i = 0; i < g.nx; ++i)
    for (int j = 0; j < g.ny; ++j) {
      const double xxx = std::pow(g.xpd, 2) * g.kx[i] / nx;
      const double yyy = std::pow(g.ypd, 2) * g.ky[j] / ny;
      const double rsqr = std::pow(xxx, 2) + std::pow(yyy, 2);
      double v = 0.0;
      for (int k = 0; k + 1 < n; ++k) {
        if (rsqr >= domain_sqr[k] && rsqr < domain_sqr[k + 1]) {
          const double d1 = std::sqrt(domain_sqr[k]), d2 = std::sqrt(domain_sqr[k + 1]);
          v = mtf[k] + (mtf[k + 1] - mtf[k]) * (std::sqrt(rsqr) - d1) / (d2 - d1);
          double arg = xxx / resolution;
          const double sx = arg != 0 ? std::sin(arg) / arg : 1;
          arg = yyy / resolution;
          const double sy = arg != 0 ? std::sin(arg) / arg : 1;
          v = v * sx * sy;
        }
      }
      out[2 * ((size_t)i * g.ny + j)] = v;
    }
  return out;
}

}  // namespace msf
