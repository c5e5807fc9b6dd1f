/* CPU restatement of the reference's multislice path (see msf_oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY -- the oracle, never the product.  FP64 throughout,
 * compiled with -ffp-contract=off so scalar set-up values (lambda, gamma,
 * domains, cut-offs, bin boundaries, pixel snaps) are bit-identical to the
 * reference's.  Citations are to the reference sources (src/ implied). */
#include "msf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OR_PI 3.14159265369 /* adfstem.hpp:55, func.hpp:34 (quirk: not pi) */

static const double kirkland[103][12] = {
#include "../ms-stem-fem_b200/csrc/kirkland_table.inc"
};

/* ------------------------------------------------------------- FFT -------
 * Unnormalised complex DFT with FFTW's sign convention (the reference's
 * fftw_mpi_plan_dft_2d calls): sign -1 forward, +1 backward.  Radix-2 for
 * power-of-two lengths, direct DFT otherwise. */
static void fft1d(double* re, double* im, size_t n, int sign, const double* tw) {
  if (n <= 1) return;
  const double two_pi = 6.283185307179586476925286766559;
  if ((n & (n - 1)) == 0) {
    size_t bits = 0;
    while (((size_t)1 << bits) < n) ++bits;
    for (size_t k = 0; k < n; ++k) {
      size_t r = 0;
      for (size_t b = 0; b < bits; ++b) r |= ((k >> b) & 1) << (bits - 1 - b);
      if (r > k) {
        double t = re[k]; re[k] = re[r]; re[r] = t;
        t = im[k]; im[k] = im[r]; im[r] = t;
      }
    }
    for (size_t len = 2; len <= n; len <<= 1) {
      size_t half = len >> 1, step = n / len;
      for (size_t s = 0; s < n; s += len)
        for (size_t k = 0; k < half; ++k) {
          double wr = tw[2 * k * step], wi = tw[2 * k * step + 1];
          size_t a = s + k, b = a + half;
          double tr = re[b] * wr - im[b] * wi;
          double ti = re[b] * wi + im[b] * wr;
          re[b] = re[a] - tr; im[b] = im[a] - ti;
          re[a] += tr; im[a] += ti;
        }
    }
    return;
  }
  double* out = (double*)malloc(2 * n * sizeof(double));
  for (size_t k = 0; k < n; ++k) {
    double sr = 0.0, si = 0.0;
    for (size_t m = 0; m < n; ++m) {
      size_t idx = (k * m) % n;
      double c = tw[2 * idx], s = tw[2 * idx + 1];
      sr += re[m] * c - im[m] * s;
      si += re[m] * s + im[m] * c;
    }
    out[2 * k] = sr; out[2 * k + 1] = si;
  }
  for (size_t k = 0; k < n; ++k) { re[k] = out[2 * k]; im[k] = out[2 * k + 1]; }
  free(out);
  (void)two_pi;
}

/* e^{sign 2 pi i k / n} for k < n, interleaved (libm cos/sin in FP64). */
static double* twiddles(size_t n, int sign) {
  const double two_pi = 6.283185307179586476925286766559;
  double* tw = (double*)malloc(2 * (n ? n : 1) * sizeof(double));
  for (size_t k = 0; k < n; ++k) {
    tw[2 * k] = cos(two_pi * (double)k / (double)n);
    tw[2 * k + 1] = (double)sign * sin(two_pi * (double)k / (double)n);
  }
  return tw;
}

/* 2-D transform of an interleaved [n0][n1] array (n1 fastest). */
static void fft2d(double* d, size_t n0, size_t n1, int sign) {
  size_t m = n0 > n1 ? n0 : n1;
  double* re = (double*)malloc(m * sizeof(double));
  double* im = (double*)malloc(m * sizeof(double));
  double* tw1 = twiddles(n1, sign);
  double* tw0 = twiddles(n0, sign);
  for (size_t i = 0; i < n0; ++i) {
    double* row = d + 2 * i * n1;
    for (size_t j = 0; j < n1; ++j) { re[j] = row[2 * j]; im[j] = row[2 * j + 1]; }
    fft1d(re, im, n1, sign, tw1);
    for (size_t j = 0; j < n1; ++j) { row[2 * j] = re[j]; row[2 * j + 1] = im[j]; }
  }
  for (size_t j = 0; j < n1; ++j) {
    for (size_t i = 0; i < n0; ++i) { re[i] = d[2 * (i * n1 + j)]; im[i] = d[2 * (i * n1 + j) + 1]; }
    fft1d(re, im, n0, sign, tw0);
    for (size_t i = 0; i < n0; ++i) { d[2 * (i * n1 + j)] = re[i]; d[2 * (i * n1 + j) + 1] = im[i]; }
  }
  free(re); free(im); free(tw1); free(tw0);
}

/* ------------------------------------------------------- set-up ---------- */
void or_constants(double VV, double* lambda, double* gamma) {
  /* tem.cpp:424-438, same operation order */
  const double m_e0 = 9.109e-31, cc = 299792458, ee = 1.60217662e-19;
  const double hh = 6.62607004e-34;
  *lambda = hh * cc * pow(10, 10) / sqrt(ee * VV * (2.0 * m_e0 * cc * cc + ee * VV));
  *gamma = (hh * pow(10, 10) / *lambda) * (hh * pow(10, 10) / *lambda) *
           (m_e0 * cc * cc + ee * VV) / ((2 * m_e0 * cc * cc + ee * VV) * ee * VV * m_e0);
}

typedef struct {
  size_t nx, ny;
  double *xx, *yy, *kx, *ky;
  double bw_pap, bw_t, lambda, gamma, s; /* s = sqrtNxNy (adfstem.cpp:196-198) */
  double nxny;
} grid_t;

static void grid_init(grid_t* g, const or_job* job) {
  g->nx = (size_t)job->nx; g->ny = (size_t)job->ny;
  g->xx = (double*)malloc(g->nx * sizeof(double));
  g->yy = (double*)malloc(g->ny * sizeof(double));
  g->kx = (double*)malloc(g->nx * sizeof(double));
  g->ky = (double*)malloc(g->ny * sizeof(double));
  const double xpd = job->xperiod_duped, ypd = job->yperiod_duped;
  const long Nx = job->nx, Ny = job->ny;
  /* tem.cpp:756-788 with func.cpp:92-106 and 147-167 */
  const double dx = xpd / Nx, dy = ypd / Ny, dkx = 1.0 / xpd, dky = 1.0 / ypd;
  const double kxp = Nx / xpd, kyp = Ny / ypd;
  for (int i = 0; i < Nx; ++i) g->xx[i] = job->xmin + (i * dx);
  for (int i = 0; i < Ny; ++i) g->yy[i] = job->ymin + (i * dy);
  for (int i = 0; i < Nx / 2; ++i) g->kx[i] = i * dkx;
  for (int i = Nx / 2; i < Nx; ++i) g->kx[i] = i * dkx - kxp;
  for (int i = 0; i < Ny / 2; ++i) g->ky[i] = i * dky;
  for (int i = Ny / 2; i < Ny; ++i) g->ky[i] = i * dky - kyp;
  /* tem.cpp:683-695 */
  if (Nx / (2 * xpd) < Ny / (2 * ypd)) g->bw_pap = Nx / (2 * xpd);
  else g->bw_pap = Ny / (2 * ypd);
  g->bw_t = (2.0 / 3.0) * g->bw_pap;
  or_constants(job->voltage, &g->lambda, &g->gamma);
  g->nxny = (double)(Nx * Ny);
  g->s = (Nx == Ny) ? (double)Nx : sqrt(g->nxny); /* tem.cpp:407-408 */
}

static void grid_free(grid_t* g) { free(g->xx); free(g->yy); free(g->kx); free(g->ky); }

int64_t or_snap(const double* grid, int64_t n, double q, double half,
                int64_t fallback) {
  for (int64_t i = 0; i < n; ++i)
    if (grid[i] - q >= half) return i - 1; /* i == 0 -> -1: size_t wrap */
  return fallback;
}

/* scatterer.hpp:192 comparator; ties keep index order (std::sort is not
 * stable, but members of a z tie always share a slice and a mean). */
static const double* g_sort_q;
static int cmp_z(const void* a, const void* b) {
  int64_t ia = *(const int64_t*)a, ib = *(const int64_t*)b;
  double za = g_sort_q[3 * ia + 2], zb = g_sort_q[3 * ib + 2];
  if (za < zb) return -1;
  if (zb < za) return 1;
  return (ia > ib) - (ia < ib);
}

int64_t or_slice_atoms(int64_t n, const double* q, double zmin, double zperiod,
                       double min_thickness, int64_t* order, int64_t* start,
                       double* lower, double* thick) {
  /* slice.cpp:469-980 */
  if (n == 0) { /* slice.cpp:632-639: one empty slice spanning zperiod */
    start[0] = 0; start[1] = 0; lower[0] = zmin; thick[0] = zperiod;
    return 1;
  }
  for (int64_t i = 0; i < n; ++i) order[i] = i;
  g_sort_q = q;
  qsort(order, (size_t)n, sizeof(int64_t), cmp_z);
  int64_t ns = 0;
  start[0] = 0;
  lower[0] = 0.0;
  double first = q[3 * order[0] + 2];
  for (int64_t k = 0; k < n; ++k) {
    double z = q[3 * order[k] + 2];
    if (z - first <= min_thickness) {
      lower[ns] += z;
    } else {
      ++ns;
      start[ns] = k;
      lower[ns] = z;
      first = z;
    }
  }
  ++ns;
  start[ns] = n;
  for (int64_t s = 0; s < ns; ++s)
    lower[s] = lower[s] / (double)(size_t)(start[s + 1] - start[s]);
  for (int64_t s = 0; s < ns; ++s) {
    if (s + 1 == ns)
      thick[s] = q[3 * order[start[s + 1] - 1] + 2] + min_thickness - lower[s];
    else
      thick[s] = lower[s + 1] - lower[s];
  }
  return ns;
}

/* Per-species real-space projected-potential LUT: scatterer_pap.hpp:45-230
 * with sigmaVz_single_scatterer / f_ej_single_scatterer
 * (projected_atomic_potential.cpp:169-220).  2*nx*ny interleaved. */
static void build_lut(const grid_t* g, const or_job* job, uint32_t Z, double ab_inv,
                      double* lut) {
  const double* p = kirkland[Z - 1];
  const double *a = p, *b = p + 3, *c = p + 6, *d = p + 9;
  const double cutoffsq = g->bw_pap * g->bw_pap;
  for (size_t i = 0; i < g->nx; ++i)
    for (size_t j = 0; j < g->ny; ++j) {
      double* v = lut + 2 * (j + i * g->ny);
      v[0] = 0.0; v[1] = 0.0;
      if (pow(g->kx[i], 2) + pow(g->ky[j], 2) < cutoffsq) {
        double kx = g->kx[i], ky = g->ky[j];
        double ksq = (kx * kx) + (ky * ky);
        double f = a[0] / (ksq + b[0]) + a[1] / (ksq + b[1]) + a[2] / (ksq + b[2]) +
                   c[0] * exp(-d[0] * ksq) + c[1] * exp(-d[1] * ksq) + c[2] * exp(-d[2] * ksq);
        double trig = 2 * OR_PI * (kx * job->xmin + ky * job->ymin);
        v[0] += g->lambda * g->gamma * ab_inv * f * cos(trig);
        v[1] += g->lambda * g->gamma * ab_inv * f * sin(trig);
      }
    }
  fft2d(lut, g->nx, g->ny, +1);
  const double s = sqrt((double)(g->nx * g->ny));
  for (size_t k = 0; k < 2 * g->nx * g->ny; ++k) lut[k] = lut[k] / s;
}

/* bw_limit.cpp:30-47 */
static void bw_limit(const grid_t* g, double* d, double cutoff) {
  const double cutoffsq = pow(cutoff, 2);
  for (size_t i = 0; i < g->nx; ++i)
    for (size_t j = 0; j < g->ny; ++j)
      if (pow(g->kx[i], 2) + pow(g->ky[j], 2) >= cutoffsq) {
        d[2 * (j + i * g->ny)] = 0.0;
        d[2 * (j + i * g->ny) + 1] = 0.0;
      }
}

typedef struct {
  int64_t n;           /* slices */
  int64_t *order, *start;
  double *lower, *thick;
} slicing_t;

static int slice_specimen(const or_job* job, const or_atoms* at, slicing_t* sl) {
  int64_t n = at->n_atoms;
  sl->order = (int64_t*)malloc((size_t)(n + 1) * sizeof(int64_t));
  sl->start = (int64_t*)malloc((size_t)(n + 2) * sizeof(int64_t));
  sl->lower = (double*)calloc((size_t)(n + 1), sizeof(double));
  sl->thick = (double*)calloc((size_t)(n + 1), sizeof(double));
  sl->n = or_slice_atoms(n, at->q, 0.0, 0.0, job->min_slice, sl->order, sl->start,
                         sl->lower, sl->thick);
  return 0;
}

static void slicing_free(slicing_t* sl) {
  free(sl->order); free(sl->start); free(sl->lower); free(sl->thick);
}

/* One slice's transmission function: slice.cpp:1451-1757. */
static int build_transmission(const grid_t* g, const or_atoms* at, const slicing_t* sl,
                              int64_t s, double* const* luts, const uint32_t* lut_z,
                              int n_species, double* t) {
  const size_t nx = g->nx, ny = g->ny;
  memset(t, 0, 2 * nx * ny * sizeof(double));
  const double half_dx = 0.5 * (g->xx[1] - g->xx[0]);
  const double half_dy = 0.5 * (g->yy[1] - g->yy[0]);
  for (int64_t k = sl->start[s]; k < sl->start[s + 1]; ++k) {
    int64_t a = sl->order[k];
    const double* lut = NULL;
    for (int sp = 0; sp < n_species; ++sp)
      if (lut_z[sp] == at->z[a]) lut = luts[sp];
    if (!lut) return 1;
    int64_t sx = or_snap(g->xx, (int64_t)nx, at->q[3 * a], half_dx, 0);
    int64_t sy = or_snap(g->yy, (int64_t)ny, at->q[3 * a + 1], half_dy, 0);
    if (sx < 0 || sy < 0) return 2; /* reference would index out of bounds */
    for (size_t i = 0; i < nx; ++i) {
      size_t ix = (i < (size_t)sx) ? i + nx - (size_t)sx : i - (size_t)sx;
      for (size_t j = 0; j < ny; ++j) {
        size_t iy = (j < (size_t)sy) ? j + ny - (size_t)sy : j - (size_t)sy;
        t[2 * (j + i * ny)] += lut[2 * (iy + ix * ny)];
        t[2 * (j + i * ny) + 1] += lut[2 * (iy + ix * ny) + 1];
      }
    }
  }
  for (size_t p = 0; p < nx * ny; ++p) { /* slice.cpp:1700-1725 */
    double e = exp(-(t[2 * p + 1]));
    double re = t[2 * p];
    t[2 * p] = e * cos(re);
    t[2 * p + 1] = e * sin(re);
  }
  fft2d(t, nx, ny, -1); /* slice.cpp:1730-1748 */
  bw_limit(g, t, g->bw_t);
  fft2d(t, nx, ny, +1);
  for (size_t p = 0; p < 2 * nx * ny; ++p) t[p] = t[p] / g->nxny;
  return 0;
}

/* slice.cpp:1293-1363 */
static void build_propagator(const grid_t* g, double thickness, double* pxr, double* pxi,
                             double* pyr, double* pyi) {
  for (size_t i = 0; i < g->nx; ++i) {
    if (g->kx[i] < g->bw_t && g->kx[i] > -1.0 * g->bw_t) {
      double arg = OR_PI * g->lambda * thickness * pow(g->kx[i], 2);
      pxr[i] = cos(arg); pxi[i] = -sin(arg);
    } else { pxr[i] = 0.0; pxi[i] = 0.0; }
  }
  for (size_t j = 0; j < g->ny; ++j) {
    if (g->ky[j] < g->bw_t && g->ky[j] > -1.0 * g->bw_t) {
      double arg = OR_PI * g->lambda * thickness * pow(g->ky[j], 2);
      pyr[j] = cos(arg); pyi[j] = -sin(arg);
    } else { pyr[j] = 0.0; pyi[j] = 0.0; }
  }
}

/* adfstem.cpp:586-817 with probe_wavefunction.cpp:37-137 / 139-239,
 * lenses.cpp:249-290 and probe_wavefunction.cpp:287-315. */
static void build_probe(const grid_t* g, const or_job* job, double* pr) {
  const double lambda = g->lambda, lsq = lambda * lambda;
  const double amax_sq = job->alpha_max * job->alpha_max;
  const double x0 = g->xx[0], y0 = g->yy[0];
  for (size_t i = 0; i < g->nx; ++i)
    for (size_t j = 0; j < g->ny; ++j) {
      double* v = pr + 2 * (j + i * g->ny);
      double kx = g->kx[i], ky = g->ky[j];
      double ksqr = kx * kx + ky * ky;
      if (lsq * ksqr < amax_sq) {
        double chi;
        if (job->corrected) {
          double kl = ksqr * lsq;
          chi = OR_PI * lambda * ksqr *
                (-job->defocus + 0.5 * job->cs3 * kl + (1.0 / 3.0) * job->cs5 * pow(kl, 2));
        } else {
          chi = OR_PI * lambda * ksqr * (0.5 * job->cs3 * lsq * ksqr - job->defocus);
        }
        double trig = chi + 2 * OR_PI * ((kx * x0) + (ky * y0));
        v[0] = cos(trig);
        v[1] = -1.0 * sin(trig);
      } else { v[0] = 0.0; v[1] = 0.0; }
    }
  fft2d(pr, g->nx, g->ny, +1);
  for (size_t p = 0; p < 2 * g->nx * g->ny; ++p) pr[p] = pr[p] / g->s;
  double ap = 0.0;
  for (size_t p = 0; p < g->nx * g->ny; ++p)
    ap += pr[2 * p] * pr[2 * p] + pr[2 * p + 1] * pr[2 * p + 1];
  ap = 1.0 / sqrt(ap);
  for (size_t p = 0; p < 2 * g->nx * g->ny; ++p) pr[p] = ap * pr[p];
}

int or_probe(const or_job* job, double* probe_out) {
  grid_t g;
  grid_init(&g, job);
  build_probe(&g, job, probe_out);
  grid_free(&g);
  return 0;
}

/* Species list in ascending Z (tem.cpp:944-972) and their LUTs. */
static int make_luts(const grid_t* g, const or_job* job, const or_atoms* at,
                     uint32_t* zs, double** luts) {
  int ns = 0;
  for (int64_t a = 0; a < at->n_atoms; ++a) {
    int seen = 0;
    for (int k = 0; k < ns; ++k) seen |= (zs[k] == at->z[a]);
    if (!seen) {
      if (at->z[a] < 1 || at->z[a] > 103) return -1;
      zs[ns++] = at->z[a];
    }
  }
  const double ab_inv = 1 / (job->xperiod_duped * job->yperiod_duped);
  for (int k = 0; k < ns; ++k) {
    luts[k] = (double*)malloc(2 * g->nx * g->ny * sizeof(double));
    build_lut(g, job, zs[k], ab_inv, luts[k]);
  }
  return ns;
}

int or_transmission(const or_job* job, const or_atoms* at, int32_t slice, double* t_out) {
  grid_t g;
  grid_init(&g, job);
  uint32_t zs[128];
  double* luts[128];
  int ns = make_luts(&g, job, at, zs, luts);
  if (ns < 0) { grid_free(&g); return 1; }
  slicing_t sl;
  slice_specimen(job, at, &sl);
  int rc = (slice < 0 || slice >= sl.n) ? 3
           : build_transmission(&g, at, &sl, slice, luts, zs, ns, t_out);
  for (int k = 0; k < ns; ++k) free(luts[k]);
  slicing_free(&sl);
  grid_free(&g);
  return rc;
}

/* Ring bin of every pixel (adfstem.cpp:947-1062, variance.cpp:64-300):
 * bin(k^2) = smallest ii with k^2 <= b_{ii+1}^2, or -1 beyond the last. */
static void ring_bins(const grid_t* g, double dr, int32_t* n_k, double** bounds,
                      int32_t** bin, int32_t** counts) {
  double dk = dr * sqrt((g->kx[1] - g->kx[0]) * (g->kx[1] - g->kx[0]) +
                        (g->ky[1] - g->ky[0]) * (g->ky[1] - g->ky[0]));
  unsigned int nk = (unsigned int)(g->bw_t / dk);
  *n_k = (int32_t)nk;
  *bounds = (double*)malloc((nk + 1) * sizeof(double));
  for (unsigned int ii = 0; ii < nk + 1; ++ii) (*bounds)[ii] = ii * dk;
  *bin = (int32_t*)malloc(g->nx * g->ny * sizeof(int32_t));
  *counts = (int32_t*)calloc(nk ? nk : 1, sizeof(int32_t));
  for (size_t i = 0; i < g->nx; ++i)
    for (size_t j = 0; j < g->ny; ++j) {
      double ksq = g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j];
      int32_t b = -1;
      for (unsigned int ii = 0; ii < nk; ++ii) {
        double ub = (*bounds)[ii + 1];
        if (ksq <= ub * ub) { b = (int32_t)ii; break; }
      }
      (*bin)[j + i * g->ny] = b;
      if (b >= 0) (*counts)[b] += 1;
    }
}

/* Ring sums over a real per-pixel array, summed in ascending k^2 order
 * (variance.cpp:303-510 walks the k^2-sorted pixel list). */
typedef struct { double ksq; int64_t p; } kpix_t;
static int cmp_kpix(const void* a, const void* b) {
  const kpix_t *x = (const kpix_t*)a, *y = (const kpix_t*)b;
  if (x->ksq < y->ksq) return -1;
  if (y->ksq < x->ksq) return 1;
  return (x->p > y->p) - (x->p < y->p);
}

static void ring_sum(const kpix_t* sorted, size_t npix, const int32_t* bin,
                     const double* val, int32_t nk, double* out) {
  for (int32_t k = 0; k < nk; ++k) out[k] = 0.0;
  for (size_t q = 0; q < npix; ++q) {
    int32_t b = bin[sorted[q].p];
    if (b >= 0) out[b] += val[sorted[q].p];
  }
}

int or_run(const or_job* job, const or_atoms* at, or_result* out) {
  grid_t g;
  grid_init(&g, job);
  const size_t nx = g.nx, ny = g.ny, np = nx * ny;
  uint32_t zs[128];
  double* luts[128];
  int ns = make_luts(&g, job, at, zs, luts);
  if (ns < 0) { grid_free(&g); return 1; }
  slicing_t sl;
  slice_specimen(job, at, &sl);
  out->n_slices = (int32_t)sl.n;

  double** trans = (double**)malloc((size_t)sl.n * sizeof(double*));
  double* prop = (double*)malloc((size_t)sl.n * 2 * (nx + ny) * sizeof(double));
  for (int64_t s = 0; s < sl.n; ++s) {
    trans[s] = (double*)malloc(2 * np * sizeof(double));
    int rc = build_transmission(&g, at, &sl, s, luts, zs, ns, trans[s]);
    if (rc) { grid_free(&g); return 10 + rc; }
    double* p = prop + s * 2 * (nx + ny);
    build_propagator(&g, sl.thick[s], p, p + nx, p + 2 * nx, p + 2 * nx + ny);
  }
  for (int k = 0; k < ns; ++k) free(luts[k]);

  double* probe = (double*)malloc(2 * np * sizeof(double));
  build_probe(&g, job, probe);

  const int fem = (job->flags & ~OR_ADF) != 0;
  int32_t nk = 0, *bin = NULL, *cnt = NULL;
  double* bounds = NULL;
  kpix_t* sorted = NULL;
  if (fem) {
    ring_bins(&g, job->dr, &nk, &bounds, &bin, &cnt);
    sorted = (kpix_t*)malloc(np * sizeof(kpix_t));
    for (size_t i = 0; i < nx; ++i)
      for (size_t j = 0; j < ny; ++j) {
        sorted[j + i * ny].ksq = g.kx[i] * g.kx[i] + g.ky[j] * g.ky[j];
        sorted[j + i * ny].p = (int64_t)(j + i * ny);
      }
    qsort(sorted, np, sizeof(kpix_t), cmp_kpix);
    out->n_k = nk;
    if (nk > out->cap_k) return 20;
    for (int32_t k = 0; k < nk; ++k) {
      if (out->k_lower) out->k_lower[k] = bounds[k];
      if (out->bin_counts) out->bin_counts[k] = cnt[k];
    }
  }
  /* bins whose outer edge lies inside the aperture are zeroed
   * (adfstem.cpp:2518-2533 and the equivalent blocks after it) */
  int* inside = (int*)calloc((size_t)(nk > 0 ? nk : 1), sizeof(int));
  for (int32_t k = 0; k < nk; ++k)
    inside[k] = (g.lambda * bounds[k + 1] <= job->alpha_max);

  double *sumA = (double*)calloc(nk + 1, sizeof(double));
  double *sumA2 = (double*)calloc(nk + 1, sizeof(double));
  double *var_sum = (double*)calloc(nk + 1, sizeof(double));
  double *ring = (double*)calloc(nk + 1, sizeof(double));
  double *ring2 = (double*)calloc(nk + 1, sizeof(double));
  const int pix = (job->flags & (OR_D3 | OR_D4 | OR_GT17 | OR_RVA)) != 0;
  double* mag_sum = pix ? (double*)calloc(np, sizeof(double)) : NULL;
  double* mag_sqr_sum = pix ? (double*)calloc(np, sizeof(double)) : NULL;
  double* amp = (double*)malloc(np * sizeof(double));
  double* psi = (double*)malloc(2 * np * sizeof(double));
  const double k1 = job->det_inner / g.lambda, k2 = job->det_outer / g.lambda;
  const double half_dx = 0.5 * (g.xx[1] - g.xx[0]);
  const double half_dy = 0.5 * (g.yy[1] - g.yy[0]);
  const double bwt_sq = g.bw_t * g.bw_t;
  int64_t sx = 0, sy = 0; /* adfstem.cpp:1525-1528: persist across probes */
  const size_t n_raster = (size_t)job->n_rx * (size_t)job->n_ry;

  for (int32_t px = 0; px < job->n_rx; ++px) {
    for (int32_t py = 0; py < job->n_ry; ++py) {
      /* adfstem.cpp:1590-1606 */
      sx = or_snap(g.xx, (int64_t)nx, job->x_p[px], half_dx, sx);
      sy = or_snap(g.yy, (int64_t)ny, job->y_p[py], half_dy, sy);
      if (sx < 0 || sy < 0) return 30;
      /* adfstem.cpp:1632-1671 */
      for (size_t i = 0; i < nx; ++i) {
        size_t ix = (i < (size_t)sx) ? i + nx - (size_t)sx : i - (size_t)sx;
        for (size_t j = 0; j < ny; ++j) {
          size_t iy = (j < (size_t)sy) ? j + ny - (size_t)sy : j - (size_t)sy;
          psi[2 * (j + i * ny)] = probe[2 * (iy + ix * ny)];
          psi[2 * (j + i * ny) + 1] = probe[2 * (iy + ix * ny) + 1];
        }
      }
      fft2d(psi, nx, ny, -1); /* adfstem.cpp:1831-1837 */
      for (size_t p = 0; p < 2 * np; ++p) psi[p] = psi[p] / g.s;
      for (int64_t s = 0; s < sl.n; ++s) { /* adfstem.cpp:1866-2132 */
        fft2d(psi, nx, ny, +1);
        const double* t = trans[s];
        for (size_t p = 0; p < np; ++p) { /* quirk Q1, adfstem.cpp:1922-1952 */
          psi[2 * p] = (t[2 * p] * psi[2 * p] - t[2 * p + 1] * psi[2 * p + 1]) / g.s;
          psi[2 * p + 1] = (t[2 * p] * psi[2 * p + 1] + t[2 * p + 1] * psi[2 * p]) / g.s;
        }
        fft2d(psi, nx, ny, -1);
        for (size_t p = 0; p < 2 * np; ++p) psi[p] = psi[p] / g.s;
        bw_limit(&g, psi, g.bw_t);
        const double* pp = prop + s * 2 * (nx + ny); /* slice.cpp:1366-1421 */
        const double *pxr = pp, *pxi = pp + nx, *pyr = pp + 2 * nx, *pyi = pp + 2 * nx + ny;
        for (size_t i = 0; i < nx; ++i)
          for (size_t j = 0; j < ny; ++j) {
            double* v = psi + 2 * (j + i * ny);
            double ksq = pow(g.kx[i], 2) + pow(g.ky[j], 2);
            if (ksq < bwt_sq) {
              double pr = pxr[i] * pyr[j] - pxi[i] * pyi[j];
              double pi = pxr[i] * pyi[j] + pxi[i] * pyr[j];
              double vr = v[0], vi = v[1];
              v[0] = (pr * vr - pi * vi);
              v[1] = (pr * vi + pi * vr);
            } else { v[0] = 0.0; v[1] = 0.0; }
          }
      }
      if ((job->flags & OR_ADF) && out->adf_image) { /* func.cpp:2593-2640 */
        double det = 0.0;
        for (size_t i = 0; i < nx; ++i)
          for (size_t j = 0; j < ny; ++j) {
            double ksq = g.kx[i] * g.kx[i] + g.ky[j] * g.ky[j];
            if (ksq > k1 && ksq <= k2)
              det += psi[2 * (j + i * ny)] * psi[2 * (j + i * ny)] +
                     psi[2 * (j + i * ny) + 1] * psi[2 * (j + i * ny) + 1];
          }
        out->adf_image[py + (size_t)px * job->n_ry] = det;
      }
      if (fem) {
        for (size_t p = 0; p < np; ++p)
          amp[p] = sqrt((psi[2 * p] * psi[2 * p]) + (psi[2 * p + 1] * psi[2 * p + 1]));
        ring_sum(sorted, np, bin, amp, nk, ring); /* variance.cpp:64-300 */
        for (int32_t k = 0; k < nk; ++k) if (inside[k]) ring[k] = 0.0;
        if (job->flags & OR_D1) /* adfstem.cpp:2585-2601 */
          for (int32_t k = 0; k < nk; ++k) {
            sumA2[k] += (ring[k] * ring[k]) / (cnt[k] * cnt[k]);
            sumA[k] += ring[k] / cnt[k];
          }
        if (job->flags & OR_D2) { /* adfstem.cpp:2688-2750 */
          for (size_t p = 0; p < np; ++p)
            amp[p] = (psi[2 * p] * psi[2 * p]) + (psi[2 * p + 1] * psi[2 * p + 1]);
          ring_sum(sorted, np, bin, amp, nk, ring2);
          for (int32_t k = 0; k < nk; ++k) if (inside[k]) ring2[k] = 0.0;
          for (int32_t k = 0; k < nk; ++k)
            var_sum[k] += ((ring2[k] / cnt[k]) /
                           ((ring[k] * ring[k]) / (cnt[k] * cnt[k]))) - 1.0;
        }
        if (pix) /* adfstem.cpp:2753-2781 */
          for (size_t p = 0; p < np; ++p) {
            mag_sum[p] += sqrt(psi[2 * p] * psi[2 * p] + psi[2 * p + 1] * psi[2 * p + 1]);
            mag_sqr_sum[p] += psi[2 * p] * psi[2 * p] + psi[2 * p + 1] * psi[2 * p + 1];
          }
      }
    }
  }
  if (out->last_psi) memcpy(out->last_psi, psi, 2 * np * sizeof(double));

  /* post-raster FEM, adfstem.cpp:2822-3612 */
  if (fem && (job->flags & OR_D1) && out->v_omega)
    for (int32_t k = 0; k < nk; ++k) {
      if (sumA[k] == 0.0) out->v_omega[k] = 0.0;
      else out->v_omega[k] = (n_raster * sumA2[k] / (sumA[k] * sumA[k])) - 1.0;
    }
  if (fem && (job->flags & OR_D2) && out->vbar_r)
    for (int32_t k = 0; k < nk; ++k) out->vbar_r[k] = var_sum[k] / n_raster;
  if (fem && pix) {
    double* mean_sq = (double*)malloc(np * sizeof(double));
    for (size_t p = 0; p < np; ++p) {
      mag_sum[p] = mag_sum[p] / n_raster;
      mean_sq[p] = mag_sum[p] * mag_sum[p];
      mag_sqr_sum[p] = mag_sqr_sum[p] / n_raster;
    }
    double *r1 = (double*)calloc(nk + 1, sizeof(double));
    double *r2 = (double*)calloc(nk + 1, sizeof(double));
    double *r3 = (double*)calloc(nk + 1, sizeof(double));
    ring_sum(sorted, np, bin, mag_sqr_sum, nk, r1);
    ring_sum(sorted, np, bin, mean_sq, nk, r2);
    ring_sum(sorted, np, bin, mag_sum, nk, r3);
    for (int32_t k = 0; k < nk; ++k)
      if (inside[k]) { r1[k] = 0.0; r2[k] = 0.0; r3[k] = 0.0; }
    for (int32_t k = 0; k < nk; ++k) {
      double c = (double)cnt[k];
      double cc = (double)(cnt[k] * cnt[k]);
      if ((job->flags & OR_GT17) && out->v_gt17) out->v_gt17[k] = (r1[k] / c) / (r2[k] / c);
      if ((job->flags & OR_D3) && out->v_re) out->v_re[k] = ((r1[k] / c) / (r3[k] * r3[k] / cc)) - 1.0;
      if ((job->flags & OR_RVA) && out->v_rbar) out->v_rbar[k] = ((r2[k] / c) / (r3[k] * r3[k] / cc)) - 1.0;
    }
    if ((job->flags & OR_D4) && out->omega_vimage) {
      const double lsq = g.lambda * g.lambda, amax_sq = job->alpha_max * job->alpha_max;
      for (size_t i = 0; i < nx; ++i)
        for (size_t j = 0; j < ny; ++j) {
          size_t p = j + ny * i;
          mean_sq[p] = (mag_sqr_sum[p] / (mag_sum[p] * mag_sum[p])) - 1.0;
          double ksqr = pow(g.kx[i], 2) + pow(g.ky[j], 2);
          if (lsq * ksqr <= amax_sq) mean_sq[p] = 0.0;
        }
      ring_sum(sorted, np, bin, mean_sq, nk, r1);
      for (int32_t k = 0; k < nk; ++k) {
        if (inside[k]) r1[k] = 0.0;
        out->omega_vimage[k] = r1[k] / cnt[k];
      }
    }
    free(r1); free(r2); free(r3); free(mean_sq);
  }

  for (int64_t s = 0; s < sl.n; ++s) free(trans[s]);
  free(trans); free(prop); free(probe); free(psi); free(amp);
  free(sumA); free(sumA2); free(var_sum); free(ring); free(ring2); free(inside);
  free(mag_sum); free(mag_sqr_sum);
  free(bin); free(cnt); free(bounds); free(sorted);
  slicing_free(&sl);
  grid_free(&g);
  return 0;
}

int32_t or_ring_bins(const or_job* job, int32_t* bins_out, int32_t* counts_out,
                     double* bounds_out, int32_t cap) {
  grid_t g;
  grid_init(&g, job);
  int32_t nk = 0, *bin = NULL, *cnt = NULL;
  double* bounds = NULL;
  ring_bins(&g, job->dr, &nk, &bounds, &bin, &cnt);
  if (bins_out) memcpy(bins_out, bin, g.nx * g.ny * sizeof(int32_t));
  for (int32_t k = 0; k < nk && k < cap; ++k) {
    if (counts_out) counts_out[k] = cnt[k];
    if (bounds_out) bounds_out[k] = bounds[k];
  }
  free(bin); free(cnt); free(bounds);
  grid_free(&g);
  return nk;
}
