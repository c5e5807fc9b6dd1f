// Implementations behind oracle/shims/{mpi.h,fftw3.h,fftw3-mpi.h,tiffio.h}.
//
// Test infrastructure only.  These let the reference's own sources compile and
// run unchanged as a single-rank CPU program (the oracle binary under
// oracle/_ref/).  Nothing in the product links this file.
//
//  * MPI: one rank; broadcasts are no-ops, collectives copy send -> receive.
//  * FFTW: 2-D complex DFT in FP64 following FFTW's documented definition
//    (forward e^{-2 pi i nk/N}, backward e^{+2 pi i nk/N}, unnormalised),
//    iterative radix-2 for power-of-two lengths and a direct O(N^2) DFT
//    otherwise.  Twiddles come from libm cos/sin in double precision.
//  * libtiff: uncompressed little-endian baseline TIFF writer.
#include <algorithm>
#include <mpi.h>
#include <fftw3-mpi.h>
#include <tiffio.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <sys/time.h>
#include <vector>

// ------------------------------------------------------------------ MPI ----
static size_t mpi_type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR:
    case MPI_UNSIGNED_CHAR: return 1;
    case MPI_UNSIGNED_SHORT: return 2;
    case MPI_INT:
    case MPI_UNSIGNED: return 4;
    case MPI_UNSIGNED_LONG:
    case MPI_UNSIGNED_LONG_LONG:
    case MPI_DOUBLE: return 8;
  }
  std::fprintf(stderr, "mpi shim: unknown datatype %d\n", t);
  std::abort();
}

static void copy_elems(const void* sb, void* rb, int count, MPI_Datatype t) {
  if (sb == MPI_IN_PLACE || sb == rb || count <= 0) return;
  std::memmove(rb, sb, (size_t)count * mpi_type_size(t));
}

extern "C" {
int MPI_Init(int*, char***) { return MPI_SUCCESS; }
int MPI_Init_thread(int*, char***, int required, int* provided) {
  if (provided) *provided = required;
  return MPI_SUCCESS;
}
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
int MPI_Allgather(const void* sb, int sc, MPI_Datatype st, void* rb, int,
                  MPI_Datatype, MPI_Comm) {
  copy_elems(sb, rb, sc, st);
  return MPI_SUCCESS;
}
int MPI_Allgatherv(const void* sb, int sc, MPI_Datatype st, void* rb,
                   const int*, const int* displs, MPI_Datatype rt, MPI_Comm) {
  copy_elems(sb, (char*)rb + (size_t)displs[0] * mpi_type_size(rt), sc, st);
  return MPI_SUCCESS;
}
int MPI_Gather(const void* sb, int sc, MPI_Datatype st, void* rb, int,
               MPI_Datatype, int, MPI_Comm) {
  copy_elems(sb, rb, sc, st);
  return MPI_SUCCESS;
}
int MPI_Gatherv(const void* sb, int sc, MPI_Datatype st, void* rb, const int*,
                const int* displs, MPI_Datatype rt, int, MPI_Comm) {
  copy_elems(sb, (char*)rb + (size_t)displs[0] * mpi_type_size(rt), sc, st);
  return MPI_SUCCESS;
}
int MPI_Scatter(const void* sb, int sc, MPI_Datatype st, void* rb, int,
                MPI_Datatype, int, MPI_Comm) {
  copy_elems(sb, rb, sc, st);
  return MPI_SUCCESS;
}
int MPI_Scatterv(const void* sb, const int* scounts, const int* displs,
                 MPI_Datatype st, void* rb, int, MPI_Datatype, int, MPI_Comm) {
  copy_elems((const char*)sb + (size_t)displs[0] * mpi_type_size(st), rb,
             scounts[0], st);
  return MPI_SUCCESS;
}
int MPI_Reduce(const void* sb, void* rb, int count, MPI_Datatype t, MPI_Op,
               int, MPI_Comm) {
  copy_elems(sb, rb, count, t);
  return MPI_SUCCESS;
}
int MPI_Allreduce(const void* sb, void* rb, int count, MPI_Datatype t, MPI_Op,
                  MPI_Comm) {
  copy_elems(sb, rb, count, t);
  return MPI_SUCCESS;
}
double MPI_Wtime(void) {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return (double)tv.tv_sec + 1e-6 * (double)tv.tv_usec;
}
}  // extern "C"

// ----------------------------------------------------------------- FFTW ----
struct msf_shim_plan {
  ptrdiff_t n0, n1;
  fftw_complex* in;
  fftw_complex* out;
  int sign;
};

namespace {
struct Line1D {
  // Precomputed data for one transform length and sign.
  size_t n = 0;
  bool pow2 = false;
  std::vector<double> wr, wi;  // e^{sign 2 pi i k / n}, k < n
  std::vector<size_t> rev;     // bit reversal (pow2 only)
};

std::map<std::pair<size_t, int>, Line1D>& line_cache() {
  static std::map<std::pair<size_t, int>, Line1D> c;
  return c;
}

const Line1D& get_line(size_t n, int sign) {
  auto key = std::make_pair(n, sign);
  auto it = line_cache().find(key);
  if (it != line_cache().end()) return it->second;
  Line1D L;
  L.n = n;
  L.pow2 = (n & (n - 1)) == 0;
  L.wr.resize(n);
  L.wi.resize(n);
  const double two_pi = 6.283185307179586476925286766559;
  for (size_t k = 0; k < n; ++k) {
    double a = two_pi * (double)k / (double)n;
    L.wr[k] = std::cos(a);
    L.wi[k] = (sign < 0 ? -1.0 : 1.0) * std::sin(a);
  }
  if (L.pow2) {
    L.rev.resize(n);
    size_t bits = 0;
    while (((size_t)1 << bits) < n) ++bits;
    for (size_t k = 0; k < n; ++k) {
      size_t r = 0;
      for (size_t b = 0; b < bits; ++b) r |= ((k >> b) & 1) << (bits - 1 - b);
      L.rev[k] = r;
    }
  }
  return line_cache().emplace(key, std::move(L)).first->second;
}

// In-place 1-D transform of n complex values stored interleaved in re/im.
void transform_line(const Line1D& L, double* re, double* im,
                    std::vector<double>& scratch) {
  const size_t n = L.n;
  if (n <= 1) return;
  if (L.pow2) {
    for (size_t k = 0; k < n; ++k) {
      size_t r = L.rev[k];
      if (r > k) {
        std::swap(re[k], re[r]);
        std::swap(im[k], im[r]);
      }
    }
    for (size_t len = 2; len <= n; len <<= 1) {
      size_t half = len >> 1, step = n / len;
      for (size_t s = 0; s < n; s += len) {
        for (size_t k = 0; k < half; ++k) {
          double wr = L.wr[k * step], wi = L.wi[k * step];
          size_t a = s + k, b = a + half;
          double tr = re[b] * wr - im[b] * wi;
          double ti = re[b] * wi + im[b] * wr;
          re[b] = re[a] - tr;
          im[b] = im[a] - ti;
          re[a] += tr;
          im[a] += ti;
        }
      }
    }
    return;
  }
  scratch.assign(2 * n, 0.0);
  for (size_t k = 0; k < n; ++k) {
    double sr = 0.0, si = 0.0;
    for (size_t m = 0; m < n; ++m) {
      size_t idx = (k * m) % n;
      sr += re[m] * L.wr[idx] - im[m] * L.wi[idx];
      si += re[m] * L.wi[idx] + im[m] * L.wr[idx];
    }
    scratch[2 * k] = sr;
    scratch[2 * k + 1] = si;
  }
  for (size_t k = 0; k < n; ++k) {
    re[k] = scratch[2 * k];
    im[k] = scratch[2 * k + 1];
  }
}
}  // namespace

extern "C" {
fftw_complex* fftw_alloc_complex(size_t n) {
  void* p = nullptr;
  if (posix_memalign(&p, 64, (n ? n : 1) * sizeof(fftw_complex)) != 0)
    return nullptr;
  return (fftw_complex*)p;
}
void fftw_free(void* p) { std::free(p); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int) {}
int fftw_import_wisdom_from_filename(const char*) { return 0; }
int fftw_export_wisdom_to_filename(const char*) { return 1; }
void fftw_mpi_init(void) {}
void fftw_mpi_cleanup(void) {}
void fftw_mpi_broadcast_wisdom(MPI_Comm) {}
void fftw_mpi_gather_wisdom(MPI_Comm) {}

ptrdiff_t fftw_mpi_local_size_2d(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm,
                                 ptrdiff_t* local_n0,
                                 ptrdiff_t* local_0_start) {
  *local_n0 = n0;
  *local_0_start = 0;
  return n0 * n1;
}

fftw_plan fftw_mpi_plan_dft_2d(ptrdiff_t n0, ptrdiff_t n1, fftw_complex* in,
                               fftw_complex* out, MPI_Comm, int sign,
                               unsigned) {
  msf_shim_plan* p = new msf_shim_plan;
  p->n0 = n0;
  p->n1 = n1;
  p->in = in;
  p->out = out;
  p->sign = sign;
  return p;
}

void fftw_destroy_plan(fftw_plan p) { delete p; }

void fftw_execute(const fftw_plan p) {
  const size_t n0 = (size_t)p->n0, n1 = (size_t)p->n1;
  if (p->out != p->in)
    std::memcpy(p->out, p->in, n0 * n1 * sizeof(fftw_complex));
  double* d = &p->out[0][0];
  const Line1D& L1 = get_line(n1, p->sign);
  const Line1D& L0 = get_line(n0, p->sign);
  std::vector<double> re(std::max(n0, n1)), im(std::max(n0, n1)), scratch;
  for (size_t i = 0; i < n0; ++i) {  // transforms along the fast index
    double* row = d + 2 * i * n1;
    for (size_t j = 0; j < n1; ++j) {
      re[j] = row[2 * j];
      im[j] = row[2 * j + 1];
    }
    transform_line(L1, re.data(), im.data(), scratch);
    for (size_t j = 0; j < n1; ++j) {
      row[2 * j] = re[j];
      row[2 * j + 1] = im[j];
    }
  }
  // transforms along the slow index, a block of columns at a time: each
  // row segment of the block is one cache-line run, where gathering one
  // column at a time touches a new line per element.  Every line still
  // gets the same arithmetic as a transform of that column alone.
  const size_t CB = 16;
  std::vector<double> bre(CB * n0), bim(CB * n0);
  for (size_t j0 = 0; j0 < n1; j0 += CB) {
    const size_t nb = std::min(CB, n1 - j0);
    for (size_t i = 0; i < n0; ++i) {
      const double* src = d + 2 * (i * n1 + j0);
      for (size_t c = 0; c < nb; ++c) {
        bre[c * n0 + i] = src[2 * c];
        bim[c * n0 + i] = src[2 * c + 1];
      }
    }
    for (size_t c = 0; c < nb; ++c)
      transform_line(L0, bre.data() + c * n0, bim.data() + c * n0, scratch);
    for (size_t i = 0; i < n0; ++i) {
      double* dst = d + 2 * (i * n1 + j0);
      for (size_t c = 0; c < nb; ++c) {
        dst[2 * c] = bre[c * n0 + i];
        dst[2 * c + 1] = bim[c * n0 + i];
      }
    }
  }
}
}  // extern "C"

// ----------------------------------------------------------------- TIFF ----
struct msf_shim_tiff {
  std::string name;
  uint32 width = 0, length = 0, rows_per_strip = 0;
  uint16 bps = 8, spp = 1, photometric = 1, orientation = 1, planar = 1;
  uint16 resunit = 2, sampleformat = 0;
  bool has_sampleformat = false;
  double xres = 72.0, yres = 72.0;
  std::vector<unsigned char> data;
};

extern "C" {
TIFF* TIFFOpen(const char* name, const char* mode) {
  if (!mode || mode[0] != 'w') return nullptr;
  FILE* f = std::fopen(name, "wb");
  if (!f) return nullptr;
  std::fclose(f);
  TIFF* t = new msf_shim_tiff;
  t->name = name;
  return t;
}

int TIFFSetField(TIFF* t, uint32 tag, ...) {
  va_list ap;
  va_start(ap, tag);
  switch (tag) {
    case TIFFTAG_IMAGEWIDTH: t->width = va_arg(ap, uint32); break;
    case TIFFTAG_IMAGELENGTH: t->length = va_arg(ap, uint32); break;
    case TIFFTAG_BITSPERSAMPLE: t->bps = (uint16)va_arg(ap, int); break;
    case TIFFTAG_SAMPLESPERPIXEL: t->spp = (uint16)va_arg(ap, int); break;
    case TIFFTAG_PHOTOMETRIC: t->photometric = (uint16)va_arg(ap, int); break;
    case TIFFTAG_ORIENTATION: t->orientation = (uint16)va_arg(ap, int); break;
    case TIFFTAG_PLANARCONFIG: t->planar = (uint16)va_arg(ap, int); break;
    case TIFFTAG_RESOLUTIONUNIT: t->resunit = (uint16)va_arg(ap, int); break;
    case TIFFTAG_ROWSPERSTRIP: t->rows_per_strip = va_arg(ap, uint32); break;
    case TIFFTAG_XRESOLUTION: t->xres = va_arg(ap, double); break;
    case TIFFTAG_YRESOLUTION: t->yres = va_arg(ap, double); break;
    case TIFFTAG_SAMPLEFORMAT:
      t->sampleformat = (uint16)va_arg(ap, int);
      t->has_sampleformat = true;
      break;
    default: break;
  }
  va_end(ap);
  return 1;
}

uint32 TIFFDefaultStripSize(TIFF* t, uint32 request) {
  if ((int32_t)request >= 1) return request;
  tsize_t line = TIFFScanlineSize(t);
  uint32 rows = line > 0 ? (uint32)(8192 / line) : 1;
  return rows ? rows : 1;
}

tsize_t TIFFScanlineSize(TIFF* t) {
  return (tsize_t)t->width * t->spp * t->bps / 8;
}

int TIFFWriteScanline(TIFF* t, void* buf, uint32 row, uint16) {
  size_t line = (size_t)TIFFScanlineSize(t);
  if (t->data.size() < (size_t)(row + 1) * line)
    t->data.resize((size_t)(row + 1) * line);
  std::memcpy(t->data.data() + (size_t)row * line, buf, line);
  return 1;
}

static void put16(std::vector<unsigned char>& b, uint16 v) {
  b.push_back(v & 0xff);
  b.push_back(v >> 8);
}
static void put32(std::vector<unsigned char>& b, uint32 v) {
  for (int k = 0; k < 4; ++k) b.push_back((v >> (8 * k)) & 0xff);
}

void TIFFClose(TIFF* t) {
  if (!t) return;
  const size_t line = (size_t)TIFFScanlineSize(t);
  t->data.resize(line * t->length);
  uint32 rps = t->rows_per_strip ? t->rows_per_strip : t->length;
  if (rps == 0) rps = 1;
  uint32 nstrips = (t->length + rps - 1) / rps;
  std::vector<unsigned char> out;
  out.push_back('I');
  out.push_back('I');
  put16(out, 42);
  put32(out, 0);  // IFD offset, patched below
  std::vector<uint32> offs, counts;
  for (uint32 s = 0; s < nstrips; ++s) {
    uint32 r0 = s * rps, r1 = std::min(t->length, r0 + rps);
    offs.push_back((uint32)out.size());
    counts.push_back((uint32)((r1 - r0) * line));
    out.insert(out.end(), t->data.begin() + (size_t)r0 * line,
               t->data.begin() + (size_t)r1 * line);
  }
  if (out.size() & 1) out.push_back(0);
  auto rational = [&](double v, uint32& off) {
    off = (uint32)out.size();
    uint32 den = 10000;
    put32(out, (uint32)std::llround(v * den));
    put32(out, den);
  };
  uint32 xoff, yoff, soff = 0, coff = 0;
  rational(t->xres, xoff);
  rational(t->yres, yoff);
  if (nstrips > 1) {
    soff = (uint32)out.size();
    for (uint32 v : offs) put32(out, v);
    coff = (uint32)out.size();
    for (uint32 v : counts) put32(out, v);
  }
  struct Entry { uint16 tag, type; uint32 count, value; };
  std::vector<Entry> e;
  e.push_back({TIFFTAG_IMAGEWIDTH, 4, 1, t->width});
  e.push_back({TIFFTAG_IMAGELENGTH, 4, 1, t->length});
  e.push_back({TIFFTAG_BITSPERSAMPLE, 3, 1, t->bps});
  e.push_back({TIFFTAG_COMPRESSION, 3, 1, 1});
  e.push_back({TIFFTAG_PHOTOMETRIC, 3, 1, t->photometric});
  e.push_back({TIFFTAG_STRIPOFFSETS, 4, nstrips, nstrips > 1 ? soff : offs[0]});
  e.push_back({TIFFTAG_ORIENTATION, 3, 1, t->orientation});
  e.push_back({TIFFTAG_SAMPLESPERPIXEL, 3, 1, t->spp});
  e.push_back({TIFFTAG_ROWSPERSTRIP, 4, 1, rps});
  e.push_back({TIFFTAG_STRIPBYTECOUNTS, 4, nstrips,
               nstrips > 1 ? coff : counts[0]});
  e.push_back({TIFFTAG_XRESOLUTION, 5, 1, xoff});
  e.push_back({TIFFTAG_YRESOLUTION, 5, 1, yoff});
  e.push_back({TIFFTAG_PLANARCONFIG, 3, 1, t->planar});
  e.push_back({TIFFTAG_RESOLUTIONUNIT, 3, 1, t->resunit});
  if (t->has_sampleformat)
    e.push_back({TIFFTAG_SAMPLEFORMAT, 3, 1, t->sampleformat});
  uint32 ifd = (uint32)out.size();
  for (int k = 0; k < 4; ++k) out[4 + k] = (ifd >> (8 * k)) & 0xff;
  put16(out, (uint16)e.size());
  for (const Entry& x : e) {
    put16(out, x.tag);
    put16(out, x.type);
    put32(out, x.count);
    if (x.type == 3 && x.count == 1) {
      put16(out, (uint16)x.value);
      put16(out, 0);
    } else {
      put32(out, x.value);
    }
  }
  put32(out, 0);
  FILE* f = std::fopen(t->name.c_str(), "wb");
  if (f) {
    std::fwrite(out.data(), 1, out.size(), f);
    std::fclose(f);
  }
  delete t;
}

void* _TIFFmalloc(tsize_t s) { return std::malloc((size_t)s); }
void _TIFFfree(void* p) { std::free(p); }
}  // extern "C"
