// msf_probe_noalloc: the probe build of msf_probe with no device allocation.
//
// Some callers cannot call cudaMalloc when they need a probe: applications
// that hand every byte of device memory to their own pool at start-up and
// forbid allocation afterwards (cudaMalloc can synchronise the device and
// stall a running acquisition or serving loop), and host frameworks whose
// plug-ins only ever receive pre-sized buffers.  Such a caller passes the
// output buffer; the scratch this build needs -- the k-space domains, two
// twiddle tables and the norm accumulator -- lives in one fixed file-scope
// device array, sized for grids of at most kMaxSide x kMaxSide.
//
// Behaviour a caller must know:
//  * The first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current, and so does every
//    later call made outside a stream capture; make the first call on each
//    device before any stream capture (and again after a cudaDeviceReset).
//  * The probe equals msf_probe's to within FP64 rounding (1e-12 of its
//    largest value), not bit for bit: the twiddles here come from the
//    device's sincospi, msf_probe's from host cos/sin.
//  * Every call on a device shares the one array and leaves its contents
//    behind.  Each call overwrites every scratch entry it reads, so nothing
//    has to start at zero, but two calls whose work overlaps on the GPU (for
//    example on two streams) race on the scratch and must not be issued.
//  * Grids larger than kMaxSide on either side are rejected with
//    MSF_ERR_ARG and a message; no partial work is enqueued.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "kernels.h"
#include "msf.h"
#include "setup.hpp"

namespace msf {
void set_error(const std::string& msg);
}

namespace {

constexpr int kMaxSide = 2048;
constexpr size_t kDomainBytes = sizeof(double) * kMaxSide;       // one of kx, ky
constexpr size_t kTwiddleBytes = sizeof(double2) * kMaxSide;     // one table
constexpr size_t kScratchBytes = 2 * kDomainBytes + 2 * kTwiddleBytes + 256;

// kx | ky | twiddles(nx) | twiddles(ny) | norm accumulator
static __device__ __align__(256) unsigned char msf_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_address[kMaxDevices] = {};

// Device address of the scratch array on the current device.  Outside a
// stream capture it is looked up again on every call (a host-side query
// that allocates nothing), so a context the application tore down and
// recreated (cudaDeviceReset) cannot leave a stale address behind; the
// first call on a device must therefore not be inside a capture.
msf_status scratch_address(int device, cudaStream_t s, unsigned char** out) {
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
    msf::set_error("msf_probe_noalloc: cudaStreamIsCapturing failed");
    return MSF_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_mutex);
  if (cap == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, msf_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      msf::set_error(std::string("cudaGetSymbolAddress(msf_noalloc_scratch): ") +
                     cudaGetErrorString(e));
      return MSF_ERR_CUDA;
    }
    g_address[device] = p;
  } else if (!g_address[device]) {
    msf::set_error("msf_probe_noalloc: the first call on a device must not be captured "
                   "(the scratch address is looked up outside a capture)");
    return MSF_ERR_ARG;
  }
  *out = static_cast<unsigned char*>(g_address[device]);
  return MSF_OK;
}

// k-space domains (func.cpp:147-167) without contraction, so the values equal
// the host's make_grid bit for bit.
__global__ void noalloc_domains(double* kx, double* ky, int nx, int ny, double dkx,
                                double dky, double kxp, double kyp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nx) kx[i] = (i < nx / 2) ? __dmul_rn((double)i, dkx)
                                   : __dsub_rn(__dmul_rn((double)i, dkx), kxp);
  if (i < ny) ky[i] = (i < ny / 2) ? __dmul_rn((double)i, dky)
                                   : __dsub_rn(__dmul_rn((double)i, dky), kyp);
}

// e^{-2 pi i m / n}, m < n
__global__ void noalloc_twiddles(double2* tw, int n) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < n) {
    double s, c;
    sincospi(2.0 * (double)m / (double)n, &s, &c);
    tw[m] = make_double2(c, -s);
  }
}

// a *= 1/sqrt(sum[0]) (probe_wavefunction.cpp:287-315)
__global__ void noalloc_normalise(double2* a, int64_t n, const double* sum) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) {
    const double ap = 1.0 / sqrt(sum[0]);
    a[k] = make_double2(ap * a[k].x, ap * a[k].y);
  }
}

#define NOALLOC_CUDA(call)                                                       \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess) {                                                     \
      msf::set_error(std::string("msf_probe_noalloc: ") + cudaGetErrorString(e_)); \
      return MSF_ERR_CUDA;                                                       \
    }                                                                            \
  } while (0)

}  // namespace

extern "C" msf_status msf_probe_noalloc(const msf_grid* grid, const msf_optics* optics,
                                        double* probe_device, void* stream) {
  if (!grid || !optics || !probe_device) {
    msf::set_error("msf_probe_noalloc: null argument");
    return MSF_ERR_ARG;
  }
  const int nx = grid->nx, ny = grid->ny;
  if (nx > kMaxSide || ny > kMaxSide) {
    msf::set_error("msf_probe_noalloc: grid " + std::to_string(nx) + "x" + std::to_string(ny) +
                   " exceeds the fixed scratch limit of " + std::to_string(kMaxSide) +
                   " samples per side; use msf_probe");
    return MSF_ERR_ARG;
  }
  if (!msf::supported_length(nx) || !msf::supported_length(ny)) {
    msf::set_error("msf_probe_noalloc: each grid side must be a power of two in [64, 2048]");
    return MSF_ERR_UNSUPPORTED;
  }
  int device = 0;
  NOALLOC_CUDA(cudaGetDevice(&device));
  if (device < 0 || device >= kMaxDevices) {
    msf::set_error("msf_probe_noalloc: device ordinal out of range");
    return MSF_ERR_ARG;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned char* base = nullptr;
  msf_status st = scratch_address(device, s, &base);
  if (st != MSF_OK) return st;
  double* kx = reinterpret_cast<double*>(base);
  double* ky = reinterpret_cast<double*>(base + kDomainBytes);
  double2* twx = reinterpret_cast<double2*>(base + 2 * kDomainBytes);
  double2* twy = reinterpret_cast<double2*>(base + 2 * kDomainBytes + kTwiddleBytes);
  double* norm = reinterpret_cast<double*>(base + 2 * kDomainBytes + 2 * kTwiddleBytes);

  // scalars of tem.cpp:424-788 (no host allocation)
  const int dxf = grid->dupe_x > 0 ? grid->dupe_x : 1, dyf = grid->dupe_y > 0 ? grid->dupe_y : 1;
  const double xpd = grid->xperiod * dxf, ypd = grid->yperiod * dyf;
  double lambda = 0, gamma = 0;
  msf::wavelength(grid->voltage, &lambda, &gamma);
  const long Nx = nx, Ny = ny;
  const double sq = (Nx == Ny) ? (double)Nx : std::sqrt((double)(Nx * Ny));

  const int side = nx > ny ? nx : ny;
  noalloc_domains<<<(side + 255) / 256, 256, 0, s>>>(kx, ky, nx, ny, 1.0 / xpd, 1.0 / ypd,
                                                     Nx / xpd, Ny / ypd);
  NOALLOC_CUDA(cudaGetLastError());
  noalloc_twiddles<<<(nx + 255) / 256, 256, 0, s>>>(twx, nx);
  NOALLOC_CUDA(cudaGetLastError());
  noalloc_twiddles<<<(ny + 255) / 256, 256, 0, s>>>(twy, ny);
  NOALLOC_CUDA(cudaGetLastError());
  // probe in k-space at (xx[0], yy[0]) = (xmin, ymin) (adfstem.cpp:586-645)
  NOALLOC_CUDA(msf::launch_probe_synth(probe_device, kx, ky, nx, ny, optics->corrected,
                                       optics->cs3, optics->cs5, optics->defocus, lambda,
                                       lambda * lambda, optics->alpha_max * optics->alpha_max,
                                       grid->xmin, grid->ymin, s));
  // BACKWARD transform in place, / sqrtNxNy (adfstem.cpp:686-732)
  msf::PassArgs a;
  a.psi = probe_device;
  a.batch_stride = (int64_t)nx * ny;
  a.nb = 1;
  a.nx = nx;
  a.ny = ny;
  a.tw = twy;
  a.scale = 1.0;
  NOALLOC_CUDA(msf::launch_row(true, msf::ROW_INV, a, s));
  a.tw = twx;
  a.scale = 1.0 / sq;
  NOALLOC_CUDA(msf::launch_col(true, msf::COL_INV, a, s));
  // norm (overwrites the accumulator) and scale, all on the device
  NOALLOC_CUDA(msf::launch_norm2(probe_device, (int64_t)nx * ny, norm, s));
  const int64_t n = (int64_t)nx * ny;
  noalloc_normalise<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
      reinterpret_cast<double2*>(probe_device), n, norm);
  NOALLOC_CUDA(cudaGetLastError());
  return MSF_OK;
}
