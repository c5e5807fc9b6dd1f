// One raster over several ranks, one process per GPU.
//
// The reference runs `mpirun -np K ms-stem-fem.x` (tem.cpp:90): every rank
// builds the specimen, takes its share of the probe positions
// (adfstem.cpp:1556-1606) and the detector sums are combined with MPI
// collectives (adfstem.cpp:2256, 2489-2782).  Here a communicator joins the
// ranks:
//  * bootstrap: a TCP star through rank 0 at a rendezvous address
//    "host:port" (the MASTER_ADDR / MASTER_PORT torchrun exports); every
//    connection and every transfer has a deadline, so a rank that never
//    joins or stops answering ends the others' calls with MSF_ERR_TIMEOUT
//    instead of a hang;
//  * exchange transport: NCCL (libnccl.so.2, loaded when the communicator
//    is created, so the library itself does not depend on it) on device
//    buffers, or the TCP star ("host"), for ranks that share a GPU and for
//    machines without one.
// The exchange is the one collective step of a sharded raster: an
// all-gather of the per-probe detector rows (ring sums and ADF annulus;
// each rank's rows padded to the largest shard) and an all-gather of the
// per-pixel sums of the FEM pixel modes, which every rank adds in rank
// order (so the result does not depend on the collective's reduction
// order, and both transports give the same bits).  Every rank then
// finishes the ADF image and FEM statistics on the host.
#include <arpa/inet.h>
#include <dlfcn.h>
#include <netdb.h>
#include <netinet/in.h>
#include <netinet/tcp.h>
#include <poll.h>
#include <sys/socket.h>
#include <unistd.h>

#include <nccl.h>

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "engine.hpp"
#include "kernels.h"
#include "trace.hpp"

namespace msf {

#define MSF_CUDA(call)                                                      \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) {                                                \
      set_error(std::string("CUDA error: ") + cudaGetErrorString(e_) +      \
                " at " + __FILE__ + ":" + std::to_string(__LINE__));        \
      return MSF_ERR_CUDA;                                                  \
    }                                                                       \
  } while (0)
#define MSF_TRY(call)                \
  do {                               \
    msf_status s_ = (call);          \
    if (s_ != MSF_OK) return s_;     \
  } while (0)

msf_status raster_sums(msf_context* ctx, const RasterPlan& P, msf_results* res);

namespace {

using Clock = std::chrono::steady_clock;

// ------------------------------------------------------------- NCCL ----
// The NCCL entry points this file uses, looked up in libnccl.so.2.
struct Nccl {
  decltype(&ncclGetUniqueId) get_unique_id = nullptr;
  decltype(&ncclCommInitRank) init_rank = nullptr;
  decltype(&ncclAllGather) all_gather = nullptr;
  decltype(&ncclCommDestroy) destroy = nullptr;
  decltype(&ncclCommAbort) abort = nullptr;
  decltype(&ncclCommGetAsyncError) async_error = nullptr;
  decltype(&ncclGetErrorString) error_string = nullptr;
  bool ok = false;
  std::string why;
};

// Which libnccl.so.2: the one MSF_NCCL_LIBRARY names (a path), else one
// the process has loaded already (a framework's own NCCL: loading a second
// copy under the same soname would break that framework's later symbol
// lookups), else the system's.
const Nccl& nccl() {
  static Nccl n = [] {
    Nccl r;
    void* h = nullptr;
    if (const char* path = std::getenv("MSF_NCCL_LIBRARY"))
      if (*path) h = dlopen(path, RTLD_NOW | RTLD_GLOBAL);
    if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
    if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
    if (!h) {
      r.why = std::string("libnccl.so.2 not found: ") + dlerror();
      return r;
    }
#define MSF_NCCL_SYM(field, name)                                       \
  r.field = reinterpret_cast<decltype(r.field)>(dlsym(h, name));        \
  if (!r.field) {                                                       \
    r.why = std::string("libnccl.so.2 lacks ") + name;                  \
    return r;                                                           \
  }
    MSF_NCCL_SYM(get_unique_id, "ncclGetUniqueId")
    MSF_NCCL_SYM(init_rank, "ncclCommInitRank")
    MSF_NCCL_SYM(all_gather, "ncclAllGather")
    MSF_NCCL_SYM(destroy, "ncclCommDestroy")
    MSF_NCCL_SYM(abort, "ncclCommAbort")
    MSF_NCCL_SYM(async_error, "ncclCommGetAsyncError")
    MSF_NCCL_SYM(error_string, "ncclGetErrorString")
#undef MSF_NCCL_SYM
    r.ok = true;
    return r;
  }();
  return n;
}

// ------------------------------------------------------- TCP star ------
double remaining(Clock::time_point deadline) {
  return std::chrono::duration<double>(deadline - Clock::now()).count();
}

// Waits until fd is readable (POLLIN) or writable (POLLOUT), or the
// deadline passes.
bool wait_fd(int fd, short events, Clock::time_point deadline) {
  for (;;) {
    const double left = remaining(deadline);
    if (left <= 0) return false;
    pollfd p{fd, events, 0};
    const int r = poll(&p, 1, (int)std::min(left * 1000.0 + 1.0, 1000.0));
    if (r > 0) return true;
    if (r < 0 && errno != EINTR) return false;
  }
}

// Outcome of a transfer: done, deadline passed, or the peer closed the
// connection (or another socket error).
enum Xfer { XFER_OK = 0, XFER_TIMEOUT, XFER_LOST };

Xfer send_all(int fd, const void* buf, size_t n, Clock::time_point deadline) {
  const char* p = static_cast<const char*>(buf);
  while (n > 0) {
    if (!wait_fd(fd, POLLOUT, deadline)) return XFER_TIMEOUT;
    const ssize_t k = ::send(fd, p, n, MSG_NOSIGNAL);
    if (k < 0 && (errno == EINTR || errno == EAGAIN)) continue;
    if (k <= 0) return XFER_LOST;
    p += k;
    n -= (size_t)k;
  }
  return XFER_OK;
}

Xfer recv_all(int fd, void* buf, size_t n, Clock::time_point deadline) {
  char* p = static_cast<char*>(buf);
  while (n > 0) {
    if (!wait_fd(fd, POLLIN, deadline)) return XFER_TIMEOUT;
    const ssize_t k = ::recv(fd, p, n, 0);
    if (k < 0 && (errno == EINTR || errno == EAGAIN)) continue;
    if (k <= 0) return XFER_LOST;
    p += k;
    n -= (size_t)k;
  }
  return XFER_OK;
}

bool split_address(const std::string& addr, std::string* host, int* port) {
  const size_t c = addr.rfind(':');
  if (c == std::string::npos || c == 0) return false;
  *host = addr.substr(0, c);
  char* end = nullptr;
  const long p = std::strtol(addr.c_str() + c + 1, &end, 10);
  if (!end || *end || p <= 0 || p > 65535) return false;
  *port = (int)p;
  return true;
}

}  // namespace
}  // namespace msf

// A communicator of `world` ranks (see msf.h).
struct msf_comm {
  int rank = 0, world = 1, device = -1;
  int transport = MSF_COMM_HOST;
  double timeout_s = 60.0;
  int listen_fd = -1;
  std::vector<int> fds;      // rank 0: one socket per other rank; others: [0] to rank 0
  ncclComm_t nccl = nullptr;
  cudaStream_t stream = nullptr;
  ~msf_comm() {
    if (nccl) msf::nccl().destroy(nccl);
    if (stream) cudaStreamDestroy(stream);
    for (int fd : fds)
      if (fd >= 0) ::close(fd);
    if (listen_fd >= 0) ::close(listen_fd);
  }
  std::chrono::steady_clock::time_point deadline() const {
    return std::chrono::steady_clock::now() +
           std::chrono::milliseconds((int64_t)(timeout_s * 1000.0));
  }
};

namespace msf {
namespace {

msf_status comm_timeout(const msf_comm* c, const std::string& what) {
  set_error("rank " + std::to_string(c->rank) + " of " + std::to_string(c->world) + ": " +
            what + " did not complete within " + std::to_string(c->timeout_s) + " s");
  return MSF_ERR_TIMEOUT;
}

// A failed transfer: MSF_ERR_TIMEOUT when the deadline passed, MSF_ERR_IO
// when the other side closed the connection (its process ended).
msf_status comm_failed(const msf_comm* c, Xfer x, const std::string& what) {
  if (x == XFER_TIMEOUT) return comm_timeout(c, what);
  set_error("rank " + std::to_string(c->rank) + " of " + std::to_string(c->world) + ": " +
            what + " failed: the connection was closed (the other rank ended)");
  return MSF_ERR_IO;
}

msf_status star_connect(msf_comm* c, const std::string& address) {
  std::string host;
  int port = 0;
  if (!split_address(address, &host, &port)) {
    set_error("rendezvous address must be host:port, got '" + address + "'");
    return MSF_ERR_ARG;
  }
  const auto deadline = c->deadline();
  if (c->rank == 0) {
    c->listen_fd = ::socket(AF_INET, SOCK_STREAM, 0);
    if (c->listen_fd < 0) { set_error("socket() failed"); return MSF_ERR_IO; }
    int one = 1;
    setsockopt(c->listen_fd, SOL_SOCKET, SO_REUSEADDR, &one, sizeof one);
    sockaddr_in a{};
    a.sin_family = AF_INET;
    a.sin_port = htons((uint16_t)port);
    a.sin_addr.s_addr = htonl(INADDR_ANY);
    if (::bind(c->listen_fd, reinterpret_cast<sockaddr*>(&a), sizeof a) != 0 ||
        ::listen(c->listen_fd, c->world) != 0) {
      set_error("rank 0 could not listen on port " + std::to_string(port) + ": " +
                std::strerror(errno));
      return MSF_ERR_IO;
    }
    c->fds.assign(c->world, -1);
    for (int joined = 1; joined < c->world; ++joined) {
      if (!wait_fd(c->listen_fd, POLLIN, deadline))
        return comm_timeout(c, "waiting for " + std::to_string(c->world - joined) +
                                   " more rank(s) to join");
      const int fd = ::accept(c->listen_fd, nullptr, nullptr);
      if (fd < 0) { --joined; continue; }
      int32_t r = -1;
      if (recv_all(fd, &r, sizeof r, deadline) != XFER_OK || r <= 0 || r >= c->world ||
          c->fds[r] >= 0) {
        ::close(fd);
        set_error("a joining rank sent an invalid or repeated rank number");
        return MSF_ERR_ARG;
      }
      setsockopt(fd, IPPROTO_TCP, TCP_NODELAY, &one, sizeof one);
      c->fds[r] = fd;
    }
    return MSF_OK;
  }
  addrinfo hints{}, *res = nullptr;
  hints.ai_family = AF_INET;
  hints.ai_socktype = SOCK_STREAM;
  if (getaddrinfo(host.c_str(), std::to_string(port).c_str(), &hints, &res) != 0 || !res) {
    set_error("cannot resolve rendezvous host '" + host + "'");
    return MSF_ERR_ARG;
  }
  int fd = -1;
  while (remaining(deadline) > 0) {  // rank 0 may not be listening yet
    fd = ::socket(AF_INET, SOCK_STREAM, 0);
    if (fd >= 0 && ::connect(fd, res->ai_addr, res->ai_addrlen) == 0) break;
    if (fd >= 0) ::close(fd);
    fd = -1;
    std::this_thread::sleep_for(std::chrono::milliseconds(50));
  }
  freeaddrinfo(res);
  if (fd < 0) return comm_timeout(c, "connecting to rank 0 at " + address);
  int one = 1;
  setsockopt(fd, IPPROTO_TCP, TCP_NODELAY, &one, sizeof one);
  const int32_t r = c->rank;
  if (const Xfer x = send_all(fd, &r, sizeof r, deadline); x != XFER_OK) {
    ::close(fd);
    return comm_failed(c, x, "announcing this rank to rank 0");
  }
  c->fds.assign(1, fd);
  return MSF_OK;
}

// Every rank gets every rank's `bytes` (rank order) in recv[world * bytes];
// the blocks travel through rank 0.
msf_status star_allgather(msf_comm* c, const void* send, size_t bytes, void* recv) {
  char* out = static_cast<char*>(recv);
  std::memcpy(out + (size_t)c->rank * bytes, send, bytes);
  if (c->world == 1) return MSF_OK;
  const auto deadline = c->deadline();
  if (c->rank == 0) {
    for (int r = 1; r < c->world; ++r)
      if (const Xfer x = recv_all(c->fds[r], out + (size_t)r * bytes, bytes, deadline);
          x != XFER_OK)
        return comm_failed(c, x, "receiving rank " + std::to_string(r) + "'s block");
    for (int r = 1; r < c->world; ++r)
      if (const Xfer x = send_all(c->fds[r], out, bytes * c->world, deadline); x != XFER_OK)
        return comm_failed(c, x, "sending the gathered blocks to rank " + std::to_string(r));
    return MSF_OK;
  }
  if (const Xfer x = send_all(c->fds[0], send, bytes, deadline); x != XFER_OK)
    return comm_failed(c, x, "sending this rank's block to rank 0");
  if (const Xfer x = recv_all(c->fds[0], out, bytes * c->world, deadline); x != XFER_OK)
    return comm_failed(c, x, "receiving the gathered blocks from rank 0");
  return MSF_OK;
}

// Waits (bounded) for the NCCL work enqueued on the communicator's stream;
// on a timeout or an asynchronous NCCL error the communicator is aborted.
msf_status nccl_wait(msf_comm* c, const char* what) {
  const auto deadline = c->deadline();
  for (;;) {
    const cudaError_t q = cudaStreamQuery(c->stream);
    if (q == cudaSuccess) return MSF_OK;
    if (q != cudaErrorNotReady) {
      set_error(std::string(what) + ": " + cudaGetErrorString(q));
      return MSF_ERR_CUDA;
    }
    ncclResult_t ae = ncclSuccess;
    nccl().async_error(c->nccl, &ae);
    if (ae != ncclSuccess && ae != ncclInProgress) {
      set_error(std::string(what) + ": NCCL " + nccl().error_string(ae));
      nccl().abort(c->nccl);
      c->nccl = nullptr;
      return MSF_ERR_CUDA;
    }
    if (remaining(deadline) <= 0) {
      nccl().abort(c->nccl);
      c->nccl = nullptr;
      return comm_timeout(c, what);
    }
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

}  // namespace

// Probes [begin, end) of rank `rank`: contiguous, sizes differ by at most
// one, lower ranks take the larger shares (the reference's ranks take
// contiguous blocks of the raster, adfstem.cpp:1556-1606).
void shard_range(int64_t n, int rank, int world, int64_t* begin, int64_t* end) {
  const int64_t base = n / world, extra = n % world;
  *begin = rank * base + std::min<int64_t>(rank, extra);
  *end = *begin + base + (rank < extra ? 1 : 0);
}

msf_status run_sharded(msf_context* ctx, const msf_specimen* spec, const msf_optics* optics,
                       const msf_raster* raster, const msf_detect* det, msf_comm* comm,
                       msf_results* res, msf_shard_info* info) {
  TraceScope trace_scope("raster_sharded");
  if (!ctx || !spec || !optics || !raster || !det || !comm || !res) {
    set_error("msf_run_sharded: null argument");
    return MSF_ERR_ARG;
  }
  const bool on_device = comm->transport == MSF_COMM_NCCL;
  if (on_device && comm->device != ctx->device) {
    set_error("msf_run_sharded: the communicator's device differs from the context's");
    return MSF_ERR_ARG;
  }
  MSF_CUDA(cudaSetDevice(ctx->device));
  const int world = comm->world, rank = comm->rank;
  const int64_t n = (int64_t)raster->n_x * raster->n_y;
  if (n <= 0) { set_error("empty raster"); return MSF_ERR_ARG; }
  int64_t b = 0, e = 0;
  shard_range(n, rank, world, &b, &e);
  const int64_t rows_max = (n + world - 1) / world;
  const Grid& g = spec->g;
  const int64_t plane = (int64_t)g.nx * g.ny;
  const bool pix = det->outputs & (MSF_OUT_V_RE | MSF_OUT_OMEGA_VIMAGE | MSF_OUT_V_GT17 |
                                   MSF_OUT_V_RBAR);
  static const Rings no_rings;
  std::shared_ptr<const Rings> rings_sp;
  int n_seg = 1;  // ring bins (and correlograph cells), then the ADF annulus
  if (det->outputs & MSF_OUT_FEM_MASK) {
    rings_sp = rings_for(ctx, g, det->dr);
    n_seg = rings_sp->n_k + 1;
    if (det->outputs & MSF_OUT_CORRELOGRAPH) n_seg += rings_sp->n_k * make_cells(g, *rings_sp).n_phi;
  }
  const Rings& rings = rings_sp ? *rings_sp : no_rings;
  const size_t row_doubles = (size_t)rows_max * n_seg;  // one of amp / inten, padded

  // this rank's probes
  const auto t0 = Clock::now();
  RasterPlan P;
  msf_results part{};
  // the raster's first exit wave is rank 0's first probe; its last one is
  // the last rank's last probe, sent on to rank 0 below
  std::vector<double> last_psi;
  const bool has_last = e == n && e > b;
  if (res->first_psi && b == 0) part.first_psi = res->first_psi;
  if (res->final_psi && has_last) {
    last_psi.assign(2 * plane, 0.0);
    part.final_psi = last_psi.data();
  }
  if (e > b) {
    MSF_TRY(plan_raster(ctx, spec, optics, raster, det, &P, b, e));
    if (P.n_seg != n_seg) { set_error("segment count mismatch"); return MSF_ERR_ARG; }
    MSF_TRY(raster_sums(ctx, P, &part));
  }
  const auto t1 = Clock::now();

  std::vector<double> rows_all((size_t)world * 2 * row_doubles);
  std::vector<double> acc_a, acc_i;
  if (pix) {
    acc_a.assign(plane, 0.0);
    acc_i.assign(plane, 0.0);
  }
  if (on_device) {
    // rows and pixel sums stay on the device: NCCL all-gathers them, the
    // pixel sums are added in rank order by a kernel
    DevBuf send, recv, pix_send, pix_recv, pix_sum;
    MSF_TRY(ctx->alloc(&send, sizeof(double) * 2 * row_doubles));
    MSF_TRY(ctx->alloc(&recv, sizeof(double) * 2 * row_doubles * world));
    MSF_CUDA(cudaMemsetAsync(send.p, 0, send.bytes, ctx->stream));
    if (e > b) {
      const size_t bytes = sizeof(double) * (size_t)(e - b) * n_seg;
      MSF_CUDA(cudaMemcpyAsync(send.p, P.amp.p, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
      MSF_CUDA(cudaMemcpyAsync(send.as<double>() + row_doubles, P.inten.p, bytes,
                               cudaMemcpyDeviceToDevice, ctx->stream));
    }
    if (pix) {
      MSF_TRY(ctx->alloc(&pix_send, sizeof(double) * 2 * plane));
      MSF_TRY(ctx->alloc(&pix_recv, sizeof(double) * 2 * plane * world));
      MSF_TRY(ctx->alloc(&pix_sum, sizeof(double) * 2 * plane));
      if (e > b) {
        MSF_CUDA(cudaMemcpyAsync(pix_send.p, P.acc_a.p, sizeof(double) * plane,
                                 cudaMemcpyDeviceToDevice, ctx->stream));
        MSF_CUDA(cudaMemcpyAsync(pix_send.as<double>() + plane, P.acc_i.p,
                                 sizeof(double) * plane, cudaMemcpyDeviceToDevice, ctx->stream));
      } else {
        MSF_CUDA(cudaMemsetAsync(pix_send.p, 0, pix_send.bytes, ctx->stream));
      }
    }
    // the collectives run on the communicator's stream, after this rank's
    // raster and copies
    cudaEvent_t ready;
    MSF_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    MSF_CUDA(cudaEventRecord(ready, ctx->stream));
    MSF_CUDA(cudaStreamWaitEvent(comm->stream, ready, 0));
    cudaEventDestroy(ready);
    if (!comm->nccl) { set_error("the communicator's NCCL state was aborted"); return MSF_ERR_CUDA; }
    ncclResult_t r = nccl().all_gather(send.p, recv.p, 2 * row_doubles, ncclDouble, comm->nccl,
                                       comm->stream);
    if (r == ncclSuccess && pix)
      r = nccl().all_gather(pix_send.p, pix_recv.p, 2 * plane, ncclDouble, comm->nccl,
                            comm->stream);
    if (r != ncclSuccess) {
      set_error(std::string("ncclAllGather: ") + nccl().error_string(r));
      return MSF_ERR_CUDA;
    }
    MSF_TRY(nccl_wait(comm, "the exchange of detector rows and pixel sums"));
    MSF_CUDA(cudaMemcpyAsync(rows_all.data(), recv.p, recv.bytes, cudaMemcpyDeviceToHost,
                             comm->stream));
    if (pix) {
      MSF_CUDA(launch_rank_sum(pix_recv.as<double>(), world, 2 * plane, pix_sum.as<double>(),
                               comm->stream));
      MSF_CUDA(cudaMemcpyAsync(acc_a.data(), pix_sum.p, sizeof(double) * plane,
                               cudaMemcpyDeviceToHost, comm->stream));
      MSF_CUDA(cudaMemcpyAsync(acc_i.data(), pix_sum.as<double>() + plane,
                               sizeof(double) * plane, cudaMemcpyDeviceToHost, comm->stream));
    }
    MSF_CUDA(cudaStreamSynchronize(comm->stream));
  } else {
    std::vector<double> mine(2 * row_doubles, 0.0);
    std::vector<double> pa, pi;
    if (pix) {
      pa.assign(plane, 0.0);
      pi.assign(plane, 0.0);
    }
    if (e > b)
      MSF_TRY(download_sums(ctx, P, ctx->stream, mine.data(), mine.data() + row_doubles,
                            pix ? pa.data() : nullptr, pix ? pi.data() : nullptr));
    MSF_TRY(star_allgather(comm, mine.data(), sizeof(double) * mine.size(), rows_all.data()));
    if (pix) {
      std::vector<double> both(2 * plane), got(2 * plane * world);
      std::copy(pa.begin(), pa.end(), both.begin());
      std::copy(pi.begin(), pi.end(), both.begin() + plane);
      MSF_TRY(star_allgather(comm, both.data(), sizeof(double) * both.size(), got.data()));
      for (int r = 0; r < world; ++r)  // rank order, as the device kernel adds
        for (int64_t p = 0; p < plane; ++p) {
          acc_a[p] += got[(size_t)r * 2 * plane + p];
          acc_i[p] += got[(size_t)r * 2 * plane + plane + p];
        }
    }
  }
  if (res->final_psi) {  // the last exit wave reaches every rank
    if (world == 1) {
      std::copy(last_psi.begin(), last_psi.end(), res->final_psi);
    } else {
      // the rank holding the raster's last probe: the highest with probes
      int holder = world - 1;
      for (; holder > 0; --holder) {
        int64_t hb = 0, he = 0;
        shard_range(n, holder, world, &hb, &he);
        if (he > hb) break;
      }
      std::vector<double> got((size_t)world * 2 * plane);
      if (last_psi.empty()) last_psi.assign(2 * plane, 0.0);
      MSF_TRY(star_allgather(comm, last_psi.data(), sizeof(double) * 2 * plane, got.data()));
      std::copy(got.begin() + (size_t)holder * 2 * plane,
                got.begin() + (size_t)(holder + 1) * 2 * plane, res->final_psi);
    }
  }
  const auto t2 = Clock::now();

  // rows of all probes in raster order
  std::vector<double> amp((size_t)n * n_seg), inten((size_t)n * n_seg);
  for (int r = 0; r < world; ++r) {
    int64_t rb = 0, re = 0;
    shard_range(n, r, world, &rb, &re);
    const double* blk = rows_all.data() + (size_t)r * 2 * row_doubles;
    std::copy(blk, blk + (size_t)(re - rb) * n_seg, amp.begin() + (size_t)rb * n_seg);
    std::copy(blk + row_doubles, blk + row_doubles + (size_t)(re - rb) * n_seg,
              inten.begin() + (size_t)rb * n_seg);
  }
  MSF_TRY(finish_host(g, rings, *optics, *det, n, amp.data(), inten.data(),
                      pix ? acc_a.data() : nullptr, pix ? acc_i.data() : nullptr, res));
  const auto t3 = Clock::now();
  res->probe_slices = part.probe_slices;
  res->kernel_launches = part.kernel_launches;
  res->seconds_raster = part.seconds_raster;
  res->ms_row_pass = part.ms_row_pass;
  res->ms_col_pass = part.ms_col_pass;
  res->pass_batch = part.pass_batch;
  if (info) {
    info->p_begin = b;
    info->p_end = e;
    info->seconds_shard = std::chrono::duration<double>(t1 - t0).count();
    info->seconds_exchange = std::chrono::duration<double>(t2 - t1).count();
    info->seconds_finish = std::chrono::duration<double>(t3 - t2).count();
  }
  return MSF_OK;
}

}  // namespace msf

extern "C" {

msf_status msf_comm_create(int32_t rank, int32_t world, const char* rendezvous,
                           int32_t transport, int32_t device, double timeout_s,
                           msf_comm** out) {
  using namespace msf;
  if (!out) return MSF_ERR_ARG;
  *out = nullptr;
  if (world < 1 || rank < 0 || rank >= world) {
    set_error("msf_comm_create: rank " + std::to_string(rank) + " outside a world of " +
              std::to_string(world));
    return MSF_ERR_ARG;
  }
  if (transport != MSF_COMM_NCCL && transport != MSF_COMM_HOST) {
    set_error("msf_comm_create: transport must be MSF_COMM_NCCL or MSF_COMM_HOST");
    return MSF_ERR_ARG;
  }
  if (world > 1 && (!rendezvous || !*rendezvous)) {
    set_error("msf_comm_create: a rendezvous address host:port is needed for world > 1");
    return MSF_ERR_ARG;
  }
  auto c = std::make_unique<msf_comm>();
  c->rank = rank;
  c->world = world;
  c->device = device;
  c->transport = transport;
  c->timeout_s = timeout_s > 0 ? timeout_s : 60.0;
  if (world > 1) {
    msf_status st = star_connect(c.get(), rendezvous);
    if (st != MSF_OK) return st;
  }
  if (transport == MSF_COMM_NCCL) {
    const Nccl& N = nccl();
    if (!N.ok) {
      set_error("msf_comm_create: " + N.why);
      return MSF_ERR_UNSUPPORTED;
    }
    cudaError_t ce = cudaSetDevice(device);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) {
      set_error(std::string("msf_comm_create: ") + cudaGetErrorString(ce));
      return MSF_ERR_CUDA;
    }
    ncclUniqueId id{};
    if (rank == 0 && N.get_unique_id(&id) != ncclSuccess) {
      set_error("ncclGetUniqueId failed");
      return MSF_ERR_CUDA;
    }
    std::vector<ncclUniqueId> ids(world);  // rank 0's id reaches every rank
    msf_status st = star_allgather(c.get(), &id, sizeof id, ids.data());
    if (st != MSF_OK) return st;
    const ncclResult_t r = N.init_rank(&c->nccl, world, ids[0], rank);
    if (r != ncclSuccess) {
      c->nccl = nullptr;
      set_error(std::string("ncclCommInitRank: ") + N.error_string(r));
      return MSF_ERR_CUDA;
    }
  }
  *out = c.release();
  return MSF_OK;
}

void msf_comm_destroy(msf_comm* comm) { delete comm; }

msf_status msf_comm_allgather_host(msf_comm* comm, const void* send, int64_t bytes,
                                   void* recv) {
  if (!comm || bytes < 0 || (bytes > 0 && (!send || !recv))) return MSF_ERR_ARG;
  return msf::star_allgather(comm, send, (size_t)bytes, recv);
}

msf_status msf_run_sharded(msf_context* ctx, const msf_specimen* spec, const msf_optics* optics,
                           const msf_raster* raster, const msf_detect* detect, msf_comm* comm,
                           msf_results* results, msf_shard_info* info) {
  return msf::run_sharded(ctx, spec, optics, raster, detect, comm, results, info);
}

}  // extern "C"
