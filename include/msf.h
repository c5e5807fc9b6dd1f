/* msf.h -- C ABI of the B200 multislice ADF-STEM / FEM library (libmsf.so).
 *
 * Plain C: opaque handles, POD structs, caller-owned host buffers, integer
 * status codes (never exit()).  One CUDA stream per context; contexts are
 * independent, so separate threads may drive separate contexts.
 *
 * The reference (nickjulian/ms-stem-fem) is one MPI executable with no FFI;
 * these entry points replace its multislice path at the function boundary:
 *
 *   msf_specimen_create   replaces tem.cpp:944-1276 -- scatterer_pap_LUT
 *                         (scatterer_pap.hpp:45-230), assign_atoms_to_slices_
 *                         z_auto (slice.cpp:469-980), slice::update_propagator
 *                         (slice.cpp:1293-1363) and slice::update_transmission_
 *                         function (slice.cpp:1451-1757)
 *   msf_run               replaces TEM_NS::adfstem (adfstem.hpp:66-122,
 *                         adfstem.cpp:37-4096): probe, raster, slice loop,
 *                         ADF detection and the FEM V(k) statistics
 *   msf_parse_cmdline     replaces read_cmdline_options / read_parameter_file
 *                         / check_runtime_flags (tem_io.cpp:5277-5720,
 *                         4063-4626, 5858-6169) plus tem.cpp's defaults
 *   msf_read_specimen     replaces read_position_lammps_data_file
 *                         (tem_io.cpp:36-1028) and read_position_xyz_file
 *                         (tem_io.cpp:4627-4958)
 *   msf_write_outputs     replaces output_variance_to_txt (io_txt.cpp:30-94)
 *                         and output_stem_image (write_tif.cpp:1552-1605)
 */
#ifndef MSF_H
#define MSF_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MSF_ABI_VERSION 4

typedef enum {
  MSF_OK = 0,
  MSF_ERR_ARG = 1,         /* invalid argument or inconsistent request     */
  MSF_ERR_UNSUPPORTED = 2, /* valid for the reference, not built here      */
  MSF_ERR_CUDA = 3,        /* CUDA runtime error (message via msf_last_error) */
  MSF_ERR_NOMEM = 4,       /* device or host allocation failed             */
  MSF_ERR_IO = 5,          /* file could not be read or written            */
  MSF_ERR_PARSE = 6,       /* malformed command line / parameter / specimen */
  MSF_ERR_TIMEOUT = 7,     /* a bounded device wait gave up                */
  MSF_ERR_BUSY = 8,        /* serving queue full / budget exhausted        */
  MSF_ERR_CANCELLED = 9
} msf_status;

typedef enum { MSF_FP64 = 0, MSF_FP32 = 1 } msf_precision;

/* FEM modes (tem_io.cpp:5563-5586) and image output, as bits. */
#define MSF_OUT_ADF_IMAGE    (1u << 0) /* --images                          */
#define MSF_OUT_V_OMEGA      (1u << 1) /* --V_omega     (flags.d1)          */
#define MSF_OUT_VBAR_R       (1u << 2) /* --Vbar_r      (flags.d2)          */
#define MSF_OUT_V_RE         (1u << 3) /* --V_re        (flags.d3)          */
#define MSF_OUT_OMEGA_VIMAGE (1u << 4) /* --Omega_vimage (flags.d4)         */
#define MSF_OUT_V_GT17       (1u << 5) /* --V_gt17      (flags.gt17)        */
#define MSF_OUT_V_RBAR       (1u << 6) /* --V_rbar      (flags.rva)         */
#define MSF_OUT_CORRELOGRAPH (1u << 7) /* --correlograph (raster average)  */
#define MSF_OUT_CORRELOGRAPH_VAR (1u << 8) /* --correlograph_variance      */
#define MSF_OUT_FEM_MASK     (0x1feu)  /* every output that needs ring bins */

typedef struct msf_context msf_context;
typedef struct msf_specimen msf_specimen;

typedef struct {
  int32_t device;          /* CUDA device ordinal                              */
  int32_t precision;       /* msf_precision of wavefields and FFTs             */
  int32_t batch;           /* probes per launch; 0 = choose from free memory   */
  int32_t use_graphs;      /* capture each batch's slice stack in a CUDA graph */
  int64_t hbm_budget;      /* bytes this context may allocate; 0 = no limit    */
} msf_options;

/* Simulation cell and grid (tem.cpp:405-695). */
typedef struct {
  int32_t nx, ny;          /* -m samples_x samples_y                           */
  double voltage;          /* -m VV [V]                                        */
  double xperiod, yperiod, zperiod; /* specimen periods [A] (raster uses x,y)  */
  int32_t dupe_x, dupe_y, dupe_z;   /* --dupe period multipliers (1 1 1 if absent) */
  int32_t replicate_atoms;  /* 1: copy the atoms into every duped cell, as
                               tem.cpp:1051-1143 does for FEM runs only      */
  double xmin, ymin, zmin; /* domain origin (0 after the LAMMPS reader shift)  */
  double min_slice;        /* --minslice [A]                                   */
} msf_grid;

typedef struct {
  int64_t n_atoms;
  const double* q;         /* 3*n_atoms: x y z [A] per atom                    */
  const uint32_t* z;       /* atomic numbers 1..103                            */
} msf_atoms;

typedef struct {
  int32_t corrected;       /* 0: uncorrected chi, 1: Cs5-corrected chi         */
  double cs3, cs5;         /* [A]                                              */
  double defocus;          /* [A]                                              */
  double alpha_max;        /* probe-forming aperture [rad]                     */
} msf_optics;

typedef struct {
  int32_t n_x, n_y;        /* raster points                                    */
  const double* x_p;       /* n_x positions [A]                                */
  const double* y_p;       /* n_y positions [A]                                */
} msf_raster;

typedef struct {
  uint32_t outputs;        /* MSF_OUT_* bits                                   */
  double det_inner, det_outer; /* ADF detector angles [rad]                    */
  double dr;               /* --dr azimuthal_binning_size_factor               */
  /* Detector modulation transfer function (mtf_file + mtf_sampling_rate,
   * adfstem.cpp:236-453, 2272-2385): applied to |psi(k)| before the FEM sums
   * when n_mtf > 0 and mtf_resolution != 0.  mtf[n_mtf] and
   * mtf_domain_sqr[n_mtf] as tem.cpp:276-285 leaves them (domain squared
   * after scaling by 0.5 * mtf_resolution). */
  int32_t n_mtf;
  const double* mtf;
  const double* mtf_domain_sqr;
  double mtf_resolution;   /* [pixels per 1/A]                                */
} msf_detect;

/* Caller-owned result buffers; any pointer may be NULL when not wanted. */
typedef struct {
  double* adf_image;       /* n_x*n_y, row px, column py: [px*n_y + py]        */
  int32_t cap_k;           /* capacity of each per-bin array below            */
  int32_t n_k;             /* out: number of k bins                            */
  double* k_lower;         /* out: lower boundary of each bin [1/A]            */
  int32_t* bin_counts;     /* out: pixels per bin                              */
  double* v_omega;
  double* vbar_r;
  double* v_re;
  double* omega_vimage;
  double* v_gt17;
  double* v_rbar;
  double* final_psi;       /* 2*nx*ny: last probe's exit wave in k-space (after
                              the detector MTF when one is applied)          */
  double* mean_amplitude;  /* nx*ny: raster mean of |psi(k)| (FEM pixel modes)*/
  double* mean_intensity;  /* nx*ny: raster mean of |psi(k)|^2                */
  double* ring_amplitude;  /* n_x*n_y*cap_k: per probe, sum |psi| per ring,
                              before the aperture zeroing (FEM runs)         */
  double* ring_intensity;  /* n_x*n_y*cap_k: per probe, sum |psi|^2 per ring  */
  int64_t probe_slices;    /* out: probe*slice propagations performed          */
  int64_t kernel_launches; /* out: CUDA kernels this call launched (incl. the
                              kernels inside replayed graphs)                 */
  double seconds_setup;    /* out: specimen set-up time (msf_run: 0)           */
  double seconds_raster;   /* out: device time of the raster                   */
  /* FEM correlograph (adfstem.cpp:2603-2685, 3617-3760): per probe and ring
   * bin ii, per azimuthal bin jj, n_k * S(ii,jj) / S(ii) - 1 when that
   * ratio is >= 1 (else 0), S(ii,jj) the sum of |psi(k)| over the cell and
   * S(ii) over the ring; arrays [jj*n_k + ii], n_k*n_phi entries. */
  int32_t cap_phi;         /* capacity: phi_lower holds cap_phi + 1 values,
                              the arrays below cap_k * cap_phi (per probe)  */
  int32_t n_phi;           /* out: number of azimuthal bins                    */
  double* phi_lower;       /* out: n_phi + 1 azimuthal boundaries [rad]        */
  double* correlograph;    /* out: raster average                              */
  double* correlograph_sqr;/* out: sum over probes of the squares (variance)   */
  double* correlograph_probes; /* out: n_x*n_y blocks of n_k*n_phi, raster order */
  double* first_psi;       /* 2*nx*ny: first probe's exit wave in k-space (before
                              any detector MTF)                               */
  /* out (msf_run): device time of the slice passes of the raster's first
   * batch, timed with CUDA events on the launching stream while the raster
   * runs: mean ms of one row pass and of one column pass over the slices
   * after the first (row) and before the last (column), and the probes that
   * batch carried; 0 when the raster has fewer than three slices. */
  double ms_row_pass, ms_col_pass;
  int32_t pass_batch;
} msf_results;

/* ---- library ---------------------------------------------------------- */
int32_t msf_abi_version(void);
const char* msf_last_error(void);            /* thread-local message        */
const char* msf_status_string(msf_status s);

/* ---- context ---------------------------------------------------------- */
msf_status msf_context_create(const msf_options* opt, msf_context** out);
msf_status msf_context_destroy(msf_context* ctx);
msf_status msf_context_synchronize(msf_context* ctx);
/* Host<->device bytes this context has copied since the last reset
 * (reset != 0 zeroes the counters after reading). */
msf_status msf_context_transfer_bytes(msf_context* ctx, int64_t* h2d,
                                      int64_t* d2h, int32_t reset);

/* ---- specimen: LUTs, slicing, propagators, transmission functions ------ */
msf_status msf_specimen_create(msf_context* ctx, const msf_grid* grid,
                               const msf_atoms* atoms, msf_specimen** out);
msf_status msf_specimen_destroy(msf_specimen* spec);
/* Slice count and per-slice lower bound, thickness and atom count (any
 * pointer may be NULL; arrays hold `cap` entries). */
msf_status msf_specimen_slices(const msf_specimen* spec, int32_t* n_slices,
                               double* lower, double* thickness,
                               int64_t* atoms_per_slice, int32_t cap);
/* Copy one slice's transmission function t(x,y) to host, 2*nx*ny doubles
 * interleaved re/im, row-major [x][y] as the reference's exp_i_sigma_v. */
msf_status msf_specimen_transmission(const msf_specimen* spec, int32_t slice,
                                     double* out);
/* Bytes of device memory the specimen holds. */
int64_t msf_specimen_device_bytes(const msf_specimen* spec);
/* --paptif (slice.cpp:1660-1690): specimens built by `ctx` after
 * msf_context_keep_potentials(ctx, 1) keep a host copy of every slice's
 * projected potential sigma*V before the exponential (the sum of the
 * scatterers' shifted lookup tables); msf_specimen_potential copies slice
 * `slice`'s 2*nx*ny doubles ([x][y] complex) into `out`, MSF_ERR_ARG when
 * the specimen was built without them. */
msf_status msf_context_keep_potentials(msf_context* ctx, int32_t on);
msf_status msf_specimen_potential(const msf_specimen* spec, int32_t slice, double* out);
/* Columns (ky values) in which the band limit keeps any kx (bw_limit.cpp:
 * 30-47 with the transmission cut-off); the slice passes move no data for
 * the others, which only ever hold zeros between the passes. */
int32_t msf_specimen_live_columns(const msf_specimen* spec);

/* ---- the multislice raster (adfstem) ----------------------------------- */
msf_status msf_run(msf_context* ctx, const msf_specimen* spec,
                   const msf_optics* optics, const msf_raster* raster,
                   const msf_detect* detect, msf_results* results);
/* The same raster as msf_run, computed the plain way: one probe at a time,
 * FP64, one kernel launch per step of the reference's loop
 * (adfstem.cpp:1632-2132: place probe, FFT, / sqrt(NxNy); per slice iFFT,
 * transmission, FFT, / sqrt(NxNy), bw_limit, propagate), no graph.  The
 * comparator the batched path is measured against; FP64 contexts only. */
msf_status msf_run_plain(msf_context* ctx, const msf_specimen* spec,
                         const msf_optics* optics, const msf_raster* raster,
                         const msf_detect* detect, msf_results* results);
/* Normalised real-space probe (adfstem.cpp:586-817), 2*nx*ny doubles. */
msf_status msf_probe(msf_context* ctx, const msf_specimen* spec,
                     const msf_optics* optics, double* out);

/* The probe of msf_probe, to within FP64 rounding (1e-12 of its largest
 * value; the twiddles come from the device's sincospi rather than host
 * cos/sin, so not bit for bit), written into caller-provided device memory
 * (2*nx*ny doubles) on `stream` (a cudaStream_t, NULL for the default
 * stream), allocating no device memory.  No counterpart in the reference.
 * For callers that may not call cudaMalloc (an application that owns all
 * device memory in its own pool, a running loop that must not stall on an
 * allocation).  Its scratch is one fixed device array per device, sized for
 * grids of at most 2048 x 2048; larger grids return MSF_ERR_ARG.  The first
 * call on a device looks up that array's address (cudaGetSymbolAddress,
 * with the device current), and so does every later call made outside a
 * stream capture (a device reset then leaves nothing stale): make the first
 * call on each device before any stream capture.  Calls that overlap on the
 * GPU share the array and race. */
msf_status msf_probe_noalloc(const msf_grid* grid, const msf_optics* optics,
                             double* probe_device, void* stream);

/* ---- launch tiling autotuner (the analogue of the reference's FFTW
 * wisdom, tem.cpp:583-616 and 1748-1765) ---------------------------------- */
typedef struct {
  int32_t nx, ny;             /* grid                                          */
  int32_t batch;              /* probes per launch chosen                      */
  int32_t pipe;               /* slice-pass variants: bit 0 pipelined column
                                 pass, bit 1 pipelined row pass, bit 2 row
                                 pass with staged slice tables (FP32), bit 3
                                 the FP32 split-wave row pass on its
                                 alternative FFT radix schedule, bit 4 the
                                 plain row pass prefetching its tables into
                                 L1, bit 5 the plain row pass prefetching
                                 the wavefield rows of the CTAs one resident
                                 wave ahead into L2 (distance scaled by the
                                 MSF_ROW_AHEAD_PCT environment variable,
                                 percent of a wave, default 100), bit 6 the
                                 plain row pass giving each CTA one row of
                                 consecutive probes                         */
  double ns_per_probe_slice;  /* measured time of the two slice passes        */
} msf_tuning;
/* Times the two slice passes of `spec`'s grid (CUDA events, after a
 * warm-up) for each candidate probes-per-launch (8 .. 256, within half the
 * free memory) and each slice-pass variant the grid supports (pipelined
 * column pass or not; for FP32, staged row pass or not, in either FFT radix
 * schedule, and the plain one with or without its L1 and L2 prefetches);
 * records the fastest per probe*slice
 * in the context, where msf_run / msf_run_md / msf_run_partial use it for
 * that grid unless the context's batch or MSF_PIPE fixes the choice. */
msf_status msf_tune(msf_context* ctx, const msf_specimen* spec, msf_tuning* out);
/* The context's tuning as text, one line per grid ("msf-wisdom 1 <device
 * name> <fp32|fp64> <nx> <ny> <batch> <pipe> <ns>"): returns the length
 * (without the terminating NUL) and copies what fits into buf[cap]. */
int64_t msf_wisdom_export(const msf_context* ctx, char* buf, int64_t cap);
/* Adds the lines of `text` that were measured on this device model and
 * precision to the context's tuning; *n_imported (may be NULL) counts them. */
msf_status msf_wisdom_import(msf_context* ctx, const char* text, int32_t* n_imported);

/* ---- MD-coupled FEM (the reference's ms-stem-fem-md) -------------------- */
/* Replaces the raster loop of ftem_lammps.cpp main (1513-3610, 4077-4990):
 * every probe position is propagated through `samples` configurations of
 * the specimen, sample s through snapshots[s % n_snapshots] (samples must
 * be a multiple of n_snapshots); its exit waves (after the detector MTF
 * when one is given) are averaged coherently, psi_acc += psi / samples
 * (:3601-3610), the ADF image is the average of the samples' ADF signals
 * (:3385-3402), and the FEM statistics, correlograph and pixel means are
 * those of msf_run evaluated on psi_acc (:3686-3990).  The snapshots must
 * share the grid, voltage and lateral cell (x/y periods, duplication and
 * minima); their z extents, atoms and slicing may differ.  final_psi gets
 * the last probe's psi_acc; first_psi is not filled.  probe_slices counts
 * every propagation of every sample. */
msf_status msf_run_md(msf_context* ctx, int32_t n_snapshots,
                      const msf_specimen* const* snapshots, int32_t samples,
                      const msf_optics* optics, const msf_raster* raster,
                      const msf_detect* detect, msf_results* results);

/* ---- one raster sharded over several GPUs ------------------------------ */
/* The reference splits a raster over MPI ranks and reduces the detector
 * sums with MPI_Reduce / MPI_Allgatherv (adfstem.cpp:1556-1606, 2489-2782,
 * 2822-3612).  Here each GPU runs a contiguous range of probes with
 * msf_run_partial, the caller exchanges the per-probe rows (all-gather, in
 * probe order) and the per-pixel sums (sum), and any rank finishes with
 * msf_finish, which needs no GPU. */
/* Segments per probe: FEM ring bins, then the ADF annulus (n_k + 1). */
int32_t msf_segment_count(const msf_grid* grid, const msf_detect* detect);
/* Probes [p_begin, p_end) of the raster (pixel snaps found over the whole
 * raster, as the reference's carried-over search needs).  amp / inten get
 * (p_end - p_begin) rows of msf_segment_count doubles: per segment the sum
 * of |psi(k)| and of |psi(k)|^2; acc_a / acc_i (pixel FEM modes) nx*ny sums
 * of |psi(k)| and |psi(k)|^2 over these probes.  Any output may be NULL.
 * `info` (may be NULL) receives probe_slices, kernel_launches, n_k and
 * seconds_raster. */
msf_status msf_run_partial(msf_context* ctx, const msf_specimen* spec,
                           const msf_optics* optics, const msf_raster* raster,
                           const msf_detect* detect, int64_t p_begin, int64_t p_end,
                           double* amp, double* inten, double* acc_a, double* acc_i,
                           msf_results* info);
/* ADF image and FEM statistics of a whole raster from the rows of all its
 * probes in raster order and the summed pixel sums (host only; the same
 * arithmetic as msf_run's finish). */
msf_status msf_finish(const msf_grid* grid, const msf_optics* optics,
                      const msf_detect* detect, int64_t n_probes, const double* amp,
                      const double* inten, const double* acc_a, const double* acc_i,
                      msf_results* results);

/* ---- one raster over several ranks (the reference's mpirun -np K,
 * tem.cpp:90; probe shares adfstem.cpp:1556-1606; collective sums
 * adfstem.cpp:2256, 2489-2782) ------------------------------------------- */
typedef struct msf_comm msf_comm;
#define MSF_COMM_NCCL 1 /* exchange on device buffers through NCCL (one GPU per rank) */
#define MSF_COMM_HOST 2 /* exchange through the TCP bootstrap (ranks may share a GPU) */
/* Joins `world` ranks (one process each).  Rank 0 listens at `rendezvous`
 * ("host:port", e.g. torchrun's MASTER_ADDR:MASTER_PORT; unused when
 * world == 1), the others connect to it; with MSF_COMM_NCCL every rank then
 * creates an NCCL communicator on `device` (libnccl.so.2 is loaded at this
 * point; MSF_ERR_UNSUPPORTED when it is absent).  Every connection and
 * exchange waits at most `timeout_s` seconds (<= 0: 60) and then returns
 * MSF_ERR_TIMEOUT, so a rank that never joins or stops answering surfaces
 * as an error on the others.  Collective: every rank calls it. */
msf_status msf_comm_create(int32_t rank, int32_t world, const char* rendezvous,
                           int32_t transport, int32_t device, double timeout_s,
                           msf_comm** out);
void msf_comm_destroy(msf_comm* comm);
/* Host all-gather over the bootstrap connections: recv[world * bytes] gets
 * every rank's `bytes` of `send` in rank order.  Collective. */
msf_status msf_comm_allgather_host(msf_comm* comm, const void* send, int64_t bytes,
                                   void* recv);
typedef struct {
  int64_t p_begin, p_end;    /* out: this rank's probes (raster order)        */
  double seconds_shard;      /* out: wall time of this rank's probes           */
  double seconds_exchange;   /* out: wall time of the exchange                 */
  double seconds_finish;     /* out: wall time of the host finish              */
} msf_shard_info;
/* msf_run over the communicator's ranks: each rank runs a contiguous share
 * of the probes (sizes differ by at most one, lower ranks first), then one
 * exchange step all-gathers the per-probe detector rows and the per-pixel
 * sums of the FEM pixel modes (added in rank order on every rank), and
 * every rank finishes the same ADF image, FEM statistics and correlograph
 * into `results`; first_psi is filled on rank 0 and final_psi (the last
 * probe's exit wave, sent on from the rank that ran it) on every rank.
 * probe_slices,
 * kernel_launches, seconds_raster and the pass times describe this rank's
 * share.  With world == 1 the outputs equal msf_run's bit for bit.
 * Collective: every rank calls it with the same raster, detector and set
 * of output buffers; `info` may be NULL. */
msf_status msf_run_sharded(msf_context* ctx, const msf_specimen* spec,
                           const msf_optics* optics, const msf_raster* raster,
                           const msf_detect* detect, msf_comm* comm, msf_results* results,
                           msf_shard_info* info);

/* ---- slot batches and serving (no counterpart in the reference) -------- */
/* Several rasters at once: results[i] is what msf_run(ctx, specs[i],
 * &optics[i], &rasters[i], &detects[i], &results[i]) returns, within FP32
 * rounding (final_psi is not filled).  Rasters of the same grid size share
 * launches: each of `slots` wavefields (0: about 2 GiB of wavefields,
 * 16..256, bounded by free memory) carries one probe of any raster at its
 * own slice, and a slot whose
 * probe finished is refilled with the next waiting probe.  Grid sizes run as
 * separate lanes on separate streams that overlap on the GPU.  FP32 contexts
 * only.  results[i].seconds_raster is the device time from the start of the
 * batch to the completion of raster i; kernel_launches counts the launches
 * of its lane. */
msf_status msf_run_batch(msf_context* ctx, int32_t n, const msf_specimen* const* specs,
                         const msf_optics* optics, const msf_raster* rasters,
                         const msf_detect* detects, msf_results* results,
                         int32_t slots);

/* A simulation request: everything is copied at submission. */
typedef struct {
  msf_grid grid;
  msf_atoms atoms;
  msf_optics optics;
  msf_raster raster;
  msf_detect detect;
} msf_request;

typedef struct {
  int64_t submitted, completed, failed, running, waiting; /* failed: incl. cancelled */
  double p50_s, p99_s, max_s;  /* latency, submission to completion         */
  double probe_slices_per_s;   /* completed probe*slices / busy wall time    */
  int64_t probe_slices;
  int64_t device_bytes;        /* bytes the server holds now                */
} msf_server_stats;

typedef struct msf_server msf_server;
/* A request loop on one GPU (FP32 wavefields).  A worker thread admits
 * requests in arrival order whose estimated device bytes fit
 * `opt->hbm_budget` (0: 80 % of free memory; a request that does not fit
 * lets later ones past it for 5 s, then holds them back until it fits),
 * builds each specimen (smallest first, unless one has waited 5 s), and
 * feeds its probes into the slot lane of its grid size (`slots` wavefields
 * per lane; 0: about 2 GiB of wavefields, 16..256, by grid size); requests
 * that arrive while others run join the running launches as slots free up,
 * a lane shares its slots fairly among its rasters, and lanes of smaller
 * grids run on higher-priority streams. */
msf_status msf_server_create(const msf_options* opt, int32_t slots, msf_server** out);
/* Queue a request; returns at once with its ticket. */
msf_status msf_server_submit(msf_server* srv, const msf_request* req, uint64_t* ticket);
/* MSF_OK and the results (as msf_run fills them) when the request finished,
 * MSF_ERR_BUSY while it is queued or running after waiting up to wait_ms,
 * or the request's error status.  A finished request is forgotten after its
 * first successful poll. */
msf_status msf_server_poll(msf_server* srv, uint64_t ticket, int32_t wait_ms,
                           msf_results* results);
msf_status msf_server_stats_get(msf_server* srv, msf_server_stats* out);
/* Latency of the completed requests per grid size (submission to
 * completion, as msf_server_stats): fills up to `cap` entries in order of
 * grid size and returns how many grid sizes have completed requests. */
typedef struct {
  int32_t nx, ny;
  int64_t completed;
  double p50_s, p99_s, max_s;
} msf_server_grid_stats;
int32_t msf_server_grid_stats_get(msf_server* srv, msf_server_grid_stats* out, int32_t cap);
/* Cancels a request: one still waiting for admission is dropped at once;
 * one already admitted runs to the end of its probes (they share launches
 * with other requests) and its results are discarded; a finished one not
 * yet polled loses its results.  Its poll then returns MSF_ERR_CANCELLED.
 * MSF_ERR_ARG for an unknown, delivered or already cancelled ticket. */
msf_status msf_server_cancel(msf_server* srv, uint64_t ticket);
/* Finishes the running and queued requests, then stops the worker. */
msf_status msf_server_destroy(msf_server* srv);

/* ---- host-side set-up helpers (bit-exact with the reference) ----------- */
/* lambda [A] and gamma for an accelerating voltage (tem.cpp:424-438). */
void msf_wavelength(double voltage, double* lambda, double* gamma);
/* Scherzer conditions (scherzer.cpp:61-168); which: 0 defocus_uncorrected,
 * 1 alphamax_uncorrected, 2 defocus_corrected, 3 alphamax_corrected,
 * 4 cs3_corrected.  `aberration` is Cs3 (0,1) or Cs5 (2,3,4). */
double msf_scherzer(int32_t which, double lambda, double aberration);
/* Raster positions (func.cpp:108-127): n = floor(period/spacing). */
int32_t msf_raster_points(double period, double origin, double spacing,
                          double* out, int32_t cap);
/* Pixel snap of each raster probe with the reference's carried-over search
 * (adfstem.cpp:1590-1606); shifts[2*k] = sx, [2*k+1] = sy in raster order. */
msf_status msf_probe_shifts(const msf_grid* grid, const msf_raster* raster,
                            int64_t* shifts);
/* Ring bin of every pixel (-1 outside all bins) and bin count for --dr. */
msf_status msf_ring_bins(const msf_grid* grid, double dr, int32_t* bins,
                         int32_t* n_k);
/* Slicing alone (slice.cpp:469-980): host only.  order[n] receives atom
 * indices in slice order; lower/thickness/counts hold up to `cap` slices. */
msf_status msf_slice_atoms(int64_t n_atoms, const double* q, double zmin,
                           double zperiod, double min_slice, int32_t* n_slices,
                           double* lower, double* thickness, int64_t* counts,
                           int64_t* order, int32_t cap);

/* ---- specimen generator (no counterpart in the reference) -------------- */
/* Seeded amorphous positions: random sequential addition of n_atoms points
 * uniform in [0, box[0]) x [0, box[1]) x [0, box[2]) with a minimum periodic
 * separation min_sep [A]; proposals from std::mt19937_64(seed) mapped to
 * doubles as (x >> 11) * 2^-53.  q receives 3*n_atoms coordinates.  Fails
 * with MSF_ERR_ARG when max_proposals (0: 1000 per atom) run out first. */
msf_status msf_amorphous_positions(int64_t n_atoms, const double* box, double min_sep,
                                   uint64_t seed, int64_t max_proposals, double* q);

/* ---- measurement hook (no counterpart in the reference) ---------------- */
/* Time the two fused slice passes on a resident batch of `nb` wavefields:
 * `reps` launches of each, CUDA events on the context's stream around each
 * launch; returns the mean milliseconds per launch of the row pass and of
 * the column pass. */
msf_status msf_time_passes(msf_context* ctx, const msf_specimen* spec,
                           int32_t nb, int32_t reps, double* ms_row,
                           double* ms_col);

/* ---- drop-in front end -------------------------------------------------- */
typedef struct msf_job msf_job;   /* parsed command line + specimen         */
/* Parse argv exactly as ms-stem-fem does (tem.cpp:81-403): options,
 * --parameter_file, flag checks, specimen file, defaults.  On failure the
 * returned status is non-zero and msf_last_error() holds the message the
 * reference would print. */
msf_status msf_parse_cmdline(int32_t argc, const char* const* argv,
                             msf_job** out);
msf_status msf_job_destroy(msf_job* job);
/* Views into a parsed job (valid until msf_job_destroy). */
msf_status msf_job_describe(const msf_job* job, msf_grid* grid,
                            msf_atoms* atoms, msf_optics* optics,
                            msf_raster* raster, msf_detect* detect);
const char* msf_job_output_prefix(const msf_job* job); /* incl. _adfstem_* */
/* Read a LAMMPS data or .xyz specimen; the arrays are owned by the job. */
msf_status msf_read_specimen(const char* path, msf_job** out);
/* Write the reference's output files for a finished run: <prefix>_fem_*.txt
 * and <prefix>_stem_image_output{,_logscale}.tif (+ raw .f64 image). */
msf_status msf_write_outputs(const msf_job* job, const msf_results* res);
/* The whole drop-in program: parse, build, run, write.  Returns the process
 * exit status the reference would return (0 success, 1 failure). */
int32_t msf_main(int32_t argc, const char* const* argv,
                 const msf_options* opt);
/* The drop-in ms-stem-fem-md program (ftem_lammps.cpp main), argv as the
 * reference's, with LAMMPS replaced by a replay of LAMMPS data files: the
 * pre-TEM file's read_data gives the initial configuration (and the cell),
 * its tersoff / sw / eam pair_coeff line the element of each atom type, and
 * the i-th "run" of the MD loads entry (i - 1) mod K of the list that
 * `--md_replay <file>` names (one data file per line; with
 * --lammps_TEM_steps 0 nothing runs and every sample sees the initial
 * configuration).  lammps_TEM_samples must be a multiple of K.  Outputs go
 * under the plain output prefix, as there. */
int32_t msf_md_main(int32_t argc, const char* const* argv,
                    const msf_options* opt);

#ifdef __cplusplus
}
#endif
#endif /* MSF_H */
