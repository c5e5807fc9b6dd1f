/* CPU restatement of the reference's multislice ADF-STEM / FEM path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA path is checked
 * against: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it, and only as the checker.  Plain FP64 C, one thread, no
 * tricks; every routine cites the reference file:line it restates.
 *
 * Parity pin: the restatement is itself checked against the reference's own
 * sources compiled in this container (oracle/Makefile -> oracle/_ref/) on
 * seeded specimens; the committed golden fixtures under tests/golden/ come
 * from those runs. */
#ifndef MSF_ORACLE_H
#define MSF_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Output selection bits for or_job.flags. */
#define OR_ADF 1u      /* --images: ADF image (adfstem.cpp:2245-2267)     */
#define OR_D1 2u       /* --V_omega      (adfstem.cpp:2585-2601, 2822)    */
#define OR_D2 4u       /* --Vbar_r       (adfstem.cpp:2688-2750, 2870)    */
#define OR_D3 8u       /* --V_re         (adfstem.cpp:3324-3466)          */
#define OR_D4 16u      /* --Omega_vimage (adfstem.cpp:3468-3612)          */
#define OR_GT17 32u    /* --V_gt17       (adfstem.cpp:3169-3321)          */
#define OR_RVA 64u     /* --V_rbar       (adfstem.cpp:3324-3466)          */

typedef struct {
  int32_t nx, ny;                 /* -m samples                                 */
  double voltage;                 /* -m VV [V]                                  */
  double xperiod, yperiod;        /* specimen periods (raster uses these)       */
  double xperiod_duped, yperiod_duped; /* periods of the simulated cell         */
  double xmin, ymin;              /* domain origin                              */
  double min_slice;               /* --minslice                                 */
  int32_t corrected;              /* 0: --adfstemuncorr*, 1: --adfstemcorr*     */
  double cs3, cs5, defocus, alpha_max; /* optics (defocus/alpha already chosen) */
  double det_inner, det_outer;    /* detector angles [rad]                      */
  double dr;                      /* --dr azimuthal_binning_size_factor         */
  int32_t n_rx, n_ry;             /* raster counts                              */
  const double* x_p;              /* n_rx raster x positions                    */
  const double* y_p;              /* n_ry raster y positions                    */
  uint32_t flags;                 /* OR_* bits                                  */
} or_job;

typedef struct {
  int64_t n_atoms;
  const double* q;                /* 3*n_atoms, x y z per atom                  */
  const uint32_t* z;              /* atomic numbers                             */
} or_atoms;

typedef struct {
  double* adf_image;              /* n_rx*n_ry, [px*n_ry + py] (or NULL)        */
  int32_t cap_k;                  /* capacity of each k array below             */
  int32_t n_k;                    /* out: number of k bins                      */
  double* k_lower;                /* out: lower bin boundary per bin            */
  double* v_omega, *vbar_r, *v_re, *omega_vimage, *v_gt17, *v_rbar;
  int32_t* bin_counts;            /* out: pixels per bin (or NULL)              */
  double* last_psi;               /* out: 2*nx*ny final k-space wave of the
                                     last probe, interleaved re/im (or NULL)    */
  int32_t n_slices;               /* out                                        */
} or_result;

/* tem.cpp:424-438 */
void or_constants(double voltage, double* lambda, double* gamma);
/* Slicing, slice.cpp:469-980.  order[n] receives atom indices in slice order,
 * start[] (capacity n+1) the first position of each slice in order[], lower[]
 * and thick[] (capacity n) the slice boundaries.  Returns the slice count. */
int64_t or_slice_atoms(int64_t n, const double* q, double zmin, double zperiod,
                       double min_thickness, int64_t* order, int64_t* start,
                       double* lower, double* thick);
/* Nearest-pixel snap used for atoms (slice.cpp:1556-1572) and probes
 * (adfstem.cpp:1590-1606): (first i with grid[i] - q >= half) - 1, else
 * `fallback`.  Returns -1 where the reference's size_t would wrap. */
int64_t or_snap(const double* grid, int64_t n, double q, double half,
                int64_t fallback);
/* Whole raster job: specimen -> slices -> transmission functions -> probe ->
 * every probe through every slice -> ADF and FEM outputs.  Returns 0 on
 * success. */
int or_run(const or_job* job, const or_atoms* atoms, or_result* out);
/* Transmission function of one slice after the full build (slice.cpp:1451),
 * 2*nx*ny interleaved.  Returns 0 on success. */
int or_transmission(const or_job* job, const or_atoms* atoms, int32_t slice,
                    double* t_out);
/* FEM ring bin of every pixel (-1 outside), pixels per bin and lower bin
 * boundaries (adfstem.cpp:947-1062, variance.cpp:64-300); returns n_k. */
int32_t or_ring_bins(const or_job* job, int32_t* bins_out, int32_t* counts_out,
                     double* bounds_out, int32_t cap);
/* Normalised real-space probe (adfstem.cpp:586-817), 2*nx*ny interleaved. */
int or_probe(const or_job* job, double* probe_out);

#ifdef __cplusplus
}
#endif
#endif
