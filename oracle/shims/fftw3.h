/* Stand-in for the FFTW 3 API subset the reference calls (test infrastructure).
 *
 * FFTW itself is absent from this machine.  The transforms follow FFTW's
 * documented definition: FFTW_FORWARD computes X[k] = sum_n x[n] e^{-2 pi i nk/N},
 * FFTW_BACKWARD uses e^{+2 pi i nk/N}; neither is normalised.  Planner flags
 * are accepted and ignored; wisdom calls report "no wisdom". */
#ifndef MSF_ORACLE_SHIM_FFTW3_H
#define MSF_ORACLE_SHIM_FFTW3_H
#include <stddef.h>

typedef double fftw_complex[2];
typedef struct msf_shim_plan* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_WISDOM_ONLY (1U << 21)

#ifdef __cplusplus
extern "C" {
#endif
fftw_complex* fftw_alloc_complex(size_t n);
void fftw_free(void* p);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
int fftw_import_wisdom_from_filename(const char* filename);
int fftw_export_wisdom_to_filename(const char* filename);
#ifdef __cplusplus
}
#endif
#endif
