/* Stand-in for the FFTW-MPI API subset the reference calls (test
 * infrastructure).  With one rank the local slab is the whole grid. */
#ifndef MSF_ORACLE_SHIM_FFTW3_MPI_H
#define MSF_ORACLE_SHIM_FFTW3_MPI_H
#include <stddef.h>
#include <mpi.h>
#include "fftw3.h"

#ifdef __cplusplus
extern "C" {
#endif
void fftw_mpi_init(void);
void fftw_mpi_cleanup(void);
ptrdiff_t fftw_mpi_local_size_2d(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm comm,
                                 ptrdiff_t* local_n0, ptrdiff_t* local_0_start);
fftw_plan fftw_mpi_plan_dft_2d(ptrdiff_t n0, ptrdiff_t n1, fftw_complex* in,
                               fftw_complex* out, MPI_Comm comm, int sign,
                               unsigned flags);
void fftw_mpi_broadcast_wisdom(MPI_Comm comm);
void fftw_mpi_gather_wisdom(MPI_Comm comm);
#ifdef __cplusplus
}
#endif
#endif
