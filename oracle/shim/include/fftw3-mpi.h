/* FFTW3-MPI shim (TEST INFRASTRUCTURE), single rank.  Layouts follow FFTW's
 * documented conventions: an r2c with FFTW_MPI_TRANSPOSED_OUT writes
 * [n1][n0][n2/2+1]; a c2r with FFTW_MPI_TRANSPOSED_IN reads that layout and
 * writes real data padded to 2*(n2/2+1) per row; "many" transforms interleave
 * `howmany` components element by element. */
#ifndef SHIM_FFTW3_MPI_H
#define SHIM_FFTW3_MPI_H
#include "fftw3.h"
#include "mpi.h"
#define FFTW_MPI_DEFAULT_BLOCK 0
#define FFTW_MPI_TRANSPOSED_IN (1U << 29)
#define FFTW_MPI_TRANSPOSED_OUT (1U << 30)
#ifdef __cplusplus
extern "C" {
#endif
void fftw_mpi_init(void);
ptrdiff_t fftw_mpi_local_size_many_transposed(int rnk, const ptrdiff_t* n, ptrdiff_t howmany, ptrdiff_t block0,
                                              ptrdiff_t block1, MPI_Comm comm, ptrdiff_t* local_n0,
                                              ptrdiff_t* local_0_start, ptrdiff_t* local_n1,
                                              ptrdiff_t* local_1_start);
fftw_plan fftw_mpi_plan_dft_r2c_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, double* in, fftw_complex* out,
                                   MPI_Comm comm, unsigned flags);
fftw_plan fftw_mpi_plan_dft_c2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, fftw_complex* in, double* out,
                                   MPI_Comm comm, unsigned flags);
fftw_plan fftw_mpi_plan_many_dft_c2r(int rnk, const ptrdiff_t* n, ptrdiff_t howmany, ptrdiff_t block0,
                                     ptrdiff_t block1, fftw_complex* in, double* out, MPI_Comm comm, unsigned flags);
#ifdef __cplusplus
}
#endif
#endif
