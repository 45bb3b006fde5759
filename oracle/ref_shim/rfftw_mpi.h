/* rfftw_mpi.h -- TEST INFRASTRUCTURE ONLY.  Stand-in for the FFTW 2.x MPI real
 * multi-dimensional transforms the reference calls (fft_solver.cpp:17-42) on one
 * rank: rfftw3d_mpi_create_plan, rfftwnd_mpi_local_sizes, rfftwnd_mpi and
 * rfftwnd_mpi_destroy_plan with FFTW's conventions -- in-place on a real
 * [nx][ny][2(nz/2+1)] array, unnormalised, forward sign e^{-ikx}, the complex
 * result in transposed order [ny][nx][nz/2+1], and the inverse taking the
 * half-complex form along z (no imaginary part at kz = 0 and nz/2).  The
 * transforms themselves are project-written (ref_shim/shim.cpp); only the API
 * names and argument lists follow FFTW 2.x. */
#ifndef REF_SHIM_RFFTW_MPI_H
#define REF_SHIM_RFFTW_MPI_H
#include "mpi.h"

typedef double fftw_real;
typedef enum { FFTW_REAL_TO_COMPLEX = -1, FFTW_COMPLEX_TO_REAL = 1 } fftw_direction;
typedef enum { FFTW_NORMAL_ORDER = 0, FFTW_TRANSPOSED_ORDER = 1 } fftwnd_mpi_output_order;
#define FFTW_ESTIMATE 0
#define FFTW_MEASURE 1

typedef struct ref_rfftw_plan* rfftwnd_mpi_plan;

#ifdef __cplusplus
extern "C" {
#endif
rfftwnd_mpi_plan rfftw3d_mpi_create_plan(MPI_Comm comm, int nx, int ny, int nz, fftw_direction dir, int flags);
void rfftwnd_mpi_local_sizes(rfftwnd_mpi_plan p, int* local_nx, int* local_x_start, int* local_ny_after_transpose,
                             int* local_y_start_after_transpose, int* total_local_size);
void rfftwnd_mpi(rfftwnd_mpi_plan p, int n_fields, fftw_real* local_data, fftw_real* work,
                 fftwnd_mpi_output_order output_order);
void rfftwnd_mpi_destroy_plan(rfftwnd_mpi_plan p);
#ifdef __cplusplus
}
#endif
#endif
