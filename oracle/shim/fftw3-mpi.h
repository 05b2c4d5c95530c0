/* Stand-in for the subset of FFTW 3.3.10 + fftw3-mpi that SPM-IQC calls.
 * TEST INFRASTRUCTURE ONLY (the CPU oracle): it lets the reference's own
 * src/*.cpp compile unchanged. FFTW itself is not vendored by the reference
 * (makefile:2 points at a cluster install), so the transform under this header
 * is a project-written FP64 complex DFT (shim_fft.cpp) that implements FFTW's
 * published definition: FFTW_FORWARD = exp(-2 pi i jk/n), FFTW_BACKWARD =
 * exp(+2 pi i jk/n), both unnormalised, row-major 3D, in place.
 *
 * Call sites served: src/My_FFT.cpp:33-127 (plans, wisdom, execute);
 * src/LPsrc.cpp:126,142; src/LOBPCG.cpp:122,133,171,184 (fftw_execute);
 * fftw_free of malloc'd buffers everywhere (so fftw_free == free).
 */
#ifndef SPMIQC_ORACLE_SHIM_FFTW3_MPI_H
#define SPMIQC_ORACLE_SHIM_FFTW3_MPI_H

#include <stddef.h>
#include "mpi.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct spm_shim_plan *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_PATIENT (1U << 5)
#define FFTW_WISDOM_ONLY (1U << 21)

void *fftw_malloc(size_t n);
fftw_complex *fftw_alloc_complex(size_t n);
void fftw_free(void *p);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

void fftw_mpi_init(void);
ptrdiff_t fftw_mpi_local_size_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2,
                                 MPI_Comm comm, ptrdiff_t *local_n0,
                                 ptrdiff_t *local_0_start);
fftw_plan fftw_mpi_plan_dft_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2,
                               fftw_complex *in, fftw_complex *out, MPI_Comm comm,
                               int sign, unsigned flags);
void fftw_mpi_broadcast_wisdom(MPI_Comm comm);
int fftw_import_wisdom_from_filename(const char *filename);
int fftw_export_wisdom_to_filename(const char *filename);

/* Oracle-only controls (not FFTW API): worker threads used by fftw_execute. */
void spm_shim_fft_set_threads(int nthreads);
int spm_shim_fft_get_threads(void);

#ifdef __cplusplus
}
#endif

#endif
