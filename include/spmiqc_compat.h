/* spmiqc_compat.h -- link-time drop-in for SPM-IQC's hot-path routines.
 *
 * libspmiqc_compat.so defines the reference's own C++ functions with the
 * reference's signatures, so a program built from the reference's drivers
 * (main_SPM.cpp, grad.cpp) links against it instead of the objects of
 * src/My_FFT.cpp, src/LPsrc.cpp, src/LOBPCG.cpp and src/SPM.cpp. Each call
 * reads the reference's process globals (src/Data.cpp: N, L, Tau, Gamma, dt,
 * max_iter, u_R_local, u_F_local, tv, ...), copies the fields to the GPU,
 * runs the sm_100a implementation (libspmiqc_cuda.so, spmiqc.h) and writes the
 * results back into the reference's buffers and globals.
 *
 * The globals stay defined by the reference's Data.cpp (or by the program);
 * this header only declares the ones the drop-in reads or writes, with the
 * types of include/Data.h.
 *
 * Limits of the drop-in:
 *  - one MPI rank: the GPU holds the whole field (numprocs must be 1);
 *  - fields passed as fftw_complex are real (imaginary parts ignored), as they
 *    are everywhere in the reference; spectra are full N^3 complex arrays;
 *  - grid sizes of spm_supported_size();
 *  - hiosd_lobpcg_initialization draws its start block from a SplitMix64
 *    stream (seed from the environment variable SPMIQC_LOBPCG_SEED, default 0)
 *    instead of Eigen's unseeded MatrixXd::Random.
 */
#ifndef SPMIQC_COMPAT_H
#define SPMIQC_COMPAT_H

#include <stddef.h>

typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;

/* include/Data.h:29-41 */
struct Option {
  int k;
  int maxiter;
  int outputp;
  int outputd;
  double dt;
  double epsf;
  double betat;
  double betau;
  fftw_complex **V;
};

/* Globals of src/Data.cpp read or written by the drop-in. */
extern int N, CplxDofs, CplxDofs_local, max_iter, myid, numprocs;
extern double L, Tau, Gamma, dt;
extern fftw_complex *u_R_local, *u_F_local, *tv, *data;
extern ptrdiff_t alloc_local, local_n0, local_0_start;
extern fftw_plan plan1, plan2;

/* My_FFT.h:10-14 */
void my_fft(fftw_complex *x_R_local, fftw_complex *x_F_local);
void my_ifft(fftw_complex *x_F_local, fftw_complex *x_R_local);
void My_mpi_fft_set_up();

/* LPsrc.h:5-7 */
double get_Ene();
void get_min_u_F();
void ngrad_cam(fftw_complex *phir, fftw_complex *gradr);

/* LOBPCG.h:7-10 */
void hv_cam(fftw_complex *phir, fftw_complex *v, fftw_complex *hv);
void precond_camnew(fftw_complex *w);
void hiosd_lobpcg_initialization(Option *option, int ki);
void hiosd_lobpcg_inip(fftw_complex *x, Option *option);
void copy_option_V(Option *option1, Option *option2, int k);  /* LOBPCG.cpp:489-520 */
void copy_option_V(fftw_complex **V, Option *option2, int k);
void copy_option_V(fftw_complex *v, Option *option2, int k);

/* SPM.h:7-9 and SPM.cpp:103 (MinMax_Forces is not in SPM.h) */
void get_Tv(fftw_complex **Phi, fftw_complex *v);
void Natural_Forces(fftw_complex *x, fftw_complex *v);
void MinMax_Forces(fftw_complex *x, fftw_complex *v);
void Spring_Pairing(fftw_complex **Phi, double maxiter, double tol);
void Gs_gri_nuc(fftw_complex *v_loc, fftw_complex *phi_loc);  /* SPM.cpp:265-300 (host) */

/* Releases the drop-in's GPU context (optional; also released at exit). */
extern "C" void spmiqc_compat_release(void);

#endif /* SPMIQC_COMPAT_H */
