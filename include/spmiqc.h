/* spmiqc.h -- C ABI of the B200 (sm_100a) implementation of SPM-IQC's
 * pseudo-spectral hot path (libspmiqc_cuda.so).
 *
 * The reference (JKGroupCUDA/SPM-IQC) has no plugin API: its hot path is a set
 * of free C++ functions over process globals. Each entry point below names the
 * reference routine it replaces (file:line within the SPM-IQC project). The
 * C++ signatures themselves are kept by the link-time compat layer declared in
 * spmiqc_compat.h.
 *
 * Conventions
 *  - Every function returns an int status (SPM_OK = 0, else SPM_ERR_*); the
 *    reference returns void and aborts on MPI errors. spm_last_error() gives
 *    a message for the calling thread.
 *  - A context owns one grid size N, the model parameters and its scratch; it
 *    is bound to one CUDA device and one stream and is not re-entrant (one
 *    context per thread), like the reference's globals.
 *  - "Field" arguments are device pointers to real arrays of N^3 values of the
 *    context's precision (double for SPM_FP64, float for SPM_FP32), row-major
 *    i*N*N + j*N + k, the reference's index order (Initialization.cpp:109-120).
 *    Batched entry points take nb fields stored back to back.
 *  - "Spectrum" arguments are device pointers to the packed half spectrum:
 *    N*N*(N/2) complex values (re, im interleaved), spec[(kx*N + ky)*(N/2) + c]
 *    = X(kx, ky, c) for c >= 1 and X(kx, ky, 0) + i X(kx, ky, N/2) for c = 0,
 *    where X is the reference's spectrum, normalised by 1/N^3
 *    (My_FFT.cpp:4-13). spm_spectrum_to_full / _from_full convert to and from
 *    the reference's full N^3 complex layout.
 *  - Norms and inner products follow inpfp/nrmp: <p,q> = (1/N^3) sum p q
 *    (BasicOperators.cpp:132-172); ||grad F|| = nrmp(ngrad_cam(phi)).
 *  - Functions run asynchronously on the context's stream unless they return a
 *    host scalar, in which case they synchronise the stream.
 */
#ifndef SPMIQC_H
#define SPMIQC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct spm_ctx spm_ctx;

enum spm_status {
  SPM_OK = 0,
  SPM_ERR_ARG = 1,          /* bad argument (size, null pointer, batch) */
  SPM_ERR_CUDA = 2,         /* a CUDA runtime error */
  SPM_ERR_NOMEM = 3,        /* device allocation refused */
  SPM_ERR_NONFINITE = 4,    /* a reduction returned NaN/Inf */
  SPM_ERR_UNSUPPORTED = 5,  /* grid size or precision not built */
  SPM_ERR_STATE = 6,        /* call order (e.g. LOBPCG block not initialised) */
  SPM_ERR_CANCELLED = 7     /* a job was cancelled (job server) */
};

/* Contexts take SPM_FP64 or SPM_FP32; SPM_MIXED is a job precision of the job
 * server (FP32 transforms to a switch tolerance, then an FP64 polish). */
enum spm_precision { SPM_FP64 = 0, SPM_FP32 = 1, SPM_MIXED = 2 };

/* Per-step record of a gradient-flow run (LPsrc.cpp:52-110). */
typedef struct spm_step_stats {
  double energy;    /* get_Ene() of the state entering the step (LPsrc.cpp:54) */
  double res;       /* max_k |Re(u'_k - u_k)| (LPsrc.cpp:77-84) */
  double grad_norm; /* nrmp(ngrad_cam(phi)) of the state entering the step */
  double e1;        /* the pair-interaction part 1/2 sum G |u|^2 */
} spm_step_stats;

/* ---------------------------------------------------------------- context */

/* Creates a context for an N^3 grid. Replaces the set-up of main_SPM.cpp:29-60
 * (LPsystParameter, get_kindex_all, My_mpi_fft_set_up, get_ksquare_local,
 * get_epmckt2_local, get_ikt2_local): k^2, G(k) and the preconditioner symbol
 * are evaluated inside the kernels, so no tables are built. stream may be NULL
 * (the legacy default stream). N must satisfy spm_supported_size(N). */
int spm_ctx_create(int N, double L, double Tau, double Gamma, double dt, int precision,
                   void *stream, spm_ctx **out);
int spm_ctx_destroy(spm_ctx *ctx);
int spm_set_stream(spm_ctx *ctx, void *stream);
int spm_sync(spm_ctx *ctx);
int spm_supported_size(int N);
size_t spm_field_bytes(const spm_ctx *ctx);
size_t spm_spectrum_bytes(const spm_ctx *ctx);
const char *spm_status_str(int status);
/* Tuning knobs (no counterpart in the reference; the analogue of FFTW's plan
 * choice, My_FFT.cpp:49-97). knob "plane_cps": 1 = plane kernels stage their
 * input in shared memory (one CTA per SM), 2 = direct loads, two CTAs per SM,
 * 3 = direct loads, three CTAs per SM (fewer registers per thread), 4 = four
 * CTAs per SM for the exchanges through L2 of FP32 gradient chains (3
 * elsewhere), 5 = CTAs of 16 rows and 128 threads, four per SM, for gradient
 * chains with both exchanges through L2 (2 elsewhere), 6 = as 5 with the
 * fused plane pass software-pipelined over x-planes (each exchange's cluster
 * barrier split into arrive and wait with a neighbouring plane's work in
 * between; the same bits).
 * knob "fuse_planes": 1 (default) = chains of gradient steps join each step's
 * inverse plane pass with the next step's forward one (phi stays on chip
 * between steps; the same bits as 0), 0 = three passes per step.
 * knob "plane_xg" (0..3, plane_cps 2 to 6): the plane kernels of
 * gradient chains exchange the x-plane between the CTAs of a cluster through
 * distributed shared memory (0) or through per-CTA areas in global memory that
 * stay resident in L2 (bit 1: the forward exchange, bit 2: the inverse one;
 * the same bits either way). Nonzero allocates the areas (4 x resident CTAs x
 * 16 N complex values).
 * knob "pencil_tc" (8 or 4): the width in spectral columns of the pencil
 * passes' tiles; 4 halves a CTA's shared memory and threads so that several
 * CTAs share an SM (the same bits either way).
 * knob "batch_group" (1 or 0): spm_batch_grad_flow lets instances of the same
 * N and precision share every launch (1) or gives each its own (0).
 * knob "block_stage" (1 or 0): the LOBPCG block kernels (Grams, combinations
 * of more than 8 fields) stage their fields through shared memory with bulk
 * copies (1) or load them directly (0).
 * knob "pdl" (0 or 1): 1 = the plane and pencil kernels are launched as
 * programmatic dependents (in a stream capture, programmatic edges of the
 * graph): a launch may be set up while the previous kernel of the stream
 * completes, and its kernel waits on the device for that kernel before its
 * first memory access; 0 (default) = plain stream order. The same bits
 * either way; spm_autotune turns it on where it is at least 1 % faster.
 * spm_tune_get returns the current value or -1 for an unknown knob. */
int spm_tune(spm_ctx *ctx, const char *knob, int value);
int spm_tune_get(const spm_ctx *ctx, const char *knob);
/* Autotuner (no counterpart in the reference): times chains of `steps`
 * gradient steps on a scratch field for each candidate schedule (plane_cps
 * 1/2/3 with fused chains, plane_cps 2 without, plane_xg 1/2/3 with plane_cps
 * 2 and 3 on fused chains, plane_cps 4 for FP32, 5, 6; then pencil_tc 4 and
 * pdl 1 for the best of them), keeping a later candidate only if it is at least 1 % faster, and
 * keeps the fastest in the context; the choice is remembered per (device, N, precision), so later
 * contexts of the same kind take it without timing (FP32 twins of mixed flows
 * included). Synchronises; allocates two scratch fields while it runs. The
 * chosen knobs are returned in *plane_cps, *fuse_planes (may be NULL);
 * spm_tune_get(ctx, "plane_xg") gives the exchange route. */
int spm_autotune(spm_ctx *ctx, int steps, int *plane_cps, int *fuse_planes);
const char *spm_last_error(void);
/* Number of transform-kernel launches issued by this context so far. */
uint64_t spm_launch_count(const spm_ctx *ctx);
/* Failure-path self-test (no counterpart in the reference, which has no
 * device code): launches one CTA whose mbarrier wait cannot complete (an
 * arrival expecting 16 bytes with no copy issued) and gives it a limit of
 * `polls` polls of ~256 ns (1 <= polls <= 2^22, the limit every transform
 * kernel's waits use). The wait gives up, sets the context's error word and
 * the kernel returns; the call synchronises the stream and returns what every
 * entry point returns after such a timeout: SPM_ERR_CUDA with the message "a
 * kernel's bounded wait for its asynchronous copies timed out". The error
 * word is cleared by that read and the context stays usable. */
int spm_selftest_bounded_wait(spm_ctx *ctx, int polls);

/* ------------------------------------------------------------- transforms */

/* my_fft (My_FFT.cpp:4-13): xhat = FFT(x) / N^3, packed. */
int spm_fft(spm_ctx *ctx, const void *x, void *xhat);
/* my_ifft (My_FFT.cpp:15-21): x = unnormalised inverse of xhat. */
int spm_ifft(spm_ctx *ctx, const void *xhat, void *x);
/* Packed spectrum <-> the reference's full N^3 complex spectrum
 * (fftw_complex, interleaved, always double). */
int spm_spectrum_to_full(spm_ctx *ctx, const void *xhat, double *full);
int spm_spectrum_from_full(spm_ctx *ctx, const double *full, void *xhat);

/* ------------------------------------------------------ energy / gradient */

/* get_Ene (LPsrc.cpp:8-38) on the state (phi, uhat) as given. */
int spm_energy(spm_ctx *ctx, const void *phi, const void *uhat, double *energy);

/* get_min_u_F (LPsrc.cpp:40-117): up to max_steps semi-implicit steps on
 * (phi, uhat) in place. The loop stops after the step whose res <= 1e-16 (the
 * reference's criterion) or, when tol_grad > 0, after the first step whose
 * incoming state has ||grad F|| <= tol_grad. stats (host, may be NULL) receives
 * one record per executed step; *steps_done the number of steps executed.
 * Steps are enqueued ahead in chunks and stop on the device, so no host round
 * trip happens per step. */
int spm_grad_flow(spm_ctx *ctx, void *phi, void *uhat, int max_steps, double tol_grad,
                  spm_step_stats *stats, int *steps_done);

/* Mixed-precision get_min_u_F (no counterpart in the reference): on an FP64
 * context, runs the flow with FP32 transforms (FP64 reductions) until
 * ||grad F|| <= max(switch_tol, tol_grad) or until 512 FP32 steps bring no
 * new minimum of ||grad F|| (the FP32 rounding floor), then continues in FP64
 * from that state (phi cast to FP64, uhat = my_fft(phi)) until
 * ||grad F|| <= tol_grad. switch_tol = 0 runs FP32 as far as it goes. stats
 * (host, >= max_steps records, may be NULL) receives the FP32 steps then the
 * FP64 ones. */
int spm_grad_flow_mixed(spm_ctx *ctx, void *phi, void *uhat, int max_steps, double tol_grad, double switch_tol,
                        spm_step_stats *stats, int *steps_fp32, int *steps_fp64);

/* Batched get_min_u_F over n independent instances (no counterpart in the
 * reference; each context may have its own N, L, Tau, Gamma, dt): one
 * captured CUDA graph advances every instance by steps_per_launch gated steps
 * on parallel stream branches and is relaunched until all instances reached
 * ||grad F|| <= tol_grad (or max_steps). With switch_tol > tol_grad the
 * instances (FP64 contexts) first run with FP32 transforms to switch_tol (or
 * until 512 FP32 steps bring no new minimum of ||grad F||), then in FP64 with
 * the steps each has left. steps_done (host, n entries, may be NULL) receives
 * the steps executed per instance. The contexts' streams are synchronised
 * first. */
int spm_batch_grad_flow(spm_ctx **ctx, void **phi, void **uhat, int n, int max_steps, double tol_grad,
                        double switch_tol, int steps_per_launch, int *steps_done);

/* The asynchronous form of spm_grad_flow: enqueues exactly nsteps gated steps
 * on the context stream and returns without synchronising (the stop rule is
 * evaluated on the device; steps after it do no work). Capturable in a CUDA
 * graph. spm_grad_flow_collect synchronises and returns the records. */
int spm_grad_flow_enqueue(spm_ctx *ctx, void *phi, void *uhat, int nsteps, double tol_grad);
int spm_grad_flow_collect(spm_ctx *ctx, spm_step_stats *stats, int max_records, int *steps_done);

/* get_min_u_F with the field in host memory (the reference's u_R_local,
 * as real values): copies phi_host in, sets uhat = my_fft(phi), runs up to
 * max_steps steps and copies phi back. phi_host holds N^3 values of the
 * context precision (pinned memory recommended). */
int spm_grad_flow_host(spm_ctx *ctx, void *phi_host, int max_steps, double tol_grad,
                       spm_step_stats *stats, int *steps_done);

/* Measurement aid (phi/uhat advance): runs reps >= 2 ungated gradient steps
 * the way spm_grad_flow does, with CUDA events between the kernels. ms (4
 * entries) receives the durations of plane_fwd (ms[0]), the mean pencil pass
 * (ms[1]), the mean fused inverse -> forward plane pass (ms[2]; 0 with
 * fuse_planes = 0) and plane_inv (ms[3]). With fuse_planes = 1 the steps form
 * one chain (plane_fwd and plane_inv run once); with 0, every step runs all
 * three passes and ms[0], ms[3] are means. */
int spm_grad_step_profile(spm_ctx *ctx, void *phi, void *uhat, int reps, double *ms);

/* ngrad_cam (LPsrc.cpp:119-173): grad = -grad F(phi). If norm is non-NULL it
 * receives nrmp(grad) (synchronises). */
int spm_ngrad(spm_ctx *ctx, const void *phi, void *grad, double *norm);

/* ---------------------------------------------------- Hessian / precond */

/* hv_cam (LOBPCG.cpp:113-166) for nb vectors: hv[b] = H(phi) v[b]. */
int spm_hv(spm_ctx *ctx, const void *phi, const void *v, void *hv, int nb);
/* precond_camnew (LOBPCG.cpp:168-199), in place on nb vectors. */
int spm_precond(spm_ctx *ctx, void *w, int nb);

/* --------------------------------------------------------------- LOBPCG */

/* hiosd_lobpcg_initialization (LOBPCG.cpp:10-109): V (k fields, 1 <= k <= 8)
 * receives a random start block -- Eigen's unseeded MatrixXd::Random(k, N^3)
 * replaced by a SplitMix64 stream, V[i][j] = -1 + 2 u(seed, j*k + i) --, each
 * vector minus its mean, then Gram-Schmidt orthonormalised under inpfp. */
int spm_lobpcg_init(spm_ctx *ctx, void *V, int k, uint64_t seed);

/* hiosd_lobpcg_inip (LOBPCG.cpp:207-487): one call of maxiter LOBPCG
 * iterations for the k lowest eigenpairs of H(phi), updating V (k fields) in
 * place. Each iteration builds [V, W, P] with the reference's order and 1e-8
 * dropping rule and solves the Rayleigh-Ritz problem; block inner products
 * run on the FP64 tensor cores. If tol > 0 the call also stops when every
 * residual ||H v_i - lambda_i v_i|| is <= tol. On return evals[i] =
 * <v_i, H v_i> and resid[i] the residual of the returned block (host arrays
 * of k, may be NULL), *iters the iterations done. */
int spm_lobpcg(spm_ctx *ctx, const void *phi, void *V, int k, int maxiter, double tol, double *evals,
               double *resid, int *iters);
/* spm_lobpcg with guard vectors, for solves run to a tolerance: V holds
 * k + guard fields (k + guard <= 8, start block from spm_lobpcg_init of
 * k + guard) and the iteration runs on the whole block, but the stop test
 * takes only the first k residuals. Where the k-th eigenvalue has a close
 * neighbour above it, a block of k converges slowly (its last vector mixes
 * with the neighbour); the guards hold the neighbours. evals and resid (may
 * be NULL) receive k + guard entries. guard = 0 is spm_lobpcg. */
int spm_lobpcg_guarded(spm_ctx *ctx, const void *phi, void *V, int k, int guard, int maxiter, double tol,
                       double *evals, double *resid, int *iters);

/* ------------------------------------------------------------------ SPM */

/* get_Tv (SPM.cpp:15-32): v = (phi1 - phi0) / nrmp(phi1 - phi0). */
int spm_get_tv(spm_ctx *ctx, const void *phi0, const void *phi1, void *v);
/* Natural_Forces (SPM.cpp:34-99) and MinMax_Forces (SPM.cpp:103-168): one
 * semi-implicit force step on x in place along the unit tangent v. */
int spm_natural_forces(spm_ctx *ctx, void *x, const void *v);
int spm_minmax_forces(spm_ctx *ctx, void *x, const void *v);
/* Spring_Pairing (SPM.cpp:170-263) on the replica pair (phi0, phi1) in place:
 * up to maxiter iterations while res = max_i nrmp(ngrad(phi_i)) > tol.
 * res_hist (host, may be NULL, >= maxiter entries) receives res per
 * iteration; *iters the iterations done. */
int spm_spring_pairing(spm_ctx *ctx, void *phi0, void *phi1, int maxiter, double tol, double *res_hist,
                       int *iters);
/* Rest length of the spring between the SPM replicas (default 0: the
 * reference's spring, whose rest length spring_d = 0.001 is computed into
 * kd = ks (dd - spring_d) but never applied, SPM.cpp:179, 206-212). With
 * rest > 0 both spring updates of an iteration apply the force
 * ks (dd - rest) along (phi1 - phi0) / dd, dd = nrmp(phi1 - phi0) measured
 * after the natural-force step, so the pair settles at distance ~rest
 * around the saddle instead of collapsing onto it. Applies to
 * spm_spring_pairing and spm_spring_pairing_mixed on this context. */
int spm_set_spring_length(spm_ctx *ctx, double rest);
/* Mixed-precision Spring_Pairing (no counterpart in the reference): on an
 * FP64 context, the natural-force and min-max steps run with FP32 transforms
 * (FP64 reductions) until res <= max(switch_tol, tol) or until 256 FP32
 * iterations bring no new minimum of res, then continue in FP64 from the
 * cast replicas until res <= tol. res_hist (host, >= maxiter entries, may be
 * NULL) receives the FP32 iterations' residuals, then the FP64 ones. */
int spm_spring_pairing_mixed(spm_ctx *ctx, void *phi0, void *phi1, int maxiter, double tol, double switch_tol,
                             double *res_hist, int *iters_fp32, int *iters_fp64);

/* hiosd_lobpcg_sieh (HISD.cpp:86-485): k-index saddle dynamics from x along
 * the k directions V (k fields, 1 <= k <= 8), both updated in place, with the
 * reference's options dt, betat, betau (Barzilai-Borwein step clamp), epsf
 * (stop when ||grad F|| < epsf) and maxiter (critical_point_HISD,
 * HISD.cpp:13-31, uses 0.8, 8.0, 0.02, 1e-7, 10000). res_hist (host, may be
 * NULL, >= maxiter entries) receives ||grad F|| per iteration. */
int spm_hisd(spm_ctx *ctx, void *x, void *V, int k, double dt, double betat, double betau, double epsf,
             int maxiter, double *res_hist, int *iters);
/* hiosd_lobpcg_sieh_V0 (GOSD.cpp:123-531): spm_hisd with the directions V
 * also kept orthogonal to k0 fixed orthonormal fields V0 (1 <= k0 <= 24), as
 * critical_point (GOSD.cpp:13-56) does with the zero modes of a structure. */
int spm_gosd(spm_ctx *ctx, void *x, void *V, int k, const void *V0, int k0, double dt, double betat, double betau,
             double epsf, int maxiter, double *res_hist, int *iters);

/* ------------------------------------------------------------ BLAS-1 */

/* inpfp (BasicOperators.cpp:132-143): <p, q> = (1/N^3) sum p q. */
int spm_inpfp(spm_ctx *ctx, const void *p, const void *q, double *out);

/* Block of inner products, the Gram of LOBPCG.cpp:336-358 (UUm * YYm^T /
 * N^3): G[a*mb + b] = <X[a], Y[b]> for a < ma, b < mb (1 <= ma, mb <= 24;
 * X and Y are host arrays of device field pointers, which may repeat fields
 * or share them between X and Y; each distinct field is read once), G a host
 * array of ma*mb doubles. Runs on the FP64 tensor cores; the sums are in a
 * fixed order (identical results on every call). Synchronises the context's
 * stream. */
int spm_block_gram(spm_ctx *ctx, const void *const *X, int ma, const void *const *Y, int mb, double *G);

/* Block combination, the Ritz-vector update of LOBPCG.cpp:403-418 (Vm =
 * eta1^T UUm): Y[q] = sum_p C[p*nout + q] X[p] + d[q] for q < nout (1 <= nin
 * <= 32, 1 <= nout <= 24; X, Y host arrays of device field pointers; C a host
 * array of nin*nout doubles, d of nout doubles or NULL for zeros). A point's
 * inputs are all read before any of its outputs is written, so Y may alias X
 * (an in-place update); a field may not appear twice in Y (SPM_ERR_ARG).
 * Enqueued on the context's stream. */
int spm_block_combine(spm_ctx *ctx, const void *const *X, int nin, void *const *Y, int nout, const double *C,
                      const double *d);

/* Allocation-free batch of inner products; no counterpart in the reference.
 * For callers that cannot allocate device memory when they need the result
 * (their device memory is fully reserved by their own pool, or a cudaMalloc's
 * implicit synchronisation would stall their other streams): needs no context
 * and allocates nothing. out[b] = (1/n) sum_i p[b*n + i] * q[b*n + i] for
 * b < nb, with p, q device arrays of nb*n values (double for SPM_FP64, float
 * for SPM_FP32) and out a device array of nb doubles, enqueued on stream.
 * nb is limited to 16 (SPM_ERR_ARG above): the reduction's scratch is a fixed
 * ~77 KB array in the library's device memory, resident on every device that
 * loads the library until exit. Calls share that array: calls that overlap on
 * the GPU race and must be ordered. The stream and the pointers must belong to
 * the device that is current at the call. The first call on a device looks up
 * the array's address and keeps it; make it before any stream capture begins,
 * and do not call this entry point on a device after a cudaDeviceReset (the
 * array may then have moved). */
int spm_inpfp_batch_noalloc(size_t n, int nb, int precision, const void *p, const void *q,
                            double *out, void *stream);

/* ------------------------------------------------------------ field I/O */

/* Save_phi / Save_Option_V (File_Op.cpp:8-49): count values of a host array,
 * one per line as "%.16e \n" (k eigenvectors: k*N^3 values back to back). */
int spm_save_field_txt(const char *path, const double *x, size_t count);
/* load_phi / load_Option_V (File_Op.cpp:51-89): reads count values ("%lf");
 * SPM_ERR_STATE if the file holds fewer. */
int spm_load_field_txt(const char *path, double *x, size_t count);

/* Binary checkpoint (no counterpart in the reference): nfields host fields of
 * N^3 doubles with the model parameters and a step count; a checksum is
 * verified on load. The file is written under a temporary name and renamed. */
typedef struct spm_checkpoint_info {
  int N, nfields, precision;
  double L, Tau, Gamma, dt;
  int64_t step;
} spm_checkpoint_info;
int spm_checkpoint_save(const char *path, const spm_checkpoint_info *info, const double *fields);
/* fields may be NULL to read the header only; capacity in doubles. */
int spm_checkpoint_load(const char *path, spm_checkpoint_info *info, double *fields, size_t capacity);

/* get_initial_value (Initialization.cpp:242-339) on one initData file: full
 * (host, 2*N^3 doubles, interleaved) receives the reference's u_F: 0.1 x the
 * amplitude of each listed mode at k = round(k_file / l * L) (wrapped), where
 * l is the shell scale the reference pairs with the phase (1 DIS/LAM, sqrt 2
 * BCC/HPC, sqrt 3 FCC, sqrt 6 DG). */
int spm_initdata_spectrum(const char *path, int N, double L, double l, double *full);
/* The real initial field of that spectrum on the device: phi = Re(my_ifft(u_F)). */
int spm_initial_field(spm_ctx *ctx, const char *path, double l, void *phi);

/* ------------------------------------------------------------ job server */

/* A job server (no counterpart in the reference, whose drivers run one job
 * per process: main_SPM.cpp, grad.cpp): relaxation, eigenmode and saddle
 * jobs of any supported grid sizes share one GPU. Submitted jobs wait in
 * arrival order; the oldest waiting job whose device-memory footprint fits in
 * the free part of the budget and for which a slot is free starts at once, on
 * its own stream and context, while the others run (smaller jobs may pass a
 * large one that does not fit yet). Reductions are deterministic, so a job's
 * result is the same alone and among others. */
typedef struct spm_server spm_server;

enum spm_job_kind {
  SPM_JOB_RELAX = 0,  /* get_min_u_F to ||grad F|| <= tol (max_steps cap) */
  SPM_JOB_LOBPCG = 1, /* hiosd_lobpcg_initialization(seed) + inip at phi0, k modes */
  SPM_JOB_SPM = 2     /* Spring_Pairing of the replicas (phi0, phi1) to res <= tol */
};

typedef struct spm_job_desc {
  int kind;        /* spm_job_kind */
  int N;           /* grid size (spm_supported_size) */
  int precision;   /* SPM_FP64, SPM_FP32 or SPM_MIXED (relaxation and SPM) */
  int k;           /* LOBPCG block size, 1..8 */
  int max_steps;   /* step / iteration cap */
  int guard;       /* LOBPCG guard vectors (spm_lobpcg_guarded), k + guard <= 8; 0 for other jobs */
  double L, Tau, Gamma, dt;
  double tol;        /* ||grad F|| (relaxation), residual (LOBPCG, SPM) */
  double switch_tol; /* SPM_MIXED: FP32 until this tolerance (0: as far as FP32 goes) */
  uint64_t seed;     /* LOBPCG start block */
} spm_job_desc;

typedef struct spm_job_result {
  int status;        /* SPM_OK, SPM_ERR_CANCELLED, SPM_ERR_NOMEM, ... */
  int steps;         /* steps / iterations executed */
  double energy;     /* relaxation: final energy; SPM: energy of phi1 */
  double residual;   /* final ||grad F||, max LOBPCG residual or SPM res */
  double evals[8];   /* LOBPCG eigenvalues */
  double t_submit, t_start, t_end; /* seconds since the server was created */
  char message[128];  /* spm_last_error() of a failed job, else empty */
} spm_job_result;

typedef struct spm_server_config {
  size_t budget_bytes;  /* device bytes jobs may hold at once (0: 90% of free) */
  int max_slots;        /* jobs running at once */
  int fake_device;      /* nonzero: no GPU work; a job sleeps fake_ms_per_munit
                           ms per million grid points per step */
  double fake_ms_per_munit;
  size_t fake_device_bytes; /* fake device memory; an allocation beyond it is
                               refused (0: unlimited) */
  int max_bypass;       /* times later jobs may start before a waiting job
                           that does not fit (0: 8) */
} spm_server_config;

typedef struct spm_server_stats {
  int64_t completed, failed, cancelled, pending;
  int running, peak_running;
  size_t peak_bytes, budget_bytes;
  double p50_s, p99_s;  /* submit-to-end latency of completed jobs */
  double elapsed_s;     /* since the server was created */
} spm_server_stats;

int spm_server_create(const spm_server_config *cfg, spm_server **out);
/* Device bytes the server reserves for a job while it runs. */
size_t spm_job_footprint(const spm_job_desc *job);
/* phi0 (and phi1 for SPM_JOB_SPM) are host arrays of N^3 doubles, copied at
 * submission. A job larger than the whole budget is refused (SPM_ERR_NOMEM). */
int spm_server_submit(spm_server *srv, const spm_job_desc *job, const double *phi0, const double *phi1,
                      int64_t *job_id);
/* Cancels a waiting job, or asks a running one to stop at its next host
 * check (between chunks of steps); its status becomes SPM_ERR_CANCELLED. */
int spm_server_cancel(spm_server *srv, int64_t job_id);
/* Waits for a job (block != 0) or polls it (SPM_ERR_STATE while unfinished).
 * field (may be NULL) receives the result as doubles: the relaxed phi (N^3),
 * the k eigenvectors (k N^3) or the replica phi1 (N^3). */
int spm_server_wait(spm_server *srv, int64_t job_id, int block, spm_job_result *result, double *field);
/* Drops the record of a finished job (its result field and times). */
int spm_server_release(spm_server *srv, int64_t job_id);
int spm_server_get_stats(spm_server *srv, spm_server_stats *stats);
/* Waits for every submitted job, then releases the server. */
int spm_server_destroy(spm_server *srv);

#ifdef __cplusplus
}
#endif

#endif /* SPMIQC_H */
