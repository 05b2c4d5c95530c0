// Harness around SPM-IQC's own hot-path sources, compiled unchanged from the
// reference tree against the shim headers in oracle/shim/.
// TEST INFRASTRUCTURE ONLY: this is the CPU oracle (built into oracle/_ref/
// by oracle/Makefile). Only the tests, __graft_entry__.smoke() and bench.py's
// CPU-baseline / reference arm load it, as the checker. The product never does.
//
// The set-up replays main_SPM.cpp:25-62 with the parameters passed in instead
// of the hard-coded ones of LPsystParameter (src/Initialization.cpp:7-42):
// LPsystParameter runs first, then N, L, Tau, Gamma, dt, CplxDofs and the
// 1/L projection are overwritten. Each exported function then calls exactly
// one reference routine on the reference's own globals (src/Data.cpp).
//
// Fields cross this boundary as real double[N^3] (row-major i*N*N + j*N + k);
// spectra as interleaved (re, im) double[2*N^3], the reference's own layout.
#include <fcntl.h>
#include <unistd.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "BasicOperators.h"
#include "Data.h"
#include "File_Op.h"
#include "GOSD.h"
#include "HISD.h"
#include "Initialization.h"
#include "LOBPCG.h"
#include "LPsrc.h"
#include "Memfree.h"
#include "My_FFT.h"
#include "SPM.h"

extern void MinMax_Forces(fftw_complex *x, fftw_complex *v);  // src/SPM.cpp:103 (not in SPM.h)
extern "C" void spm_shim_eigen_seed(uint64_t seed);

namespace {
bool g_ready = false;
int g_quiet = 1;
int g_saved_fd = -1;
Option *g_opt = nullptr;

void mute() {
  if (!g_quiet) return;
  fflush(stdout);
  g_saved_fd = dup(1);
  int fd = open("/dev/null", O_WRONLY);
  dup2(fd, 1);
  close(fd);
}
void unmute() {
  if (g_saved_fd < 0) return;
  fflush(stdout);
  dup2(g_saved_fd, 1);
  close(g_saved_fd);
  g_saved_fd = -1;
}
struct Mute {
  Mute() { mute(); }
  ~Mute() { unmute(); }
};

void to_cplx(const double *r, fftw_complex *c) {
  for (int i = 0; i < CplxDofs_local; i++) { c[i][0] = r[i]; c[i][1] = 0.0; }
}
void to_real(const fftw_complex *c, double *r) {
  for (int i = 0; i < CplxDofs_local; i++) r[i] = c[i][0];
}
fftw_complex *alloc_c() { return (fftw_complex *)calloc((size_t)CplxDofs_local, sizeof(fftw_complex)); }

void free_option() {
  if (!g_opt) return;
  for (int i = 0; i < g_opt->k; i++) free(g_opt->V[i]);
  free(g_opt->V);
  free(g_opt);
  g_opt = nullptr;
}
}  // namespace

extern "C" {

void ref_set_quiet(int q) { g_quiet = q; }
void ref_set_threads(int n) { spm_shim_fft_set_threads(n); }
int ref_get_threads(void) { return spm_shim_fft_get_threads(); }

void ref_teardown(void) {
  if (!g_ready) return;
  free_option();
  fftw_destroy_plan(plan1);
  fftw_destroy_plan(plan2);
  fftw_free(data);
  Memfree_local_kspace();
  Memfree_local_data();
  Memfree_global_data();
  g_ready = false;
}

// main_SPM.cpp:20-62 without the initial-value file (the caller sets fields).
int ref_setup(int n, double l, double tau, double gamma, double step) {
  if (n < 2 || n > 512) return 1;
  ref_teardown();
  Mute m;
  MPI_Init(nullptr, nullptr);
  fftw_mpi_init();
  MPI_Comm_size(MPI_COMM_WORLD, &numprocs);
  MPI_Comm_rank(MPI_COMM_WORLD, &myid);
  LPsystParameter();
  N = n;
  CplxDofs = N * N * N;
  L = l;
  Tau = tau;
  Gamma = gamma;
  dt = step;
  for (int j = 0; j < dimCpt; j++) ProjMatrix[j][j] = 1.0 / L;
  for (int i = 0; i < dimCpt; i++) NCpt[i] = N;
  memAllocation_all();
  get_kindex_all();
  My_mpi_fft_set_up();
  memAllocation_local();
  // k_square_local is malloc'd and accumulated with += (Initialization.cpp:54,145)
  memset(k_square_local, 0, sizeof(double) * (size_t)CplxDofs_local);
  Distribute_C(kindex, kindex_local);
  get_ksquare_local();
  get_epmckt2_local();
  get_ikt2_local();
  Memfree_global_kspace();
  memset(u_R_local, 0, sizeof(fftw_complex) * (size_t)CplxDofs_local);
  memset(u_F_local, 0, sizeof(fftw_complex) * (size_t)CplxDofs_local);
  g_ready = true;
  return 0;
}

int ref_ready(void) { return g_ready ? N : 0; }

// Tables the reference builds at set-up (Initialization.cpp:150-174, :123-129).
void ref_get_tables(double *G, double *ikt2) {
  if (G) memcpy(G, epmckt2_local, sizeof(double) * (size_t)CplxDofs_local);
  if (ikt2) memcpy(ikt2, ikt2_local, sizeof(double) * (size_t)CplxDofs_local);
}
double ref_get_GK(double k2) { return get_GK(k2); }

// u_R = phi; u_F = my_fft(u_R) (the state main_SPM.cpp:73 establishes).
void ref_set_state(const double *phi) {
  to_cplx(phi, u_R_local);
  my_fft(u_R_local, u_F_local);
}
// u_R = phi; u_F given (interleaved), as after a restart from both globals.
void ref_set_state2(const double *phi, const double *uF) {
  to_cplx(phi, u_R_local);
  memcpy(u_F_local, uF, sizeof(fftw_complex) * (size_t)CplxDofs_local);
}
void ref_get_state(double *phi, double *uF) {
  if (phi) to_real(u_R_local, phi);
  if (uF) memcpy(uF, u_F_local, sizeof(fftw_complex) * (size_t)CplxDofs_local);
}

// src/My_FFT.cpp:4-21
void ref_my_fft(const double *x_ri, double *xf_ri) {
  my_fft((fftw_complex *)x_ri, (fftw_complex *)xf_ri);
}
void ref_my_ifft(const double *xf_ri, double *x_ri) {
  my_ifft((fftw_complex *)xf_ri, (fftw_complex *)x_ri);
}

// src/LPsrc.cpp:8-38 on the current globals.
double ref_get_Ene(void) {
  Mute m;
  return get_Ene();
}

// src/LPsrc.cpp:40-117, one iteration per call (max_iter = 1); the state
// persists in u_R_local/u_F_local between calls. Per step this records the
// energy the step computes (get_Ene on the same state), ||grad F|| =
// nrmp(ngrad_cam(u_R)) at that state, and res = max|Re(u_F' - u_F)|, which is
// recomputed from the two spectra with the expression of LPsrc.cpp:79-84.
int ref_grad_steps(int nsteps, double *E, double *res, double *gnorm) {
  Mute m;
  fftw_complex *g = alloc_c();
  fftw_complex *old = alloc_c();
  for (int s = 0; s < nsteps; s++) {
    if (E) E[s] = get_Ene();
    if (gnorm) {
      ngrad_cam(u_R_local, g);
      gnorm[s] = nrmp(g);
    }
    memcpy(old, u_F_local, sizeof(fftw_complex) * (size_t)CplxDofs_local);
    max_iter = 1;
    get_min_u_F();
    if (res) {
      double r = 0.0;
      for (int i = 0; i < CplxDofs_local; i++) {
        double d = (u_F_local[i][0] - old[i][0]) * (u_F_local[i][0] - old[i][0]);
        d = sqrt(d);
        if (r < d) r = d;
      }
      res[s] = r;
    }
  }
  free(g);
  free(old);
  return 0;
}

// Full get_min_u_F loop (LPsrc.cpp:52) with the given iteration cap.
void ref_get_min_u_F(int maxit) {
  Mute m;
  max_iter = maxit;
  get_min_u_F();
}

// src/LPsrc.cpp:119-173
void ref_ngrad(const double *phi, double *grad) {
  fftw_complex *p = alloc_c(), *g = alloc_c();
  to_cplx(phi, p);
  ngrad_cam(p, g);
  to_real(g, grad);
  free(p);
  free(g);
}

// src/LOBPCG.cpp:113-166
void ref_hv(const double *phi, const double *v, double *hv) {
  fftw_complex *p = alloc_c(), *vv = alloc_c(), *h = alloc_c();
  to_cplx(phi, p);
  to_cplx(v, vv);
  hv_cam(p, vv, h);
  to_real(h, hv);
  free(p);
  free(vv);
  free(h);
}

// src/LOBPCG.cpp:168-199 (in place)
void ref_precond(double *w) {
  fftw_complex *c = alloc_c();
  to_cplx(w, c);
  precond_camnew(c);
  to_real(c, w);
  free(c);
}

// src/BasicOperators.cpp:132-143, 174-185
double ref_inpfp(const double *p, const double *q) {
  return inpfp(const_cast<double *>(p), const_cast<double *>(q));
}
double ref_rayleighq(const double *phi, const double *v) {
  fftw_complex *p = alloc_c(), *vv = alloc_c();
  to_cplx(phi, p);
  to_cplx(v, vv);
  double r = rayleighq(p, vv);
  free(p);
  free(vv);
  return r;
}

// src/LOBPCG.cpp:10-109 with MatrixXd::Random seeded; V_out is k x N^3.
void ref_lobpcg_init(int k, uint64_t seed, double *V_out) {
  free_option();
  spm_shim_eigen_seed(seed);
  g_opt = (Option *)malloc(sizeof(Option));
  {
    Mute m;
    hiosd_lobpcg_initialization(g_opt, k);
  }
  if (V_out)
    for (int i = 0; i < k; i++) to_real(g_opt->V[i], V_out + (size_t)i * CplxDofs_local);
}

// src/LOBPCG.cpp:207-487: one call (maxiter iterations) on the block V (k x N^3, in/out).
void ref_lobpcg_inip(const double *phi, int k, int maxiter, double *V) {
  if (!g_opt || g_opt->k != k) {
    free_option();
    spm_shim_eigen_seed(0);
    g_opt = (Option *)malloc(sizeof(Option));
    Mute m;
    hiosd_lobpcg_initialization(g_opt, k);
  }
  for (int i = 0; i < k; i++) to_cplx(V + (size_t)i * CplxDofs_local, g_opt->V[i]);
  g_opt->maxiter = maxiter;
  fftw_complex *x = alloc_c();
  to_cplx(phi, x);
  {
    Mute m;
    hiosd_lobpcg_inip(x, g_opt);
  }
  for (int i = 0; i < k; i++) to_real(g_opt->V[i], V + (size_t)i * CplxDofs_local);
  free(x);
}

// src/SPM.cpp:15-32
void ref_get_Tv(const double *phi0, const double *phi1, double *v) {
  fftw_complex *P[2] = {alloc_c(), alloc_c()}, *t = alloc_c();
  to_cplx(phi0, P[0]);
  to_cplx(phi1, P[1]);
  get_Tv(P, t);
  to_real(t, v);
  free(P[0]);
  free(P[1]);
  free(t);
}

// src/SPM.cpp:34-99 and :103-168 (x updated in place)
void ref_natural_forces(double *x, const double *v) {
  fftw_complex *xc = alloc_c(), *vc = alloc_c();
  to_cplx(x, xc);
  to_cplx(v, vc);
  Natural_Forces(xc, vc);
  to_real(xc, x);
  free(xc);
  free(vc);
}
void ref_minmax_forces(double *x, const double *v) {
  fftw_complex *xc = alloc_c(), *vc = alloc_c();
  to_cplx(x, xc);
  to_cplx(v, vc);
  MinMax_Forces(xc, vc);
  to_real(xc, x);
  free(xc);
  free(vc);
}

// src/SPM.cpp:170-263 on the global replica pair Phi0 and tangent tv.
void ref_spring_pairing(double *phi0, double *phi1, double maxiter, double tol) {
  to_cplx(phi0, Phi0[0]);
  to_cplx(phi1, Phi0[1]);
  {
    Mute m;
    Spring_Pairing(Phi0, maxiter, tol);
  }
  to_real(Phi0[0], phi0);
  to_real(Phi0[1], phi1);
}

// HISD.cpp:86-485 on (x, V) in place with the given options.
void ref_hisd(double *xr, int k, double *V, double dt, double betat, double betau, double epsf, int maxiter) {
  if (!g_opt || g_opt->k != k) {
    free_option();
    spm_shim_eigen_seed(0);
    g_opt = (Option *)malloc(sizeof(Option));
    Mute m;
    hiosd_lobpcg_initialization(g_opt, k);
  }
  for (int i = 0; i < k; i++) to_cplx(V + (size_t)i * CplxDofs_local, g_opt->V[i]);
  g_opt->dt = dt;
  g_opt->betat = betat;
  g_opt->betau = betau;
  g_opt->epsf = epsf;
  g_opt->maxiter = maxiter;
  g_opt->outputp = 100;
  g_opt->outputd = 1000;
  fftw_complex *x = alloc_c();
  to_cplx(xr, x);
  {
    Mute m;
    hiosd_lobpcg_sieh(x, g_opt);
  }
  to_real(x, xr);
  for (int i = 0; i < k; i++) to_real(g_opt->V[i], V + (size_t)i * CplxDofs_local);
  free(x);
}

// GOSD.cpp:123-531 (hiosd_lobpcg_sieh_V0) on (x, V) with k0 fixed fields V0.
void ref_gosd(double *xr, int k, double *V, int k0, const double *V0r, double dt, double betat, double betau,
              double epsf, int maxiter) {
  if (!g_opt || g_opt->k != k) {
    free_option();
    spm_shim_eigen_seed(0);
    g_opt = (Option *)malloc(sizeof(Option));
    Mute m;
    hiosd_lobpcg_initialization(g_opt, k);
  }
  for (int i = 0; i < k; i++) to_cplx(V + (size_t)i * CplxDofs_local, g_opt->V[i]);
  g_opt->dt = dt;
  g_opt->betat = betat;
  g_opt->betau = betau;
  g_opt->epsf = epsf;
  g_opt->maxiter = maxiter;
  g_opt->outputp = 100;
  g_opt->outputd = 1000;
  fftw_complex **V0 = (fftw_complex **)malloc(sizeof(fftw_complex *) * k0);
  for (int i = 0; i < k0; i++) {
    V0[i] = alloc_c();
    to_cplx(V0r + (size_t)i * CplxDofs_local, V0[i]);
  }
  fftw_complex *x = alloc_c();
  to_cplx(xr, x);
  {
    Mute m;
    hiosd_lobpcg_sieh_V0(x, g_opt, V0, k0);
  }
  to_real(x, xr);
  for (int i = 0; i < k; i++) to_real(g_opt->V[i], V + (size_t)i * CplxDofs_local);
  for (int i = 0; i < k0; i++) free(V0[i]);
  free(V0);
  free(x);
}

// File_Op.cpp:40-61 (Save_phi / load_phi) on a real field.
void ref_save_phi(const double *phi, const char *path) {
  Mute m;
  const size_t n = (size_t)CplxDofs;
  fftw_complex *x = (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
  for (size_t i = 0; i < n; i++) {
    x[i][0] = phi[i];
    x[i][1] = 0.0;
  }
  Save_phi(x, const_cast<char *>(path));
  fftw_free(x);
}
void ref_load_phi(const char *path, double *phi) {
  Mute m;
  const size_t n = (size_t)CplxDofs;
  fftw_complex *x = (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
  load_phi(x, const_cast<char *>(path));
  for (size_t i = 0; i < n; i++) phi[i] = x[i][0];
  fftw_free(x);
}
// File_Op.cpp:8-38, 63-89 (Save_Option_V / load_Option_V) on k fields.
void ref_save_option_v(int k, const double *V, const char *path) {
  Mute m;
  Option opt;
  memset(&opt, 0, sizeof(opt));
  opt.k = k;
  const size_t n = (size_t)CplxDofs_local;
  opt.V = (fftw_complex **)malloc(sizeof(fftw_complex *) * k);
  for (int i = 0; i < k; i++) {
    opt.V[i] = (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
    for (size_t j = 0; j < n; j++) {
      opt.V[i][j][0] = V[i * n + j];
      opt.V[i][j][1] = 0.0;
    }
  }
  Save_Option_V(&opt, const_cast<char *>(path));
  for (int i = 0; i < k; i++) fftw_free(opt.V[i]);
  free(opt.V);
}
void ref_load_option_v(int k, const char *path, double *V) {
  Mute m;
  Option opt;
  memset(&opt, 0, sizeof(opt));
  opt.k = k;
  const size_t n = (size_t)CplxDofs_local;
  opt.V = (fftw_complex **)malloc(sizeof(fftw_complex *) * k);
  for (int i = 0; i < k; i++) opt.V[i] = (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
  load_Option_V(&opt, const_cast<char *>(path));
  for (int i = 0; i < k; i++) {
    for (size_t j = 0; j < n; j++) V[i * n + j] = opt.V[i][j][0];
    fftw_free(opt.V[i]);
  }
  free(opt.V);
}
// get_initial_value (Initialization.cpp:242-339): reads ./initData/<phase>
// relative to `root` (the directory holding initData/); uF_ri receives u_F.
int ref_initial_value(int choice, const char *root, double *uF_ri) {
  char cwd[4096];
  if (!getcwd(cwd, sizeof(cwd)) || chdir(root) != 0) return 1;
  const size_t n = (size_t)CplxDofs;
  fftw_complex *u = (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
  {
    Mute m;
    get_initial_value(u, choice, 0.0);
  }
  memcpy(uF_ri, u, sizeof(fftw_complex) * n);
  fftw_free(u);
  return chdir(cwd) == 0 ? 0 : 1;
}

}  // extern "C"
