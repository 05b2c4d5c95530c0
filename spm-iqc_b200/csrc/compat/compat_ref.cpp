// Link-time drop-in for SPM-IQC's hot-path routines (include/spmiqc_compat.h):
// the reference's own C++ signatures, implemented on the C ABI of
// libspmiqc_cuda.so. Each routine reads the reference's globals, moves the
// fields to the GPU (real parts of fftw_complex fields; full <-> packed
// spectra), calls the sm_100a implementation and writes back.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "spmiqc.h"
#include "spmiqc_compat.h"

namespace {

spm_ctx *g_ctx = nullptr;
int g_N = 0;
double g_L = 0, g_tau = 0, g_gamma = 0, g_dt = 0;
std::vector<void *> g_dev;   // device fields, grown on demand
double *g_full = nullptr;    // device full N^3 complex spectrum (staging)
double *g_host = nullptr;    // pinned real field (staging)

void die(const char *what) {
  std::fprintf(stderr, "spmiqc compat: %s: %s\n", what, spm_last_error());
  std::abort();
}
void ck(int s, const char *what) {
  if (s != SPM_OK) die(what);
}
void ckc(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "spmiqc compat: %s: %s\n", what, cudaGetErrorString(e));
    std::abort();
  }
}

size_t n3() { return (size_t)N * N * N; }

// Context for the current globals; (re)created when N or a parameter changed.
void ensure() {
  if (numprocs > 1) die("the GPU drop-in runs with one MPI rank");
  if (g_ctx && g_N == N && g_L == L && g_tau == Tau && g_gamma == Gamma && g_dt == dt) return;
  spmiqc_compat_release();
  ck(spm_ctx_create(N, L, Tau, Gamma, dt, SPM_FP64, nullptr, &g_ctx), "context");
  g_N = N;
  g_L = L;
  g_tau = Tau;
  g_gamma = Gamma;
  g_dt = dt;
  ckc(cudaMalloc(&g_full, sizeof(double) * 2 * n3()), "spectrum staging");
  ckc(cudaMallocHost(&g_host, sizeof(double) * n3()), "host staging");
}

// i-th device field (N^3 doubles)
double *dev(int i) {
  while ((int)g_dev.size() <= i) {
    void *p = nullptr;
    ckc(cudaMalloc(&p, sizeof(double) * n3()), "device field");
    g_dev.push_back(p);
  }
  return (double *)g_dev[i];
}

void put_real(double *d, const fftw_complex *x) {
  const size_t n = n3();
  for (size_t i = 0; i < n; i++) g_host[i] = x[i][0];
  ckc(cudaMemcpy(d, g_host, sizeof(double) * n, cudaMemcpyHostToDevice), "upload");
}
void get_real(fftw_complex *x, const double *d) {
  const size_t n = n3();
  ckc(cudaMemcpy(g_host, d, sizeof(double) * n, cudaMemcpyDeviceToHost), "download");
  for (size_t i = 0; i < n; i++) {
    x[i][0] = g_host[i];
    x[i][1] = 0.0;
  }
}
void put_spec(double *d, const fftw_complex *xf) {
  ckc(cudaMemcpy(g_full, xf, sizeof(double) * 2 * n3(), cudaMemcpyHostToDevice), "spectrum upload");
  ck(spm_spectrum_from_full(g_ctx, g_full, d), "pack spectrum");
}
void get_spec(fftw_complex *xf, const double *d) {
  ck(spm_spectrum_to_full(g_ctx, d, g_full), "unpack spectrum");
  ckc(cudaMemcpy(xf, g_full, sizeof(double) * 2 * n3(), cudaMemcpyDeviceToHost), "spectrum download");
}

}  // namespace

extern "C" void spmiqc_compat_release(void) {
  if (g_ctx) spm_ctx_destroy(g_ctx);
  g_ctx = nullptr;
  for (void *p : g_dev) cudaFree(p);
  g_dev.clear();
  if (g_full) cudaFree(g_full);
  if (g_host) cudaFreeHost(g_host);
  g_full = nullptr;
  g_host = nullptr;
}

// ---------------------------------------------------------------- My_FFT.cpp
void My_mpi_fft_set_up() {
  // the reference's slab bookkeeping for one rank (My_FFT.cpp:80-84)
  alloc_local = (ptrdiff_t)N * N * N;
  local_n0 = N;
  local_0_start = 0;
  CplxDofs_local = N * N * N;
  if (!data) data = (fftw_complex *)std::calloc((size_t)alloc_local, sizeof(fftw_complex));
  plan1 = nullptr;
  plan2 = nullptr;
  ensure();
}

void my_fft(fftw_complex *x_R_local, fftw_complex *x_F_local) {
  ensure();
  put_real(dev(0), x_R_local);
  ck(spm_fft(g_ctx, dev(0), dev(1)), "my_fft");
  get_spec(x_F_local, dev(1));
}

void my_ifft(fftw_complex *x_F_local, fftw_complex *x_R_local) {
  ensure();
  put_spec(dev(1), x_F_local);
  ck(spm_ifft(g_ctx, dev(1), dev(0)), "my_ifft");
  get_real(x_R_local, dev(0));
}

// ---------------------------------------------------------------- LPsrc.cpp
double get_Ene() {
  ensure();
  put_real(dev(0), u_R_local);
  put_spec(dev(1), u_F_local);
  double e = 0;
  ck(spm_energy(g_ctx, dev(0), dev(1), &e), "get_Ene");
  return e;
}

void get_min_u_F() {
  ensure();
  put_real(dev(0), u_R_local);
  put_spec(dev(1), u_F_local);
  const int maxit = max_iter > 0 ? max_iter : 0;
  std::vector<spm_step_stats> st((size_t)(maxit > 0 ? maxit : 1));
  int done = 0;
  ck(spm_grad_flow(g_ctx, dev(0), dev(1), maxit, 0.0, st.data(), &done), "get_min_u_F");
  if (myid == 0)  // the reference's progress line every 10 iterations (LPsrc.cpp:96-100)
    for (int i = 0; i < done; i += 10)
      std::printf("\nmyid : %d ,\t iter : %d \t res: %.3e \t E: %.3e \t", myid, i, st[i].res, st[i].energy);
  get_real(u_R_local, dev(0));
  get_spec(u_F_local, dev(1));
}

void ngrad_cam(fftw_complex *phir, fftw_complex *gradr) {
  ensure();
  put_real(dev(0), phir);
  ck(spm_ngrad(g_ctx, dev(0), dev(2), nullptr), "ngrad_cam");
  get_real(gradr, dev(2));
}

// ---------------------------------------------------------------- LOBPCG.cpp
void hv_cam(fftw_complex *phir, fftw_complex *v, fftw_complex *hv) {
  ensure();
  put_real(dev(0), phir);
  put_real(dev(2), v);
  ck(spm_hv(g_ctx, dev(0), dev(2), dev(3), 1), "hv_cam");
  get_real(hv, dev(3));
}

void precond_camnew(fftw_complex *w) {
  ensure();
  put_real(dev(2), w);
  ck(spm_precond(g_ctx, dev(2), 1), "precond_camnew");
  get_real(w, dev(2));
}

void hiosd_lobpcg_initialization(Option *option, int ki) {
  ensure();
  // option defaults of LOBPCG.cpp:12-19
  option->k = ki;
  option->maxiter = 21;
  option->dt = 0.1;
  option->epsf = 1e-7;
  option->betat = 1.0;
  option->betau = 1.0;
  option->outputp = 1;
  option->outputd = 1;
  option->V = (fftw_complex **)std::malloc(sizeof(fftw_complex *) * (size_t)ki);
  for (int i = 0; i < ki; i++) option->V[i] = (fftw_complex *)std::malloc(sizeof(fftw_complex) * n3());
  const char *s = std::getenv("SPMIQC_LOBPCG_SEED");
  const uint64_t seed = s ? (uint64_t)std::strtoull(s, nullptr, 10) : 0;
  double *blk = nullptr;
  ckc(cudaMalloc(&blk, sizeof(double) * n3() * (size_t)ki), "start block");
  ck(spm_lobpcg_init(g_ctx, blk, ki, seed), "hiosd_lobpcg_initialization");
  for (int i = 0; i < ki; i++) get_real(option->V[i], blk + n3() * (size_t)i);
  cudaFree(blk);
}

void hiosd_lobpcg_inip(fftw_complex *x, Option *option) {
  ensure();
  const int k = option->k;
  put_real(dev(0), x);
  double *blk = nullptr;
  ckc(cudaMalloc(&blk, sizeof(double) * n3() * (size_t)k), "block");
  for (int i = 0; i < k; i++) put_real(blk + n3() * (size_t)i, option->V[i]);
  std::vector<double> ev((size_t)k);
  int it = 0;
  ck(spm_lobpcg(g_ctx, dev(0), blk, k, option->maxiter, 0.0, ev.data(), nullptr, &it), "hiosd_lobpcg_inip");
  for (int i = 0; i < k; i++) get_real(option->V[i], blk + n3() * (size_t)i);
  cudaFree(blk);
}

// copy_option_V (LOBPCG.cpp:489-520): host copies of the real parts.
void copy_option_V(Option *o1, Option *o2, int k) {
  for (int i = 0; i < k; i++)
    for (int j = 0; j < CplxDofs_local; j++) {
      o2->V[i][j][0] = o1->V[i][j][0];
      o2->V[i][j][1] = 0.0;
    }
}
void copy_option_V(fftw_complex **V, Option *o2, int k) {
  for (int i = 0; i < k; i++)
    for (int j = 0; j < CplxDofs_local; j++) {
      o2->V[i][j][0] = V[i][j][0];
      o2->V[i][j][1] = 0.0;
    }
}
void copy_option_V(fftw_complex *v, Option *o2, int k) {
  for (int j = 0; j < CplxDofs_local; j++) {
    o2->V[k][j][0] = v[j][0];
    o2->V[k][j][1] = 0.0;
  }
}

// ---------------------------------------------------------------- SPM.cpp
// Gs_gri_nuc (SPM.cpp:265-300, unused by the drivers): Gaussian window
// exp(-18 r^2) on [-1, 1)^3 times phi, on the host.
void Gs_gri_nuc(fftw_complex *v_loc, fftw_complex *phi_loc) {
  const double h = 2.0 / N, alpha = 18;
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++)
      for (int k = 0; k < N; k++) {
        const double x = -1 + i * h, y = -1 + j * h, z = -1 + k * h;
        const size_t s = ((size_t)i * N + j) * N + k;
        v_loc[s][0] = std::exp(-alpha * (std::pow(x, 2) + std::pow(y, 2) + std::pow(z, 2))) * phi_loc[s][0];
        v_loc[s][1] = 0.0;
      }
}

void get_Tv(fftw_complex **Phi, fftw_complex *v) {
  ensure();
  put_real(dev(4), Phi[0]);
  put_real(dev(5), Phi[1]);
  ck(spm_get_tv(g_ctx, dev(4), dev(5), dev(2)), "get_Tv");
  get_real(v, dev(2));
}

void Natural_Forces(fftw_complex *x, fftw_complex *v) {
  ensure();
  put_real(dev(4), x);
  put_real(dev(2), v);
  ck(spm_natural_forces(g_ctx, dev(4), dev(2)), "Natural_Forces");
  get_real(x, dev(4));
}

void MinMax_Forces(fftw_complex *x, fftw_complex *v) {
  ensure();
  put_real(dev(4), x);
  put_real(dev(2), v);
  ck(spm_minmax_forces(g_ctx, dev(4), dev(2)), "MinMax_Forces");
  get_real(x, dev(4));
}

void Spring_Pairing(fftw_complex **Phi, double maxiter, double tol) {
  ensure();
  put_real(dev(4), Phi[0]);
  put_real(dev(5), Phi[1]);
  const int mi = maxiter > 0 ? (int)maxiter : 0;
  std::vector<double> hist((size_t)(mi > 0 ? mi : 1));
  int it = 0;
  ck(spm_spring_pairing(g_ctx, dev(4), dev(5), mi, tol, hist.data(), &it), "Spring_Pairing");
  if (myid == 0)  // the reference's progress line every 10 iterations (SPM.cpp:248-254)
    for (int i = 9; i < it; i += 10) std::printf("\n iter = %d , res =  %.3e \n", i + 1, hist[i]);
  get_real(Phi[0], dev(4));
  get_real(Phi[1], dev(5));
  if (tv) get_Tv(Phi, tv);  // SPM.cpp:258
}
