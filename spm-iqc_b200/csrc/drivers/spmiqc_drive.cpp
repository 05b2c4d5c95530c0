// spmiqc_drive: the reference's two driver programs replayed on the C ABI.
//
//   spmiqc_drive stage1 [options]   main_SPM.cpp:15-163 — relax the initial
//       phase (get_min_u_F), energy, LOBPCG k=2 (10 calls of 21 iterations),
//       SPM from (phi, phi + 0.001 v0) (Spring_Pairing, 30000 iterations,
//       tol 1e-9), energy of the transition state, save S1.txt.
//   spmiqc_drive stage2 [options]   grad.cpp:14-182 — load S1.txt, energy,
//       LOBPCG k=3 (20 calls, or load V1_saddle.txt when it exists, else save
//       it), phi + 0.001 v0, get_min_u_F, energy of the relaxed minimum, save
//       Min.txt, 25 more LOBPCG calls, save V0_Min.txt.
//
// Fields stay on the GPU; files use the reference's ASCII format
// (spm_save_field_txt). Options (defaults are the reference's
// LPsystParameter values, Initialization.cpp:7-42):
//   --N 256 --L 26 --Tau -0.0061 --Gamma 0.30 --dt 0.3 --max-iter 100000
//   --tol-grad 0        extra stop of get_min_u_F at ||grad F|| <= tol (0: off)
//   --init FILE --l X   initData file and its shell scale (stage 1; default
//                       phi = 0, the reference's DIS phase)
//   --init-txt FILE     start from a field file instead (stage 1)
//   --result DIR        where S1.txt, V1_saddle.txt, Min.txt, V0_Min.txt go (./result)
//   --lobpcg-calls n    calls of hiosd_lobpcg_inip (10 in stage 1, 20 + 25 in stage 2)
//   --lobpcg-iters 21   iterations per call (Option maxiter, LOBPCG.cpp:12-19)
//   --spm-maxiter 30000 --spm-tol 1e-9 --seed 0
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "spmiqc.h"

namespace {

struct Opts {
  std::string stage;
  int N = 256;
  double L = 26, Tau = -0.0061, Gamma = 0.30, dt = 0.3;
  int max_iter = 100000;
  double tol_grad = 0;
  std::string init, init_txt, result = "./result";
  double l = 1.0;
  int lobpcg_calls = -1, lobpcg_calls2 = 25, lobpcg_iters = 21;
  int spm_maxiter = 30000;
  double spm_tol = 1e-9;
  unsigned long long seed = 0;
};

[[noreturn]] void die(const char *what, int rc) {
  std::fprintf(stderr, "spmiqc_drive: %s: %s (%s)\n", what, spm_status_str(rc), spm_last_error());
  std::exit(2);
}
#define CHECK(x)                  \
  do {                            \
    int _rc = (x);                \
    if (_rc != SPM_OK) die(#x, _rc); \
  } while (0)

double num(const char *opt, const char *v) {
  char *end = nullptr;
  const double x = std::strtod(v, &end);
  if (end == v || *end != '\0') {
    std::fprintf(stderr, "spmiqc_drive: %s needs a number, got '%s'\n", opt, v);
    std::exit(1);
  }
  return x;
}

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Dev {
  std::vector<void *> p;
  void *alloc(size_t bytes) {
    void *q = nullptr;
    if (cudaMalloc(&q, bytes) != cudaSuccess || cudaMemset(q, 0, bytes) != cudaSuccess) {
      std::fprintf(stderr, "spmiqc_drive: device allocation of %zu bytes failed\n", bytes);
      std::exit(2);
    }
    p.push_back(q);
    return q;
  }
  ~Dev() {
    for (void *q : p) cudaFree(q);
  }
};

// get_min_u_F with the reference's progress line every 10 iterations (LPsrc.cpp:93-96)
void relax(spm_ctx *c, void *phi, void *uh, const Opts &o) {
  std::vector<spm_step_stats> st((size_t)o.max_iter);
  int done = 0;
  CHECK(spm_grad_flow(c, phi, uh, o.max_iter, o.tol_grad, st.data(), &done));
  for (int i = 0; i < done; i += 10)
    std::printf("\nmyid : 0 ,\t iter : %d \t res: %.3e \t E: %.3e \t", i, st[i].res, st[i].energy);
  if (done > 0)
    std::printf("\nget_min_u_F: %d iterations, res %.3e, ||grad F|| %.3e\n", done, st[done - 1].res,
                st[done - 1].grad_norm);
}

void lobpcg_calls(spm_ctx *c, void *phi, void *V, int k, int calls, const Opts &o) {
  double ev[8], rs[8];
  int it = 0;
  for (int i = 0; i < calls; i++) CHECK(spm_lobpcg(c, phi, V, k, o.lobpcg_iters, 0.0, ev, rs, &it));
  std::printf("\nLOBPCG (k = %d, %d calls):", k, calls);
  for (int i = 0; i < k; i++) std::printf(" lambda_%d = %.15e (residual %.3e)", i, ev[i], rs[i]);
  std::printf("\n");
}

void save(const std::string &path, const void *dev, size_t count) {
  std::vector<double> h(count);
  if (cudaMemcpy(h.data(), dev, count * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) {
    std::fprintf(stderr, "spmiqc_drive: download failed\n");
    std::exit(2);
  }
  CHECK(spm_save_field_txt(path.c_str(), h.data(), count));
  std::printf("save : %s\n", path.c_str());
}

void load(const std::string &path, void *dev, size_t count) {
  std::vector<double> h(count);
  CHECK(spm_load_field_txt(path.c_str(), h.data(), count));
  if (cudaMemcpy(dev, h.data(), count * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    std::fprintf(stderr, "spmiqc_drive: upload failed\n");
    std::exit(2);
  }
  std::printf("load: %s\n", path.c_str());
}

// x += a * y on the device through the host (driver-level glue, once per stage)
void axpy(void *x, double a, const void *y, size_t n) {
  std::vector<double> hx(n), hy(n);
  cudaMemcpy(hx.data(), x, n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaMemcpy(hy.data(), y, n * sizeof(double), cudaMemcpyDeviceToHost);
  for (size_t i = 0; i < n; i++) hx[i] = hx[i] + a * hy[i];  // FuncsLinear2Cplx order (BasicOperators.cpp:110-119)
  cudaMemcpy(x, hx.data(), n * sizeof(double), cudaMemcpyHostToDevice);
}

int stage1(spm_ctx *c, const Opts &o) {
  const size_t n = (size_t)o.N * o.N * o.N, fb = n * sizeof(double);
  Dev d;
  void *phi = d.alloc(fb), *uh = d.alloc(fb), *phi1 = d.alloc(fb), *V = d.alloc(2 * fb);
  if (!o.init.empty()) CHECK(spm_initial_field(c, o.init.c_str(), o.l, phi));
  else if (!o.init_txt.empty()) load(o.init_txt, phi, n);
  const double t0 = now();
  CHECK(spm_fft(c, phi, uh));
  relax(c, phi, uh, o);
  const double t1 = now();
  double E = 0;
  CHECK(spm_fft(c, phi, uh));
  CHECK(spm_energy(c, phi, uh, &E));
  const double t2 = now();
  CHECK(spm_lobpcg_init(c, V, 2, o.seed));
  std::printf("\n--------------Calculating eigenvalues--------------------------\n");
  lobpcg_calls(c, phi, V, 2, o.lobpcg_calls >= 0 ? o.lobpcg_calls : 10, o);
  const double t3 = now();
  std::printf("\nEnergy of metastable state :  %.15e\n", E);
  std::printf("\n =========================SPM================================= \n ");
  cudaMemcpy(phi1, phi, fb, cudaMemcpyDeviceToDevice);
  axpy(phi1, 0.001, V, n);  // Phi1 = phi + 0.001 v0 (main_SPM.cpp:103-112)
  std::vector<double> hist((size_t)std::max(o.spm_maxiter, 1));
  int its = 0;
  CHECK(spm_spring_pairing(c, phi, phi1, o.spm_maxiter, o.spm_tol, hist.data(), &its));
  std::printf("\nSpring_Pairing: %d iterations, res %.3e\n", its, its ? hist[its - 1] : 0.0);
  double Es = 0;
  CHECK(spm_fft(c, phi1, uh));
  CHECK(spm_energy(c, phi1, uh, &Es));
  const double t4 = now();
  std::printf("\nEnergy of transition state ： %.15e\n", Es);
  save(o.result + "/S1.txt", phi1, n);
  std::printf("\nRunning time of the whole program %f s \n", t4 - t0);
  std::printf("minimum %f s, LOBPCG %f s, SPM %f s\n", t1 - t0, t3 - t2, t4 - t3);
  return 0;
}

int stage2(spm_ctx *c, const Opts &o) {
  const size_t n = (size_t)o.N * o.N * o.N, fb = n * sizeof(double);
  Dev d;
  void *phi = d.alloc(fb), *uh = d.alloc(fb), *V = d.alloc(3 * fb);
  const double t0 = now();
  load(o.result + "/S1.txt", phi, n);
  CHECK(spm_fft(c, phi, uh));
  double E = 0;
  CHECK(spm_energy(c, phi, uh, &E));
  std::printf("\nEnergy of transition state : %.15e\n", E);
  const double t2 = now();
  CHECK(spm_lobpcg_init(c, V, 3, o.seed));
  const std::string vs = o.result + "/V1_saddle.txt";
  if (FILE *f = std::fopen(vs.c_str(), "r")) {  // resume by cache (grad.cpp:93-112)
    std::fclose(f);
    std::printf("File  exists. Skipping LOBPCG calculation.\n");
    load(vs, V, 3 * n);
  } else {
    std::printf("File does not exist. Performing LOBPCG calculation.\n");
    lobpcg_calls(c, phi, V, 3, o.lobpcg_calls >= 0 ? o.lobpcg_calls : 20, o);
    save(vs, V, 3 * n);
  }
  const double t3 = now();
  axpy(phi, 0.001, V, n);  // FuncsLinear2Cplx(u_R, 1, u_R, 0.001, V[0]) (grad.cpp:118)
  CHECK(spm_fft(c, phi, uh));
  relax(c, phi, uh, o);
  const double t4 = now();
  CHECK(spm_energy(c, phi, uh, &E));
  std::printf("\nEnergy of relaxed minimum ：%.15e\n", E);
  save(o.result + "/Min.txt", phi, n);
  lobpcg_calls(c, phi, V, 3, o.lobpcg_calls2, o);
  save(o.result + "/V0_Min.txt", V, 3 * n);
  const double t5 = now();
  std::printf("Running time of the whole program %f s \n", t5 - t0);
  std::printf("Running time of the calculate  minimum point program %f s \n", t4 - t3);
  std::printf("Running time of the LOBPCG program %f s \n", t3 - t2);
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 2 || (std::strcmp(argv[1], "stage1") && std::strcmp(argv[1], "stage2"))) {
    std::fprintf(stderr, "usage: spmiqc_drive stage1|stage2 [--N n] [--L x] [--Tau x] [--Gamma x] [--dt x] "
                         "[--max-iter n] [--tol-grad x] [--init file --l x] [--init-txt file] [--result dir] "
                         "[--lobpcg-calls n] [--lobpcg-calls2 n] [--lobpcg-iters n] [--spm-maxiter n] "
                         "[--spm-tol x] [--seed n]\n");
    return 1;
  }
  Opts o;
  o.stage = argv[1];
  for (int i = 2; i + 1 < argc; i += 2) {
    const std::string k = argv[i];
    const char *v = argv[i + 1];
    if (k == "--N") o.N = (int)num(k.c_str(), v);
    else if (k == "--L") o.L = num(k.c_str(), v);
    else if (k == "--Tau") o.Tau = num(k.c_str(), v);
    else if (k == "--Gamma") o.Gamma = num(k.c_str(), v);
    else if (k == "--dt") o.dt = num(k.c_str(), v);
    else if (k == "--max-iter") o.max_iter = (int)num(k.c_str(), v);
    else if (k == "--tol-grad") o.tol_grad = num(k.c_str(), v);
    else if (k == "--init") o.init = v;
    else if (k == "--l") o.l = num(k.c_str(), v);
    else if (k == "--init-txt") o.init_txt = v;
    else if (k == "--result") o.result = v;
    else if (k == "--lobpcg-calls") o.lobpcg_calls = (int)num(k.c_str(), v);
    else if (k == "--lobpcg-calls2") o.lobpcg_calls2 = (int)num(k.c_str(), v);
    else if (k == "--lobpcg-iters") o.lobpcg_iters = (int)num(k.c_str(), v);
    else if (k == "--spm-maxiter") o.spm_maxiter = (int)num(k.c_str(), v);
    else if (k == "--spm-tol") o.spm_tol = num(k.c_str(), v);
    else if (k == "--seed") o.seed = (unsigned long long)num(k.c_str(), v);
    else {
      std::fprintf(stderr, "spmiqc_drive: unknown option %s\n", k.c_str());
      return 1;
    }
  }
  std::printf("\nset parameter: Tau = %f, Gamma = %f \n", o.Tau, o.Gamma);
  std::printf("\nset parameter: L = %f, N = %d \n", o.L, o.N);
  spm_ctx *c = nullptr;
  CHECK(spm_ctx_create(o.N, o.L, o.Tau, o.Gamma, o.dt, SPM_FP64, nullptr, &c));
  const int rc = o.stage == "stage1" ? stage1(c, o) : stage2(c, o);
  spm_ctx_destroy(c);
  std::fflush(stdout);
  return rc;
}
