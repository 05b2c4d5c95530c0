// Host side of the C ABI (include/spmiqc.h): contexts, scratch, launches and
// the chains of kernels that make up each reference routine.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/spmiqc.h"
#include "blas1.cuh"
#include "spm_internal.h"
#include "spm_table.h"

using namespace spm;

// ------------------------------------------------------------------ errors
static thread_local std::string g_err;

int spm_fail(int status, const char *what) {
  g_err = what ? what : "";
  return status;
}
int spm_fail_cuda(cudaError_t e, const char *what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? SPM_ERR_NOMEM : SPM_ERR_CUDA;
}

extern "C" const char *spm_last_error(void) { return g_err.c_str(); }

extern "C" const char *spm_status_str(int s) {
  switch (s) {
    case SPM_OK: return "ok";
    case SPM_ERR_ARG: return "invalid argument";
    case SPM_ERR_CUDA: return "CUDA error";
    case SPM_ERR_NOMEM: return "device memory exhausted";
    case SPM_ERR_NONFINITE: return "non-finite result";
    case SPM_ERR_UNSUPPORTED: return "unsupported size or precision";
    case SPM_ERR_STATE: return "invalid call order";
    default: return "unknown status";
  }
}

extern "C" int spm_supported_size(int N) {
  switch (N) {
    case 32: case 64: case 96: case 128: case 160: case 192: case 256: return 1;
    default: return 0;
  }
}

// ------------------------------------------------------------------ dispatch
const OpsTable *spm_table_of(const spm_ctx *c) {
  switch (c->N) {
    case 32: return spm_table_32(c->prec);
    case 64: return spm_table_64(c->prec);
    case 96: return spm_table_96(c->prec);
    case 128: return spm_table_128(c->prec);
    case 160: return spm_table_160(c->prec);
    case 192: return spm_table_192(c->prec);
    case 256: return spm_table_256(c->prec);
    default: return nullptr;
  }
}

#define SPM_TRY(x)             \
  do {                         \
    int _s = (x);              \
    if (_s != SPM_OK) return _s; \
  } while (0)

// ------------------------------------------------------------------ context
KParams spm_params(const spm_ctx *c) {
  KParams p;
  std::memset(&p, 0, sizeof(p));
  p.m = c->m;
  p.tw = c->tw;
  p.partials = c->partials;
  p.tickets = c->tickets;
  p.scal = c->scal;
  p.flow = c->gate;
  return p;
}

int spm_ensure_scratch(spm_ctx *c, int nb) {
  if (nb <= c->scratch_cap) return SPM_OK;
  if (c->bufA) cudaFree(c->bufA);
  if (c->bufB) cudaFree(c->bufB);
  c->bufA = c->bufB = nullptr;
  c->scratch_cap = 0;
  const size_t bytes = c->field_bytes * (size_t)nb;
  cudaError_t e = cudaMalloc(&c->bufA, bytes);
  if (e != cudaSuccess) return spm_fail_cuda(e, "scratch A");
  e = cudaMalloc(&c->bufB, bytes);
  if (e != cudaSuccess) {
    cudaFree(c->bufA);
    c->bufA = nullptr;
    return spm_fail_cuda(e, "scratch B");
  }
  c->scratch_cap = nb;
  return SPM_OK;
}

char *spm_bufA(spm_ctx *c, int b) { return (char *)c->bufA + c->field_bytes * (size_t)b; }
char *spm_bufB(spm_ctx *c, int b) { return (char *)c->bufB + c->field_bytes * (size_t)b; }

int spm_read_scal(spm_ctx *c, int nb) {
  cudaError_t e = cudaMemcpyAsync(c->host_scal, c->scal, sizeof(double) * kScal * nb, cudaMemcpyDeviceToHost,
                                  c->stream);
  if (e != cudaSuccess) return spm_fail_cuda(e, "scalar read");
  e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? SPM_OK : spm_fail_cuda(e, "stream sync");
}

extern "C" int spm_ctx_create(int N, double L, double Tau, double Gamma, double dt, int precision, void *stream,
                              spm_ctx **out) {
  if (!out) return spm_fail(SPM_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (!spm_supported_size(N)) return spm_fail(SPM_ERR_UNSUPPORTED, "grid size not built");
  if (precision != SPM_FP64 && precision != SPM_FP32) return spm_fail(SPM_ERR_UNSUPPORTED, "precision");
  if (!(L > 0) || !std::isfinite(L) || !std::isfinite(Tau) || !std::isfinite(Gamma) || !std::isfinite(dt))
    return spm_fail(SPM_ERR_ARG, "model parameters");
  spm_ctx *c = new spm_ctx();
  c->N = N;
  c->prec = precision;
  c->stream = (cudaStream_t)stream;
  cudaGetDevice(&c->device);
  const double n3 = (double)N * N * N;
  c->m.Tau = Tau;
  c->m.Gamma = Gamma;
  c->m.dt = dt;
  c->m.invL = 1.0 / L;
  c->m.inv_n3 = 1.0 / n3;
  c->m.n3 = n3;
  {  // G(0) and the preconditioner symbol at k = 0 (Initialization.cpp:123-166)
    const double ph = 0.568809, s2 = ph * ph, k2 = 0.0;
    c->m.G0 = std::exp(-0.5 * k2 / s2) * 1.969182919080340 + 0.08;
    c->m.ikt0 = 1.0 / (c->m.G0 + std::fabs(Tau) + 0.02);
  }
  c->m.tol_grad = 0.0;
  c->m.factor = 1.0;
  const size_t real_sz = precision == SPM_FP64 ? 8 : 4;
  c->field_bytes = (size_t)N * N * N * real_sz;
  // twiddle table exp(-2 pi i j / N)
  {
    std::vector<double> twd(2 * N);
    std::vector<float> twf(2 * N);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int j = 0; j < N; j++) {
      long double a = 2.0L * pi * (long double)j / (long double)N;
      twd[2 * j] = (double)cosl(a);
      twd[2 * j + 1] = (double)(-sinl(a));
      twf[2 * j] = (float)cosl(a);
      twf[2 * j + 1] = (float)(-sinl(a));
    }
    const size_t bytes = 2 * N * real_sz;
    cudaError_t e = cudaMalloc(&c->tw, bytes);
    if (e != cudaSuccess) { delete c; return spm_fail_cuda(e, "twiddles"); }
    e = cudaMemcpy(c->tw, precision == SPM_FP64 ? (const void *)twd.data() : (const void *)twf.data(), bytes,
                   cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { spm_ctx_destroy(c); return spm_fail_cuda(e, "twiddles"); }
  }
  cudaError_t e = cudaMalloc(&c->partials, sizeof(double) * kPartStride * kRedMax * kMaxBatch);
  if (e == cudaSuccess) e = cudaMalloc(&c->tickets, sizeof(unsigned) * kMaxBatch);
  if (e == cudaSuccess) e = cudaMemset(c->tickets, 0, sizeof(unsigned) * kMaxBatch);
  if (e == cudaSuccess) e = cudaMalloc(&c->scal, sizeof(double) * kScal * kMaxBatch);
  if (e == cudaSuccess) e = cudaMemset(c->scal, 0, sizeof(double) * kScal * kMaxBatch);
  if (e == cudaSuccess) e = cudaMalloc(&c->flow, sizeof(int) * 8);
  if (e == cudaSuccess) e = cudaMallocHost(&c->host_scal, sizeof(double) * kScal * kMaxBatch);
  if (e == cudaSuccess) e = cudaMallocHost(&c->host_flow, sizeof(int) * 8);
  if (e != cudaSuccess) {
    spm_ctx_destroy(c);
    return spm_fail_cuda(e, "context buffers");
  }
  *out = c;
  return SPM_OK;
}

extern "C" int spm_ctx_destroy(spm_ctx *c) {
  if (!c) return SPM_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  else cudaDeviceSynchronize();
  spm_free_extra(c);
  cudaFree(c->tw);
  cudaFree(c->partials);
  cudaFree(c->tickets);
  cudaFree(c->scal);
  cudaFree(c->flow);
  cudaFree(c->stats);
  cudaFree(c->bufA);
  cudaFree(c->bufB);
  cudaFree(c->host_phi);
  cudaFree(c->host_uhat);
  if (c->host_scal) cudaFreeHost(c->host_scal);
  if (c->host_flow) cudaFreeHost(c->host_flow);
  delete c;
  return SPM_OK;
}

extern "C" int spm_set_stream(spm_ctx *c, void *stream) {
  if (!c) return spm_fail(SPM_ERR_ARG, "ctx is NULL");
  c->stream = (cudaStream_t)stream;
  return SPM_OK;
}

extern "C" int spm_sync(spm_ctx *c) {
  if (!c) return spm_fail(SPM_ERR_ARG, "ctx is NULL");
  cudaError_t e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? SPM_OK : spm_fail_cuda(e, "stream sync");
}

extern "C" size_t spm_field_bytes(const spm_ctx *c) { return c ? c->field_bytes : 0; }
extern "C" size_t spm_spectrum_bytes(const spm_ctx *c) { return c ? c->field_bytes : 0; }
extern "C" uint64_t spm_launch_count(const spm_ctx *c) { return c ? c->launches : 0; }

// ------------------------------------------------------------------ transforms
extern "C" int spm_fft(spm_ctx *c, const void *x, void *xhat) {
  if (!c || !x || !xhat) return spm_fail(SPM_ERR_ARG, "null argument");
  SPM_TRY(spm_ensure_scratch(c, 1));
  return spm_table_of(c)->fft(c, x, xhat);
}

extern "C" int spm_ifft(spm_ctx *c, const void *xhat, void *x) {
  if (!c || !x || !xhat) return spm_fail(SPM_ERR_ARG, "null argument");
  SPM_TRY(spm_ensure_scratch(c, 1));
  return spm_table_of(c)->ifft(c, xhat, x);
}

extern "C" int spm_spectrum_to_full(spm_ctx *c, const void *xhat, double *full) {
  if (!c || !xhat || !full) return spm_fail(SPM_ERR_ARG, "null argument");
  c->launches++;
  if (c->prec == SPM_FP64)
    packed_to_full_kernel<double><<<1184, 256, 0, c->stream>>>((const double2 *)xhat, (double2 *)full, c->N);
  else
    packed_to_full_kernel<float><<<1184, 256, 0, c->stream>>>((const float2 *)xhat, (double2 *)full, c->N);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SPM_OK : spm_fail_cuda(e, "packed_to_full");
}

extern "C" int spm_spectrum_from_full(spm_ctx *c, const double *full, void *xhat) {
  if (!c || !xhat || !full) return spm_fail(SPM_ERR_ARG, "null argument");
  c->launches++;
  if (c->prec == SPM_FP64)
    full_to_packed_kernel<double><<<1184, 256, 0, c->stream>>>((const double2 *)full, (double2 *)xhat, c->N);
  else
    full_to_packed_kernel<float><<<1184, 256, 0, c->stream>>>((const double2 *)full, (float2 *)xhat, c->N);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SPM_OK : spm_fail_cuda(e, "full_to_packed");
}

// ------------------------------------------------------------------ energy, gradient
extern "C" int spm_energy(spm_ctx *c, const void *phi, const void *uhat, double *energy) {
  if (!c || !phi || !uhat || !energy) return spm_fail(SPM_ERR_ARG, "null argument");
  SPM_TRY(spm_table_of(c)->energy(c, phi, uhat));
  SPM_TRY(spm_read_scal(c, 1));
  *energy = c->host_scal[SC_E1] + c->host_scal[SC_E2];
  if (!std::isfinite(*energy)) return spm_fail(SPM_ERR_NONFINITE, "energy is not finite");
  return SPM_OK;
}

static __global__ void flow_init_kernel(int *flow) {
  flow[FW_GO] = 1;
  flow[FW_PENDING] = 0;
  flow[FW_ITER] = 0;
  flow[3] = 0;
}

static int ensure_stats(spm_ctx *c, int n) {
  if (c->stats_cap >= n) return SPM_OK;
  if (c->stats) cudaStreamSynchronize(c->stream);
  cudaFree(c->stats);
  c->stats = nullptr;
  c->stats_cap = 0;
  const int cap = std::max(n, 1024);
  cudaError_t e = cudaMalloc(&c->stats, sizeof(double) * 4 * (size_t)cap);
  if (e != cudaSuccess) return spm_fail_cuda(e, "stats buffer");
  c->stats_cap = cap;
  return SPM_OK;
}

extern "C" int spm_grad_flow_enqueue(spm_ctx *c, void *phi, void *uhat, int nsteps, double tol_grad) {
  if (!c || !phi || !uhat || nsteps < 0) return spm_fail(SPM_ERR_ARG, "bad argument");
  SPM_TRY(spm_ensure_scratch(c, 1));
  SPM_TRY(ensure_stats(c, nsteps));
  c->launches++;
  flow_init_kernel<<<1, 1, 0, c->stream>>>(c->flow);
  const OpsTable *t = spm_table_of(c);
  c->m.tol_grad = tol_grad;
  int rc = SPM_OK;
  for (int i = 0; i < nsteps && rc == SPM_OK; i++) rc = t->grad_step(c, phi, uhat);
  c->m.tol_grad = 0.0;
  return rc;
}

extern "C" int spm_grad_flow_collect(spm_ctx *c, spm_step_stats *stats, int max_records, int *steps_done) {
  if (!c) return spm_fail(SPM_ERR_ARG, "ctx is NULL");
  cudaError_t e = cudaMemcpyAsync(c->host_flow, c->flow, sizeof(int) * 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return spm_fail_cuda(e, "grad flow");
  const int done = c->host_flow[FW_ITER];
  if (steps_done) *steps_done = done;
  const int n = std::min(done, max_records);
  if (stats && n > 0) {
    e = cudaMemcpy(stats, c->stats, sizeof(double) * 4 * (size_t)n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return spm_fail_cuda(e, "stats read");
    for (int i = 0; i < n; i++)
      if (!std::isfinite(stats[i].energy) || !std::isfinite(stats[i].grad_norm))
        return spm_fail(SPM_ERR_NONFINITE, "non-finite energy or gradient norm");
  }
  return SPM_OK;
}

extern "C" int spm_grad_flow(spm_ctx *c, void *phi, void *uhat, int max_steps, double tol_grad,
                             spm_step_stats *stats, int *steps_done) {
  if (!c || !phi || !uhat || max_steps < 0) return spm_fail(SPM_ERR_ARG, "bad argument");
  if (steps_done) *steps_done = 0;
  if (max_steps == 0) return SPM_OK;
  SPM_TRY(spm_ensure_scratch(c, 1));
  SPM_TRY(ensure_stats(c, max_steps));
  c->launches++;
  flow_init_kernel<<<1, 1, 0, c->stream>>>(c->flow);
  const OpsTable *t = spm_table_of(c);
  c->m.tol_grad = tol_grad;
  int enq = 0, chunk = 8, rc = SPM_OK;
  cudaError_t e = cudaSuccess;
  while (enq < max_steps) {
    const int n = std::min(chunk, max_steps - enq);
    for (int i = 0; i < n && rc == SPM_OK; i++) rc = t->grad_step(c, phi, uhat);
    if (rc != SPM_OK) break;
    enq += n;
    e = cudaMemcpyAsync(c->host_flow, c->flow, sizeof(int) * 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { rc = spm_fail_cuda(e, "grad flow"); break; }
    if (c->host_flow[FW_GO] == 0) break;
    chunk = std::min(chunk * 2, 256);
  }
  c->m.tol_grad = 0.0;
  if (rc != SPM_OK) return rc;
  return spm_grad_flow_collect(c, stats, max_steps, steps_done);
}

extern "C" int spm_grad_flow_host(spm_ctx *c, void *phi_host, int max_steps, double tol_grad,
                                  spm_step_stats *stats, int *steps_done) {
  if (!c || !phi_host || max_steps < 0) return spm_fail(SPM_ERR_ARG, "bad argument");
  if (!c->host_phi) {
    cudaError_t e = cudaMalloc(&c->host_phi, c->field_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&c->host_uhat, c->field_bytes);
    if (e != cudaSuccess) return spm_fail_cuda(e, "host-path buffers");
  }
  cudaError_t e = cudaMemcpyAsync(c->host_phi, phi_host, c->field_bytes, cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return spm_fail_cuda(e, "phi upload");
  SPM_TRY(spm_fft(c, c->host_phi, c->host_uhat));
  SPM_TRY(spm_grad_flow(c, c->host_phi, c->host_uhat, max_steps, tol_grad, stats, steps_done));
  e = cudaMemcpyAsync(phi_host, c->host_phi, c->field_bytes, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? SPM_OK : spm_fail_cuda(e, "phi download");
}

extern "C" int spm_grad_step_profile(spm_ctx *c, void *phi, void *uhat, int reps, double *ms) {
  if (!c || !phi || !uhat || !ms || reps < 1) return spm_fail(SPM_ERR_ARG, "bad argument");
  SPM_TRY(spm_ensure_scratch(c, 1));
  SPM_TRY(ensure_stats(c, reps));
  c->launches++;
  flow_init_kernel<<<1, 1, 0, c->stream>>>(c->flow);
  cudaEvent_t ev[4];
  for (int i = 0; i < 4; i++) cudaEventCreate(&ev[i]);
  double acc[3] = {0, 0, 0};
  int rc = SPM_OK;
  const OpsTable *t = spm_table_of(c);
  for (int r = 0; r < reps && rc == SPM_OK; r++) {
    rc = t->grad_step_ev(c, phi, uhat, (void *const *)ev);
    if (rc != SPM_OK) break;
    cudaError_t e = cudaEventSynchronize(ev[3]);
    if (e != cudaSuccess) { rc = spm_fail_cuda(e, "profile"); break; }
    for (int k = 0; k < 3; k++) {
      float f = 0;
      cudaEventElapsedTime(&f, ev[k], ev[k + 1]);
      acc[k] += f;
    }
  }
  for (int i = 0; i < 4; i++) cudaEventDestroy(ev[i]);
  for (int k = 0; k < 3; k++) ms[k] = acc[k] / reps;
  return rc;
}

extern "C" int spm_ngrad(spm_ctx *c, const void *phi, void *grad, double *norm) {
  if (!c || !phi || !grad) return spm_fail(SPM_ERR_ARG, "null argument");
  SPM_TRY(spm_ensure_scratch(c, 1));
  SPM_TRY(spm_table_of(c)->ngrad(c, phi, grad));
  if (norm) {
    SPM_TRY(spm_read_scal(c, 1));
    *norm = std::sqrt(c->host_scal[SC_GN2]);
    if (!std::isfinite(*norm)) return spm_fail(SPM_ERR_NONFINITE, "gradient norm is not finite");
  }
  return SPM_OK;
}

extern "C" int spm_hv(spm_ctx *c, const void *phi, const void *v, void *hv, int nb) {
  if (!c || !phi || !v || !hv || nb < 1) return spm_fail(SPM_ERR_ARG, "bad argument");
  for (int b0 = 0; b0 < nb; b0 += kMaxBatch) {
    const int n = std::min(kMaxBatch, nb - b0);
    SPM_TRY(spm_ensure_scratch(c, n));
    const void *vv[kMaxBatch];
    void *hh[kMaxBatch];
    for (int b = 0; b < n; b++) {
      vv[b] = (const char *)v + c->field_bytes * (size_t)(b0 + b);
      hh[b] = (char *)hv + c->field_bytes * (size_t)(b0 + b);
    }
    SPM_TRY(spm_table_of(c)->hv(c, phi, vv, hh, n));
  }
  return SPM_OK;
}

extern "C" int spm_precond(spm_ctx *c, void *w, int nb) {
  if (!c || !w || nb < 1) return spm_fail(SPM_ERR_ARG, "bad argument");
  for (int b0 = 0; b0 < nb; b0 += kMaxBatch) {
    const int n = std::min(kMaxBatch, nb - b0);
    SPM_TRY(spm_ensure_scratch(c, n));
    void *ww[kMaxBatch];
    for (int b = 0; b < n; b++) ww[b] = (char *)w + c->field_bytes * (size_t)(b0 + b);
    SPM_TRY(spm_table_of(c)->precond(c, ww, n));
  }
  return SPM_OK;
}

extern "C" int spm_inpfp(spm_ctx *c, const void *pp, const void *qq, double *out) {
  if (!c || !pp || !qq || !out) return spm_fail(SPM_ERR_ARG, "null argument");
  SPM_TRY(spm_table_of(c)->dot(c, pp, qq));
  SPM_TRY(spm_read_scal(c, 1));
  *out = c->host_scal[SC_SUM0];
  return SPM_OK;
}
