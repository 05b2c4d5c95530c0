// Host side of the C ABI (include/spmiqc.h): contexts, scratch, launches and
// the chains of kernels that make up each reference routine.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
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
    case SPM_ERR_CANCELLED: return "cancelled";
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
  p.gtab = reinterpret_cast<const double4 *>(c->gtab);
  p.err = c->flow + FW_ERR;
  p.xg = c->xg;
  p.xg_cap = c->xg_cap;
  p.xg_regions = c->xg ? spm::kXgRegions : 0;
  return p;
}

// One area per resident CTA of a plane kernel, exchange and region (two
// regions per exchange, for the software-pipelined fused pass): at most
// min(SMs x CTAs per SM, N x CL) CTAs, the CTAs per SM bounded by the plane
// kernels' shared memory and 8 blocks of 256 threads.
int spm_ensure_xg(spm_ctx *c) {
  if (!c->plane_xg || c->xg) return SPM_OK;
  int sms = 0, smem_sm = 0;
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c->device);
  if (e != cudaSuccess) return spm_fail_cuda(e, "device attributes");
  const size_t cplx = c->prec == SPM_FP64 ? 16 : 8;
  const size_t units = 16 * (size_t)c->N;  // PLANE_UNITS
  const size_t smem = cplx * (c->N + c->N / 2 + units) + 16 + 8 * 32 * spm::kRedMax + 128 + 1024;
  int per_sm = (int)(smem_sm / smem);
  per_sm = per_sm < 1 ? 1 : (per_sm > 8 ? 8 : per_sm);
  const int most = c->N * (c->N / spm::kRows);
  const int cap = sms * per_sm < most ? sms * per_sm : most;
  e = cudaMalloc(&c->xg, (size_t)spm::kXgRegions * cap * units * cplx);
  if (e != cudaSuccess) {
    c->xg = nullptr;
    return spm_fail_cuda(e, "plane exchange areas");
  }
  c->xg_cap = cap;
  return SPM_OK;
}

int spm_ensure_scratch(spm_ctx *c, int nb) {
  SPM_TRY(spm_ensure_xg(c));
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

// ------------------------------------------------------------------ tensor maps
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  });
  return fn;
}

int spm_tensor_map(spm_ctx *c, const void *ptr, int kind, CUtensorMap *out) {
  for (size_t i = c->tmaps.size(); i-- > 0;)
    if (c->tmaps[i].ptr == ptr && c->tmaps[i].kind == kind) {
      *out = c->tmaps[i].map;
      return SPM_OK;
    }
  if (((uintptr_t)ptr & 15u) != 0) return spm_fail(SPM_ERR_ARG, "spectrum buffers must be 16-byte aligned");
  auto fn = encode_fn();
  if (!fn) return spm_fail(SPM_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  const int N = c->N;
  const size_t es = c->prec == SPM_FP64 ? 8 : 4;
  const cuuint64_t dims[3] = {(cuuint64_t)N, (cuuint64_t)N, (cuuint64_t)N};  // N reals = N/2 complex per row
  const cuuint64_t strides[2] = {(cuuint64_t)N * es, (cuuint64_t)N * N * es};
  cuuint32_t box[3];
  if (kind == TM_PENCIL || kind == TM_PENCIL4) {
    box[0] = kind == TM_PENCIL ? 16 : 8;  // 8 or 4 complex columns
    box[1] = 1;
    box[2] = (cuuint32_t)N;
  } else {
    box[0] = 32;  // 16 complex columns
    box[1] = (cuuint32_t)N;
    box[2] = 1;
  }
  const cuuint32_t estr[3] = {1, 1, 1};
  TmEntry e;
  e.ptr = ptr;
  e.kind = kind;
  CUresult r = fn(&e.map, es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                  const_cast<void *>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return spm_fail(SPM_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  if (c->tmaps.size() >= 64) c->tmaps.erase(c->tmaps.begin());
  c->tmaps.push_back(e);
  *out = e.map;
  return SPM_OK;
}

// Reads (and clears) the error word that bounded waits set on timeout.
int spm_check_device_error(spm_ctx *c) {
  int err = 0;
  cudaError_t e = cudaMemcpy(&err, c->flow + FW_ERR, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return spm_fail_cuda(e, "error word read");
  if (err) {
    cudaMemset(c->flow + FW_ERR, 0, sizeof(int));
    return spm_fail(SPM_ERR_CUDA, "a kernel's bounded wait for its asynchronous copies timed out");
  }
  return SPM_OK;
}

// The failure path of the bounded waits, run on purpose: one thread arrives
// on an mbarrier expecting 16 bytes of transactions and no copy is issued, so
// the phase cannot complete; the wait gives up after `polls` polls, the CTA
// reports through the context's error word and returns. Nothing is in flight
// when it returns (no copy was issued), so the context stays usable.
static __global__ void bounded_wait_selftest_kernel(int *err, long polls) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_err;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    s_err = 0;
    fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_expect_tx(&bar, 16);
  __syncthreads();
  mbar_wait_n(&bar, 0, &s_err, polls);
  __syncthreads();
  if (threadIdx.x == 0 && s_err) atomicExch(err, 1);
}

extern "C" int spm_selftest_bounded_wait(spm_ctx *c, int polls) {
  if (!c || polls < 1 || polls > (int)kSpinLimit) return spm_fail(SPM_ERR_ARG, "polls must be in [1, 2^22]");
  c->launches++;
  bounded_wait_selftest_kernel<<<1, 32, 0, c->stream>>>(c->flow + FW_ERR, (long)polls);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return spm_fail_cuda(e, "bounded-wait self-test");
  return spm_check_device_error(c);
}

int spm_read_scal(spm_ctx *c, int nb) {
  // the scalars and the error word of the bounded waits in one round trip
  cudaError_t e = cudaMemcpyAsync(c->host_scal, c->scal, sizeof(double) * kScal * nb, cudaMemcpyDeviceToHost,
                                  c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(c->host_flow + FW_ERR, c->flow + FW_ERR, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  if (e != cudaSuccess) return spm_fail_cuda(e, "scalar read");
  e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return spm_fail_cuda(e, "stream sync");
  return c->host_flow[FW_ERR] ? spm_check_device_error(c) : SPM_OK;
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
  c->L = L;
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
  // Spectral symbols per K^2 = Kx^2 + Ky^2 + Kz^2 (every K in [-N/2, N/2)):
  // G(k^2) with k^2 = K^2 / L^2 (get_GK, Initialization.cpp:150-166), the
  // gradient-step factor 1/(1 + dt G) (LPsrc.cpp:64-67), the preconditioner
  // symbol 1/(G + |Tau| + 0.02) (Initialization.cpp:123-129) and the force-step
  // factor 1/(1 + G) (SPM.cpp:82-86).
  {
    const int kmax = 3 * (N / 2) * (N / 2);
    std::vector<double> tab(4 * (size_t)(kmax + 1));
    const double ph = 0.568809, s2 = ph * ph, invL = 1.0 / L;
    for (int K2 = 0; K2 <= kmax; K2++) {
      const double k2 = (double)K2 * (invL * invL);
      const double k4 = k2 * k2, k6 = k4 * k2, k8 = k6 * k2;
      const double G = std::exp(-0.5 * k2 / s2) *
                           (1.969182919080340 + -14.949858723012090 * k2 + 37.445683882581790 * k4 +
                            -38.839451762550148 * k6 + 13.999261011773505 * k8) +
                       0.08;
      tab[4 * (size_t)K2 + 0] = G;
      tab[4 * (size_t)K2 + 1] = 1.0 / (1.0 + dt * G);
      tab[4 * (size_t)K2 + 2] = 1.0 / (G + std::fabs(Tau) + 0.02);
      tab[4 * (size_t)K2 + 3] = 1.0 / (1.0 + G);
    }
    cudaError_t e = cudaMalloc(&c->gtab, sizeof(double) * tab.size());
    if (e == cudaSuccess)
      e = cudaMemcpy(c->gtab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      spm_ctx_destroy(c);
      return spm_fail_cuda(e, "symbol table");
    }
  }
  cudaError_t e = cudaMalloc(&c->partials, sizeof(double) * kPartStride * kRedMax * kMaxBatch);
  if (e == cudaSuccess) e = cudaMalloc(&c->tickets, sizeof(unsigned) * kMaxBatch);
  if (e == cudaSuccess) e = cudaMemset(c->tickets, 0, sizeof(unsigned) * kMaxBatch);
  if (e == cudaSuccess) e = cudaMalloc(&c->scal, sizeof(double) * kScal * kMaxBatch);
  if (e == cudaSuccess) e = cudaMemset(c->scal, 0, sizeof(double) * kScal * kMaxBatch);
  if (e == cudaSuccess) e = cudaMalloc(&c->flow, sizeof(int) * 8);
  if (e == cudaSuccess) e = cudaMemset(c->flow, 0, sizeof(int) * 8);
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
  if (c->twin) spm_ctx_destroy(c->twin);
  cudaFree(c->twin_buf);
  cudaFree(c->tw);
  cudaFree(c->gtab);
  cudaFree(c->partials);
  cudaFree(c->tickets);
  cudaFree(c->scal);
  cudaFree(c->flow);
  cudaFree(c->stats);
  cudaFree(c->bufA);
  cudaFree(c->bufB);
  cudaFree(c->xg);
  cudaFree(c->host_phi);
  cudaFree(c->host_uhat);
  if (c->host_scal) cudaFreeHost(c->host_scal);
  if (c->host_flow) cudaFreeHost(c->host_flow);
  delete c;
  return SPM_OK;
}

extern "C" int spm_tune(spm_ctx *c, const char *knob, int value) {
  if (!c || !knob) return spm_fail(SPM_ERR_ARG, "null argument");
  if (std::strcmp(knob, "plane_cps") == 0) {
    if (value < 1 || value > 6) return spm_fail(SPM_ERR_ARG, "plane_cps must be 1 to 6");
    c->plane_cps = value;
    return SPM_OK;
  }
  if (std::strcmp(knob, "fuse_planes") == 0) {
    if (value != 0 && value != 1) return spm_fail(SPM_ERR_ARG, "fuse_planes must be 0 or 1");
    c->fuse_planes = value;
    return SPM_OK;
  }
  if (std::strcmp(knob, "plane_xg") == 0) {
    if (value < 0 || value > 3) return spm_fail(SPM_ERR_ARG, "plane_xg must be 0..3");
    c->plane_xg = value;
    return spm_ensure_xg(c);
  }
  if (std::strcmp(knob, "batch_group") == 0) {
    if (value != 0 && value != 1) return spm_fail(SPM_ERR_ARG, "batch_group must be 0 or 1");
    c->batch_group = value;
    return SPM_OK;
  }
  if (std::strcmp(knob, "pencil_tc") == 0) {
    if (value != 8 && value != 4) return spm_fail(SPM_ERR_ARG, "pencil_tc must be 8 or 4");
    c->pencil_tc = value;
    return SPM_OK;
  }
  if (std::strcmp(knob, "block_stage") == 0) {
    if (value != 0 && value != 1) return spm_fail(SPM_ERR_ARG, "block_stage must be 0 or 1");
    c->block_stage = value;
    return SPM_OK;
  }
  if (std::strcmp(knob, "pdl") == 0) {
    if (value != 0 && value != 1) return spm_fail(SPM_ERR_ARG, "pdl must be 0 or 1");
    c->pdl = value;
    return SPM_OK;
  }
  return spm_fail(SPM_ERR_ARG, "unknown tuning knob");
}

extern "C" int spm_tune_get(const spm_ctx *c, const char *knob) {
  if (!c || !knob) return -1;
  if (std::strcmp(knob, "plane_cps") == 0) return c->plane_cps;
  if (std::strcmp(knob, "fuse_planes") == 0) return c->fuse_planes;
  if (std::strcmp(knob, "plane_xg") == 0) return c->plane_xg;
  if (std::strcmp(knob, "batch_group") == 0) return c->batch_group;
  if (std::strcmp(knob, "pencil_tc") == 0) return c->pencil_tc;
  if (std::strcmp(knob, "block_stage") == 0) return c->block_stage;
  if (std::strcmp(knob, "pdl") == 0) return c->pdl;
  return -1;
}

extern "C" int spm_set_stream(spm_ctx *c, void *stream) {
  if (!c) return spm_fail(SPM_ERR_ARG, "ctx is NULL");
  c->stream = (cudaStream_t)stream;
  return SPM_OK;
}

extern "C" int spm_sync(spm_ctx *c) {
  if (!c) return spm_fail(SPM_ERR_ARG, "ctx is NULL");
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return spm_fail_cuda(e, "stream sync");
  return spm_check_device_error(c);
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

int spm_flow_init(spm_ctx *c, cudaStream_t s) {
  c->launches++;
  flow_init_kernel<<<1, 1, 0, s>>>(c->flow);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SPM_OK : spm_fail_cuda(e, "flow init");
}

int spm_ensure_stats(spm_ctx *c, int n);
static int ensure_stats(spm_ctx *c, int n) { return spm_ensure_stats(c, n); }

int spm_ensure_stats(spm_ctx *c, int n) {
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
  rc = t->grad_steps(c, phi, uhat, nsteps);
  c->m.tol_grad = 0.0;
  return rc;
}

extern "C" int spm_grad_flow_collect(spm_ctx *c, spm_step_stats *stats, int max_records, int *steps_done) {
  if (!c) return spm_fail(SPM_ERR_ARG, "ctx is NULL");
  cudaError_t e = cudaMemcpyAsync(c->host_flow, c->flow, sizeof(int) * 8, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return spm_fail_cuda(e, "grad flow");
  SPM_TRY(spm_check_device_error(c));
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
    rc = t->grad_steps(c, phi, uhat, n);
    if (rc != SPM_OK) break;
    enq += n;
    e = cudaMemcpyAsync(c->host_flow, c->flow, sizeof(int) * 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { rc = spm_fail_cuda(e, "grad flow"); break; }
    if (c->host_flow[FW_GO] == 0) break;
    if (spm_cancelled(c)) { rc = spm_fail(SPM_ERR_CANCELLED, "cancelled"); break; }
    chunk = std::min(chunk * 2, 256);
  }
  c->m.tol_grad = 0.0;
  if (rc != SPM_OK) return rc;
  return spm_grad_flow_collect(c, stats, max_steps, steps_done);
}

FloorWatch::FloorWatch(double switch_at, int window) : sw(switch_at), short_win(window), long_win(16 * window) {}

// One more FP32 residual; true when the FP32 phase should hand over to FP64.
// A new best counts only if it is 0.5 % below the previous one. Flows are
// not monotone at first (a structure forming from a random field can raise
// ||grad F|| for thousands of steps), so a short stall (short_win residuals
// without a new best) ends the phase only once the best is within 10x of the
// switch point; anywhere, a long stall (long_win residuals) ends it.
bool FloorWatch::step(double r) {
  n++;
  if (r < 0.995 * best) {
    best = r;
    last = n;
    return false;
  }
  const int since = n - last;
  return (best < 10.0 * sw && since >= short_win) || since >= long_win;
}

int spm_ensure_twin(spm_ctx *c) {
  if (!c->twin) {
    const size_t n = (size_t)c->N * c->N * c->N;
    SPM_TRY(spm_ctx_create(c->N, c->L, c->m.Tau, c->m.Gamma, c->m.dt, SPM_FP32, c->stream, &c->twin));
    cudaError_t e = cudaMalloc(&c->twin_buf, 2 * n * sizeof(float));
    if (e != cudaSuccess) return spm_fail_cuda(e, "FP32 twin fields");
  }
  c->twin->stream = c->stream;
  c->twin->cancel = c->cancel;
  c->twin->plane_cps = c->plane_cps;
  c->twin->fuse_planes = c->fuse_planes;
  c->twin->plane_xg = c->plane_xg;
  c->twin->batch_group = c->batch_group;
  c->twin->pencil_tc = c->pencil_tc;
  c->twin->block_stage = c->block_stage;
  c->twin->pdl = c->pdl;
  c->twin->spring_len = c->spring_len;
  // an FP32 schedule chosen by spm_autotune on an FP32 context of this size wins
  spm_autotune_lookup(c->device, c->N, SPM_FP32, &c->twin->plane_cps, &c->twin->fuse_planes, &c->twin->plane_xg,
                      &c->twin->pencil_tc, &c->twin->pdl);
  return spm_ensure_xg(c->twin);
}

// Mixed precision: FP32 transforms with FP64 reductions until ||grad F|| <=
// switch_tol, then an FP64 polish from the FP32 state (phi in FP64, uhat =
// my_fft(phi) recomputed in FP64) to tol_grad.
extern "C" int spm_grad_flow_mixed(spm_ctx *c, void *phi, void *uhat, int max_steps, double tol_grad,
                                   double switch_tol, spm_step_stats *stats, int *steps_fp32, int *steps_fp64) {
  if (!c || !phi || !uhat || max_steps < 0 || !(tol_grad > 0)) return spm_fail(SPM_ERR_ARG, "bad argument");
  if (c->prec != SPM_FP64) return spm_fail(SPM_ERR_ARG, "mixed precision runs on an FP64 context");
  if (steps_fp32) *steps_fp32 = 0;
  if (steps_fp64) *steps_fp64 = 0;
  const size_t n = (size_t)c->N * c->N * c->N;
  SPM_TRY(spm_ensure_twin(c));
  float *phi32 = (float *)c->twin_buf, *uh32 = phi32 + n;
  c->launches += 2;
  cast_kernel<double, float><<<1184, 256, 0, c->stream>>>((const double *)phi, phi32, n);
  cast_kernel<double, float><<<1184, 256, 0, c->stream>>>((const double *)uhat, uh32, n);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return spm_fail_cuda(e, "cast");
  int n32 = 0, n64 = 0;
  const double sw = switch_tol > tol_grad ? switch_tol : tol_grad;
  // FP32 in windows of kWindow steps until ||grad F|| <= sw, or until FP32
  // stops making progress (its rounding floor): see FloorWatch.
  constexpr int kWindow = 512;
  std::vector<spm_step_stats> rec(kWindow);
  FloorWatch watch(sw, kWindow);
  while (n32 < max_steps) {
    const int chunk = std::min(kWindow, max_steps - n32);
    int done = 0;
    spm_step_stats *out = stats ? stats + n32 : rec.data();
    SPM_TRY(spm_grad_flow(c->twin, phi32, uh32, chunk, sw, out, &done));
    n32 += done;
    if (done == 0) break;
    if (done < chunk || out[done - 1].grad_norm <= sw || out[done - 1].res <= 1e-16) break;
    bool stop = false;
    for (int i = 0; i < done && !stop; i++) stop = watch.step(out[i].grad_norm);
    if (stop) break;
  }
  c->launches += c->twin->launches;
  c->twin->launches = 0;
  c->launches++;
  cast_kernel<float, double><<<1184, 256, 0, c->stream>>>(phi32, (double *)phi, n);
  e = cudaGetLastError();
  if (e != cudaSuccess) return spm_fail_cuda(e, "cast");
  SPM_TRY(spm_fft(c, phi, uhat));
  const int left = max_steps - n32;
  if (left > 0) SPM_TRY(spm_grad_flow(c, phi, uhat, left, tol_grad, stats ? stats + n32 : nullptr, &n64));
  if (steps_fp32) *steps_fp32 = n32;
  if (steps_fp64) *steps_fp64 = n64;
  return SPM_OK;
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
  if (!c || !phi || !uhat || !ms || reps < 2) return spm_fail(SPM_ERR_ARG, "bad argument (reps >= 2)");
  SPM_TRY(spm_ensure_scratch(c, 1));
  SPM_TRY(ensure_stats(c, reps));
  c->launches++;
  flow_init_kernel<<<1, 1, 0, c->stream>>>(c->flow);
  const OpsTable *t = spm_table_of(c);
  int rc = SPM_OK;
  for (int k = 0; k < 4; k++) ms[k] = 0.0;
  auto elapsed = [](cudaEvent_t a, cudaEvent_t b) {
    float f = 0;
    cudaEventElapsedTime(&f, a, b);
    return (double)f;
  };
  if (c->fuse_planes) {
    // one chain: plane_fwd, reps x (pencil, plane_inv_fwd), the last plane pass plane_inv
    std::vector<cudaEvent_t> ev(2 * (size_t)reps + 2);
    for (auto &e : ev) cudaEventCreate(&e);
    rc = t->grad_steps_ev(c, phi, uhat, reps, (void *const *)ev.data());
    if (rc == SPM_OK) {
      cudaError_t e = cudaEventSynchronize(ev.back());
      if (e != cudaSuccess) rc = spm_fail_cuda(e, "profile");
    }
    if (rc == SPM_OK) {
      ms[0] = elapsed(ev[0], ev[1]);
      for (int k = 0; k < reps; k++) ms[1] += elapsed(ev[1 + 2 * k], ev[2 + 2 * k]) / reps;
      for (int k = 0; k + 1 < reps; k++) ms[2] += elapsed(ev[2 + 2 * k], ev[3 + 2 * k]) / (reps - 1);
      ms[3] = elapsed(ev[2 * reps], ev[2 * reps + 1]);
    }
    for (auto &e : ev) cudaEventDestroy(e);
    return rc;
  }
  cudaEvent_t ev[4];
  for (int i = 0; i < 4; i++) cudaEventCreate(&ev[i]);
  double acc[3] = {0, 0, 0};
  for (int r = 0; r < reps && rc == SPM_OK; r++) {
    rc = t->grad_step_ev(c, phi, uhat, (void *const *)ev);
    if (rc != SPM_OK) break;
    cudaError_t e = cudaEventSynchronize(ev[3]);
    if (e != cudaSuccess) { rc = spm_fail_cuda(e, "profile"); break; }
    for (int k = 0; k < 3; k++) acc[k] += elapsed(ev[k], ev[k + 1]);
  }
  for (int i = 0; i < 4; i++) cudaEventDestroy(ev[i]);
  ms[0] = acc[0] / reps;
  ms[1] = acc[1] / reps;
  ms[3] = acc[2] / reps;
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
