// Context layout and helpers shared by the host translation units of
// libspmiqc_cuda.so (not part of the public ABI).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "fft_core.cuh"

// Box shapes of the tensor copies over a packed spectrum [x][ky][2*(N/2) reals].
enum TmKind {
  TM_PENCIL = 0,     // 8 complex columns x 1 ky row x all N x
  TM_PLANE_INV = 1,  // 16 complex columns x all N ky x 1 x-plane
  TM_PENCIL4 = 2     // 4 complex columns x 1 ky row x all N x (narrow pencil tiles)
};
struct TmEntry {
  const void *ptr;
  int kind;
  CUtensorMap map;
};

struct spm_ctx {
  int N = 0;
  int prec = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  spm::ModelC m{};
  double L = 0;             // box length as given
  size_t field_bytes = 0;   // bytes of one real field = bytes of one packed spectrum
  void *tw = nullptr;       // twiddle table exp(-2 pi i j/N) in the context precision
  double *partials = nullptr;
  unsigned *tickets = nullptr;
  double *scal = nullptr;
  int *flow = nullptr;
  double *stats = nullptr;
  int stats_cap = 0;
  void *bufA = nullptr;     // spectral scratch, scratch_cap fields
  void *bufB = nullptr;
  int scratch_cap = 0;
  double *host_scal = nullptr;  // pinned
  int *host_flow = nullptr;     // pinned
  uint64_t launches = 0;
  void *extra = nullptr;        // solver state (LOBPCG / SPM work arrays)
  void *host_phi = nullptr;     // device copies used by the host-buffer entry points
  void *host_uhat = nullptr;
  int *gate = nullptr;          // flow words gating every launch of a solver chain (or null)
  double *gtab = nullptr;       // spectral symbols per K^2 (4 doubles each)
  std::vector<TmEntry> tmaps;   // tensor-map cache (most recent last)
  int plane_cps = 2;            // plane-kernel variant: CTAs per SM (1 staged; 2, 3 direct; 4 FP32 chains)
  int fuse_planes = 1;          // gradient chains use the fused inverse -> forward plane pass
  int plane_xg = 0;             // gradient-chain plane kernels: exchanges through L2 (spm::kXgFwd | kXgInv bits)
  void *xg = nullptr;           // their global exchange areas (2 x xg_cap CTAs x 16 N complex)
  int xg_cap = 0;
  int batch_group = 1;          // spm_batch_grad_flow: same-size instances share launches (knob "batch_group")
  int pencil_tc = 8;            // pencil tile width in complex columns: 8 or 4 (knob "pencil_tc")
  int block_stage = 1;          // solver Grams stage their fields through shared memory (knob "block_stage")
  int pdl = 0;                  // plane and pencil kernels launched as programmatic dependents (knob "pdl")
  double spring_len = 0.0;      // SPM spring rest length (0: the reference's zero-length spring)
  spm_ctx *twin = nullptr;      // FP32 twin of an FP64 context (mixed-precision flows)
  void *twin_buf = nullptr;     // FP32 phi and uhat of the twin
  const volatile int *cancel = nullptr;  // host flag polled between chunks of steps (job server)
};

inline bool spm_cancelled(const spm_ctx *c) { return c->cancel && *c->cancel; }

int spm_fail(int status, const char *what);
int spm_fail_cuda(cudaError_t e, const char *what);
spm::KParams spm_params(const spm_ctx *c);
int spm_ensure_scratch(spm_ctx *c, int nb);
// Allocates the global exchange areas when c->plane_xg asks for them.
int spm_ensure_xg(spm_ctx *c);
char *spm_bufA(spm_ctx *c, int b);
char *spm_bufB(spm_ctx *c, int b);
int spm_read_scal(spm_ctx *c, int nb);
int spm_check_device_error(spm_ctx *c);
int spm_flow_init(spm_ctx *c, cudaStream_t s);    // go = 1, iter = 0
int spm_ensure_stats(spm_ctx *c, int n);          // per-step record capacity
// Tensor map of kind `kind` over the packed spectrum at ptr (cached per context).
int spm_tensor_map(spm_ctx *c, const void *ptr, int kind, CUtensorMap *out);
void spm_free_extra(spm_ctx *c);
// Creates (once) the FP32 twin context and its two FP32 fields, and binds it
// to the context's stream, cancel flag and tuning.
int spm_ensure_twin(spm_ctx *c);
// Decides when the FP32 phase of a mixed-precision run has reached its
// rounding floor, from its sequence of residuals (||grad F|| or the SPM
// residual); switch_at is the residual at which the phase hands over anyway.
struct FloorWatch {
  double sw, best = 1e300;
  int short_win, long_win, n = 0, last = 0;
  FloorWatch(double switch_at, int window);
  bool step(double r);
};

// The autotuner's remembered choice for (device, N, precision), if any.
bool spm_autotune_lookup(int device, int N, int prec, int *plane_cps, int *fuse_planes, int *plane_xg,
                         int *pencil_tc = nullptr, int *pdl = nullptr);
const struct OpsTable *spm_table_of(const spm_ctx *c);
