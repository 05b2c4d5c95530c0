// Batched gradient flows of independent instances (grids of any supported
// sizes and parameters): one CUDA graph holds `steps_per_launch` gated steps of
// every instance, so one graph launch advances all of them. Instances of the
// same grid size and precision form groups of up to 16 that share every
// launch (one launch per pass for the whole group, blockIdx.y = instance,
// each instance with its own model, symbols and flow words); each group runs
// on its own stream branch, so groups of different sizes overlap on the
// device. (With the context knob "batch_group" = 0 on the first instance,
// every instance gets its own branch and launches instead.) Instances stop
// on the device (convergence or their step cap); the graph is relaunched until
// every instance has stopped. With switch_tol > 0 the instances first run on
// their FP32 twins (FP32 transforms, FP64 reductions) to switch_tol, then on
// FP64 to tol_grad.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/spmiqc.h"
#include "blas1.cuh"
#include "spm_internal.h"
#include "spm_table.h"

using namespace spm;

#define SPM_TRY(x)               \
  do {                           \
    int _s = (x);                \
    if (_s != SPM_OK) return _s; \
  } while (0)

namespace {

struct Streams {
  std::vector<cudaStream_t> s;
  std::vector<cudaEvent_t> ev;
  ~Streams() {
    for (auto x : s) cudaStreamDestroy(x);
    for (auto e : ev) cudaEventDestroy(e);
  }
};

// Instances grouped by (N, precision), at most kMaxBatch per group, in order
// of first appearance; with `group` false every instance is its own group.
std::vector<std::vector<int>> make_groups(spm_ctx *const *ctx, int n, bool group) {
  std::vector<std::vector<int>> g;
  for (int i = 0; i < n; i++) {
    bool placed = false;
    if (group)
      for (auto &grp : g)
        if ((int)grp.size() < kMaxBatch && ctx[grp[0]]->N == ctx[i]->N && ctx[grp[0]]->prec == ctx[i]->prec) {
          grp.push_back(i);
          placed = true;
          break;
        }
    if (!placed) g.push_back({i});
  }
  return g;
}

// K gated steps of one group on its leader's stream.
int group_steps(spm_ctx *const *ctx, void *const *phi, void *const *uh, const std::vector<int> &grp, int K) {
  if (grp.size() == 1) return spm_table_of(ctx[grp[0]])->grad_steps(ctx[grp[0]], phi[grp[0]], uh[grp[0]], K);
  std::vector<spm_ctx *> c;
  std::vector<void *> p, u;
  for (int i : grp) {
    c.push_back(ctx[i]);
    p.push_back(phi[i]);
    u.push_back(uh[i]);
  }
  return spm_table_of(c[0])->grad_steps_group(c.data(), p.data(), u.data(), (int)grp.size(), K);
}

// Runs the flows of n contexts to tol (or max_steps each); steps[i] += done.
// With stall > 0 an instance is also stopped (between graph launches) once
// FloorWatch (windows of `stall` steps, switch point tol) sees its FP32
// rounding floor.
// caps (may be null) gives each instance its own step budget (<= max_steps).
int run_phase(spm_ctx *const *ctx, void *const *phi, void *const *uh, int n, int max_steps, double tol, int K,
              int *steps, int stall = 0, const int *caps = nullptr) {
  const auto groups = make_groups(ctx, n, ctx[0]->batch_group != 0);
  const int ng = (int)groups.size();
  Streams st;
  st.s.resize(ng + 1);
  st.ev.resize(ng + 1);
  for (int i = 0; i <= ng; i++) {
    if (cudaStreamCreateWithFlags(&st.s[i], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&st.ev[i], cudaEventDisableTiming) != cudaSuccess)
      return spm_fail(SPM_ERR_CUDA, "batch streams");
  }
  cudaStream_t s0 = st.s[ng];
  std::vector<cudaStream_t> saved(n);
  for (int i = 0; i < n; i++) {
    saved[i] = ctx[i]->stream;
    cudaStreamSynchronize(saved[i]);  // earlier work of the instance is complete
    SPM_TRY(spm_ensure_scratch(ctx[i], 1));
    SPM_TRY(spm_ensure_stats(ctx[i], max_steps + K));
    SPM_TRY(spm_flow_init(ctx[i], s0));
    ctx[i]->m.tol_grad = tol;
    ctx[i]->m.max_steps = caps ? caps[i] : max_steps;
  }
  // one step of every group outside the capture sets up kernel attributes
  // and tensor maps; it counts as the first step of the flow
  for (int i = 0; i < n; i++) ctx[i]->stream = s0;
  for (const auto &grp : groups) SPM_TRY(group_steps(ctx, phi, uh, grp, 1));
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaError_t e = cudaStreamBeginCapture(s0, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) return spm_fail_cuda(e, "graph capture");
  e = cudaEventRecord(st.ev[ng], s0);
  int rc = SPM_OK;
  for (int g = 0; g < ng && rc == SPM_OK && e == cudaSuccess; g++) {
    e = cudaStreamWaitEvent(st.s[g], st.ev[ng], 0);
    for (int i : groups[g]) ctx[i]->stream = st.s[g];
    rc = group_steps(ctx, phi, uh, groups[g], K);
    if (e == cudaSuccess) e = cudaEventRecord(st.ev[g], st.s[g]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s0, st.ev[g], 0);
  }
  cudaError_t e2 = cudaStreamEndCapture(s0, &graph);
  if (rc != SPM_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
  if (e != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return spm_fail_cuda(e, "graph instantiate");
  }
  std::vector<int> host(8 * (size_t)n);
  std::vector<double> rec;
  std::vector<int> seen(n, 1);  // the step outside the graph is record 0
  std::vector<FloorWatch> watch(n, FloorWatch(tol, stall > 0 ? stall : 1));
  static const int kZero = 0;
  const int launches = (max_steps + K - 1) / K;
  for (int l = 0; l < launches && rc == SPM_OK; l++) {
    e = cudaGraphLaunch(exec, s0);
    if (e != cudaSuccess) {
      rc = spm_fail_cuda(e, "graph launch");
      break;
    }
    for (int i = 0; i < n; i++)
      cudaMemcpyAsync(&host[8 * (size_t)i], ctx[i]->flow, sizeof(int) * 8, cudaMemcpyDeviceToHost, s0);
    e = cudaStreamSynchronize(s0);
    if (e != cudaSuccess) {
      rc = spm_fail_cuda(e, "batch run");
      break;
    }
    bool all = true;
    for (int i = 0; i < n; i++) {
      if (host[8 * (size_t)i + FW_ERR]) rc = spm_fail(SPM_ERR_CUDA, "a bounded wait timed out in a batched flow");
      if (stall > 0 && host[8 * (size_t)i + FW_GO] != 0) {
        const int it = host[8 * (size_t)i + FW_ITER];
        if (it > seen[i]) {
          rec.resize(4 * (size_t)(it - seen[i]));
          e = cudaMemcpy(rec.data(), ctx[i]->stats + 4 * (size_t)seen[i], sizeof(double) * rec.size(),
                         cudaMemcpyDeviceToHost);
          if (e != cudaSuccess) {
            rc = spm_fail_cuda(e, "batch records");
            break;
          }
          bool stop = false;
          for (int s = 0; s < it - seen[i] && !stop; s++) stop = watch[i].step(rec[4 * (size_t)s + 2]);
          seen[i] = it;
          if (stop) {  // the instance stops before the next launch
            e = cudaMemcpyAsync(ctx[i]->flow + FW_GO, &kZero, sizeof(int), cudaMemcpyHostToDevice, s0);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s0);
            if (e != cudaSuccess) {
              rc = spm_fail_cuda(e, "batch stop");
              break;
            }
            host[8 * (size_t)i + FW_GO] = 0;
          }
        }
      }
      all = all && host[8 * (size_t)i + FW_GO] == 0;
    }
    if (all || rc != SPM_OK) break;
  }
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  for (int i = 0; i < n; i++) {
    ctx[i]->stream = saved[i];
    ctx[i]->m.tol_grad = 0.0;
    ctx[i]->m.max_steps = 0.0;
    steps[i] += host[8 * (size_t)i + FW_ITER];
  }
  return rc;
}

}  // namespace

extern "C" int spm_batch_grad_flow(spm_ctx **ctx, void **phi, void **uhat, int n, int max_steps, double tol_grad,
                                   double switch_tol, int steps_per_launch, int *steps_done) {
  if (!ctx || !phi || !uhat || n < 1 || max_steps < 1 || steps_per_launch < 1 || !(tol_grad > 0))
    return spm_fail(SPM_ERR_ARG, "bad argument");
  for (int i = 0; i < n; i++)
    if (!ctx[i] || !phi[i] || !uhat[i]) return spm_fail(SPM_ERR_ARG, "null instance");
  std::vector<int> steps(n, 0);
  if (switch_tol > tol_grad) {
    for (int i = 0; i < n; i++)
      if (ctx[i]->prec != SPM_FP64) return spm_fail(SPM_ERR_ARG, "mixed batches run on FP64 contexts");
    std::vector<spm_ctx *> tw(n);
    std::vector<void *> p32(n), u32(n);
    for (int i = 0; i < n; i++) {
      spm_ctx *c = ctx[i];
      const size_t m = (size_t)c->N * c->N * c->N;
      SPM_TRY(spm_ensure_twin(c));
      tw[i] = c->twin;
      p32[i] = c->twin_buf;
      u32[i] = (float *)c->twin_buf + m;
      cast_kernel<double, float><<<1184, 256, 0, c->stream>>>((const double *)phi[i], (float *)p32[i], m);
      cast_kernel<double, float><<<1184, 256, 0, c->stream>>>((const double *)uhat[i], (float *)u32[i], m);
      c->launches += 2;
    }
    SPM_TRY(run_phase(tw.data(), p32.data(), u32.data(), n, max_steps, switch_tol, steps_per_launch,
                      steps.data(), 512));
    for (int i = 0; i < n; i++) {
      spm_ctx *c = ctx[i];
      const size_t m = (size_t)c->N * c->N * c->N;
      cast_kernel<float, double><<<1184, 256, 0, c->stream>>>((const float *)p32[i], (double *)phi[i], m);
      c->launches++;
      SPM_TRY(spm_fft(c, phi[i], uhat[i]));
    }
  }
  // FP64 phase: each instance with steps left continues with its own budget
  std::vector<spm_ctx *> c64;
  std::vector<void *> p64, u64;
  std::vector<int> caps, idx, s64;
  for (int i = 0; i < n; i++)
    if (max_steps - steps[i] > 0) {
      c64.push_back(ctx[i]);
      p64.push_back(phi[i]);
      u64.push_back(uhat[i]);
      caps.push_back(max_steps - steps[i]);
      idx.push_back(i);
    }
  if (!c64.empty()) {
    const int most = *std::max_element(caps.begin(), caps.end());
    s64.assign(c64.size(), 0);
    SPM_TRY(run_phase(c64.data(), p64.data(), u64.data(), (int)c64.size(), most, tol_grad, steps_per_launch,
                      s64.data(), 0, caps.data()));
    for (size_t j = 0; j < idx.size(); j++) steps[idx[j]] += s64[j];
  }
  for (int i = 0; i < n; i++) {
    cudaError_t e = cudaStreamSynchronize(ctx[i]->stream);
    if (e != cudaSuccess) return spm_fail_cuda(e, "batch");
    if (steps_done) steps_done[i] = steps[i];
  }
  return SPM_OK;
}
