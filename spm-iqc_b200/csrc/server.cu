// Job server: relaxation, eigenmode and saddle jobs of mixed grid sizes share
// one GPU (the reference runs one job per MPI program: main_SPM.cpp,
// grad.cpp). max_slots worker threads each take the oldest waiting job whose
// device-memory footprint fits in the free part of the budget, so jobs that
// arrive while others are running start as soon as a slot and memory free
// up, and their kernels overlap on the device (each job has its own stream
// and context). A small job may pass a large one that does not fit yet, but
// only max_bypass times: after that the large job holds the queue until it
// fits, so it cannot starve. Reductions are deterministic and persistent
// grids are sized from the device, not from the load, so a job's result does
// not depend on what runs beside it.
//
// In fake-device mode (scheduler tests without a GPU) a job sleeps in
// proportion to its work, and "allocates" from a fake device memory that
// refuses allocations beyond its size.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/spmiqc.h"
#include "spm_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

enum JobState { JS_PENDING = 0, JS_RUNNING = 1, JS_DONE = 2 };

struct Job {
  int64_t id = 0;
  spm_job_desc d{};
  std::vector<double> phi0, phi1, out;
  spm_job_result r{};
  size_t footprint = 0;
  int state = JS_PENDING;
  int bypassed = 0;         // times a later job started before this one
  volatile int cancel = 0;  // polled by the solvers between chunks of steps
  Clock::time_point t_submit, t_start, t_end;
};

double secs(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

size_t npts(int N) { return (size_t)N * N * N; }

// Device bytes a job holds while it runs, in fields of N^3 doubles: the
// job's own arrays, the solver work arrays and the context scratch (two
// spectral buffers per batched vector), plus the context's tables.
size_t footprint_of(const spm_job_desc &d) {
  const double fb = (double)npts(d.N) * (d.precision == SPM_FP32 ? 4 : 8);
  double fields = 0;
  const bool mixed = d.precision == SPM_MIXED;
  switch (d.kind) {
    case SPM_JOB_RELAX:  // phi, uhat, gradient; scratch 2; FP32 twin: 2 half fields + scratch
      fields = 3 + 2 + (mixed ? 1 + 1 : 0);
      break;
    case SPM_JOB_LOBPCG: {  // phi, V (k + guard), work 6 per vector, scratch 2 per batched vector
      const double kb = d.k + d.guard;
      fields = 1 + kb + 6.0 * kb + 2.0 * kb + 1;
      break;
    }
    case SPM_JOB_SPM:  // replicas 2, uhat, v/vhat/Gv, scratch 2 x 2; twin half of that
      fields = 2 + 1 + 3 + 4 + (mixed ? 1 + 3.5 : 0);
      break;
    default: fields = 4;
  }
  // an FP32 twin may take the plane exchange areas of an earlier FP32
  // autotune in this process: at most 2 x (N x N/32 CTAs) x 16 N FP32 complex
  // values = one FP64 field
  if (mixed) fields += 1;
  const double tables = (3.0 * (d.N / 2) * (d.N / 2) + 1) * 32 + d.N * 16.0;
  return (size_t)(fields * fb + tables) + (8u << 20);
}

}  // namespace

struct spm_server {
  spm_server_config cfg{};
  std::mutex mu;
  std::condition_variable work_cv, done_cv;
  std::deque<Job *> pending;
  std::map<int64_t, Job *> jobs;
  std::vector<std::thread> workers;
  size_t used = 0, peak = 0, fake_used = 0;
  int running = 0, peak_running = 0, max_bypass = 8;
  int device = 0;
  bool stop = false;
  int64_t next_id = 1, completed = 0, failed = 0, cancelled = 0;
  Clock::time_point t0;
  std::vector<double> latencies;
};

namespace {

// Device arrays of one job, released in every exit path.
struct JobRes {
  cudaStream_t st = nullptr;
  spm_ctx *c = nullptr;
  void *buf = nullptr;
  ~JobRes() {
    if (st) cudaStreamSynchronize(st);
    if (c) spm_ctx_destroy(c);
    if (buf) cudaFree(buf);
    if (st) cudaStreamDestroy(st);
  }
};

int run_job_gpu(spm_server *S, Job *j) {
  cudaSetDevice(S->device);
  const spm_job_desc &d = j->d;
  const bool f32 = d.precision == SPM_FP32, mixed = d.precision == SPM_MIXED;
  const size_t n = npts(d.N);
  const size_t rb = f32 ? 4 : 8;
  JobRes R;
  cudaError_t e = cudaStreamCreateWithFlags(&R.st, cudaStreamNonBlocking);
  if (e != cudaSuccess) return spm_fail_cuda(e, "job stream");
  int rc = spm_ctx_create(d.N, d.L, d.Tau, d.Gamma, d.dt, f32 ? SPM_FP32 : SPM_FP64, R.st, &R.c);
  if (rc != SPM_OK) return rc;
  spm_ctx *c = R.c;
  c->cancel = &j->cancel;
  const size_t fb = n * rb;
  const int nf = d.kind == SPM_JOB_LOBPCG ? 1 + d.k + d.guard : 3;  // phi and V (with its guard vectors)
  e = cudaMalloc(&R.buf, fb * (size_t)nf);
  if (e != cudaSuccess) return spm_fail(SPM_ERR_NOMEM, "job fields");
  char *b = (char *)R.buf;
  std::vector<float> tmp;
  auto upload = [&](void *dst, const std::vector<double> &src) -> int {
    cudaError_t e2;
    if (!f32) {
      e2 = cudaMemcpyAsync(dst, src.data(), fb, cudaMemcpyHostToDevice, R.st);
    } else {
      tmp.assign(src.begin(), src.end());
      e2 = cudaMemcpyAsync(dst, tmp.data(), fb, cudaMemcpyHostToDevice, R.st);
    }
    if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(R.st);
    return e2 == cudaSuccess ? SPM_OK : spm_fail_cuda(e2, "job upload");
  };
  auto download = [&](const void *src, size_t count) -> int {
    j->out.resize(count);
    cudaError_t e2;
    if (!f32) {
      e2 = cudaMemcpyAsync(j->out.data(), src, count * 8, cudaMemcpyDeviceToHost, R.st);
      if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(R.st);
    } else {
      tmp.resize(count);
      e2 = cudaMemcpyAsync(tmp.data(), src, count * 4, cudaMemcpyDeviceToHost, R.st);
      if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(R.st);
      for (size_t i = 0; i < count; i++) j->out[i] = tmp[i];
    }
    return e2 == cudaSuccess ? SPM_OK : spm_fail_cuda(e2, "job download");
  };
#define JOB_TRY(x)                  \
  do {                              \
    int _s = (x);                   \
    if (_s != SPM_OK) return _s;    \
  } while (0)
  JOB_TRY(upload(b, j->phi0));
  if (d.kind == SPM_JOB_RELAX) {
    void *phi = b, *uh = b + fb, *g = b + 2 * fb;
    JOB_TRY(spm_fft(c, phi, uh));
    int n32 = 0, n64 = 0;
    if (mixed)
      JOB_TRY(spm_grad_flow_mixed(c, phi, uh, d.max_steps, d.tol, d.switch_tol, nullptr,
                                  &n32, &n64));
    else
      JOB_TRY(spm_grad_flow(c, phi, uh, d.max_steps, d.tol, nullptr, &n64));
    j->r.steps = n32 + n64;
    JOB_TRY(spm_energy(c, phi, uh, &j->r.energy));
    JOB_TRY(spm_ngrad(c, phi, g, &j->r.residual));
    JOB_TRY(download(phi, n));
  } else if (d.kind == SPM_JOB_LOBPCG) {
    void *phi = b, *V = b + fb;
    JOB_TRY(spm_lobpcg_init(c, V, d.k + d.guard, d.seed));
    double rs[8] = {0};
    JOB_TRY(spm_lobpcg_guarded(c, phi, V, d.k, d.guard, d.max_steps, d.tol, j->r.evals, rs, &j->r.steps));
    for (int i = 0; i < d.k; i++) j->r.residual = std::max(j->r.residual, rs[i]);
    JOB_TRY(download(V, n * (size_t)d.k));
  } else {
    void *p0 = b, *p1 = b + fb, *uh = b + 2 * fb;
    JOB_TRY(upload(p1, j->phi1));
    std::vector<double> hist((size_t)std::max(d.max_steps, 1));
    int n32 = 0, n64 = 0;
    if (mixed)
      JOB_TRY(spm_spring_pairing_mixed(c, p0, p1, d.max_steps, d.tol, d.switch_tol,
                                       hist.data(), &n32, &n64));
    else
      JOB_TRY(spm_spring_pairing(c, p0, p1, d.max_steps, d.tol, hist.data(), &n64));
    j->r.steps = n32 + n64;
    j->r.residual = j->r.steps > 0 ? hist[j->r.steps - 1] : 0.0;
    JOB_TRY(spm_fft(c, p1, uh));
    JOB_TRY(spm_energy(c, p1, uh, &j->r.energy));
    JOB_TRY(download(p1, n));
  }
#undef JOB_TRY
  e = cudaStreamSynchronize(R.st);
  return e == cudaSuccess ? SPM_OK : spm_fail_cuda(e, "job");
}

int run_job_fake(spm_server *S, Job *j) {
  const spm_job_desc &d = j->d;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->cfg.fake_device_bytes && S->fake_used + j->footprint > S->cfg.fake_device_bytes)
      return SPM_ERR_NOMEM;  // the device refused the allocation
    S->fake_used += j->footprint;
  }
  const double units = (double)npts(d.N) / 1e6 * std::max(d.max_steps, 0) * (d.kind == SPM_JOB_LOBPCG ? d.k + d.guard : 1);
  const auto end = Clock::now() + std::chrono::duration<double, std::milli>(S->cfg.fake_ms_per_munit * units);
  int rc = SPM_OK;
  while (Clock::now() < end) {
    if (j->cancel) {
      rc = SPM_ERR_CANCELLED;
      break;
    }
    std::this_thread::sleep_for(std::chrono::microseconds(500));
  }
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->fake_used -= j->footprint;
  }
  if (rc == SPM_OK) {
    j->r.steps = d.max_steps;
    j->r.energy = (double)d.N;
    const std::vector<double> &src = d.kind == SPM_JOB_SPM ? j->phi1 : j->phi0;
    const int copies = d.kind == SPM_JOB_LOBPCG ? d.k : 1;
    j->out.clear();
    for (int i = 0; i < copies; i++) j->out.insert(j->out.end(), src.begin(), src.end());
  }
  return rc;
}

// Oldest admissible waiting job, or null. Called with the lock held.
Job *admit(spm_server *S) {
  for (auto it = S->pending.begin(); it != S->pending.end(); ++it) {
    Job *j = *it;
    if (S->used + j->footprint > S->cfg.budget_bytes) {
      if (j->bypassed >= S->max_bypass) return nullptr;  // it holds the queue until it fits
      continue;
    }
    for (auto p = S->pending.begin(); p != it; ++p) (*p)->bypassed++;
    S->pending.erase(it);
    return j;
  }
  return nullptr;
}

void worker_loop(spm_server *S) {
  if (!S->cfg.fake_device) cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    Job *j = nullptr;
    S->work_cv.wait(lk, [&] { return (j = admit(S)) != nullptr || (S->stop && S->pending.empty()); });
    if (!j) return;
    S->used += j->footprint;
    S->peak = std::max(S->peak, S->used);
    S->running++;
    S->peak_running = std::max(S->peak_running, S->running);
    j->state = JS_RUNNING;
    j->t_start = Clock::now();
    lk.unlock();
    int rc = S->cfg.fake_device ? run_job_fake(S, j) : run_job_gpu(S, j);
    if (rc != SPM_OK && j->cancel) rc = SPM_ERR_CANCELLED;
    if (rc != SPM_OK) {
      const char *m = rc == SPM_ERR_CANCELLED ? "cancelled" : spm_last_error();
      std::snprintf(j->r.message, sizeof(j->r.message), "%s", m ? m : "");
    }
    lk.lock();
    j->t_end = Clock::now();
    j->r.status = rc;
    j->r.t_submit = secs(S->t0, j->t_submit);
    j->r.t_start = secs(S->t0, j->t_start);
    j->r.t_end = secs(S->t0, j->t_end);
    j->state = JS_DONE;
    j->phi0.clear();
    j->phi0.shrink_to_fit();
    j->phi1.clear();
    j->phi1.shrink_to_fit();
    S->used -= j->footprint;
    S->running--;
    if (rc == SPM_OK) {
      S->completed++;
      S->latencies.push_back(secs(j->t_submit, j->t_end));
    } else if (rc == SPM_ERR_CANCELLED) {
      S->cancelled++;
    } else {
      S->failed++;
    }
    S->work_cv.notify_all();
    S->done_cv.notify_all();
  }
}

}  // namespace

extern "C" size_t spm_job_footprint(const spm_job_desc *d) { return d ? footprint_of(*d) : 0; }

extern "C" int spm_server_create(const spm_server_config *cfg, spm_server **out) {
  if (!cfg || !out || cfg->max_slots < 1 || cfg->max_slots > 64) return spm_fail(SPM_ERR_ARG, "bad argument");
  spm_server *S = new spm_server();
  S->cfg = *cfg;
  if (cfg->max_bypass > 0) S->max_bypass = cfg->max_bypass;
  if (!cfg->fake_device) {
    cudaError_t e = cudaGetDevice(&S->device);
    if (e != cudaSuccess) {
      delete S;
      return spm_fail_cuda(e, "no device");
    }
    if (S->cfg.budget_bytes == 0) {
      size_t fr = 0, tot = 0;
      e = cudaMemGetInfo(&fr, &tot);
      if (e != cudaSuccess) {
        delete S;
        return spm_fail_cuda(e, "cudaMemGetInfo");
      }
      S->cfg.budget_bytes = fr / 10 * 9;
    }
  } else if (S->cfg.budget_bytes == 0) {
    delete S;
    return spm_fail(SPM_ERR_ARG, "a fake device needs a budget");
  }
  S->t0 = Clock::now();
  for (int i = 0; i < S->cfg.max_slots; i++) S->workers.emplace_back(worker_loop, S);
  *out = S;
  return SPM_OK;
}

extern "C" int spm_server_submit(spm_server *S, const spm_job_desc *d, const double *phi0, const double *phi1,
                                 int64_t *job_id) {
  if (!S || !d || !phi0 || !job_id) return spm_fail(SPM_ERR_ARG, "null argument");
  if (!spm_supported_size(d->N)) return spm_fail(SPM_ERR_UNSUPPORTED, "grid size not built");
  if (d->kind < SPM_JOB_RELAX || d->kind > SPM_JOB_SPM) return spm_fail(SPM_ERR_ARG, "unknown job kind");
  if (d->precision < SPM_FP64 || d->precision > SPM_MIXED) return spm_fail(SPM_ERR_ARG, "unknown precision");
  if (d->kind == SPM_JOB_LOBPCG && (d->k < 1 || d->guard < 0 || d->k + d->guard > 8))
    return spm_fail(SPM_ERR_ARG, "LOBPCG jobs need k >= 1, guard >= 0 and k + guard <= 8");
  if (d->kind != SPM_JOB_LOBPCG && d->guard != 0) return spm_fail(SPM_ERR_ARG, "guard is for LOBPCG jobs");
  if (d->kind == SPM_JOB_LOBPCG && d->precision == SPM_MIXED)
    return spm_fail(SPM_ERR_ARG, "LOBPCG jobs run in FP64 or FP32");
  if (d->kind == SPM_JOB_SPM && !phi1) return spm_fail(SPM_ERR_ARG, "a saddle search needs two replicas");
  if (d->max_steps < 0 || !(d->tol >= 0) || !(d->L > 0) || !(d->dt > 0)) return spm_fail(SPM_ERR_ARG, "bad job");
  if ((d->precision == SPM_MIXED || d->kind == SPM_JOB_SPM) && !(d->tol > 0))
    return spm_fail(SPM_ERR_ARG, "this job needs tol > 0");
  const size_t fp = footprint_of(*d);
  if (fp > S->cfg.budget_bytes)
    return spm_fail(SPM_ERR_NOMEM, "the job needs more device memory than the server's budget");
  Job *j = new Job();
  j->d = *d;
  const size_t n = npts(d->N);
  j->phi0.assign(phi0, phi0 + n);
  if (d->kind == SPM_JOB_SPM) j->phi1.assign(phi1, phi1 + n);
  j->footprint = fp;
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->stop) {
    delete j;
    return spm_fail(SPM_ERR_STATE, "server is shutting down");
  }
  j->id = S->next_id++;
  j->t_submit = Clock::now();
  S->jobs[j->id] = j;
  S->pending.push_back(j);
  *job_id = j->id;
  S->work_cv.notify_all();
  return SPM_OK;
}

extern "C" int spm_server_cancel(spm_server *S, int64_t id) {
  if (!S) return spm_fail(SPM_ERR_ARG, "null server");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->jobs.find(id);
  if (it == S->jobs.end()) return spm_fail(SPM_ERR_ARG, "unknown job");
  Job *j = it->second;
  if (j->state == JS_PENDING) {
    S->pending.erase(std::find(S->pending.begin(), S->pending.end(), j));
    j->state = JS_DONE;
    j->t_start = j->t_end = Clock::now();
    j->r.status = SPM_ERR_CANCELLED;
    std::snprintf(j->r.message, sizeof(j->r.message), "cancelled before it started");
    j->r.t_submit = secs(S->t0, j->t_submit);
    j->r.t_start = j->r.t_end = secs(S->t0, j->t_end);
    S->cancelled++;
    S->work_cv.notify_all();
    S->done_cv.notify_all();
  } else if (j->state == JS_RUNNING) {
    j->cancel = 1;
  }
  return SPM_OK;
}

extern "C" int spm_server_wait(spm_server *S, int64_t id, int block, spm_job_result *res, double *field) {
  if (!S) return spm_fail(SPM_ERR_ARG, "null server");
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->jobs.find(id);
  if (it == S->jobs.end()) return spm_fail(SPM_ERR_ARG, "unknown job");
  Job *j = it->second;
  if (block) S->done_cv.wait(lk, [&] { return j->state == JS_DONE; });
  if (j->state != JS_DONE) return SPM_ERR_STATE;
  if (res) *res = j->r;
  if (field && !j->out.empty()) std::memcpy(field, j->out.data(), j->out.size() * sizeof(double));
  return SPM_OK;
}

extern "C" int spm_server_release(spm_server *S, int64_t id) {
  if (!S) return spm_fail(SPM_ERR_ARG, "null server");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->jobs.find(id);
  if (it == S->jobs.end()) return spm_fail(SPM_ERR_ARG, "unknown job");
  if (it->second->state != JS_DONE) return spm_fail(SPM_ERR_STATE, "job not finished");
  delete it->second;
  S->jobs.erase(it);
  return SPM_OK;
}

extern "C" int spm_server_get_stats(spm_server *S, spm_server_stats *out) {
  if (!S || !out) return spm_fail(SPM_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  std::memset(out, 0, sizeof(*out));
  out->completed = S->completed;
  out->failed = S->failed;
  out->cancelled = S->cancelled;
  out->pending = (int64_t)S->pending.size();
  out->running = S->running;
  out->peak_running = S->peak_running;
  out->peak_bytes = S->peak;
  out->budget_bytes = S->cfg.budget_bytes;
  std::vector<double> l = S->latencies;
  std::sort(l.begin(), l.end());
  if (!l.empty()) {
    // nearest-rank percentiles
    out->p50_s = l[(size_t)std::ceil(0.50 * l.size()) - 1];
    out->p99_s = l[(size_t)std::ceil(0.99 * l.size()) - 1];
  }
  out->elapsed_s = secs(S->t0, Clock::now());
  return SPM_OK;
}

extern "C" int spm_server_destroy(spm_server *S) {
  if (!S) return SPM_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    S->work_cv.notify_all();
  }
  for (auto &t : S->workers) t.join();
  for (auto &kv : S->jobs) delete kv.second;
  delete S;
  return SPM_OK;
}
