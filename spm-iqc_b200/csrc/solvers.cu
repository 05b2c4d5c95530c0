// Host-driven solvers on the transform kernels:
//  * LOBPCG for the lowest Hessian eigenpairs (hiosd_lobpcg_initialization /
//    hiosd_lobpcg_inip, LOBPCG.cpp:10-109, 207-487);
//  * the Spring Pair Method (get_Tv, Natural_Forces, MinMax_Forces,
//    Spring_Pairing, SPM.cpp:15-263).
// Fields stay on the device. Block inner products run on the FP64 tensor cores
// (gram_kernel); the small dense algebra (Cholesky, the Rayleigh-Ritz
// eigenproblem of size <= 3k) runs on the host in FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/spmiqc.h"
#include "blas1.cuh"
#include "blockops.cuh"
#include "spm_internal.h"
#include "spm_table.h"

using namespace spm;

#define SPM_TRY(x)                 \
  do {                             \
    int _s = (x);                  \
    if (_s != SPM_OK) return _s;   \
  } while (0)

namespace {

struct Solver {
  double *gram_part = nullptr;  // [kGramBlocks][kBlkMax^2]
  unsigned *gram_ticket = nullptr;
  double *gram_out = nullptr;   // kBlkMax^2
  double *h_gram = nullptr;     // pinned
  void *lob = nullptr;          // LOBPCG work fields: U, W, Y, P, Up, Vn (k each)
  int lob_k = 0;
  void *spm = nullptr;          // SPM: v, vhat, Gv
  double *spm_stats = nullptr;
  int spm_cap = 0;
  void *hisd = nullptr;         // HiSD: f, 2 PV(f), g, gp, Dx, Dg
};

Solver *solver(spm_ctx *c) {
  if (!c->extra) c->extra = new Solver();
  return reinterpret_cast<Solver *>(c->extra);
}

int ensure_base(spm_ctx *c) {
  Solver *s = solver(c);
  if (s->gram_part) return SPM_OK;
  cudaError_t e = cudaMalloc(&s->gram_part, sizeof(double) * kGramBlocks * kBlkMax * kBlkMax);
  if (e == cudaSuccess) e = cudaMalloc(&s->gram_ticket, sizeof(unsigned) * 4);
  if (e == cudaSuccess) e = cudaMemset(s->gram_ticket, 0, sizeof(unsigned) * 4);
  if (e == cudaSuccess) e = cudaMalloc(&s->gram_out, sizeof(double) * (kBlkMax * kBlkMax + 8));
  if (e == cudaSuccess) e = cudaMallocHost(&s->h_gram, sizeof(double) * (kBlkMax * kBlkMax + 8));
  if (e != cudaSuccess) return spm_fail_cuda(e, "solver buffers");
  return SPM_OK;
}

inline size_t npts(const spm_ctx *c) { return (size_t)c->N * c->N * c->N; }
inline void *fld(const spm_ctx *c, void *base, int i) { return (char *)base + c->field_bytes * (size_t)i; }

// Shared memory of the staged Gram: the stage ring, its mbarriers, and (after
// the loop, over the same bytes) the per-warp tiles of the CTA total.
static size_t gram_staged_smem(const GramP &p) {
  const size_t ring = (size_t)p.stages * p.nf * (p.chunk_bytes + 16) + 16 * (size_t)p.stages;
  const size_t tiles = sizeof(double) * kStageWarps * (size_t)(8 * ((p.ma + 7) / 8)) * (8 * ((p.mb + 7) / 8));
  return std::max(ring, tiles) + 128;
}
constexpr size_t kGramStagedSmemMax = 200 * 1024 + 1024;

// The staged Gram (gram_staged_kernel): the distinct fields of X and Y, and a
// chunk size and ring depth that keep about 200 KB of copies per SM in flight.
static int gram_staged(spm_ctx *c, GramP &p, int ma, int mb) {
  int nf = 0;
  auto slot = [&](const void *f) {
    for (int i = 0; i < nf; i++)
      if (p.F[i] == f) return i;
    p.F[nf] = f;
    return nf++;
  };
  for (int a = 0; a < ma; a++) p.xf[a] = (unsigned char)slot(p.X[a]);
  for (int b = 0; b < mb; b++) p.yf[b] = (unsigned char)slot(p.Y[b]);
  p.nf = nf;
  // bytes per field and chunk x buffers: 8 KB x 3 (<= 8 fields), 4 KB x 3
  // (<= 16), 4 KB x 2 (<= 24), 2 KB x 3 (<= 32), 2 KB x 2 (<= 48): the largest
  // copies that leave two buffers (bulk copies of 1-2 KB held the 24- and
  // 48-field Grams to 3.2-4.9 TB/s at 256^3, 4 and 2 KB copies run them at
  // 6.4 and 5.8); every field (N^3 points, N a multiple of 32) is a whole
  // number of chunks
  if (nf <= 8) p.chunk_bytes = 8192, p.stages = 3;
  else if (nf <= 16) p.chunk_bytes = 4096, p.stages = 3;
  else if (nf <= 24) p.chunk_bytes = 4096, p.stages = 2;
  else if (nf <= 32) p.chunk_bytes = 2048, p.stages = 3;
  else p.chunk_bytes = 2048, p.stages = 2;
  const size_t esz = c->prec == SPM_FP64 ? sizeof(double) : sizeof(float);
  if ((p.n * esz) % (size_t)p.chunk_bytes != 0)
    return spm_fail(SPM_ERR_ARG, "field size is not a whole number of Gram chunks");
  p.err = c->flow + FW_ERR;
  const size_t smem = gram_staged_smem(p);
  const int TA = (ma + 7) / 8, TB = (mb + 7) / 8;
  cudaError_t e = cudaSuccess;
  auto launch = [&](auto kern) {
    // (a host-side attribute write, made at every call: all kernels of this
    // family have one function type, so a cache per lambda type would be shared)
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGramStagedSmemMax);
    if (e == cudaSuccess) kern<<<kStageBlocks, (kStageWarps + 1) * 32, smem, c->stream>>>(p);
  };
  auto pick = [&](auto kd, auto kf) {
    if (c->prec == SPM_FP64) launch(kd);
    else launch(kf);
  };
#define SPM_GRAM_STAGED(A, B) \
  if (TA == A && TB == B) pick(gram_staged_kernel<double, A, B>, gram_staged_kernel<float, A, B>);
  SPM_GRAM_STAGED(1, 1) else SPM_GRAM_STAGED(1, 2) else SPM_GRAM_STAGED(1, 3)
  else SPM_GRAM_STAGED(2, 1) else SPM_GRAM_STAGED(2, 2) else SPM_GRAM_STAGED(2, 3)
  else SPM_GRAM_STAGED(3, 1) else SPM_GRAM_STAGED(3, 2) else SPM_GRAM_STAGED(3, 3)
#undef SPM_GRAM_STAGED
  if (e == cudaSuccess) e = cudaGetLastError();
  return e == cudaSuccess ? SPM_OK : spm_fail_cuda(e, "staged gram launch");
}

// G = X^T Y / N^3 (ma x mb, row-major) into host memory (synchronises).
int gram(spm_ctx *c, void *const *X, int ma, void *const *Y, int mb, std::vector<double> &G) {
  if (ma < 1 || mb < 1 || ma > kBlkMax || mb > kBlkMax) return spm_fail(SPM_ERR_ARG, "gram size");
  Solver *s = solver(c);
  GramP p;
  std::memset(&p, 0, sizeof(p));
  for (int i = 0; i < ma; i++) p.X[i] = X[i];
  for (int i = 0; i < mb; i++) p.Y[i] = Y[i];
  p.ma = ma;
  p.mb = mb;
  p.n = npts(c);
  p.inv_n = c->m.inv_n3;
  p.partials = s->gram_part;
  p.ticket = s->gram_ticket;
  p.out = s->gram_out;
  c->launches++;
  if (c->block_stage) {
    SPM_TRY(gram_staged(c, p, ma, mb));
    cudaError_t e = cudaMemcpyAsync(s->h_gram, s->gram_out, sizeof(double) * (ma * mb + 1), cudaMemcpyDeviceToHost,
                                    c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return spm_fail_cuda(e, "gram");
    if (s->h_gram[ma * mb] != 0.0) return spm_check_device_error(c);
    G.assign(s->h_gram, s->h_gram + ma * mb);
    for (double v : G)
      if (!std::isfinite(v)) return spm_fail(SPM_ERR_NONFINITE, "non-finite Gram entry");
    return SPM_OK;
  }
  // blocks of up to 8 / 16 vectors: four k-steps per loop iteration; up to 24: two
  const int tiles = (std::max(ma, mb) + 7) / 8;
  // Y = X[8 yt .. 8 yt + mb) (whole tiles): Y's fields are not read again
  int yt = -1;
  if (mb % 8 == 0)
    for (int off = 0; off + mb <= ma && yt < 0; off += 8) {
      bool same = true;
      for (int b = 0; b < mb && same; b++) same = (Y[b] == X[off + b]);
      if (same) yt = off / 8;
    }
  auto launch = [&](auto kd, auto kf) {
    if (c->prec == SPM_FP64) kd<<<kGramBlocks, kGramWarps * 32, 0, c->stream>>>(p);
    else kf<<<kGramBlocks, kGramWarps * 32, 0, c->stream>>>(p);
  };
  if (tiles == 1) {
    if (yt == 0) launch(gram_kernel<double, 4, 1, 0>, gram_kernel<float, 4, 1, 0>);
    else launch(gram_kernel<double, 4, 1>, gram_kernel<float, 4, 1>);
  } else if (tiles == 2) {
    if (yt == 0) launch(gram_kernel<double, 4, 2, 0>, gram_kernel<float, 4, 2, 0>);
    else if (yt == 1) launch(gram_kernel<double, 4, 2, 1>, gram_kernel<float, 4, 2, 1>);
    else launch(gram_kernel<double, 4, 2>, gram_kernel<float, 4, 2>);
  } else {
    if (yt == 0) launch(gram_kernel<double, 2, 3, 0>, gram_kernel<float, 2, 3, 0>);
    else if (yt == 1) launch(gram_kernel<double, 2, 3, 1>, gram_kernel<float, 2, 3, 1>);
    else if (yt == 2) launch(gram_kernel<double, 2, 3, 2>, gram_kernel<float, 2, 3, 2>);
    else launch(gram_kernel<double, 2, 3>, gram_kernel<float, 2, 3>);
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s->h_gram, s->gram_out, sizeof(double) * ma * mb, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return spm_fail_cuda(e, "gram");
  G.assign(s->h_gram, s->h_gram + ma * mb);
  for (double v : G)
    if (!std::isfinite(v)) return spm_fail(SPM_ERR_NONFINITE, "non-finite Gram entry");
  return SPM_OK;
}

// Y_q = (acc ? Y_q : 0) + sum_p C[p*nout + q] X_p + d[q]
// norms (optional, host, nout entries): the outputs' squared norms under
// inpfp, summed by the combination itself where it is staged (the call then
// synchronises); on the other paths a Gram of the outputs supplies them.
int combine(spm_ctx *c, void *const *X, int nin, void *const *Y, int nout, const std::vector<double> &C,
            const std::vector<double> *d, bool acc, double *norms = nullptr) {
  if (nin > kBlkMax + 8 || nout > kBlkMax) return spm_fail(SPM_ERR_ARG, "combine size");
  CombP p;
  std::memset(&p, 0, sizeof(p));
  for (int i = 0; i < nin; i++) p.X[i] = X[i];
  for (int i = 0; i < nout; i++) p.Y[i] = Y[i];
  p.nin = nin;
  p.nout = nout;
  p.n = npts(c);
  std::copy(C.begin(), C.begin() + (size_t)nin * nout, p.C);
  if (d) std::copy(d->begin(), d->begin() + nout, p.d);
  p.accumulate = acc ? 1 : 0;
  cudaError_t e = cudaSuccess;
  c->launches++;
  if (c->block_stage && !acc && nout <= 8 && nin > 8) {
    // staged through shared memory (combine_staged_kernel): the distinct
    // inputs, the coefficients repacked with row stride kBlkMax. (Eight or
    // fewer inputs, as the in-place 8 -> 8 update of the new block, stream
    // about as fast through combine_kernel: 5.9 against 5.5 TB/s at 256^3.)
    int nf = 0;
    for (int i = 0; i < nin; i++) {
      int f = 0;
      while (f < nf && p.F[f] != X[i]) f++;
      if (f == nf) p.F[nf++] = X[i];
      p.xf[i] = (unsigned char)f;
    }
    p.nf = nf;
    std::fill(p.C, p.C + (kBlkMax + 8) * kBlkMax, 0.0);
    for (int i = 0; i < nin; i++)
      for (int q = 0; q < nout; q++) p.C[i * kBlkMax + q] = C[(size_t)i * nout + q];
    // about 200 KB of buffers; a chunk has at least a point per thread of a group
    if (nf <= 8) p.chunk_bytes = 4096, p.stages = 6;
    else if (nf <= 16) p.chunk_bytes = 2048, p.stages = 6;
    else if (nf <= 24) p.chunk_bytes = 2048, p.stages = 4;
    else p.chunk_bytes = 2048, p.stages = 3;
    const size_t esz = c->prec == SPM_FP64 ? sizeof(double) : sizeof(float);
    if ((p.n * esz) % (size_t)p.chunk_bytes != 0)
      return spm_fail(SPM_ERR_ARG, "field size is not a whole number of combination chunks");
    p.err = c->flow + FW_ERR;
    Solver *sv = solver(c);
    if (norms) {
      p.norms = sv->gram_out;  // kBlkMax^2 + 8 doubles; the Gram buffers are idle between Grams
      p.partials = sv->gram_part;
      p.ticket = sv->gram_ticket;
      p.inv_n = c->m.inv_n3;
    }
    const size_t ring = (size_t)p.stages * nf * (p.chunk_bytes + 16) + 16 * (size_t)p.stages;
    const size_t red = norms ? sizeof(double) * 8 * (kCombWarps + 1) * 32 : 0;
    const size_t smem = std::max(ring, red) + 128;
    auto launch_s = [&](auto kern) {
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGramStagedSmemMax);
      if (e == cudaSuccess) kern<<<kStageBlocks, (kCombWarps + 1) * 32, smem, c->stream>>>(p);
    };
    auto pick = [&](auto kd, auto kf) {
      if (c->prec == SPM_FP64) launch_s(kd);
      else launch_s(kf);
    };
    if (nin <= 16) pick(combine_staged_kernel<double, 16, 8>, combine_staged_kernel<float, 16, 8>);
    else pick(combine_staged_kernel<double, kBlkMax + 8, 8>, combine_staged_kernel<float, kBlkMax + 8, 8>);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return spm_fail_cuda(e, "staged combine launch");
    if (!norms) return SPM_OK;
    e = cudaMemcpyAsync(sv->h_gram, sv->gram_out, sizeof(double) * (nout + 1), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return spm_fail_cuda(e, "combination norms");
    if (sv->h_gram[nout] != 0.0) return spm_check_device_error(c);
    std::copy(sv->h_gram, sv->h_gram + nout, norms);
    return SPM_OK;
  }
  // register-bounded variants by block shape (two points per thread where they fit)
  auto launch = [&](auto kd, auto kf) {
    if (c->prec == SPM_FP64) kd<<<1184, 256, 0, c->stream>>>(p);
    else kf<<<1184, 256, 0, c->stream>>>(p);
  };
  if (nin <= 8 && nout <= 8) launch(combine_kernel<double, 8, 8, 2>, combine_kernel<float, 8, 8, 2>);
  else if (nin <= 16 && nout <= 8) launch(combine_kernel<double, 16, 8, 1>, combine_kernel<float, 16, 8, 1>);
  else if (nout <= 8) launch(combine_kernel<double, kBlkMax + 8, 8, 1>, combine_kernel<float, kBlkMax + 8, 8, 1>);
  else launch(combine_kernel<double, kBlkMax + 8, kBlkMax, 1>, combine_kernel<float, kBlkMax + 8, kBlkMax, 1>);
  e = cudaGetLastError();
  if (e != cudaSuccess) return spm_fail_cuda(e, "combine launch");
  if (norms) {
    std::vector<double> G;
    SPM_TRY(gram(c, Y, nout, Y, nout, G));
    for (int q = 0; q < nout; q++) norms[q] = G[(size_t)q * nout + q];
  }
  return SPM_OK;
}

// Means of n fields (mean_Cplx, BasicOperators.cpp:121-130) into host memory.
int means(spm_ctx *c, void *const *X, int n, std::vector<double> &out) {
  out.assign(n, 0.0);
  for (int b0 = 0; b0 < n; b0 += kMaxBatch) {
    const int nb = std::min(kMaxBatch, n - b0);
    KParams p = spm_params(c);
    for (int b = 0; b < nb; b++) p.in[b] = X[b0 + b];
    const size_t npairs = npts(c) / 2;
    c->launches++;
    if (c->prec == SPM_FP64)
      field_reduce_kernel<double, ProSum<double>><<<dim3(kReduceBlocks, nb), kThreads, 0, c->stream>>>(p, npairs);
    else
      field_reduce_kernel<float, ProSum<float>><<<dim3(kReduceBlocks, nb), kThreads, 0, c->stream>>>(p, npairs);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return spm_fail_cuda(e, "mean launch");
    SPM_TRY(spm_read_scal(c, nb));
    for (int b = 0; b < nb; b++) out[b0 + b] = c->host_scal[b * kScal + SC_SUM0];
  }
  return SPM_OK;
}

// The LOBPCG block's Hessian products (hv_cam, LOBPCG.cpp:113-166) without
// their final mean removal: hv[b] = H v_b + mu_b, mu_b the constant hv_cam
// subtracts. The block uses them where that constant cancels or is applied
// exactly: the Rayleigh-Ritz Gram against mean-free vectors, and the residual
// combination W = H V - alpha V, which subtracts mu. With mu / vhv (host, n
// entries) the call returns mu_b and <v_b, H v_b> (after the mean removal) and
// synchronises.
int hv_many(spm_ctx *c, const void *phi, void *const *v, void *const *hv, int n, double *mu = nullptr,
            double *vhv = nullptr) {
  const OpsTable *t = spm_table_of(c);
  for (int b0 = 0; b0 < n; b0 += kMaxBatch) {
    const int nb = std::min(kMaxBatch, n - b0);
    SPM_TRY(spm_ensure_scratch(c, nb));
    SPM_TRY(t->hv_raw(c, phi, (const void *const *)(v + b0), hv + b0, nb));
    if (mu || vhv) {
      SPM_TRY(spm_read_scal(c, nb));
      for (int b = 0; b < nb; b++) {
        const double *sc = c->host_scal + (size_t)b * kScal;
        if (mu) mu[b0 + b] = sc[SC_MU];
        if (vhv) vhv[b0 + b] = sc[SC_SUM1] - sc[SC_MU] * sc[SC_SUM2];
      }
    }
  }
  return SPM_OK;
}

int precond_many(spm_ctx *c, void *const *w, int n) {
  const OpsTable *t = spm_table_of(c);
  for (int b0 = 0; b0 < n; b0 += kMaxBatch) {
    const int nb = std::min(kMaxBatch, n - b0);
    SPM_TRY(spm_ensure_scratch(c, nb));
    SPM_TRY(t->precond(c, w + b0, nb));
  }
  return SPM_OK;
}

// --------------------------------------------------------------- small algebra
// Gram-Schmidt in the metric G (Cholesky with column dropping): column j is
// dropped when its norm orthogonal to the kept columns before it is <= thr
// (the nrmW / nrmVpi > 1e-8 tests of LOBPCG.cpp:298, 319). Returns the
// coefficients B (k x k, row-major, B[p*k + q]) with X_new_q = sum_p B[p][q] X_p,
// orthonormal for kept columns and zero for dropped ones.
void gs_coefficients(const std::vector<double> &G, int k, double thr, std::vector<int> &keep,
                     std::vector<double> &B, std::vector<double> *pivots = nullptr) {
  std::vector<double> R((size_t)k * k, 0.0);
  if (pivots) pivots->assign(k, 0.0);
  for (int j = 0; j < k; j++) {
    if (!keep[j]) continue;
    double r2 = G[(size_t)j * k + j];
    for (int i = 0; i < j; i++) {
      if (!keep[i]) continue;
      double s = G[(size_t)i * k + j];
      for (int l = 0; l < i; l++)
        if (keep[l]) s -= R[(size_t)l * k + i] * R[(size_t)l * k + j];
      R[(size_t)i * k + j] = s / R[(size_t)i * k + i];
      r2 -= R[(size_t)i * k + j] * R[(size_t)i * k + j];
    }
    if (!(r2 > thr * thr)) {
      keep[j] = 0;
      continue;
    }
    R[(size_t)j * k + j] = std::sqrt(r2);
    if (pivots) (*pivots)[j] = r2;
  }
  // B = R^{-1} on the kept index set (upper triangular back-substitution)
  B.assign((size_t)k * k, 0.0);
  for (int q = 0; q < k; q++) {
    if (!keep[q]) continue;
    B[(size_t)q * k + q] = 1.0 / R[(size_t)q * k + q];
    for (int p = q - 1; p >= 0; p--) {
      if (!keep[p]) continue;
      double s = 0.0;
      for (int l = p + 1; l <= q; l++)
        if (keep[l]) s += R[(size_t)p * k + l] * B[(size_t)l * k + q];
      B[(size_t)p * k + q] = -s / R[(size_t)p * k + p];
    }
  }
}

// Symmetric eigenproblem by cyclic Jacobi; eigenvalues ascending, vectors as
// columns of V (row-major n x n). Replaces Eigen's EigenSolver on the
// symmetrised Rayleigh-Ritz matrix (LOBPCG.cpp:357-382), whose spectrum is real.
// A pair (p, q) is rotated only while |a_pq| exceeds 1e-17 sqrt(|a_pp a_qq|)
// (the relative test that keeps Jacobi's relative accuracy for the small
// eigenvalues of a graded matrix); the sweeps stop when none is rotated. The
// Rayleigh-Ritz matrices span many orders of magnitude (the W block's large
// Hessian components against the wanted eigenvalues near zero), where a test
// on the whole off-diagonal norm kept every pair rotating for a dozen sweeps.
void sym_eig(std::vector<double> A, int n, std::vector<double> &vals, std::vector<double> &V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) V[(size_t)i * n + i] = 1.0;
  double *a = A.data(), *v = V.data();
  for (int sweep = 0; sweep < 100; sweep++) {
    int rotated = 0;
    for (int p = 0; p < n - 1; p++)
      for (int q = p + 1; q < n; q++) {
        const double apq = a[(size_t)p * n + q];
        const double app = a[(size_t)p * n + p], aqq = a[(size_t)q * n + q];
        if (!(std::fabs(apq) > 1e-17 * std::sqrt(std::fabs(app * aqq))) || apq == 0.0) continue;
        rotated++;
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
        for (int k = 0; k < n; k++) {  // columns p, q
          double *rk = a + (size_t)k * n;
          const double akp = rk[p], akq = rk[q];
          rk[p] = cs * akp - sn * akq;
          rk[q] = sn * akp + cs * akq;
        }
        double *rp = a + (size_t)p * n, *rq = a + (size_t)q * n;
        for (int k = 0; k < n; k++) {  // rows p, q
          const double apk = rp[k], aqk = rq[k];
          rp[k] = cs * apk - sn * aqk;
          rq[k] = sn * apk + cs * aqk;
        }
        for (int k = 0; k < n; k++) {
          double *vk = v + (size_t)k * n;
          const double vkp = vk[p], vkq = vk[q];
          vk[p] = cs * vkp - sn * vkq;
          vk[q] = sn * vkp + cs * vkq;
        }
      }
    if (!rotated) break;
  }
  auto at = [&](int i, int j) { return a[(size_t)i * n + j]; };
  std::vector<int> idx(n);
  for (int i = 0; i < n; i++) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return at(x, x) < at(y, y); });
  std::vector<double> Vs((size_t)n * n);
  vals.resize(n);
  for (int j = 0; j < n; j++) {
    vals[j] = at(idx[j], idx[j]);
    for (int i = 0; i < n; i++) Vs[(size_t)i * n + j] = V[(size_t)i * n + idx[j]];
  }
  V = Vs;
}

// X (k fields) <- orthonormal basis of their span, in order (the Gram-Schmidt
// loops of LOBPCG.cpp:81-93, 262-267, 443-449), by two Cholesky-QR passes.
int orthonormalize(spm_ctx *c, void *const *X, int k) {
  std::vector<double> G, B;
  for (int pass = 0; pass < 2; pass++) {
    SPM_TRY(gram(c, X, k, X, k, G));
    std::vector<int> keep(k, 1);
    gs_coefficients(G, k, 0.0, keep, B);
    for (int j = 0; j < k; j++)
      if (!keep[j]) return spm_fail(SPM_ERR_NONFINITE, "block vectors are linearly dependent");
    SPM_TRY(combine(c, X, k, X, k, B, nullptr, false));
  }
  return SPM_OK;
}

// X (n fields) <- X - Q (Q^T X), twice (block classical Gram-Schmidt).
int project_out(spm_ctx *c, void *const *Q, int nq, void *const *X, int n) {
  std::vector<double> T;
  for (int pass = 0; pass < 2; pass++) {
    SPM_TRY(gram(c, Q, nq, X, n, T));
    for (double &v : T) v = -v;
    SPM_TRY(combine(c, Q, nq, X, n, T, nullptr, true));
  }
  return SPM_OK;
}

// Orthonormalise X in order with dropping (threshold thr), then once more
// on the kept vectors; dropped vectors become zero. keep is in/out.
int orth_with_drop(spm_ctx *c, void *const *X, int k, double thr, std::vector<int> &keep) {
  std::vector<double> G, B;
  SPM_TRY(gram(c, X, k, X, k, G));
  gs_coefficients(G, k, thr, keep, B);
  SPM_TRY(combine(c, X, k, X, k, B, nullptr, false));
  SPM_TRY(gram(c, X, k, X, k, G));
  std::vector<int> keep2 = keep;
  gs_coefficients(G, k, 0.0, keep2, B);
  SPM_TRY(combine(c, X, k, X, k, B, nullptr, false));
  return SPM_OK;
}

// X (k fields) <- X orthogonalised against Q (nq orthonormal fields, zero
// fields allowed) and among its own columns in order: block classical
// Gram-Schmidt with a Cholesky factorisation of the Schur complement, one or
// two passes of one Gram [Q X]^T X and one combination [Q X] -> X each. In the
// first pass a column whose norm after projecting out Q and the columns before
// it is <= thr is dropped (zeroed, keep[j] = 0): the 1e-8 tests of
// LOBPCG.cpp:298, 319, which follow the same projections (Orthoi_v2V against V
// (and W), Orthoi_Vi against the earlier columns) one column at a time. The
// second pass re-orthogonalises, and is skipped when no column is dropped and
// every column keeps at least half its squared norm through the projections
// (its Cholesky pivot against its first-pass norm: "twice is enough", the
// first pass is then orthogonal to working precision) -- the usual case for
// the preconditioned residuals W, not for P (the previous block, nearly in the
// span of the new one).
int block_orth(spm_ctx *c, void *const *Q, int nq, void *const *X, int k, double thr, std::vector<int> &keep) {
  std::vector<void *> QX(Q, Q + nq);
  QX.insert(QX.end(), X, X + k);
  const int m = nq + k;
  std::vector<double> G, S((size_t)k * k), B, Cf;
  for (int pass = 0; pass < 2; pass++) {
    SPM_TRY(gram(c, QX.data(), m, X, k, G));  // G[a * k + j] = <QX_a, X_j>
    for (int i = 0; i < k; i++)
      for (int j = 0; j < k; j++) {
        double v = G[(size_t)(nq + i) * k + j];
        for (int q = 0; q < nq; q++) v -= G[(size_t)q * k + i] * G[(size_t)q * k + j];
        S[(size_t)i * k + j] = v;
      }
    std::vector<double> piv;
    gs_coefficients(S, k, pass == 0 ? thr : 0.0, keep, B, &piv);
    bool enough = pass == 0;
    for (int j = 0; j < k && enough; j++)
      enough = keep[j] && piv[j] >= 0.5 * G[(size_t)(nq + j) * k + j];
    // X_new = X B - Q (C B), C = Q^T X
    Cf.assign((size_t)m * k, 0.0);
    for (int q = 0; q < nq; q++)
      for (int j = 0; j < k; j++) {
        double v = 0.0;
        for (int l = 0; l < k; l++) v += G[(size_t)q * k + l] * B[(size_t)l * k + j];
        Cf[(size_t)q * k + j] = -v;
      }
    for (int l = 0; l < k; l++)
      for (int j = 0; j < k; j++) Cf[(size_t)(nq + l) * k + j] = B[(size_t)l * k + j];
    SPM_TRY(combine(c, QX.data(), m, X, k, Cf, nullptr, false));
    if (enough) break;
  }
  return SPM_OK;
}

int zero_fields(spm_ctx *c, void *dst, int k) {
  cudaError_t e = cudaMemsetAsync(dst, 0, c->field_bytes * (size_t)k, c->stream);
  return e == cudaSuccess ? SPM_OK : spm_fail_cuda(e, "zero");
}

int copy_fields(spm_ctx *c, void *dst, const void *src, int k) {
  if (dst == src) return SPM_OK;
  cudaError_t e = cudaMemcpyAsync(dst, src, c->field_bytes * (size_t)k, cudaMemcpyDeviceToDevice, c->stream);
  return e == cudaSuccess ? SPM_OK : spm_fail_cuda(e, "field copy");
}

}  // namespace

void spm_free_extra(spm_ctx *c) {
  if (!c->extra) return;
  Solver *s = solver(c);
  cudaFree(s->gram_part);
  cudaFree(s->gram_ticket);
  cudaFree(s->gram_out);
  cudaFree(s->lob);
  cudaFree(s->spm);
  cudaFree(s->spm_stats);
  cudaFree(s->hisd);
  if (s->h_gram) cudaFreeHost(s->h_gram);
  delete s;
  c->extra = nullptr;
}

extern "C" int spm_block_gram(spm_ctx *c, const void *const *X, int ma, const void *const *Y, int mb, double *G) {
  if (!c || !X || !Y || !G || ma < 1 || mb < 1 || ma > kBlkMax || mb > kBlkMax)
    return spm_fail(SPM_ERR_ARG, "bad argument (1 <= ma, mb <= 24)");
  for (int i = 0; i < ma; i++)
    if (!X[i]) return spm_fail(SPM_ERR_ARG, "null field in X");
  for (int i = 0; i < mb; i++)
    if (!Y[i]) return spm_fail(SPM_ERR_ARG, "null field in Y");
  SPM_TRY(ensure_base(c));
  std::vector<double> out;
  SPM_TRY(gram(c, const_cast<void *const *>(X), ma, const_cast<void *const *>(Y), mb, out));
  std::copy(out.begin(), out.end(), G);
  return SPM_OK;
}

extern "C" int spm_block_combine(spm_ctx *c, const void *const *X, int nin, void *const *Y, int nout, const double *C,
                                 const double *d) {
  if (!c || !X || !Y || !C || nin < 1 || nout < 1 || nin > kBlkMax + 8 || nout > kBlkMax)
    return spm_fail(SPM_ERR_ARG, "bad argument (1 <= nin <= 32, 1 <= nout <= 24)");
  for (int i = 0; i < nin; i++)
    if (!X[i]) return spm_fail(SPM_ERR_ARG, "null field in X");
  for (int i = 0; i < nout; i++) {
    if (!Y[i]) return spm_fail(SPM_ERR_ARG, "null field in Y");
    for (int j = 0; j < i; j++)
      if (Y[j] == Y[i]) return spm_fail(SPM_ERR_ARG, "a field appears twice in Y");
  }
  const std::vector<double> Cv(C, C + (size_t)nin * nout);
  std::vector<double> dv;
  if (d) dv.assign(d, d + nout);
  return combine(c, const_cast<void *const *>(X), nin, Y, nout, Cv, d ? &dv : nullptr, false);
}

// ------------------------------------------------------------------ LOBPCG
extern "C" int spm_lobpcg_init(spm_ctx *c, void *V, int k, uint64_t seed) {
  if (!c || !V || k < 1 || k > kBlkMax / 3) return spm_fail(SPM_ERR_ARG, "k must be in [1, 8]");
  SPM_TRY(ensure_base(c));
  c->launches++;
  if (c->prec == SPM_FP64)
    lobpcg_random_kernel<double><<<1184, 256, 0, c->stream>>>((double *)V, k, npts(c), seed);
  else
    lobpcg_random_kernel<float><<<1184, 256, 0, c->stream>>>((float *)V, k, npts(c), seed);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return spm_fail_cuda(e, "random block");
  std::vector<void *> X(k);
  for (int i = 0; i < k; i++) X[i] = fld(c, V, i);
  // each row minus its mean (LOBPCG.cpp:67-79), then Gram-Schmidt (:81-93)
  std::vector<double> mu;
  SPM_TRY(means(c, X.data(), k, mu));
  std::vector<double> I((size_t)k * k, 0.0), d(k);
  for (int i = 0; i < k; i++) {
    I[(size_t)i * k + i] = 1.0;
    d[i] = -mu[i];
  }
  SPM_TRY(combine(c, X.data(), k, X.data(), k, I, &d, false));
  return orthonormalize(c, X.data(), k);
}

// The blocks of one LOBPCG run: V (current), U = H V, W (preconditioned
// residuals), Y = H W, P (previous V), Up = H P, Vn (scratch for the new V).
struct LobBlocks {
  std::vector<void *> Vc, U, W, Y, P, Up, Vn;
};

static int lob_blocks(spm_ctx *c, void *V, int k, LobBlocks &B) {
  Solver *s = solver(c);
  if (s->lob_k < k) {
    cudaFree(s->lob);
    s->lob = nullptr;
    s->lob_k = 0;
    cudaError_t e = cudaMalloc(&s->lob, c->field_bytes * (size_t)(6 * k));
    if (e != cudaSuccess) return spm_fail_cuda(e, "LOBPCG work fields");
    s->lob_k = k;
  }
  B = LobBlocks{};
  for (int i = 0; i < k; i++) {
    B.Vc.push_back(fld(c, V, i));
    B.U.push_back(fld(c, s->lob, i));
    B.W.push_back(fld(c, s->lob, k + i));
    B.Y.push_back(fld(c, s->lob, 2 * k + i));
    B.P.push_back(fld(c, s->lob, 3 * k + i));
    B.Up.push_back(fld(c, s->lob, 4 * k + i));
    B.Vn.push_back(fld(c, s->lob, 5 * k + i));
  }
  return SPM_OK;
}

// First half of an iteration (LOBPCG.cpp:270-286): U = H V (kept before its
// mean removal, see hv_many), alpha = <V, H V>, W = H V - alpha V and
// res_i = ||W_i||.
static int lob_residual(spm_ctx *c, const void *phi, LobBlocks &B, int k, std::vector<double> &alpha,
                        std::vector<double> &res) {
  // U = H V + mu (the Hessian products before their mean removal); alpha_i =
  // <V_i, H V_i> and mu_i summed by the products' epilogue
  std::vector<double> mu(k);
  SPM_TRY(hv_many(c, phi, B.Vc.data(), B.U.data(), k, mu.data(), alpha.data()));
  {
    std::vector<void *> X(2 * k);
    std::vector<double> C((size_t)2 * k * k, 0.0), d(k);
    for (int i = 0; i < k; i++) {
      X[i] = B.U[i];
      X[k + i] = B.Vc[i];
      C[(size_t)i * k + i] = 1.0;
      C[(size_t)(k + i) * k + i] = -alpha[i];
      d[i] = -mu[i];
    }
    // W = H V - alpha V; res_i = ||W_i||, summed by the combination that forms W
    std::vector<double> nrm(k);
    SPM_TRY(combine(c, X.data(), 2 * k, B.W.data(), k, C, &d, false, nrm.data()));
    for (int i = 0; i < k; i++) res[i] = std::sqrt(std::max(0.0, nrm[i]));
  }
  return SPM_OK;
}

// Second half (LOBPCG.cpp:287-449): W = P0(precond(W)) perp V with
// Gram-Schmidt and the 1e-8 dropping, Y = H W; P perp [V, W], dropping,
// Up = H P; Rayleigh-Ritz on [V; W; P]; P <- V; V <- the k lowest Ritz
// vectors, mean removed and Gram-Schmidt orthonormalised. The products U, Y,
// Up carry the constant that hv_cam's mean removal subtracts (hv_many); the
// Rayleigh-Ritz Gram pairs them with the mean-free V, W, P, where a constant
// adds nothing.
// With V0 (k0 fixed orthonormal fields, GOSD.cpp) W, P and the new V are also
// kept orthogonal to V0.
static int lob_update(spm_ctx *c, const void *phi, LobBlocks &B, int k, bool &have_p, void *const *V0 = nullptr,
                      int k0 = 0) {
  std::vector<double> G;
  if (k0 == 0) {
    // W: preconditioned residuals against V and in order, P against [V W],
    // each by two block Gram-Schmidt passes; then Rayleigh-Ritz on [V W P]
    SPM_TRY(precond_many(c, B.W.data(), k));
    std::vector<int> keepW(k, 1), keepP(k, 0);
    SPM_TRY(block_orth(c, B.Vc.data(), k, B.W.data(), k, 1e-8, keepW));
    SPM_TRY(hv_many(c, phi, B.W.data(), B.Y.data(), k));
    if (have_p) {
      std::vector<void *> VW(2 * k);
      for (int i = 0; i < k; i++) {
        VW[i] = B.Vc[i];
        VW[k + i] = B.W[i];
      }
      keepP.assign(k, 1);
      SPM_TRY(block_orth(c, VW.data(), 2 * k, B.P.data(), k, 1e-8, keepP));
      SPM_TRY(hv_many(c, phi, B.P.data(), B.Up.data(), k));
    }
    std::vector<void *> S, HS;
    for (int i = 0; i < k; i++) {
      S.push_back(B.Vc[i]);
      HS.push_back(B.U[i]);
    }
    for (int i = 0; i < k; i++)
      if (keepW[i]) {
        S.push_back(B.W[i]);
        HS.push_back(B.Y[i]);
      }
    for (int i = 0; i < k; i++)
      if (keepP[i]) {
        S.push_back(B.P[i]);
        HS.push_back(B.Up[i]);
      }
    const int m = (int)S.size();
    SPM_TRY(gram(c, S.data(), m, HS.data(), m, G));
    std::vector<double> Gs((size_t)m * m), vals, vecs;
    for (int i = 0; i < m; i++)
      for (int j = 0; j < m; j++) Gs[(size_t)i * m + j] = (G[(size_t)j * m + i] + G[(size_t)i * m + j]) * 0.5;
    sym_eig(Gs, m, vals, vecs);
    std::vector<double> C((size_t)m * k);
    for (int p = 0; p < m; p++)
      for (int q = 0; q < k; q++) C[(size_t)p * k + q] = vecs[(size_t)p * m + q];
    SPM_TRY(combine(c, S.data(), m, B.Vn.data(), k, C, nullptr, false));
    std::swap(B.P, B.Vc);   // P holds the old V
    std::swap(B.Vc, B.Vn);  // V holds the new block
    have_p = true;
    // each row minus its mean, then Gram-Schmidt (LOBPCG.cpp:443-449), in one
    // pass: <V_i - mu_i, V_j - mu_j> = <V_i, V_j> - mu_i mu_j, and the
    // combination subtracts mu B from B's columns (the Ritz block is already
    // orthonormal to rounding, so one Cholesky pass suffices)
    std::vector<double> mu, Bc;
    SPM_TRY(means(c, B.Vc.data(), k, mu));
    SPM_TRY(gram(c, B.Vc.data(), k, B.Vc.data(), k, G));
    for (int i = 0; i < k; i++)
      for (int j = 0; j < k; j++) G[(size_t)i * k + j] -= mu[i] * mu[j];
    std::vector<int> keep(k, 1);
    gs_coefficients(G, k, 0.0, keep, Bc);
    for (int j = 0; j < k; j++)
      if (!keep[j]) return spm_fail(SPM_ERR_NONFINITE, "block vectors are linearly dependent");
    std::vector<double> d(k, 0.0);
    for (int j = 0; j < k; j++)
      for (int p = 0; p < k; p++) d[j] -= mu[p] * Bc[(size_t)p * k + j];
    return combine(c, B.Vc.data(), k, B.Vc.data(), k, Bc, &d, false);
  }
  // with fixed fields V0 (GOSD): the projections one block at a time
  SPM_TRY(precond_many(c, B.W.data(), k));
  SPM_TRY(project_out(c, B.Vc.data(), k, B.W.data(), k));
  if (k0 > 0) SPM_TRY(project_out(c, V0, k0, B.W.data(), k));
  std::vector<int> keepW(k, 1), keepP(k, 0);
  SPM_TRY(orth_with_drop(c, B.W.data(), k, 1e-8, keepW));
  SPM_TRY(hv_many(c, phi, B.W.data(), B.Y.data(), k));
  if (have_p) {
    std::vector<void *> VW(2 * k);
    for (int i = 0; i < k; i++) {
      VW[i] = B.Vc[i];
      VW[k + i] = B.W[i];
    }
    SPM_TRY(project_out(c, VW.data(), 2 * k, B.P.data(), k));
    if (k0 > 0) SPM_TRY(project_out(c, V0, k0, B.P.data(), k));
    keepP.assign(k, 1);
    SPM_TRY(orth_with_drop(c, B.P.data(), k, 1e-8, keepP));
    SPM_TRY(hv_many(c, phi, B.P.data(), B.Up.data(), k));
  }
  std::vector<void *> S, HS;
  for (int i = 0; i < k; i++) {
    S.push_back(B.Vc[i]);
    HS.push_back(B.U[i]);
  }
  for (int i = 0; i < k; i++)
    if (keepW[i]) {
      S.push_back(B.W[i]);
      HS.push_back(B.Y[i]);
    }
  for (int i = 0; i < k; i++)
    if (keepP[i]) {
      S.push_back(B.P[i]);
      HS.push_back(B.Up[i]);
    }
  const int m = (int)S.size();
  SPM_TRY(gram(c, S.data(), m, HS.data(), m, G));
  std::vector<double> Gs((size_t)m * m), vals, vecs;
  for (int i = 0; i < m; i++)
    for (int j = 0; j < m; j++) Gs[(size_t)i * m + j] = (G[(size_t)j * m + i] + G[(size_t)i * m + j]) * 0.5;
  sym_eig(Gs, m, vals, vecs);
  std::vector<double> C((size_t)m * k);
  for (int p = 0; p < m; p++)
    for (int q = 0; q < k; q++) C[(size_t)p * k + q] = vecs[(size_t)p * m + q];
  SPM_TRY(combine(c, S.data(), m, B.Vn.data(), k, C, nullptr, false));
  std::swap(B.P, B.Vc);   // P holds the old V
  std::swap(B.Vc, B.Vn);  // V holds the new block
  have_p = true;
  std::vector<double> mu;
  SPM_TRY(means(c, B.Vc.data(), k, mu));
  std::vector<double> I((size_t)k * k, 0.0), d(k);
  for (int i = 0; i < k; i++) {
    I[(size_t)i * k + i] = 1.0;
    d[i] = -mu[i];
  }
  SPM_TRY(combine(c, B.Vc.data(), k, B.Vc.data(), k, I, &d, false));
  if (k0 > 0) SPM_TRY(project_out(c, V0, k0, B.Vc.data(), k));
  return orthonormalize(c, B.Vc.data(), k);
}

// The LOBPCG iteration on a block of kb vectors, stopping when the first
// nconv residuals are <= tol (nconv = kb: the reference's block; nconv < kb:
// the others are guard vectors).
static int lobpcg_run(spm_ctx *c, const void *phi, void *V, int kb, int nconv, int maxiter, double tol,
                      double *evals, double *resid, int *iters) {
  SPM_TRY(ensure_base(c));
  LobBlocks B;
  SPM_TRY(lob_blocks(c, V, kb, B));
  std::vector<double> alpha(kb, 0.0), res(kb, 0.0);
  SPM_TRY(orthonormalize(c, B.Vc.data(), kb));  // LOBPCG.cpp:262-267
  int it = 0;
  bool have_p = false;
  for (;; it++) {
    SPM_TRY(lob_residual(c, phi, B, kb, alpha, res));
    double rmax = 0.0;
    for (int i = 0; i < nconv; i++) rmax = std::max(rmax, res[i]);
    if (it >= maxiter || (tol > 0 && rmax <= tol)) break;
    if (spm_cancelled(c)) return spm_fail(SPM_ERR_CANCELLED, "cancelled");
    SPM_TRY(lob_update(c, phi, B, kb, have_p));
  }
  // the caller's buffer receives the final block
  for (int i = 0; i < kb; i++) SPM_TRY(copy_fields(c, fld(c, V, i), B.Vc[i], 1));
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return spm_fail_cuda(e, "lobpcg");
  if (evals) std::copy(alpha.begin(), alpha.end(), evals);
  if (resid) std::copy(res.begin(), res.end(), resid);
  if (iters) *iters = it;
  return SPM_OK;
}

extern "C" int spm_lobpcg(spm_ctx *c, const void *phi, void *V, int k, int maxiter, double tol, double *evals,
                          double *resid, int *iters) {
  if (!c || !phi || !V || k < 1 || k > kBlkMax / 3 || maxiter < 0)
    return spm_fail(SPM_ERR_ARG, "bad argument (k must be in [1, 8])");
  return lobpcg_run(c, phi, V, k, k, maxiter, tol, evals, resid, iters);
}

extern "C" int spm_lobpcg_guarded(spm_ctx *c, const void *phi, void *V, int k, int guard, int maxiter, double tol,
                                  double *evals, double *resid, int *iters) {
  if (!c || !phi || !V || k < 1 || guard < 0 || k + guard > kBlkMax / 3 || maxiter < 0)
    return spm_fail(SPM_ERR_ARG, "bad argument (k >= 1, guard >= 0, k + guard <= 8)");
  return lobpcg_run(c, phi, V, k + guard, k, maxiter, tol, evals, resid, iters);
}

// ------------------------------------------------------------------ SPM
static int ensure_spm(spm_ctx *c, int cap) {
  SPM_TRY(ensure_base(c));
  Solver *s = solver(c);
  if (!s->spm) {
    cudaError_t e = cudaMalloc(&s->spm, c->field_bytes * 3);
    if (e != cudaSuccess) return spm_fail_cuda(e, "SPM work fields");
  }
  if (s->spm_cap < cap) {
    cudaFree(s->spm_stats);
    s->spm_stats = nullptr;
    s->spm_cap = 0;
    cudaError_t e = cudaMalloc(&s->spm_stats, sizeof(double) * (size_t)std::max(cap, 1024));
    if (e != cudaSuccess) return spm_fail_cuda(e, "SPM stats");
    s->spm_cap = std::max(cap, 1024);
  }
  return spm_ensure_scratch(c, 2);
}

extern "C" int spm_get_tv(spm_ctx *c, const void *phi0, const void *phi1, void *v) {
  if (!c || !phi0 || !phi1 || !v) return spm_fail(SPM_ERR_ARG, "null argument");
  SPM_TRY(ensure_spm(c, 0));
  Solver *s = solver(c);
  return spm_table_of(c)->tangent(c, phi0, phi1, v, fld(c, s->spm, 1), fld(c, s->spm, 2));
}

static int force_step(spm_ctx *c, void *x, const void *v, double factor) {
  if (!c || !x || !v) return spm_fail(SPM_ERR_ARG, "null argument");
  SPM_TRY(ensure_spm(c, 0));
  Solver *s = solver(c);
  const OpsTable *t = spm_table_of(c);
  SPM_TRY(t->tangent(c, nullptr, v, nullptr, fld(c, s->spm, 1), fld(c, s->spm, 2)));
  void *xs[1] = {x};
  return t->force(c, xs, 1, v, fld(c, s->spm, 1), fld(c, s->spm, 2), factor);
}

extern "C" int spm_natural_forces(spm_ctx *c, void *x, const void *v) { return force_step(c, x, v, 1.0); }
extern "C" int spm_minmax_forces(spm_ctx *c, void *x, const void *v) { return force_step(c, x, v, 2.0); }

static __global__ void spm_flow_init_kernel(int *flow) {
  flow[FW_GO] = 1;
  flow[FW_PENDING] = 0;
  flow[FW_ITER] = 0;
}

// One Spring_Pairing iteration (SPM.cpp:191-255), gated by c->gate.
static int spm_iteration(spm_ctx *c, void *phi0, void *phi1, double tol, int cap) {
  Solver *s = solver(c);
  const OpsTable *t = spm_table_of(c);
  void *v = fld(c, s->spm, 0), *vh = fld(c, s->spm, 1), *gv = fld(c, s->spm, 2);
  void *X[2] = {phi0, phi1};
  const size_t n = npts(c);
  const double dt = 0.001, ks = 1.0;  // SPM.cpp:177-178
  SPM_TRY(t->tangent(c, phi0, phi1, v, vh, gv));
  SPM_TRY(t->force(c, X, 2, v, vh, gv, 1.0));
  // a spring with a rest length: dd = ||phi1 - phi0|| after the natural-force
  // step (SPM.cpp:199-200), used by both spring updates of the iteration
  const double *dd2 = nullptr;
  if (c->spring_len > 0) {
    KParams p = spm_params(c);
    p.in[0] = phi0;
    p.aux0[0] = phi1;
    c->launches++;
    if (c->prec == SPM_FP64)
      field_reduce_kernel<double, ProDist<double>><<<dim3(kReduceBlocks, 1), kThreads, 0, c->stream>>>(p, n / 2);
    else
      field_reduce_kernel<float, ProDist<float>><<<dim3(kReduceBlocks, 1), kThreads, 0, c->stream>>>(p, n / 2);
    dd2 = c->scal + SC_DD;
  }
  auto spring = [&]() {
    c->launches++;
    if (c->prec == SPM_FP64)
      spring_kernel<double><<<1184, 256, 0, c->stream>>>((double *)phi0, (double *)phi1, n, dt, ks, c->gate, dd2,
                                                         c->spring_len);
    else
      spring_kernel<float><<<1184, 256, 0, c->stream>>>((float *)phi0, (float *)phi1, n, dt, ks, c->gate, dd2,
                                                        c->spring_len);
  };
  spring();
  SPM_TRY(t->tangent(c, phi0, phi1, v, vh, gv));
  SPM_TRY(t->force(c, X, 2, v, vh, gv, 2.0));
  SPM_TRY(t->gnorm(c, (const void *const *)X, 2));
  c->launches++;
  spring();
  spm_check_kernel<<<1, 1, 0, c->stream>>>(c->scal, c->gate, s->spm_stats, tol, cap);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SPM_OK : spm_fail_cuda(e, "spm iteration");
}

extern "C" int spm_set_spring_length(spm_ctx *c, double rest) {
  if (!c || !(rest >= 0) || !std::isfinite(rest)) return spm_fail(SPM_ERR_ARG, "rest length must be finite and >= 0");
  c->spring_len = rest;
  if (c->twin) c->twin->spring_len = rest;
  return SPM_OK;
}

extern "C" int spm_spring_pairing(spm_ctx *c, void *phi0, void *phi1, int maxiter, double tol, double *res_hist,
                                  int *iters) {
  if (!c || !phi0 || !phi1 || maxiter < 0) return spm_fail(SPM_ERR_ARG, "bad argument");
  if (iters) *iters = 0;
  if (maxiter == 0) return SPM_OK;
  SPM_TRY(ensure_spm(c, maxiter));
  Solver *s = solver(c);
  c->launches++;
  spm_flow_init_kernel<<<1, 1, 0, c->stream>>>(c->flow);
  c->gate = c->flow;
  int enq = 0, chunk = 4, rc = SPM_OK;
  cudaError_t e = cudaSuccess;
  while (enq < maxiter && rc == SPM_OK) {
    const int n = std::min(chunk, maxiter - enq);
    for (int i = 0; i < n && rc == SPM_OK; i++) rc = spm_iteration(c, phi0, phi1, tol, s->spm_cap);
    if (rc != SPM_OK) break;
    enq += n;
    e = cudaMemcpyAsync(c->host_flow, c->flow, sizeof(int) * 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
      rc = spm_fail_cuda(e, "spring pairing");
      break;
    }
    if (c->host_flow[FW_GO] == 0) break;
    if (spm_cancelled(c)) {
      rc = spm_fail(SPM_ERR_CANCELLED, "cancelled");
      break;
    }
    chunk = std::min(chunk * 2, 64);
  }
  c->gate = nullptr;
  if (rc != SPM_OK) return rc;
  const int done = c->host_flow[FW_ITER];
  if (iters) *iters = done;
  if (res_hist && done > 0) {
    e = cudaMemcpy(res_hist, s->spm_stats, sizeof(double) * (size_t)done, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return spm_fail_cuda(e, "spm stats");
    for (int i = 0; i < done; i++)
      if (!std::isfinite(res_hist[i])) return spm_fail(SPM_ERR_NONFINITE, "non-finite SPM residual");
  }
  return SPM_OK;
}

// Mixed precision: the replica pair runs on the FP32 twin (FP32 transforms,
// FP64 reductions) until res <= switch_tol, then in FP64 from the cast
// replicas until res <= tol.
extern "C" int spm_spring_pairing_mixed(spm_ctx *c, void *phi0, void *phi1, int maxiter, double tol,
                                        double switch_tol, double *res_hist, int *iters_fp32, int *iters_fp64) {
  if (!c || !phi0 || !phi1 || maxiter < 0 || !(tol > 0)) return spm_fail(SPM_ERR_ARG, "bad argument");
  if (c->prec != SPM_FP64) return spm_fail(SPM_ERR_ARG, "mixed precision runs on an FP64 context");
  if (iters_fp32) *iters_fp32 = 0;
  if (iters_fp64) *iters_fp64 = 0;
  const size_t n = npts(c);
  SPM_TRY(spm_ensure_twin(c));
  float *a = (float *)c->twin_buf, *b = a + n;
  c->launches += 2;
  cast_kernel<double, float><<<1184, 256, 0, c->stream>>>((const double *)phi0, a, n);
  cast_kernel<double, float><<<1184, 256, 0, c->stream>>>((const double *)phi1, b, n);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return spm_fail_cuda(e, "cast");
  int n32 = 0, n64 = 0;
  const double sw = switch_tol > tol ? switch_tol : tol;
  // FP32 in windows of kWindow iterations until res <= sw, or until FP32
  // stops making progress (its rounding floor, FloorWatch)
  constexpr int kWindow = 256;
  std::vector<double> rec(kWindow);
  FloorWatch watch(sw, kWindow);
  while (n32 < maxiter) {
    const int chunk = std::min(kWindow, maxiter - n32);
    int done = 0;
    double *out = res_hist ? res_hist + n32 : rec.data();
    SPM_TRY(spm_spring_pairing(c->twin, a, b, chunk, sw, out, &done));
    n32 += done;
    if (done == 0 || done < chunk || out[done - 1] <= sw) break;
    bool stop = false;
    for (int i = 0; i < done && !stop; i++) stop = watch.step(out[i]);
    if (stop) break;
  }
  c->launches += c->twin->launches + 2;
  c->twin->launches = 0;
  cast_kernel<float, double><<<1184, 256, 0, c->stream>>>(a, (double *)phi0, n);
  cast_kernel<float, double><<<1184, 256, 0, c->stream>>>(b, (double *)phi1, n);
  e = cudaGetLastError();
  if (e != cudaSuccess) return spm_fail_cuda(e, "cast");
  const int left = maxiter - n32;
  if (left > 0) SPM_TRY(spm_spring_pairing(c, phi0, phi1, left, tol, res_hist ? res_hist + n32 : nullptr, &n64));
  if (iters_fp32) *iters_fp32 = n32;
  if (iters_fp64) *iters_fp64 = n64;
  return SPM_OK;
}

// ------------------------------------------------------------------ HiSD
// hiosd_lobpcg_sieh (HISD.cpp:86-485): k-index saddle dynamics. Per iteration
// a Barzilai-Borwein step size beta from the last position change Dx and the
// change of the reflected force g = f - 2 PV(f) (clamped to [betau dt,
// betat dt]); the semi-implicit position step along g (spectrum made real,
// k = 0 removed, as the reference does); one LOBPCG iteration of the k
// unstable directions V at the new position (the previous V kept as the P
// block); then f = ngrad(x) and res = nrmp(f), stopping when res < epsf.
static int hisd_run(spm_ctx *c, void *x, void *V, int k, const void *V0p, int k0, double dt, double betat,
                    double betau, double epsf, int maxiter, double *res_hist, int *iters) {
  if (!c || !x || !V || k < 1 || k > kBlkMax / 3 || maxiter < 0 || k0 < 0 || k0 > kBlkMax || (k0 && !V0p))
    return spm_fail(SPM_ERR_ARG, "bad argument");
  std::vector<void *> V0(k0);
  for (int i = 0; i < k0; i++) V0[i] = fld(c, const_cast<void *>(V0p), i);
  if (iters) *iters = 0;
  SPM_TRY(ensure_base(c));
  SPM_TRY(spm_ensure_scratch(c, 1));  // the transform chains below (ngrad, the position step) use it
  Solver *s = solver(c);
  if (!s->hisd) {
    cudaError_t e = cudaMalloc(&s->hisd, c->field_bytes * 6);
    if (e != cudaSuccess) return spm_fail_cuda(e, "HiSD work fields");
  }
  void *f = fld(c, s->hisd, 0), *tm = fld(c, s->hisd, 1), *g = fld(c, s->hisd, 2), *gp = fld(c, s->hisd, 3),
       *Dx = fld(c, s->hisd, 4), *Dg = fld(c, s->hisd, 5);
  const OpsTable *t = spm_table_of(c);
  LobBlocks B;
  SPM_TRY(lob_blocks(c, V, k, B));
  std::vector<double> alpha(k, 0.0), res(k, 0.0), G;
  auto pv = [&](double scale) -> int {  // tm = scale * sum_i <f, v_i> v_i (PV_Cplx, BasicOperators.cpp:360-371)
    SPM_TRY(gram(c, B.Vc.data(), k, &f, 1, G));
    std::vector<double> C(k);
    for (int i = 0; i < k; i++) C[i] = scale * G[i];
    return combine(c, B.Vc.data(), k, &tm, 1, C, nullptr, false);
  };
  auto lin2 = [&](void *out, double a, void *p, double b, void *q) -> int {  // FuncsLinear2Cplx
    void *X[2] = {p, q};
    std::vector<double> C = {a, b};
    return combine(c, X, 2, &out, 1, C, nullptr, false);
  };
  SPM_TRY(orthonormalize(c, B.Vc.data(), k));  // HISD.cpp:151-157
  SPM_TRY(t->ngrad(c, x, f));
  SPM_TRY(zero_fields(c, gp, 1));
  SPM_TRY(pv(1.0));
  SPM_TRY(lin2(Dx, 1.0, f, -2.0, tm));
  {  // FuncRealAddAConst(Dx, dt) (HISD.cpp:180)
    std::vector<double> I = {1.0}, d = {dt};
    SPM_TRY(combine(c, &Dx, 1, &Dx, 1, I, &d, false));
  }
  bool have_p = false;
  int it = 0;
  for (; it < maxiter;) {
    SPM_TRY(pv(2.0));
    SPM_TRY(lin2(g, 1.0, f, -1.0, tm));
    SPM_TRY(lin2(Dg, 1.0, g, -1.0, gp));
    SPM_TRY(copy_fields(c, gp, g, 1));
    void *DD[2] = {Dx, Dg};
    SPM_TRY(gram(c, DD, 2, &Dg, 1, G));  // <Dx, Dg>, <Dg, Dg>
    double bta = std::fabs(G[0] / G[1]);
    bta = std::min(bta, betat * dt);
    bta = std::max(bta, betau * dt);
    SPM_TRY(t->hisd_step(c, x, tm, Dx, bta));
    SPM_TRY(lob_residual(c, x, B, k, alpha, res));
    SPM_TRY(lob_update(c, x, B, k, have_p, V0.data(), k0));
    double gn = 0;
    SPM_TRY(spm_ngrad(c, x, f, &gn));
    if (res_hist) res_hist[it] = gn;
    it++;
    if (spm_cancelled(c)) return spm_fail(SPM_ERR_CANCELLED, "cancelled");
    if (gn < epsf) break;
  }
  for (int i = 0; i < k; i++) SPM_TRY(copy_fields(c, fld(c, V, i), B.Vc[i], 1));
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return spm_fail_cuda(e, "hisd");
  if (iters) *iters = it;
  return SPM_OK;
}

extern "C" int spm_hisd(spm_ctx *c, void *x, void *V, int k, double dt, double betat, double betau, double epsf,
                        int maxiter, double *res_hist, int *iters) {
  return hisd_run(c, x, V, k, nullptr, 0, dt, betat, betau, epsf, maxiter, res_hist, iters);
}

// hiosd_lobpcg_sieh_V0 (GOSD.cpp:123-531): HiSD with the unstable directions
// also kept orthogonal to a fixed orthonormal subspace V0 (k0 fields, e.g. the
// zero modes of a structure, critical_point, GOSD.cpp:13-56).
extern "C" int spm_gosd(spm_ctx *c, void *x, void *V, int k, const void *V0, int k0, double dt, double betat,
                        double betau, double epsf, int maxiter, double *res_hist, int *iters) {
  if (k0 < 1 || !V0) return spm_fail(SPM_ERR_ARG, "GOSD needs k0 >= 1 fixed fields");
  return hisd_run(c, x, V, k, V0, k0, dt, betat, betau, epsf, maxiter, res_hist, iters);
}
