// Kernel chains of each hot-path routine for one grid size N and real type T.
// Instantiated once per (N, T) in inst_<N>.cu; the host API reaches them
// through the OpsTable of the context.
#pragma once

#include <atomic>
#include <type_traits>

#include "../../include/spmiqc.h"
#include "blas1.cuh"
#include "spm_internal.h"
#include "spm_table.h"

namespace spm {

#define SPM_TRY(x)               \
  do {                           \
    int _s = (x);                \
    if (_s != 0) return _s;      \
  } while (0)

// Sets the dynamic shared-memory limit of a kernel once per device. Tag makes
// the "done" bits distinct per kernel (the kernels share one function type).
template <class Tag, class K> static cudaError_t prepare(K kern, size_t smem, int dev) {
  // one bit per device (first 32); contexts on several host threads may race
  // here, which at worst sets the attribute twice
  static std::atomic<unsigned> done{0};
  if (dev < 32 && (done.load(std::memory_order_acquire) >> dev) & 1u) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess && dev < 32) done.fetch_or(1u << dev, std::memory_order_release);
  return e;
}

// Programmatic dependent launches (knob "pdl"); a stream capture turns them
// into programmatic edges of the graph.
static inline bool pdl_on(const spm_ctx *c) { return c->pdl != 0; }

// Persistent cluster launch: as many clusters as can be resident at once
// (queried once per kernel and device), at most one per x-plane. With
// pdl_on the launch is a programmatic dependent one: its CTAs may be placed
// while the previous kernel of the stream finishes, and wait for it in
// grid_dep_sync.
template <class Tag, int N, class K, int RW = kRows>
static int launch_cluster(spm_ctx *c, K kern, size_t smem, const KParams &p, int nb, const char *what,
                          bool xg = false, int regions = 2) {
  constexpr int CLr = N / RW;
  cudaError_t e = prepare<Tag>(kern, smem, c->device);
  if (e == cudaSuccess && CLr > 8) {  // clusters of up to 16 CTAs (16-row CTAs at N = 256)
    static std::atomic<unsigned> np{0};
    const int dev = c->device < 32 ? c->device : 0;
    if (!((np.load(std::memory_order_acquire) >> dev) & 1u)) {
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
      if (e == cudaSuccess) np.fetch_or(1u << dev, std::memory_order_release);
    }
  }
  if (e != cudaSuccess) return spm_fail_cuda(e, what);
  cudaLaunchConfig_t cfg = {};
  cfg.blockDim = dim3(8 * RW, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c->stream;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CLr;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  // the grid depends only on the kernel and the device (never on the load),
  // so the reductions' partial sums, and hence the results, do not either
  static std::atomic<int> ncl[32] = {};
  const int dev = c->device < 32 ? c->device : 0;
  int nc = ncl[dev].load(std::memory_order_relaxed);
  if (nc == 0) {
    cfg.gridDim = dim3(CLr * N, 1, 1);
    int n = 0;
    e = cudaOccupancyMaxActiveClusters(&n, kern, &cfg);
    if (e != cudaSuccess || n < 1) return spm_fail_cuda(e != cudaSuccess ? e : cudaErrorInvalidConfiguration, what);
    nc = n < N ? n : N;
    ncl[dev].store(nc, std::memory_order_relaxed);
  }
  cfg.gridDim = dim3(CLr * nc, nb, 1);
  cfg.numAttrs = pdl_on(c) ? 2 : 1;  // the kernels begin with grid_dep_sync
  // a kernel exchanging through global areas needs one per CTA (nb == 1)
  if (xg && (!p.xg || nb != 1 || CLr * nc > p.xg_cap * (kRows / RW) || p.xg_regions < regions))
    return spm_fail(SPM_ERR_STATE, "plane exchange areas missing or too small");
  c->launches++;
  e = cudaLaunchKernelEx(&cfg, kern, p);
  return e == cudaSuccess ? 0 : spm_fail_cuda(e, what);
}

// Gradient-chain kernels (the nonlinear prologue and the flow epilogue) may
// exchange through the global areas (c->plane_xg, autotuned); other chains
// (batched Hv, preconditioner, ...) always use distributed shared memory.
template <class X> struct XgOk : std::false_type {};
template <class T> struct XgOk<ProGrad<T>> : std::true_type {};
template <class T> struct XgOk<EpiFlow<T>> : std::true_type {};
// plane_cps 5: gradient chains with both exchanges through L2 run 16-row CTAs
// (128 threads, four per SM, 128 registers each); other chains run as with 2.
// plane_cps 6: the same, with the fused pass software-pipelined over planes.
static inline bool cps_rw16(const spm_ctx *c) { return c->plane_cps == 5 || c->plane_cps == 6; }
static inline int eff_cps(const spm_ctx *c) { return cps_rw16(c) ? 2 : c->plane_cps; }
static inline int xg_bits(const spm_ctx *c, int nb) { return (c->xg && nb == 1 && eff_cps(c) >= 2) ? c->plane_xg : 0; }
static inline bool rw16(const spm_ctx *c, int nb) { return cps_rw16(c) && xg_bits(c, nb) == (kXgFwd | kXgInv); }
// Four CTAs per SM (64 registers per thread): FP32 gradient chains only.
template <class T> static inline bool cps4(const spm_ctx *c) { return sizeof(T) == 4 && eff_cps(c) == 4; }

// The plane kernels come in four variants (c->plane_cps): 1 = staged, one CTA
// per SM; 2 = direct loads, two CTAs per SM; 3 = direct, three CTAs per SM;
// 4 = direct, four CTAs per SM for FP32 gradient chains (3 elsewhere).
template <int N, class T, class Pro> static int plane_fwd(spm_ctx *c, const KParams &p, int nb) {
  if constexpr (XgOk<Pro>::value) {
    if (xg_bits(c, nb) & kXgFwd) {
      if (rw16(c, nb)) {
        struct Tag16 {};
        return launch_cluster<Tag16, N, decltype(&plane_fwd_kernel<N, T, Pro, 4, kXgFwd, 16>), 16>(
            c, plane_fwd_kernel<N, T, Pro, 4, kXgFwd, 16>, plane_smem<N, T, 4, 16>(), p, nb, "plane_fwd", true);
      }
      if constexpr (sizeof(T) == 4) {
        if (cps4<T>(c)) {
          struct Tag4x {};
          return launch_cluster<Tag4x, N>(c, plane_fwd_kernel<N, T, Pro, 4, kXgFwd>, plane_smem<N, T, 4>(), p, nb,
                                          "plane_fwd", true);
        }
      }
      if (eff_cps(c) >= 3) {
        struct Tag3x {};
        return launch_cluster<Tag3x, N>(c, plane_fwd_kernel<N, T, Pro, 3, kXgFwd>, plane_smem<N, T, 3>(), p, nb,
                                        "plane_fwd", true);
      }
      struct Tag2x {};
      return launch_cluster<Tag2x, N>(c, plane_fwd_kernel<N, T, Pro, 2, kXgFwd>, plane_smem<N, T, 2>(), p, nb,
                                      "plane_fwd", true);
    }
  }
  if (eff_cps(c) >= 3) {
    struct Tag3 {};
    return launch_cluster<Tag3, N>(c, plane_fwd_kernel<N, T, Pro, 3>, plane_smem<N, T, 3>(), p, nb, "plane_fwd");
  }
  if (eff_cps(c) == 2) {
    struct Tag2 {};
    return launch_cluster<Tag2, N>(c, plane_fwd_kernel<N, T, Pro, 2>, plane_smem<N, T, 2>(), p, nb, "plane_fwd");
  }
  struct Tag1 {};
  return launch_cluster<Tag1, N>(c, plane_fwd_kernel<N, T, Pro, 1>, plane_smem<N, T, 1>(), p, nb, "plane_fwd");
}
template <int N, class T, class Epi> static int plane_inv(spm_ctx *c, const KParams &p0, int nb) {
  if constexpr (XgOk<Epi>::value) {
    if (xg_bits(c, nb) & kXgInv) {
      if (rw16(c, nb)) {
        struct Tag16 {};
        return launch_cluster<Tag16, N, decltype(&plane_inv_kernel<N, T, Epi, 4, kXgInv, 16>), 16>(
            c, plane_inv_kernel<N, T, Epi, 4, kXgInv, 16>, plane_smem<N, T, 4, 16>(), p0, nb, "plane_inv", true);
      }
      if constexpr (sizeof(T) == 4) {
        if (cps4<T>(c)) {
          struct Tag4x {};
          return launch_cluster<Tag4x, N>(c, plane_inv_kernel<N, T, Epi, 4, kXgInv>, plane_smem<N, T, 4>(), p0, nb,
                                          "plane_inv", true);
        }
      }
      if (eff_cps(c) >= 3) {
        struct Tag3x {};
        return launch_cluster<Tag3x, N>(c, plane_inv_kernel<N, T, Epi, 3, kXgInv>, plane_smem<N, T, 3>(), p0, nb,
                                        "plane_inv", true);
      }
      struct Tag2x {};
      return launch_cluster<Tag2x, N>(c, plane_inv_kernel<N, T, Epi, 2, kXgInv>, plane_smem<N, T, 2>(), p0, nb,
                                      "plane_inv", true);
    }
  }
  if (eff_cps(c) >= 3) {
    struct Tag3 {};
    return launch_cluster<Tag3, N>(c, plane_inv_kernel<N, T, Epi, 3>, plane_smem<N, T, 3>(), p0, nb, "plane_inv");
  }
  if (eff_cps(c) == 2) {
    struct Tag2 {};
    return launch_cluster<Tag2, N>(c, plane_inv_kernel<N, T, Epi, 2>, plane_smem<N, T, 2>(), p0, nb, "plane_inv");
  }
  struct Tag1 {};
  KParams p = p0;
  for (int b = 0; b < nb; b++) SPM_TRY(spm_tensor_map(c, p.in[b], TM_PLANE_INV, &p.tmi[b]));
  return launch_cluster<Tag1, N>(c, plane_inv_kernel<N, T, Epi, 1>, plane_smem<N, T, 1>(), p, nb, "plane_inv");
}
// The fused inverse -> forward plane pass (direct loads; two CTAs per SM, or
// three with plane_cps = 3), with the exchange routes XG.
template <int N, class T, class Epi, class Pro, int XG>
static int plane_inv_fwd_xg(spm_ctx *c, const KParams &p, int nb) {
  if constexpr (sizeof(T) == 4 && XG != 0) {
    if (cps4<T>(c)) {
      struct Tag4 {};
      return launch_cluster<Tag4, N>(c, plane_inv_fwd_kernel<N, T, Epi, Pro, 4, XG>, plane_smem<N, T, 4>(), p, nb,
                                     "plane_inv_fwd", true);
    }
  }
  if (eff_cps(c) >= 3) {
    struct Tag3 {};
    return launch_cluster<Tag3, N>(c, plane_inv_fwd_kernel<N, T, Epi, Pro, 3, XG>, plane_smem<N, T, 3>(), p, nb,
                                   "plane_inv_fwd", XG != 0);
  }
  struct Tag2 {};
  return launch_cluster<Tag2, N>(c, plane_inv_fwd_kernel<N, T, Epi, Pro, 2, XG>, plane_smem<N, T, 2>(), p, nb,
                                 "plane_inv_fwd", XG != 0);
}
template <int N, class T, class Epi, class Pro> static int plane_inv_fwd(spm_ctx *c, const KParams &p, int nb) {
  if constexpr (XgOk<Pro>::value && XgOk<Epi>::value) {
    if (rw16(c, nb)) {
      constexpr int XG = kXgFwd | kXgInv;
      if (c->plane_cps == 6) {
        struct Tag16p {};
        return launch_cluster<Tag16p, N, decltype(&plane_inv_fwd_pipe_kernel<N, T, Epi, Pro, 4, 16>), 16>(
            c, plane_inv_fwd_pipe_kernel<N, T, Epi, Pro, 4, 16>, plane_smem<N, T, 4, 16>(), p, nb,
            "plane_inv_fwd (pipelined)", true, 4);
      }
      struct Tag16 {};
      return launch_cluster<Tag16, N, decltype(&plane_inv_fwd_kernel<N, T, Epi, Pro, 4, XG, 16>), 16>(
          c, plane_inv_fwd_kernel<N, T, Epi, Pro, 4, XG, 16>, plane_smem<N, T, 4, 16>(), p, nb, "plane_inv_fwd", true);
    }
    switch (xg_bits(c, nb)) {
      case kXgFwd: return plane_inv_fwd_xg<N, T, Epi, Pro, kXgFwd>(c, p, nb);
      case kXgInv: return plane_inv_fwd_xg<N, T, Epi, Pro, kXgInv>(c, p, nb);
      case kXgFwd | kXgInv: return plane_inv_fwd_xg<N, T, Epi, Pro, kXgFwd | kXgInv>(c, p, nb);
      default: break;
    }
  }
  return plane_inv_fwd_xg<N, T, Epi, Pro, 0>(c, p, nb);
}
// Persistent pencil launch: resident CTAs (queried once), at most one per tile;
// tiles of 8 columns, or 4 (knob "pencil_tc"); programmatic dependent with pdl_on.
template <int N, class T, class Op, int TC> static int pencil_tc(spm_ctx *c, const KParams &p0, int nb) {
  using PG = PencilGeo<N, TC>;
  KParams p = p0;
  const int kind = TC == 8 ? TM_PENCIL : TM_PENCIL4;
  for (int b = 0; b < nb; b++) {
    if (Op::FI) SPM_TRY(spm_tensor_map(c, p.in[b], kind, &p.tmi[b]));
    if (Op::SI) SPM_TRY(spm_tensor_map(c, p.st[b], kind, &p.tms[b]));
  }
  auto kern = pencil_kernel<N, T, Op, TC>;
  constexpr size_t smem = pencil_smem<N, T, TC>((Op::FI ? 1 : 0) + (Op::SI ? 1 : 0), Op::SYM >= 0);
  static_assert(smem_ctas_per_sm(smem) >= 1, "pencil shared memory above the 227 KB a CTA may use");
  struct Tag {};
  cudaError_t e = prepare<Tag>(kern, smem, c->device);
  if (e != cudaSuccess) return spm_fail_cuda(e, "pencil attribute");
  static std::atomic<int> nblk[32] = {};
  const int dev = c->device < 32 ? c->device : 0;
  int nbk = nblk[dev].load(std::memory_order_relaxed);
  if (nbk == 0) {
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, PG::TH, smem);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    if (e != cudaSuccess || per_sm < 1) return spm_fail_cuda(e != cudaSuccess ? e : cudaErrorInvalidConfiguration,
                                                             "pencil occupancy");
    nbk = per_sm * sms < PG::PTILES ? per_sm * sms : PG::PTILES;
    nblk[dev].store(nbk, std::memory_order_relaxed);
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nbk, nb, 1);
  cfg.blockDim = dim3(PG::TH, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_on(c) ? 1 : 0;  // the kernel begins with grid_dep_sync
  c->launches++;
  e = cudaLaunchKernelEx(&cfg, kern, p);
  return e == cudaSuccess ? 0 : spm_fail_cuda(e, "pencil launch");
}
template <int N, class T, class Op> static int pencil(spm_ctx *c, const KParams &p, int nb) {
  if (c->pencil_tc == 4) return pencil_tc<N, T, Op, 4>(c, p, nb);
  return pencil_tc<N, T, Op, 8>(c, p, nb);
}
template <int N, class T, class F> static int reduce(spm_ctx *c, const KParams &p, int nb) {
  constexpr size_t npairs = (size_t)N * N * N / 2;
  constexpr int blocks = (int)((npairs + kThreads - 1) / kThreads < (size_t)kReduceBlocks
                                   ? (npairs + kThreads - 1) / kThreads
                                   : (size_t)kReduceBlocks);
  c->launches++;
  field_reduce_kernel<T, F><<<dim3(blocks, nb, 1), kThreads, 0, c->stream>>>(p, npairs);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : spm_fail_cuda(e, "reduce launch");
}

// Every chain that goes through the spectral scratch checks that the caller
// made room for its batch (spm_ensure_scratch) instead of writing through an
// unallocated buffer.
#define SPM_NEED_SCRATCH(c, nb)                                                         \
  do {                                                                                  \
    if ((c)->scratch_cap < (nb) || !(c)->bufA || !(c)->bufB)                            \
      return spm_fail(SPM_ERR_STATE, "spectral scratch not allocated for this batch"); \
  } while (0)

template <int N, class T> struct Impl {
  static int fft(spm_ctx *c, const void *x, void *xhat) {
    SPM_NEED_SCRATCH(c, 1);
    KParams p = spm_params(c);
    p.in[0] = x;
    p.out[0] = spm_bufA(c, 0);
    SPM_TRY((plane_fwd<N, T, ProIdent<T>>(c, p, 1)));
    KParams q = spm_params(c);
    q.in[0] = spm_bufA(c, 0);
    q.sto[0] = xhat;
    return pencil<N, T, OpFwd<T>>(c, q, 1);
  }

  static int ifft(spm_ctx *c, const void *xhat, void *x) {
    SPM_NEED_SCRATCH(c, 1);
    KParams q = spm_params(c);
    q.st[0] = xhat;
    q.out[0] = spm_bufB(c, 0);
    SPM_TRY((pencil<N, T, OpInv<T>>(c, q, 1)));
    KParams p = spm_params(c);
    p.in[0] = spm_bufB(c, 0);
    p.out[0] = x;
    return plane_inv<N, T, EpiStore<T>>(c, p, 1);
  }

  // E2 -> scal[SC_E2], E1 -> scal[SC_E1]
  static int energy(spm_ctx *c, const void *phi, const void *uhat) {
    KParams p = spm_params(c);
    p.in[0] = phi;
    SPM_TRY((reduce<N, T, ProGrad<T>>(c, p, 1)));
    KParams q = spm_params(c);
    q.st[0] = uhat;
    return pencil<N, T, OpE1<T>>(c, q, 1);
  }

  // One fused semi-implicit step, gated by the flow words. With ev non-null,
  // records ev[0..3] around the three passes (for per-kernel timing).
  static int grad_step_ev(spm_ctx *c, void *phi, void *uhat, void *const *ev) {
    SPM_NEED_SCRATCH(c, 1);
    auto rec = [&](int i) {
      if (ev) cudaEventRecord((cudaEvent_t)ev[i], c->stream);
    };
    KParams p = spm_params(c);
    p.flow = c->flow;
    p.stats = c->stats;
    p.in[0] = phi;
    p.out[0] = spm_bufA(c, 0);
    rec(0);
    SPM_TRY((plane_fwd<N, T, ProGrad<T>>(c, p, 1)));
    rec(1);
    KParams q = spm_params(c);
    q.flow = c->flow;
    q.stats = c->stats;
    q.in[0] = spm_bufA(c, 0);
    q.st[0] = uhat;
    q.sto[0] = uhat;
    q.out[0] = spm_bufB(c, 0);
    SPM_TRY((pencil<N, T, OpGrad<T>>(c, q, 1)));
    rec(2);
    KParams r = spm_params(c);
    r.flow = c->flow;
    r.stats = c->stats;
    r.in[0] = spm_bufB(c, 0);
    r.out[0] = phi;
    SPM_TRY((plane_inv<N, T, EpiFlow<T>>(c, r, 1)));
    rec(3);
    return 0;
  }
  static int grad_step(spm_ctx *c, void *phi, void *uhat) { return grad_step_ev(c, phi, uhat, nullptr); }

  // K gated steps as one chain: plane_fwd, then per step a pencil pass and
  // the fused inverse -> forward plane pass (the last step ends with
  // plane_inv), so phi is read and written once per chain.
  // With ev non-null (2K + 2 events) the chain records ev[0] before the head,
  // ev[1] after it and ev[2 + 2k], ev[3 + 2k] after step k's pencil and plane
  // pass (for per-kernel timing).
  static int grad_steps_ev(spm_ctx *c, void *phi, void *uhat, int K, void *const *ev) {
    SPM_NEED_SCRATCH(c, 1);
    if (K <= 0) return 0;
    auto rec = [&](int i) {
      if (ev) cudaEventRecord((cudaEvent_t)ev[i], c->stream);
    };
    if (!c->fuse_planes || K == 1) {
      for (int k = 0; k < K; k++) SPM_TRY(grad_step(c, phi, uhat));
      return 0;
    }
    rec(0);
    KParams p = spm_params(c);
    p.flow = c->flow;
    p.stats = c->stats;
    p.in[0] = phi;
    p.out[0] = spm_bufA(c, 0);
    SPM_TRY((plane_fwd<N, T, ProGrad<T>>(c, p, 1)));
    rec(1);
    for (int k = 0; k < K; k++) {
      KParams q = spm_params(c);
      q.flow = c->flow;
      q.stats = c->stats;
      q.in[0] = spm_bufA(c, 0);
      q.st[0] = uhat;
      q.sto[0] = uhat;
      q.out[0] = spm_bufB(c, 0);
      SPM_TRY((pencil<N, T, OpGrad<T>>(c, q, 1)));
      rec(2 + 2 * k);
      KParams r = spm_params(c);
      r.flow = c->flow;
      r.stats = c->stats;
      r.in[0] = spm_bufB(c, 0);
      if (k + 1 < K) {
        r.out[0] = spm_bufA(c, 0);
        r.sto[0] = phi;
        SPM_TRY((plane_inv_fwd<N, T, EpiFlow<T>, ProGrad<T>>(c, r, 1)));
      } else {
        r.out[0] = phi;
        SPM_TRY((plane_inv<N, T, EpiFlow<T>>(c, r, 1)));
      }
      rec(3 + 2 * k);
    }
    return 0;
  }
  static int grad_steps(spm_ctx *c, void *phi, void *uhat, int K) { return grad_steps_ev(c, phi, uhat, K, nullptr); }

  // K gated steps of n <= kMaxBatch independent instances of this grid size
  // and precision as one chain of batched launches: one launch per pass
  // covers every instance (blockIdx.y = instance). Instance b keeps its own
  // fields, scratch, model, symbol table, flow words and step records
  // (ctx[b]); the partial sums, tickets and scalars use one slot per instance
  // in ctx[0]'s buffers, and ctx[0]'s stream, tuning and tensor-map cache
  // serve the launches. A stopped instance's CTAs return at once. The
  // per-instance arithmetic is that of grad_steps on its own context, but the
  // plane kernels exchange through distributed shared memory (the L2 areas
  // are per context), and results carry the reduction order of a launch of
  // this size.
  static int grad_steps_group(spm_ctx *const *ctx, void *const *phi, void *const *uhat, int n, int K) {
    if (n < 1 || n > kMaxBatch) return spm_fail(SPM_ERR_ARG, "a group holds 1 to 16 instances");
    spm_ctx *c = ctx[0];
    for (int b = 0; b < n; b++) {
      if (ctx[b]->N != N || ctx[b]->prec != c->prec) return spm_fail(SPM_ERR_ARG, "a group shares N and precision");
      SPM_NEED_SCRATCH(ctx[b], 1);
    }
    if (K <= 0) return 0;
    auto base = [&]() {
      KParams p = spm_params(c);
      p.batched = 1;
      for (int b = 0; b < n; b++) {
        p.mb[b] = ctx[b]->m;
        p.gtabs[b] = reinterpret_cast<const double4 *>(ctx[b]->gtab);
        p.flows[b] = ctx[b]->flow;
        p.statss[b] = ctx[b]->stats;
      }
      return p;
    };
    auto head = [&]() {
      KParams p = base();
      for (int b = 0; b < n; b++) {
        p.in[b] = phi[b];
        p.out[b] = spm_bufA(ctx[b], 0);
      }
      return plane_fwd<N, T, ProGrad<T>>(c, p, n);
    };
    SPM_TRY(head());
    for (int k = 0; k < K; k++) {
      KParams q = base();
      for (int b = 0; b < n; b++) {
        q.in[b] = spm_bufA(ctx[b], 0);
        q.st[b] = uhat[b];
        q.sto[b] = uhat[b];
        q.out[b] = spm_bufB(ctx[b], 0);
      }
      SPM_TRY((pencil<N, T, OpGrad<T>>(c, q, n)));
      KParams r = base();
      for (int b = 0; b < n; b++) r.in[b] = spm_bufB(ctx[b], 0);
      if (c->fuse_planes && k + 1 < K) {
        for (int b = 0; b < n; b++) {
          r.out[b] = spm_bufA(ctx[b], 0);
          r.sto[b] = phi[b];
        }
        SPM_TRY((plane_inv_fwd<N, T, EpiFlow<T>, ProGrad<T>>(c, r, n)));
      } else {
        for (int b = 0; b < n; b++) r.out[b] = phi[b];
        SPM_TRY((plane_inv<N, T, EpiFlow<T>>(c, r, n)));
        if (k + 1 < K) SPM_TRY(head());
      }
    }
    return 0;
  }

  // -grad F(phi) -> grad, ||grad||^2 -> scal[SC_GN2]
  static int ngrad(spm_ctx *c, const void *phi, void *grad) {
    SPM_NEED_SCRATCH(c, 1);
    KParams p = spm_params(c);
    p.in[0] = phi;
    p.out[0] = spm_bufA(c, 0);
    SPM_TRY((plane_fwd<N, T, ProNgrad<T>>(c, p, 1)));
    KParams q = spm_params(c);
    q.in[0] = spm_bufA(c, 0);
    q.out[0] = spm_bufB(c, 0);
    SPM_TRY((pencil<N, T, OpGmul<T, true>>(c, q, 1)));
    KParams r = spm_params(c);
    r.in[0] = spm_bufB(c, 0);
    r.aux0[0] = phi;
    r.out[0] = grad;
    return plane_inv<N, T, EpiNgrad<T>>(c, r, 1);
  }

  // n <= kMaxBatch Hessian-vector products sharing phi.
  static int hv(spm_ctx *c, const void *phi, const void *const *v, void *const *hv, int n) {
    SPM_NEED_SCRATCH(c, n);
    KParams p = spm_params(c), q = spm_params(c), r = spm_params(c);
    for (int b = 0; b < n; b++) {
      p.in[b] = v[b];
      p.aux0[b] = phi;
      p.out[b] = spm_bufA(c, b);
      q.in[b] = spm_bufA(c, b);
      q.out[b] = spm_bufB(c, b);
      r.in[b] = spm_bufB(c, b);
      r.aux0[b] = phi;
      r.aux1[b] = v[b];
      r.out[b] = hv[b];
    }
    SPM_TRY((plane_fwd<N, T, ProHv<T>>(c, p, n)));
    SPM_TRY((pencil<N, T, OpGmul<T, false>>(c, q, n)));
    return plane_inv<N, T, EpiHv<T>>(c, r, n);
  }

  // n <= kMaxBatch Hessian products without their mean removal (EpiHvRaw):
  // v is transformed as it is, so phi is read once, by the epilogue.
  static int hv_raw(spm_ctx *c, const void *phi, const void *const *v, void *const *hv, int n) {
    SPM_NEED_SCRATCH(c, n);
    KParams p = spm_params(c), q = spm_params(c), r = spm_params(c);
    for (int b = 0; b < n; b++) {
      p.in[b] = v[b];
      p.out[b] = spm_bufA(c, b);
      q.in[b] = spm_bufA(c, b);
      q.out[b] = spm_bufB(c, b);
      r.in[b] = spm_bufB(c, b);
      r.aux0[b] = phi;
      r.aux1[b] = v[b];
      r.out[b] = hv[b];
    }
    SPM_TRY((plane_fwd<N, T, ProIdent<T>>(c, p, n)));
    SPM_TRY((pencil<N, T, OpGmul<T, false>>(c, q, n)));
    return plane_inv<N, T, EpiHvRaw<T>>(c, r, n);
  }

  // n <= kMaxBatch preconditioner applications, in place.
  static int precond(spm_ctx *c, void *const *w, int n) {
    SPM_NEED_SCRATCH(c, n);
    KParams p = spm_params(c), q = spm_params(c), r = spm_params(c);
    for (int b = 0; b < n; b++) {
      p.in[b] = w[b];
      p.out[b] = spm_bufA(c, b);
      q.in[b] = spm_bufA(c, b);
      q.out[b] = spm_bufB(c, b);
      r.in[b] = spm_bufB(c, b);
      r.out[b] = w[b];
    }
    SPM_TRY((plane_fwd<N, T, ProPrecond<T>>(c, p, n)));
    SPM_TRY((pencil<N, T, OpPrecond<T>>(c, q, n)));
    return plane_inv<N, T, EpiPrecond<T>>(c, r, n);
  }

  // <p, q> -> scal[SC_SUM0]
  static int dot(spm_ctx *c, const void *pp, const void *qq) {
    KParams p = spm_params(c);
    p.in[0] = pp;
    p.aux0[0] = qq;
    return reduce<N, T, ProDot<T>>(c, p, 1);
  }

  // Tangent preparation (get_Tv, SPM.cpp:15-32, plus what the force steps
  // need): with phi0 set, d = phi1 - phi0 is normalised and v = d/||d|| is
  // written to v_out; with phi0 null, phi1 is the tangent as given. Always
  // writes vhat = FFT(v)/N^3 (packed) and Gv = IFFT(G vhat, k = 0 removed).
  static int tangent(spm_ctx *c, const void *phi0, const void *phi1, void *v_out, void *vhat, void *gv) {
    SPM_NEED_SCRATCH(c, 1);
    KParams p = spm_params(c);
    p.in[0] = phi1;
    p.aux0[0] = phi0;
    p.out[0] = spm_bufA(c, 0);
    SPM_TRY((plane_fwd<N, T, ProTangent<T>>(c, p, 1)));
    KParams q = spm_params(c);
    q.in[0] = spm_bufA(c, 0);
    q.sto[0] = vhat;
    q.out[0] = spm_bufB(c, 0);
    if (phi0) SPM_TRY((pencil<N, T, OpTangent<T, true>>(c, q, 1)));
    else SPM_TRY((pencil<N, T, OpTangent<T, false>>(c, q, 1)));
    KParams r = spm_params(c);
    r.in[0] = spm_bufB(c, 0);
    r.aux0[0] = phi0;
    r.aux1[0] = phi1;
    r.sto[0] = phi0 ? v_out : nullptr;
    r.out[0] = gv;
    return plane_inv<N, T, EpiTangent<T>>(c, r, 1);
  }

  // Natural_Forces (factor 1) / MinMax_Forces (factor 2) on n fields in place,
  // all along the tangent (v, vhat, Gv) from tangent().
  static int force(spm_ctx *c, void *const *x, int n, const void *v, const void *vhat, const void *gv,
                   double factor) {
    SPM_NEED_SCRATCH(c, n);
    KParams p = spm_params(c), q = spm_params(c), r = spm_params(c);
    p.m.factor = factor;
    for (int b = 0; b < n; b++) {
      p.in[b] = x[b];
      p.aux0[b] = v;
      p.aux1[b] = gv;
      p.out[b] = spm_bufA(c, b);
      q.in[b] = spm_bufA(c, b);
      q.st[b] = vhat;
      q.out[b] = spm_bufB(c, b);
      r.in[b] = spm_bufB(c, b);
      r.out[b] = x[b];
    }
    SPM_TRY((plane_fwd<N, T, ProForce<T>>(c, p, n)));
    SPM_TRY((pencil<N, T, OpForce<T>>(c, q, n)));
    return plane_inv<N, T, EpiStore<T>>(c, r, n);
  }

  // HiSD position step: x <- IFFT(Re(FFT(x + beta (N(x) - t)) / N^3 / (1 + beta G))), dx = x' - x.
  static int hisd_step(spm_ctx *c, void *x, const void *t, void *dx, double beta) {
    SPM_NEED_SCRATCH(c, 1);
    KParams p = spm_params(c);
    p.m.factor = beta;
    p.in[0] = x;
    p.aux0[0] = t;
    p.out[0] = spm_bufA(c, 0);
    SPM_TRY((plane_fwd<N, T, ProHisd<T>>(c, p, 1)));
    KParams q = spm_params(c);
    q.m.factor = beta;
    q.in[0] = spm_bufA(c, 0);
    q.out[0] = spm_bufB(c, 0);
    SPM_TRY((pencil<N, T, OpHisd<T>>(c, q, 1)));
    KParams r = spm_params(c);
    r.in[0] = spm_bufB(c, 0);
    r.aux1[0] = x;
    r.sto[0] = dx;
    r.out[0] = x;
    return plane_inv<N, T, EpiHisd<T>>(c, r, 1);
  }

  // ||ngrad(x_b)||^2 -> scal[b][SC_GN2] without storing the gradient.
  static int gnorm(spm_ctx *c, const void *const *x, int n) {
    SPM_NEED_SCRATCH(c, n);
    KParams p = spm_params(c), q = spm_params(c), r = spm_params(c);
    for (int b = 0; b < n; b++) {
      p.in[b] = x[b];
      p.out[b] = spm_bufA(c, b);
      q.in[b] = spm_bufA(c, b);
      q.out[b] = spm_bufB(c, b);
      r.in[b] = spm_bufB(c, b);
      r.aux0[b] = x[b];
      r.out[b] = nullptr;
    }
    SPM_TRY((plane_fwd<N, T, ProNgrad<T>>(c, p, n)));
    SPM_TRY((pencil<N, T, OpGmul<T, true>>(c, q, n)));
    return plane_inv<N, T, EpiNgrad<T>>(c, r, n);
  }

  static const OpsTable *table() {
    static const OpsTable t = {&fft, &ifft, &energy, &grad_step, &grad_steps, &grad_steps_ev, &grad_step_ev, &ngrad, &hv, &precond, &dot,
                               &tangent, &force, &gnorm, &hisd_step, &grad_steps_group, &hv_raw};
    return &t;
  }
};

}  // namespace spm
