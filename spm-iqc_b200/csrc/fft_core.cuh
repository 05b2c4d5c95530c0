// Building blocks of the sm_100a pseudo-spectral kernels: complex helpers,
// in-register mixed-radix DFTs (radix 2, 3, 4, 5 and their products up to 16),
// deterministic block / grid reductions, and the shared parameter block.
//
// The 3D transform replaces FFTW's C2C (src/My_FFT.cpp:4-21 of SPM-IQC) with a
// real-to-complex transform in "packed" layout: for a real N^3 field the
// spectrum is stored as N x N x (N/2) complex values, spec[kx][ky][c]:
//   c >= 1 : X(kx, ky, kz = c)                        (the half spectrum)
//   c == 0 : X(kx, ky, 0) + i * X(kx, ky, N/2)        (both planes Hermitian)
// so a spectrum takes exactly as many bytes as the real field. The forward
// transform is unnormalised here; ops apply the reference's 1/N^3.
#pragma once

#include <cooperative_groups.h>
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace cg = cooperative_groups;

namespace spm {

#include "tw240.inc"

constexpr int kThreads = 256;   // threads per CTA in every transform kernel
constexpr int kRows = 32;       // z-lines (rows of an x-plane) per CTA, plane kernels
constexpr int kCols = 16;       // y-lines (spectral columns) per CTA, plane kernels
// Exchange routes of the plane kernels (template XG): the forward exchange
// (R2C rows -> forward y columns) and the inverse one (inverse y columns ->
// C2R rows) go through distributed shared memory, or, with these bits, through
// per-CTA global areas that stay resident in L2.
constexpr int kXgFwd = 1, kXgInv = 2;
constexpr int kXgRegions = 4;   // exchange-area regions: two per exchange
constexpr int kMaxBatch = 16;   // fields per launch
constexpr int kScal = 16;       // scalars per field in the scalar block
constexpr int kRedMax = 8;      // reduction slots per field and CTA
constexpr int kPartStride = 2048;  // CTAs per field reserved in the partials buffer

// Scalar-block slots (per field): results of reductions, inputs of later kernels.
enum Slot {
  SC_E2 = 0,    // mean of the local free-energy density (LPsrc.cpp:19-24)
  SC_E1 = 1,    // 1/2 sum_k G |u_k|^2 (LPsrc.cpp:27-35)
  SC_RES = 2,   // max |Re(u'_k - u_k)| (LPsrc.cpp:77-84)
  SC_GN2 = 3,   // ||grad F||^2
  SC_MU = 4,    // mean removed by an epilogue (the P0 projector)
  SC_S = 5,     // <f, v> projection coefficient of the SPM force steps
  SC_NRM2 = 6,  // squared norm (tangent)
  SC_DD = 7,    // ||phi1 - phi0||^2 of an SPM replica pair (spring with a rest length)
  SC_SUM0 = 8,  // raw sums for host-side use
  SC_SUM1 = 9,
  SC_SUM2 = 10,
  SC_SUM3 = 11,
};

template <class T> struct V2;
template <> struct V2<double> { using type = double2; };
template <> struct V2<float> { using type = float2; };
template <class T> using c2 = typename V2<T>::type;

template <class T2> using base_t = decltype(T2::x);

// Rounded product and fused multiply-add, never re-contracted by the
// compiler. Sums of two products (complex products, rotations) are written
// with them so every kernel rounds the same operation the same way: the
// fused and the separate plane passes then produce identical bits.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }

template <class T2> __device__ __forceinline__ T2 cadd(T2 a, T2 b) { return {a.x + b.x, a.y + b.y}; }
template <class T2> __device__ __forceinline__ T2 csub(T2 a, T2 b) { return {a.x - b.x, a.y - b.y}; }
template <class T2> __device__ __forceinline__ T2 cmul(T2 a, T2 b) {
  return {fma_rn(a.x, b.x, -mul_rn(a.y, b.y)), fma_rn(a.x, b.y, mul_rn(a.y, b.x))};
}
template <class T2> __device__ __forceinline__ T2 cmulc(T2 a, T2 b) {  // a * conj(b)
  return {fma_rn(a.x, b.x, mul_rn(a.y, b.y)), fma_rn(a.y, b.x, -mul_rn(a.x, b.y))};
}
template <class T2> __device__ __forceinline__ T2 cconj(T2 a) { return {a.x, -a.y}; }
template <class T2, class S> __device__ __forceinline__ T2 cscale(T2 a, S s) {
  return {a.x * s, a.y * s};
}
// a * (D * i), D = +-1
template <int D, class T2> __device__ __forceinline__ T2 mul_di(T2 a) {
  if constexpr (D > 0) return {-a.y, a.x};
  else return {a.y, -a.x};
}

// compile-time loop: f(std::integral_constant<int, I>) for I in [B, E)
template <int B, int E, class F> __device__ __forceinline__ void sfor(F &&f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    sfor<B + 1, E>(f);
  }
}
#define SPM_CI(x) decltype(x)::value

// v * exp(DIR * 2 pi i * E / P) with E, P compile-time; exact for multiples of pi/2.
template <int DIR, int P, int E, class T2> __device__ __forceinline__ T2 twc(T2 v) {
  constexpr int e = ((E % P) + P) % P;
  if constexpr (e == 0) {
    return v;
  } else if constexpr (4 * e == P) {
    return mul_di<DIR>(v);
  } else if constexpr (2 * e == P) {
    return {-v.x, -v.y};
  } else if constexpr (4 * e == 3 * P) {
    return mul_di<-DIR>(v);
  } else {
    static_assert(240 % P == 0, "radix must divide 240");
    using T = base_t<T2>;
    constexpr T c = (T)kTw240[e * (240 / P)][0];
    constexpr T s = (T)(DIR * kTw240[e * (240 / P)][1]);
    return {fma_rn(v.x, c, -mul_rn(v.y, s)), fma_rn(v.x, s, mul_rn(v.y, c))};
  }
}

// In-place DFT of P register values, natural order in and out:
//   X[k] = sum_j v[j] exp(DIR * 2 pi i j k / P).
template <int DIR, int P, class T2> struct Dft;

template <int DIR, class T2> struct Dft<DIR, 1, T2> {
  static __device__ __forceinline__ void run(T2 (&)[1]) {}
};
template <int DIR, class T2> struct Dft<DIR, 2, T2> {
  static __device__ __forceinline__ void run(T2 (&v)[2]) {
    T2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};
template <int DIR, class T2> struct Dft<DIR, 3, T2> {
  static __device__ __forceinline__ void run(T2 (&v)[3]) {
    using T = base_t<T2>;
    constexpr T h = (T)0.8660254037844386467637232;  // sqrt(3)/2
    T2 t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
    T2 x0 = cadd(v[0], t1);
    T2 m = {fma_rn((T)-0.5, t1.x, v[0].x), fma_rn((T)-0.5, t1.y, v[0].y)};
    T2 n = mul_di<DIR>(T2{mul_rn(t2.x, h), mul_rn(t2.y, h)});
    v[0] = x0;
    v[1] = cadd(m, n);
    v[2] = csub(m, n);
  }
};
template <int DIR, class T2> struct Dft<DIR, 4, T2> {
  static __device__ __forceinline__ void run(T2 (&v)[4]) {
    T2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    T2 t2 = cadd(v[1], v[3]), t3 = mul_di<DIR>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[1] = cadd(t1, t3);
    v[2] = csub(t0, t2);
    v[3] = csub(t1, t3);
  }
};
template <int DIR, class T2> struct Dft<DIR, 5, T2> {
  static __device__ __forceinline__ void run(T2 (&v)[5]) {
    using T = base_t<T2>;
    constexpr T c1 = (T)kTw240[48][0], c2 = (T)kTw240[96][0];
    constexpr T s1 = (T)kTw240[48][1], s2 = (T)kTw240[96][1];
    T2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    T2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    T2 x0 = cadd(v[0], cadd(t1, t2));
    T2 b1 = {fma_rn(c2, t2.x, fma_rn(c1, t1.x, v[0].x)), fma_rn(c2, t2.y, fma_rn(c1, t1.y, v[0].y))};
    T2 b2 = {fma_rn(c1, t2.x, fma_rn(c2, t1.x, v[0].x)), fma_rn(c1, t2.y, fma_rn(c2, t1.y, v[0].y))};
    T2 d1 = mul_di<DIR>(T2{fma_rn(s1, t3.x, mul_rn(s2, t4.x)), fma_rn(s1, t3.y, mul_rn(s2, t4.y))});
    T2 d2 = mul_di<DIR>(T2{fma_rn(s2, t3.x, -mul_rn(s1, t4.x)), fma_rn(s2, t3.y, -mul_rn(s1, t4.y))});
    v[0] = x0;
    v[1] = cadd(b1, d1);
    v[4] = csub(b1, d1);
    v[2] = cadd(b2, d2);
    v[3] = csub(b2, d2);
  }
};
// Composite P = A * B (Cooley-Tukey): j = j1*B + j2, k = k1 + A*k2.
template <int DIR, int P, class T2> struct Dft {
  static constexpr int A = (P % 4 == 0 && P > 4) ? 4 : (P % 2 == 0 ? 2 : (P % 3 == 0 ? 3 : 5));
  static constexpr int B = P / A;
  static_assert(A * B == P && B > 1, "unsupported radix");
  static __device__ __forceinline__ void run(T2 (&v)[P]) {
    T2 u[A][B];
    sfor<0, B>([&](auto J2) {
      constexpr int j2 = SPM_CI(J2);
      T2 t[A];
      sfor<0, A>([&](auto J1) { t[SPM_CI(J1)] = v[SPM_CI(J1) * B + j2]; });
      Dft<DIR, A, T2>::run(t);
      sfor<0, A>([&](auto K1) {
        constexpr int k1 = SPM_CI(K1);
        u[k1][j2] = twc<DIR, P, k1 * j2>(t[k1]);
      });
    });
    sfor<0, A>([&](auto K1) {
      constexpr int k1 = SPM_CI(K1);
      T2 t[B];
      sfor<0, B>([&](auto J2) { t[SPM_CI(J2)] = u[k1][SPM_CI(J2)]; });
      Dft<DIR, B, T2>::run(t);
      sfor<0, B>([&](auto K2) { v[k1 + A * SPM_CI(K2)] = t[SPM_CI(K2)]; });
    });
  }
};

// ------------------------------------------------------------------ reductions
// Slot r of a reduction is a max when bit r of MAXM is set, otherwise a sum.
template <int NR, unsigned MAXM>
__device__ __forceinline__ void combine(double (&a)[NR], const double (&b)[NR]) {
#pragma unroll
  for (int r = 0; r < NR; r++) a[r] = ((MAXM >> r) & 1u) ? fmax(a[r], b[r]) : a[r] + b[r];
}

// FP32 partial sums of the FP32 kernels. A policy with FACC = true takes
// its accumulator array as a template parameter; in FP32 kernels a thread then
// sums the contributions of one batch of its points (16 to 32 values) in FP32
// and folds that partial into its FP64 accumulator, in place of an FP32 ->
// FP64 conversion and FP64 arithmetic per point (FP64 kernels accumulate in
// FP64 as before).
template <class X, class = void> struct HasFacc : std::false_type {};
template <class X> struct HasFacc<X, std::void_t<decltype(X::FACC)>> : std::bool_constant<X::FACC> {};
template <class T, class X> constexpr bool use_facc() { return sizeof(T) == 4 && HasFacc<X>::value; }

template <int NR, unsigned MAXM> __device__ __forceinline__ void facc_init(float (&a)[NR]) {
#pragma unroll
  for (int r = 0; r < NR; r++) a[r] = ((MAXM >> r) & 1u) ? -3.0e38f : 0.0f;
}
template <int NR, unsigned MAXM> __device__ __forceinline__ void facc_fold(double (&acc)[NR], const float (&a)[NR]) {
#pragma unroll
  for (int r = 0; r < NR; r++) acc[r] = ((MAXM >> r) & 1u) ? fmax(acc[r], (double)a[r]) : acc[r] + (double)a[r];
}

// Deterministic block reduction (fixed butterfly + fixed warp order).
// The result is valid in thread 0. scratch: 32 * NR doubles of shared memory.
template <int NR, unsigned MAXM>
__device__ __forceinline__ void block_reduce(double (&a)[NR], double *scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    double b[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) b[r] = __shfl_xor_sync(0xffffffffu, a[r], off);
    combine<NR, MAXM>(a, b);
  }
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int r = 0; r < NR; r++) scratch[warp * NR + r] = a[r];
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
    for (int w = 1; w < nw; w++) {
      double b[NR];
#pragma unroll
      for (int r = 0; r < NR; r++) b[r] = scratch[w * NR + r];
      combine<NR, MAXM>(a, b);
    }
  }
}

// Grid reduction: every CTA writes its block total to partials[bidx]; the CTA
// that finishes last sums all partials in fixed index order (so the result does
// not depend on scheduling) and returns true in its thread 0 with tot filled.
template <int NR, unsigned MAXM>
__device__ __forceinline__ bool grid_reduce(double (&acc)[NR], double *scratch, double *partials,
                                            unsigned *ticket, int nblk, int bidx, double (&tot)[NR]) {
  __shared__ int s_last;
  block_reduce<NR, MAXM>(acc, scratch);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int r = 0; r < NR; r++) partials[(size_t)bidx * kRedMax + r] = acc[r];
    __threadfence();
    unsigned prev = atomicAdd(ticket, 1u);
    s_last = (prev == (unsigned)nblk - 1u);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  double a[NR];
#pragma unroll
  for (int r = 0; r < NR; r++) a[r] = ((MAXM >> r) & 1u) ? -1.0e308 : 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
    double b[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) b[r] = __ldcg(&partials[(size_t)i * kRedMax + r]);
    combine<NR, MAXM>(a, b);
  }
  block_reduce<NR, MAXM>(a, scratch);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int r = 0; r < NR; r++) tot[r] = a[r];
    *ticket = 0u;
    return true;
  }
  return false;
}

// ------------------------------------------------------------------ async copies
// Bulk global->shared copies completing on an mbarrier (the non-tensor TMA
// path), and bounded waits: a wait that does not complete within ~1 s sets
// the CTA's error word and reports failure instead of spinning forever.
__device__ __forceinline__ uint32_t smem_u32(const void *ptr) {
  return (uint32_t)__cvta_generic_to_shared(ptr);
}
// Programmatic dependent launch. A kernel launched with the programmatic
// stream-serialisation attribute may be set up while the previous kernel of
// its stream completes; the wait blocks until that kernel has completed and
// its writes are visible, so every kernel launched that way runs this before
// its first global-memory access (a no-op in a plain launch). No kernel
// triggers its dependents early (griddepcontrol.launch_dependents): with the
// trigger at the top of each kernel, CTAs of the next launch were placed on
// the SMs as this grid's CTAs retired, and 256^3 gradient chains ran 20-25 %
// slower.
__device__ __forceinline__ void grid_dep_sync() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// Before an mbarrier's shared memory is used for anything else.
__device__ __forceinline__ void mbar_inval(uint64_t *bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// One arrival (release: the thread's earlier shared-memory accesses are
// ordered before a waiter's acquire of the completed phase).
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// One 16-byte global -> shared copy that bypasses registers and L1
// (both addresses 16-byte aligned); completes at cp_async_wait_all(), or
// by commit groups.
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)),
               "l"(__cvta_generic_to_global(src))
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// all but the most recently committed group complete
__device__ __forceinline__ void cp_async_wait_all_but_last() {
  asm volatile("cp.async.wait_group 1;" ::: "memory");
}
// Asks for `bytes` at src (16-byte aligned, a multiple of 16) to be brought
// into L2; no registers, shared memory or completion tracking involved.
__device__ __forceinline__ void prefetch_l2(const void *src, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}
// Accesses of the plane kernels' global exchange areas with an L2
// "evict last" policy, so the areas (a few tens of MB, rewritten every plane)
// stay in L2 while the streamed fields pass through it; the loads bypass L1
// (ld.global.cg: other SMs rewrite the areas between planes).
__device__ __forceinline__ uint64_t l2_keep_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ void st_keep(double2 *p, double2 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(p), "d"(v.x), "d"(v.y), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void st_keep(float2 *p, float2 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(p), "f"(v.x), "f"(v.y), "l"(pol)
               : "memory");
}
__device__ __forceinline__ double2 ld_keep(const double2 *p, uint64_t pol) {
  double2 v;
  asm volatile("ld.global.cg.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float2 ld_keep(const float2 *p, uint64_t pol) {
  float2 v;
  asm volatile("ld.global.cg.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(p), "l"(pol));
  return v;
}

// Streamed field data (read or written once per pass) with an L2 "evict
// first" policy, so it does not push the exchange areas out of L2.
__device__ __forceinline__ uint64_t l2_stream_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ double2 ld_stream(const double2 *p, uint64_t pol) {
  double2 v;
  asm volatile("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float2 ld_stream(const float2 *p, uint64_t pol) {
  float2 v;
  asm volatile("ld.global.nc.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ void st_stream(double2 *p, double2 v, uint64_t pol) { st_keep(p, v, pol); }
__device__ __forceinline__ void st_stream(float2 *p, float2 v, uint64_t pol) { st_keep(p, v, pol); }

// Cluster barrier halves. arrive_relaxed orders nothing: use it where a CTA
// only signals that it has finished READING other CTAs' shared memory (every
// loaded value already consumed by an instruction before it), so that they
// may overwrite it after their wait.
__device__ __forceinline__ void cluster_arrive_relaxed() {
  asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.aligned;" ::: "memory"); }
// Arrive with release semantics (the default of barrier.cluster.arrive): the
// CTA's earlier writes are visible to every thread of the cluster after its
// matching wait (acquire).
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.aligned;" ::: "memory"); }

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Tiled 3D tensor copy global->shared (coordinates innermost first, in
// elements; the innermost coordinate times the element size is a multiple of
// 16 bytes at every call site).
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}
constexpr long kSpinLimit = 4L << 20;  // polls of ~256 ns: about 1 s
// Returns false (and sets *err) when the phase did not complete within
// `limit` polls.
__device__ __forceinline__ bool mbar_wait_n(uint64_t *bar, unsigned parity, int *err, long limit) {
  if (*((volatile int *)err)) return false;
  for (long i = 0; i < limit; i++) {
    if (mbar_try_wait(bar, parity)) return true;
    if (i > 16) __nanosleep(256);
  }
  atomicExch(err, 1);
  return false;
}
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, int *err) {
  return mbar_wait_n(bar, parity, err, kSpinLimit);
}

// ------------------------------------------------------------------ parameters
struct ModelC {
  double Tau, Gamma, dt;
  double invL;     // 1/L, the reference's projection entry (Initialization.cpp:35-38)
  double inv_n3;   // 1/N^3
  double n3;
  double G0;       // G(k = 0)
  double ikt0;     // 1/(G0 + |Tau| + 0.02)
  double tol_grad; // grad-flow stop threshold on ||grad F|| (<= 0: off)
  double factor;   // SPM projection factor: 1 natural force, 2 min-max
  double max_steps;  // grad-flow step cap evaluated on the device (<= 0: off)
};

// Grad-flow control words in device memory.
enum FlowWord { FW_GO = 0, FW_PENDING = 1, FW_ITER = 2, FW_ERR = 4 };

struct KParams {
  // Tensor maps of the strided inputs: tmi[b] over p.in[b], tms[b] over p.st[b]
  // (filled by the launcher for the kernels that stage through TMA).
  CUtensorMap tmi[kMaxBatch];
  CUtensorMap tms[kMaxBatch];
  ModelC m;
  const void *in[kMaxBatch];
  void *out[kMaxBatch];
  const void *aux0[kMaxBatch];
  const void *aux1[kMaxBatch];
  const void *st[kMaxBatch];
  void *sto[kMaxBatch];
  const void *tw;       // T2[N]: exp(-2 pi i j / N)
  double *partials;     // [nb][blocks per field][kRedMax]
  unsigned *tickets;    // [nb]
  double *scal;         // [nb][kScal]
  int *flow;            // grad-flow control words (or null)
  double *stats;        // grad-flow per-step records (or null)
  const double4 *gtab;  // per K^2 = Kx^2+Ky^2+Kz^2: {G, 1/(1+dt G), 1/(G+|Tau|+0.02), 1/(1+G)}
  int *err;             // set when a bounded wait timed out
  void *xg;             // plane kernels with XG: global exchange areas, xg_regions x xg_cap CTAs x PLANE_UNITS complex
  int xg_cap;
  int xg_regions;
  int nb;
  // Launches that batch independent instances of one grid size (gradient
  // chains of a batched relaxation) set `batched`: field b then takes its
  // model, symbol table, flow words and step records from the arrays below
  // instead of m, gtab, flow and stats.
  int batched;
  ModelC mb[kMaxBatch];
  const double4 *gtabs[kMaxBatch];
  int *flows[kMaxBatch];
  double *statss[kMaxBatch];
};

// Per-field views of the model, symbols, flow words and records (see `batched`).
__device__ __forceinline__ const ModelC &model(const KParams &p, int b) { return p.batched ? p.mb[b] : p.m; }
__device__ __forceinline__ const double4 *gtab_of(const KParams &p, int b) { return p.batched ? p.gtabs[b] : p.gtab; }
__device__ __forceinline__ int *flow_of(const KParams &p, int b) { return p.batched ? p.flows[b] : p.flow; }
__device__ __forceinline__ double *stats_of(const KParams &p, int b) { return p.batched ? p.statss[b] : p.stats; }

// Spectral symbols of wave vector (Kx, Ky, Kz) from the per-context table.
__device__ __forceinline__ double4 symbols(const KParams &p, int Kx, int Ky, int Kz, int b = 0) {
  const double2 *t = reinterpret_cast<const double2 *>(gtab_of(p, b)) + 2 * (Kx * Kx + Ky * Ky + Kz * Kz);
  const double2 a = __ldg(t), c = __ldg(t + 1);
  return make_double4(a.x, a.y, c.x, c.y);
}

// Half `h` of the symbols at K^2 (h = 0: {G, 1/(1+dt G)}, h = 1: {1/(G+|Tau|+0.02), 1/(1+G)}).
__device__ __forceinline__ double2 symbols_half(const KParams &p, int k2, int h, int b = 0) {
  return __ldg(reinterpret_cast<const double2 *>(gtab_of(p, b)) + 2 * k2 + h);
}

// Signed wave number of index i on an N grid (Initialization.cpp:97-107).
__device__ __forceinline__ int wave(int i, int N) { return i < N / 2 ? i : i - N; }

}  // namespace spm
