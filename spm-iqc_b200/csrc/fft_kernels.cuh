// The three streaming passes of a fused pseudo-spectral step on an N^3 grid.
//
//   plane_fwd : one thread-block cluster per x-plane (CL = N/32 CTAs). Each CTA
//               loads 32 z-rows of the real field, applies a pointwise prologue
//               (the nonlinear term, an energy density, ...), does the R2C
//               z-transform of its rows, then the cluster exchanges columns
//               through distributed shared memory and each CTA does the
//               y-transform of 16 spectral columns and writes them out.
//   pencil    : x-transform of 16 x-pencils (two ky rows {ky, -ky} x 8 columns),
//               a per-spectral-point operator (gradient step, G multiply,
//               preconditioner, SPM force update, ...) with reductions, and the
//               inverse x-transform, all without leaving the SM.
//   plane_inv : inverse of plane_fwd (y then C2R z) with a pointwise epilogue.
//
// Line transforms are two-level: each thread holds R1 elements of a line in
// registers (radix-R1 DFT), one shared-memory exchange, then an R2 = 8 or 16
// point DFT. Twiddles come from a per-grid table in shared memory.
//
// Every kernel first checks the optional grad-flow "go" word so that a chain of
// steps enqueued ahead (or replayed from a CUDA graph) stops exactly where the
// reference's loop would (LPsrc.cpp:52).
#pragma once

#include "fft_core.cuh"

namespace spm {

template <int N> struct Geo {
  static_assert(N % 32 == 0 && N >= 32 && N <= 256, "grid size must be a multiple of 32 in [32, 256]");
  static constexpr int M = N / 2;           // complex points per packed z-line
  static constexpr int CL = N / kRows;      // CTAs per cluster = per x-plane
  static constexpr int N1 = M / 8;          // z stage-1 radix (z stage-2 radix is 8)
  static constexpr int M1 = N / 16;         // y/x stage-1 radix (stage-2 radix is 16)
  static constexpr int ZPAD = N1 + 1;       // padded k1 extent of the z exchange
  static constexpr int PLANE_UNITS = kRows * 8 * ZPAD > kRows * M ? kRows * 8 * ZPAD : kRows * M;
  static constexpr int PENCIL_UNITS = M1 * 16 * 16;   // = 16 N
  static constexpr int BLOCKS = N * CL;     // CTAs per field, plane kernels (= N^2/32)
  static constexpr int PBLOCKS = (N / 2) * (M / 8);   // CTAs per field, pencil kernel
  static_assert(BLOCKS <= kPartStride && PBLOCKS <= kPartStride, "partials stride");
};

template <int N, class T> constexpr size_t plane_smem() {
  return sizeof(c2<T>) * (N + Geo<N>::PLANE_UNITS) + sizeof(double) * 32 * kRedMax;
}
template <int N, class T> constexpr size_t pencil_smem() {
  return sizeof(c2<T>) * (N + Geo<N>::PENCIL_UNITS) + sizeof(double) * 32 * kRedMax;
}

__device__ __forceinline__ bool flow_stopped(const KParams &p) {
  return p.flow != nullptr && *((volatile const int *)p.flow + FW_GO) == 0;
}

// --------------------------------------------------------------- plane_fwd
// Pro: static constexpr int NR; static constexpr unsigned MAXM;
//      __device__ static T2 pro(const KParams&, int b, size_t idx, T2 x, double (&acc)[NR]);
//        (x = reals idx, idx+1 of the input field; returns the values to transform)
//      __device__ static void fin(const KParams&, int b, const double (&tot)[NR]);
template <int N, class T, class Pro>
__global__ void __launch_bounds__(kThreads) plane_fwd_kernel(const __grid_constant__ KParams p) {
  using G = Geo<N>;
  using T2 = c2<T>;
  constexpr int M = G::M, N1 = G::N1, M1 = G::M1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T2 *tw = reinterpret_cast<T2 *>(smem_raw);
  T2 *buf = tw + N;
  double *red = reinterpret_cast<double *>(buf + G::PLANE_UNITS);
  if (flow_stopped(p)) return;

  cg::cluster_group cluster = cg::this_cluster();
  const int tid = threadIdx.x;
  const int b = blockIdx.y;
  const int rank = (int)cluster.block_rank();
  const int plane = blockIdx.x / G::CL;
  for (int i = tid; i < N; i += kThreads) tw[i] = reinterpret_cast<const T2 *>(p.tw)[i];
  double acc[Pro::NR > 0 ? Pro::NR : 1];
#pragma unroll
  for (int r = 0; r < (Pro::NR > 0 ? Pro::NR : 1); r++) acc[r] = ((Pro::MAXM >> r) & 1u) ? -1.0e308 : 0.0;
  __syncthreads();

  // ---- z, stage 1: task (row r, j2), 8 threads per row; element j = j1*8 + j2
  {
    const int j2 = tid & 7, r = tid >> 3;
    const size_t rowoff = ((size_t)plane * N + (size_t)(rank * kRows + r)) * N;
    const T *src = reinterpret_cast<const T *>(p.in[b]) + rowoff;
    T2 v[N1];
    sfor<0, N1>([&](auto J1) {
      constexpr int j1 = SPM_CI(J1);
      const int j = j1 * 8 + j2;
      T2 x = __ldg(reinterpret_cast<const T2 *>(src) + j);
      v[j1] = Pro::pro(p, b, rowoff + 2 * j, x, acc);
    });
    Dft<-1, N1, T2>::run(v);
    T2 *E = buf + r * (8 * G::ZPAD) + j2 * G::ZPAD;
    sfor<0, N1>([&](auto K1) {
      constexpr int k1 = SPM_CI(K1);
      E[k1] = (k1 == 0) ? v[k1] : cmul(v[k1], tw[2 * j2 * k1]);
    });
  }
  __syncthreads();
  // ---- z, stage 2: task (r, k1), 8-point DFT over j2 -> k = k1 + N1*k2
  {
    constexpr int NT = kRows * N1;
    constexpr int TPT = (NT + kThreads - 1) / kThreads;
    T2 u[TPT][8];
#pragma unroll
    for (int t = 0; t < TPT; t++) {
      const int task = tid + t * kThreads;
      if (task < NT) {
        const int r = task / N1, k1 = task % N1;
#pragma unroll
        for (int j2 = 0; j2 < 8; j2++) u[t][j2] = buf[r * (8 * G::ZPAD) + j2 * G::ZPAD + k1];
      }
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < TPT; t++) {
      const int task = tid + t * kThreads;
      if (task < NT) {
        const int r = task / N1, k1 = task % N1;
        Dft<-1, 8, T2>::run(u[t]);
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++) buf[r * M + k1 + N1 * k2] = u[t][k2];
      }
    }
  }
  __syncthreads();
  // ---- z, real-to-complex post-processing of the packed line (pairs k, M-k)
  {
    constexpr int NT = kRows * (M / 2);
    for (int task = tid; task < NT; task += kThreads) {
      const int r = task / (M / 2), q = task % (M / 2);
      T2 *Z = buf + r * M;
      if (q == 0) {
        const T2 z0 = Z[0];
        Z[0] = T2{z0.x + z0.y, z0.x - z0.y};  // X_0 + i X_{N/2}
        const T2 a = Z[M / 2];
        const T2 e = {a.x, (T)0};            // (a + conj a)/2
        const T2 o = {a.y, (T)0};            // (a - conj a)/(2i)
        Z[M / 2] = cadd(e, cmul(tw[M / 2], o));
      } else {
        const T2 a = Z[q], c = Z[M - q];
        const T2 e1 = {(T)0.5 * (a.x + c.x), (T)0.5 * (a.y - c.y)};   // (Z_q + conj Z_{M-q})/2
        const T2 o1 = {(T)0.5 * (a.y + c.y), (T)0.5 * (c.x - a.x)};   // (Z_q - conj Z_{M-q})/(2i)
        const T2 e2 = {e1.x, -e1.y};
        const T2 o2 = {o1.x, -o1.y};
        Z[q] = cadd(e1, cmul(tw[q], o1));
        Z[M - q] = cadd(e2, cmul(tw[M - q], o2));
      }
    }
  }
  cluster.sync();
  // ---- y, stage 1: task (column c, j2); element y = 16*j1 + j2 lives in CTA y/32
  {
    const int c = tid & 15, j2 = tid >> 4;
    const int col = rank * kCols + c;
    T2 v[M1];
    sfor<0, M1>([&](auto J1) {
      constexpr int j1 = SPM_CI(J1);
      const int y = 16 * j1 + j2;
      const T2 *rem = cluster.map_shared_rank(buf, (unsigned)(y >> 5));
      v[j1] = rem[(y & 31) * M + col];
    });
    cluster.sync();
    Dft<-1, M1, T2>::run(v);
    sfor<0, M1>([&](auto K1) {
      constexpr int k1 = SPM_CI(K1);
      buf[k1 * 256 + j2 * 16 + c] = (k1 == 0) ? v[k1] : cmul(v[k1], tw[j2 * k1]);
    });
  }
  __syncthreads();
  // ---- y, stage 2: task (c, k1) -> ky = k1 + M1*k2; write the spectral column
  if (tid < 16 * M1) {
    const int c = tid & 15, k1 = tid >> 4;
    const int col = rank * kCols + c;
    T2 u[16];
#pragma unroll
    for (int j2 = 0; j2 < 16; j2++) u[j2] = buf[k1 * 256 + j2 * 16 + c];
    Dft<-1, 16, T2>::run(u);
    T2 *dst = reinterpret_cast<T2 *>(p.out[b]);
#pragma unroll
    for (int k2 = 0; k2 < 16; k2++) {
      const int ky = k1 + M1 * k2;
      dst[((size_t)plane * N + ky) * M + col] = u[k2];
    }
  }
  if constexpr (Pro::NR > 0) {
    double tot[Pro::NR];
    if (grid_reduce<Pro::NR, Pro::MAXM>(acc, red, p.partials + (size_t)b * kPartStride * kRedMax,
                                        p.tickets + b, G::BLOCKS, blockIdx.x, tot))
      Pro::fin(p, b, tot);
  }
}

// --------------------------------------------------------------- pencil
// Op: static constexpr bool FI (forward x-transform of p.in), SI (load state p.st),
//     SO (store state p.sto), INV (inverse x-transform into p.out), LIN (the op
//     acts identically on both halves of the packed c = 0 column, so no unpack);
//     static constexpr int NR; static constexpr unsigned MAXM;
//     __device__ static void point(const KParams&, int b, int Kx, int Ky, int Kz,
//         T2 f, T2 s, T2 &so, T2 &inv, double (&acc)[NR], double w);
//       f = unnormalised forward value, s = state value, w = multiplicity of the
//       point in the full N^3 spectrum (1 on the kz = 0, N/2 planes, else 2).
//     __device__ static void fin(const KParams&, int b, const double (&tot)[NR]);
template <int N, class T, class Op>
__global__ void __launch_bounds__(kThreads) pencil_kernel(const __grid_constant__ KParams p) {
  using G = Geo<N>;
  using T2 = c2<T>;
  constexpr int M = G::M, M1 = G::M1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T2 *tw = reinterpret_cast<T2 *>(smem_raw);
  T2 *ex = tw + N;
  double *red = reinterpret_cast<double *>(ex + G::PENCIL_UNITS);
  if (flow_stopped(p)) return;

  const int tid = threadIdx.x;
  const int b = blockIdx.y;
  const int t = blockIdx.x % (N / 2);
  const int c0 = (blockIdx.x / (N / 2)) * 8;
  const int pen = tid & 15, rowsel = pen >> 3, cc = pen & 7;
  const int ky0 = t, ky1 = (t == 0) ? N / 2 : N - t;
  const int ky = rowsel ? ky1 : ky0;
  const int col = c0 + cc;
  const bool dc = (c0 == 0);
  const bool has2 = (tid >> 4) < M1;  // owns a stage-2 task (pencil, k1)
  const int k1 = tid >> 4;
  for (int i = tid; i < N; i += kThreads) tw[i] = reinterpret_cast<const T2 *>(p.tw)[i];
  double acc[Op::NR > 0 ? Op::NR : 1];
#pragma unroll
  for (int r = 0; r < (Op::NR > 0 ? Op::NR : 1); r++) acc[r] = ((Op::MAXM >> r) & 1u) ? -1.0e308 : 0.0;
  __syncthreads();

  T2 F[16], S[16];
  if constexpr (Op::FI) {
    // stage 1: task (pencil, j2 = tid/16): x = 16*j1 + j2
    {
      const int j2 = tid >> 4;
      const T2 *src = reinterpret_cast<const T2 *>(p.in[b]);
      T2 v[M1];
      sfor<0, M1>([&](auto J1) {
        constexpr int j1 = SPM_CI(J1);
        const int x = 16 * j1 + j2;
        v[j1] = __ldg(src + ((size_t)x * N + ky) * M + col);
      });
      Dft<-1, M1, T2>::run(v);
      sfor<0, M1>([&](auto K1) {
        constexpr int kk = SPM_CI(K1);
        ex[kk * 256 + j2 * 16 + pen] = (kk == 0) ? v[kk] : cmul(v[kk], tw[j2 * kk]);
      });
    }
    __syncthreads();
    if (has2) {
#pragma unroll
      for (int j2 = 0; j2 < 16; j2++) F[j2] = ex[k1 * 256 + j2 * 16 + pen];
      Dft<-1, 16, T2>::run(F);  // F[k2] at kx = k1 + M1*k2
    }
  }
  if constexpr (Op::SI) {
    if (has2) {
      const T2 *st = reinterpret_cast<const T2 *>(p.st[b]);
#pragma unroll
      for (int k2 = 0; k2 < 16; k2++) S[k2] = st[((size_t)(k1 + M1 * k2) * N + ky) * M + col];
    }
  }
  // partner values at (-kx, -ky) for the packed c = 0 pencils
  T2 Fp[16], Sp[16];
  if constexpr (!Op::LIN) {
    if (dc) {
      __syncthreads();
      T2 *D = ex;  // [quantity][rowsel][kx]
      if (has2 && cc == 0) {
#pragma unroll
        for (int k2 = 0; k2 < 16; k2++) {
          const int kx = k1 + M1 * k2;
          if constexpr (Op::FI) D[(0 * 2 + rowsel) * N + kx] = F[k2];
          if constexpr (Op::SI) D[(1 * 2 + rowsel) * N + kx] = S[k2];
        }
      }
      __syncthreads();
      if (has2 && cc == 0) {
        const int pr = (t == 0) ? rowsel : 1 - rowsel;
#pragma unroll
        for (int k2 = 0; k2 < 16; k2++) {
          const int kx = k1 + M1 * k2;
          const int nk = kx ? N - kx : 0;
          if constexpr (Op::FI) Fp[k2] = D[(0 * 2 + pr) * N + nk];
          if constexpr (Op::SI) Sp[k2] = D[(1 * 2 + pr) * N + nk];
        }
      }
    }
  }
  // the per-point operator
  if (has2) {
    T2 *so = Op::SO ? reinterpret_cast<T2 *>(p.sto[b]) : nullptr;
    const int Ky = wave(ky, N);
#pragma unroll
    for (int k2 = 0; k2 < 16; k2++) {
      const int kx = k1 + M1 * k2;
      const int Kx = wave(kx, N);
      T2 f = Op::FI ? F[k2] : T2{0, 0};
      T2 s = Op::SI ? S[k2] : T2{0, 0};
      T2 o_st = {0, 0}, o_inv = {0, 0};
      if (!Op::LIN && dc && cc == 0) {
        // unpack X(., ., 0) and X(., ., N/2), apply, repack
        T2 f0 = {0, 0}, fM = {0, 0}, s0 = {0, 0}, sM = {0, 0};
        if constexpr (Op::FI) {
          const T2 q = Fp[k2];
          f0 = T2{(T)0.5 * (f.x + q.x), (T)0.5 * (f.y - q.y)};
          fM = T2{(T)0.5 * (f.y + q.y), (T)0.5 * (q.x - f.x)};
        }
        if constexpr (Op::SI) {
          const T2 q = Sp[k2];
          s0 = T2{(T)0.5 * (s.x + q.x), (T)0.5 * (s.y - q.y)};
          sM = T2{(T)0.5 * (s.y + q.y), (T)0.5 * (q.x - s.x)};
        }
        T2 so0, inv0, soM, invM;
        Op::point(p, b, Kx, Ky, 0, f0, s0, so0, inv0, acc, 1.0);
        Op::point(p, b, Kx, Ky, -N / 2, fM, sM, soM, invM, acc, 1.0);
        o_st = T2{so0.x - soM.y, so0.y + soM.x};
        o_inv = T2{inv0.x - invM.y, inv0.y + invM.x};
      } else {
        Op::point(p, b, Kx, Ky, col, f, s, o_st, o_inv, acc, dc && cc == 0 ? 1.0 : 2.0);
      }
      if constexpr (Op::SO) so[((size_t)kx * N + ky) * M + col] = o_st;
      F[k2] = o_inv;
    }
  }
  if constexpr (Op::INV) {
    __syncthreads();
    if (has2) {
      Dft<+1, 16, T2>::run(F);  // over k2 -> j2
#pragma unroll
      for (int j2 = 0; j2 < 16; j2++)
        ex[k1 * 256 + j2 * 16 + pen] = (j2 == 0 || k1 == 0) ? F[j2] : cmulc(F[j2], tw[j2 * k1]);
    }
    __syncthreads();
    {
      const int j2 = tid >> 4;
      T2 v[M1];
      sfor<0, M1>([&](auto K1) { v[SPM_CI(K1)] = ex[SPM_CI(K1) * 256 + j2 * 16 + pen]; });
      Dft<+1, M1, T2>::run(v);
      T2 *dst = reinterpret_cast<T2 *>(p.out[b]);
      sfor<0, M1>([&](auto J1) {
        constexpr int j1 = SPM_CI(J1);
        const int x = 16 * j1 + j2;
        dst[((size_t)x * N + ky) * M + col] = v[j1];
      });
    }
  }
  if constexpr (Op::NR > 0) {
    double tot[Op::NR];
    if (grid_reduce<Op::NR, Op::MAXM>(acc, red, p.partials + (size_t)b * kPartStride * kRedMax,
                                      p.tickets + b, G::PBLOCKS, blockIdx.x, tot))
      Op::fin(p, b, tot);
  }
}

// --------------------------------------------------------------- plane_inv
// Epi: static constexpr int NR; static constexpr unsigned MAXM;
//      __device__ static T2 epi(const KParams&, int b, size_t idx, T2 y, double (&acc)[NR]);
//        (y = unnormalised inverse transform at reals idx, idx+1; returns values to store)
//      __device__ static void fin(const KParams&, int b, const double (&tot)[NR]);
template <int N, class T, class Epi>
__global__ void __launch_bounds__(kThreads) plane_inv_kernel(const __grid_constant__ KParams p) {
  using G = Geo<N>;
  using T2 = c2<T>;
  constexpr int M = G::M, N1 = G::N1, M1 = G::M1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T2 *tw = reinterpret_cast<T2 *>(smem_raw);
  T2 *buf = tw + N;
  double *red = reinterpret_cast<double *>(buf + G::PLANE_UNITS);
  if (flow_stopped(p)) return;

  cg::cluster_group cluster = cg::this_cluster();
  const int tid = threadIdx.x;
  const int b = blockIdx.y;
  const int rank = (int)cluster.block_rank();
  const int plane = blockIdx.x / G::CL;
  for (int i = tid; i < N; i += kThreads) tw[i] = reinterpret_cast<const T2 *>(p.tw)[i];
  double acc[Epi::NR > 0 ? Epi::NR : 1];
#pragma unroll
  for (int r = 0; r < (Epi::NR > 0 ? Epi::NR : 1); r++) acc[r] = ((Epi::MAXM >> r) & 1u) ? -1.0e308 : 0.0;
  __syncthreads();

  // ---- inverse y, stage 1: task (c, j2), input ky = 16*j1 + j2 (natural order)
  {
    const int c = tid & 15, j2 = tid >> 4;
    const int col = rank * kCols + c;
    const T2 *src = reinterpret_cast<const T2 *>(p.in[b]);
    T2 v[M1];
    sfor<0, M1>([&](auto J1) {
      constexpr int j1 = SPM_CI(J1);
      v[j1] = __ldg(src + ((size_t)plane * N + (16 * j1 + j2)) * M + col);
    });
    Dft<+1, M1, T2>::run(v);
    sfor<0, M1>([&](auto K1) {
      constexpr int k1 = SPM_CI(K1);
      buf[k1 * 256 + j2 * 16 + c] = (k1 == 0) ? v[k1] : cmulc(v[k1], tw[j2 * k1]);
    });
  }
  __syncthreads();
  // ---- inverse y, stage 2: task (c, k1) -> y = k1 + M1*k2; keep [y][c] in smem
  {
    T2 u[16];
    const int c = tid & 15, k1 = tid >> 4;
    if (tid < 16 * M1) {
#pragma unroll
      for (int j2 = 0; j2 < 16; j2++) u[j2] = buf[k1 * 256 + j2 * 16 + c];
      Dft<+1, 16, T2>::run(u);
    }
    __syncthreads();
    if (tid < 16 * M1) {
#pragma unroll
      for (int k2 = 0; k2 < 16; k2++) buf[(k1 + M1 * k2) * 16 + c] = u[k2];
    }
  }
  cluster.sync();
  // ---- complex-to-real pre-processing: gather the pairs (q, M-q) of my rows
  {
    constexpr int NT = kRows * (M / 2);
    constexpr int TPT = NT / kThreads;  // N/32 tasks per thread
    static_assert(NT % kThreads == 0, "task count");
    T2 za[TPT], zb[TPT];
#pragma unroll
    for (int i = 0; i < TPT; i++) {
      const int task = tid + i * kThreads;
      const int r = task / (M / 2), q = task % (M / 2);
      const int y = rank * kRows + r;
      if (q == 0) {
        const T2 *r0 = cluster.map_shared_rank(buf, 0u);
        const T2 *rh = cluster.map_shared_rank(buf, (unsigned)((M / 2) / kCols));
        const T2 P = r0[y * 16 + 0];
        const T2 a = rh[y * 16 + (M / 2) % kCols];
        // Z_0 = (X0 + XM) + i (X0 - XM) from the packed value P = X0 + i XM
        za[i] = T2{P.x + P.y, P.x - P.y};
        // Z_{M/2} = (a + conj a) + i w^{-M/2} (a - conj a)
        const T2 e = {a.x + a.x, (T)0};
        const T2 o = {(T)0, a.y + a.y};
        zb[i] = cadd(e, mul_di<+1>(cmulc(o, tw[M / 2])));
      } else {
        const T2 *ra = cluster.map_shared_rank(buf, (unsigned)(q / kCols));
        const T2 *rb = cluster.map_shared_rank(buf, (unsigned)((M - q) / kCols));
        const T2 a = ra[y * 16 + q % kCols];
        const T2 c = rb[y * 16 + (M - q) % kCols];
        // Z_q = (X_q + conj X_{M-q}) + i w^{-q} (X_q - conj X_{M-q})
        const T2 e1 = {a.x + c.x, a.y - c.y}, d1 = {a.x - c.x, a.y + c.y};
        const T2 e2 = {c.x + a.x, c.y - a.y}, d2 = {c.x - a.x, c.y + a.y};
        za[i] = cadd(e1, mul_di<+1>(cmulc(d1, tw[q])));
        zb[i] = cadd(e2, mul_di<+1>(cmulc(d2, tw[M - q])));
      }
    }
    cluster.sync();
#pragma unroll
    for (int i = 0; i < TPT; i++) {
      const int task = tid + i * kThreads;
      const int r = task / (M / 2), q = task % (M / 2);
      T2 *Z = buf + r * M;
      if (q == 0) {
        Z[0] = za[i];
        Z[M / 2] = zb[i];
      } else {
        Z[q] = za[i];
        Z[M - q] = zb[i];
      }
    }
  }
  __syncthreads();
  // ---- inverse z, stage 1: task (r, j2), element j = j1*8 + j2
  {
    const int j2 = tid & 7, r = tid >> 3;
    T2 v[N1];
    sfor<0, N1>([&](auto J1) { v[SPM_CI(J1)] = buf[r * M + SPM_CI(J1) * 8 + j2]; });
    __syncthreads();
    Dft<+1, N1, T2>::run(v);
    T2 *E = buf + r * (8 * G::ZPAD) + j2 * G::ZPAD;
    sfor<0, N1>([&](auto K1) {
      constexpr int k1 = SPM_CI(K1);
      E[k1] = (k1 == 0) ? v[k1] : cmulc(v[k1], tw[2 * j2 * k1]);
    });
  }
  __syncthreads();
  // ---- inverse z, stage 2: task (r, k1) -> j = k1 + N1*k2; z_j = y_{2j} + i y_{2j+1}
  {
    constexpr int NT = kRows * N1;
    constexpr int TPT = (NT + kThreads - 1) / kThreads;
#pragma unroll
    for (int t2 = 0; t2 < TPT; t2++) {
      const int task = tid + t2 * kThreads;
      if (task < NT) {
        const int r = task / N1, k1 = task % N1;
        T2 u[8];
#pragma unroll
        for (int j2 = 0; j2 < 8; j2++) u[j2] = buf[r * (8 * G::ZPAD) + j2 * G::ZPAD + k1];
        Dft<+1, 8, T2>::run(u);
        const size_t rowoff = ((size_t)plane * N + (size_t)(rank * kRows + r)) * N;
        T *outb = reinterpret_cast<T *>(p.out[b]);  // null: reductions only
        T2 *dst = reinterpret_cast<T2 *>(outb + rowoff);
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++) {
          const int j = k1 + N1 * k2;
          const T2 val = Epi::epi(p, b, rowoff + 2 * j, u[k2], acc);
          if (outb) dst[j] = val;
        }
      }
    }
  }
  if constexpr (Epi::NR > 0) {
    double tot[Epi::NR];
    if (grid_reduce<Epi::NR, Epi::MAXM>(acc, red, p.partials + (size_t)b * kPartStride * kRedMax,
                                        p.tickets + b, G::BLOCKS, blockIdx.x, tot))
      Epi::fin(p, b, tot);
  }
}

}  // namespace spm
