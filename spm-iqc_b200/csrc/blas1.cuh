// Streaming field kernels that are not transforms: grid reductions over real
// fields (energy density, inner products) and the packed <-> full spectrum
// conversions used at the reference-compatible boundary.
#pragma once

#include "ops.cuh"

namespace spm {

constexpr int kReduceBlocks = 1184;  // 8 CTAs of 256 threads per SM on 148 SMs
static_assert(kReduceBlocks <= kPartStride, "partials stride");

// Grid-stride reduction over the real field p.in[b] (pairs of reals), with the
// prologue policy F supplying the per-element contribution and the finaliser.
template <class T, class F>
__global__ void __launch_bounds__(kThreads) field_reduce_kernel(const __grid_constant__ KParams p, size_t npairs) {
  __shared__ double red[32 * kRedMax];
  const int b = blockIdx.y;
  double acc[F::NR];
#pragma unroll
  for (int r = 0; r < F::NR; r++) acc[r] = ((F::MAXM >> r) & 1u) ? -1.0e308 : 0.0;
  const c2<T> *src = reinterpret_cast<const c2<T> *>(p.in[b]);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < npairs; i += (size_t)gridDim.x * blockDim.x)
    F::pro(p, b, 2 * i, __ldg(src + i), acc);
  double tot[F::NR];
  if (grid_reduce<F::NR, F::MAXM>(acc, red, p.partials + (size_t)b * kPartStride * kRedMax, p.tickets + b,
                                  gridDim.x, blockIdx.x, tot))
    F::fin(p, b, tot);
}

// <p, q> sums (BasicOperators.cpp:132-143): in = p, aux0 = q.
template <class T> struct ProDot {
  static constexpr int NR = 1;
  static constexpr unsigned MAXM = 0;
  __device__ static c2<T> pro(const KParams &p, int b, size_t idx, c2<T> x, double (&acc)[1]) {
    const c2<T> q = __ldg(reinterpret_cast<const c2<T> *>(reinterpret_cast<const T *>(p.aux0[b]) + idx));
    acc[0] += (double)x.x * (double)q.x + (double)x.y * (double)q.y;
    return x;
  }
  __device__ static void fin(const KParams &p, int b, const double (&tot)[1]) {
    p.scal[(size_t)b * kScal + SC_SUM0] = tot[0] * p.m.inv_n3;
  }
};

// Squared distance of an SPM replica pair, ||phi1 - phi0||^2 under inpfp
// (the dd of SPM.cpp:199-200): in = phi0, aux0 = phi1.
template <class T> struct ProDist {
  static constexpr int NR = 1;
  static constexpr unsigned MAXM = 0;
  __device__ static c2<T> pro(const KParams &p, int b, size_t idx, c2<T> x, double (&acc)[1]) {
    const c2<T> q = __ldg(reinterpret_cast<const c2<T> *>(reinterpret_cast<const T *>(p.aux0[b]) + idx));
    const double dx = (double)q.x - (double)x.x, dy = (double)q.y - (double)x.y;
    acc[0] += dx * dx + dy * dy;
    return x;
  }
  __device__ static void fin(const KParams &p, int b, const double (&tot)[1]) {
    p.scal[(size_t)b * kScal + SC_DD] = tot[0] * p.m.inv_n3;
  }
};

// Field mean (mean_Cplx, BasicOperators.cpp:121-130): scal[SC_SUM0] = sum / N^3.
template <class T> struct ProSum {
  static constexpr int NR = 1;
  static constexpr unsigned MAXM = 0;
  __device__ static c2<T> pro(const KParams &, int, size_t, c2<T> x, double (&acc)[1]) {
    acc[0] += (double)x.x + (double)x.y;
    return x;
  }
  __device__ static void fin(const KParams &p, int b, const double (&tot)[1]) {
    p.scal[(size_t)b * kScal + SC_SUM0] = tot[0] * p.m.inv_n3;
  }
};

// Precision change of a real field or packed spectrum (n scalars).
template <class Ti, class To>
__global__ void cast_kernel(const Ti *__restrict__ in, To *__restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (To)in[i];
}

// Packed spectrum -> the reference's full complex spectrum (double, interleaved).
template <class T>
__global__ void packed_to_full_kernel(const c2<T> *__restrict__ pk, double2 *__restrict__ full, int N) {
  const size_t n3 = (size_t)N * N * N;
  const int M = N / 2;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x) {
    const int kz = (int)(i % N), ky = (int)((i / N) % N), kx = (int)(i / ((size_t)N * N));
    const int nx = kx ? N - kx : 0, ny = ky ? N - ky : 0;
    double2 o;
    if (kz >= 1 && kz < M) {
      const c2<T> v = pk[((size_t)kx * N + ky) * M + kz];
      o = double2{(double)v.x, (double)v.y};
    } else if (kz > M) {
      const c2<T> v = pk[((size_t)nx * N + ny) * M + (N - kz)];
      o = double2{(double)v.x, -(double)v.y};
    } else {
      const c2<T> a = pk[((size_t)kx * N + ky) * M];
      const c2<T> c = pk[((size_t)nx * N + ny) * M];
      if (kz == 0) o = double2{0.5 * ((double)a.x + (double)c.x), 0.5 * ((double)a.y - (double)c.y)};
      else o = double2{0.5 * ((double)a.y + (double)c.y), 0.5 * ((double)c.x - (double)a.x)};
    }
    full[i] = o;
  }
}

// Full complex spectrum -> packed (takes the kz in [0, N/2] half).
template <class T>
__global__ void full_to_packed_kernel(const double2 *__restrict__ full, c2<T> *__restrict__ pk, int N) {
  const int M = N / 2;
  const size_t nh = (size_t)N * N * M;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nh; i += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % M);
    const size_t row = i / M;  // kx*N + ky
    const double2 a = full[row * N + c];
    if (c == 0) {
      const double2 h = full[row * N + M];
      pk[i] = c2<T>{(T)(a.x - h.y), (T)(a.y + h.x)};
    } else {
      pk[i] = c2<T>{(T)a.x, (T)a.y};
    }
  }
}

}  // namespace spm
