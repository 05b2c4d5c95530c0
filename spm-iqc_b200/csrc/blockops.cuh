// Block kernels of the LOBPCG and SPM solvers: the tall-skinny Gram on FP64
// tensor cores, the block combination Y = X C + d, the seeded start block, and
// the SPM spring update / stop check.
#pragma once

#include "fft_core.cuh"

namespace spm {

constexpr int kBlkMax = 24;      // vectors per block operand (3k with k <= 8)
constexpr int kGramBlocks = 296; // 2 CTAs per SM
constexpr int kGramWarps = 8;

struct GramP {
  const void *X[kBlkMax];
  const void *Y[kBlkMax];
  int ma, mb;
  size_t n;          // points per vector (multiple of 8)
  double inv_n;      // normalisation of <.,.> (1/N^3)
  double *partials;  // [kGramBlocks][kBlkMax * kBlkMax]
  unsigned *ticket;
  double *out;       // ma x mb, row-major
  const int *flow;   // optional gate
};

__device__ __forceinline__ void dmma_8x8x4(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// G[a][b] = inv_n * sum_i X_a[i] Y_b[i] for a < ma, b < mb (the Gram of
// LOBPCG.cpp:343-358 and the inner products of the block orthogonalisations).
// Each warp owns interleaved 8-point k-steps, two at a time: lane (row, tig)
// loads points 2 tig and 2 tig + 1 of the step with one vector load and feeds
// them to two MMAs (the same point order for X and Y, so the k order is
// merely permuted), accumulating the (ma x mb) product in 8x8 FP64 MMA tiles;
// CTA and grid totals are summed in a fixed order, so the result does not
// depend on scheduling.
// U = k-steps loaded per loop iteration, TM = row tiles (8 vectors each) at
// most per operand: (4, 1), (4, 2) or (2, 3) by block size.
// YT >= 0: Y's fields are X's fields from index 8 YT on (Y_b = X_{8 YT + b}),
// so a lane's B fragment of tile t is its A fragment of tile t + YT and Y is
// not read again (the Grams [Q X]^T X of the block orthogonalisations and the
// X^T X ones); YT = -1: Y is read.
template <class T, int U, int TM, int YT = -1>
__global__ void __launch_bounds__(kGramWarps * 32) gram_kernel(const __grid_constant__ GramP p) {
  __shared__ int s_last;
  if (p.flow && *((volatile const int *)p.flow) == 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gid = lane >> 2, tig = lane & 3;
  const int TA = (p.ma + 7) >> 3, TB = (p.mb + 7) >> 3;
  double acc[TM][TM][2];
#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int j = 0; j < TM; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
  using V2 = c2<T>;
  const V2 *xr[TM], *yr[TM];
#pragma unroll
  for (int t = 0; t < TM; t++) {
    const int ra = t * 8 + gid, rb = t * 8 + gid;
    xr[t] = (t < TA && ra < p.ma) ? reinterpret_cast<const V2 *>(p.X[ra]) : nullptr;
    yr[t] = (t < TB && rb < p.mb) ? reinterpret_cast<const V2 *>(p.Y[rb]) : nullptr;
  }
  const size_t steps = p.n / 8;
  const size_t gw = (size_t)blockIdx.x * kGramWarps + warp, W = (size_t)gridDim.x * kGramWarps;
  for (size_t s = gw; s < steps; s += U * W) {
    V2 a[U][TM], b[U][TM];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const size_t su = s + u * W;
      const bool in = su < steps;
#pragma unroll
      for (int t = 0; t < TM; t++) a[u][t] = (xr[t] && in) ? __ldg(xr[t] + 4 * su + tig) : V2{0, 0};
#pragma unroll
      for (int t = 0; t < TM; t++) {
        if constexpr (YT >= 0) {
          // the same lane and point mapping as the A fragment; rows beyond mb are not used
          b[u][t] = (t + YT < TM) ? a[u][t + YT] : V2{0, 0};
        } else {
          b[u][t] = (yr[t] && in) ? __ldg(yr[t] + 4 * su + tig) : V2{0, 0};
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TM; j++)
          if (i < TA && j < TB) {
            dmma_8x8x4(acc[i][j][0], acc[i][j][1], (double)a[u][i].x, (double)b[u][j].x);
            dmma_8x8x4(acc[i][j][0], acc[i][j][1], (double)a[u][i].y, (double)b[u][j].y);
          }
  }
  // CTA total in a fixed warp order: warp w writes its tiles, warp 0 sums
  __shared__ double tile[kGramWarps][kBlkMax * kBlkMax];
#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int j = 0; j < TM; j++)
      if (i < TA && j < TB) {
        const int r = i * 8 + gid, c = j * 8 + 2 * tig;
        tile[warp][r * kBlkMax + c] = acc[i][j][0];
        tile[warp][r * kBlkMax + c + 1] = acc[i][j][1];
      }
  __syncthreads();
  double *part = p.partials + (size_t)blockIdx.x * kBlkMax * kBlkMax;
  for (int e = threadIdx.x; e < kBlkMax * kBlkMax; e += blockDim.x) {
    const int r = e / kBlkMax, c = e % kBlkMax;
    if (r < TA * 8 && c < TB * 8) {
      double s = 0.0;
      for (int w = 0; w < kGramWarps; w++) s += tile[w][e];
      part[e] = s;
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(p.ticket, 1u) == gridDim.x - 1u);
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // grid total of every entry in a fixed order: each warp takes entries in
  // turn, lane l sums the partials of CTAs l, l + 32, ... (independent loads
  // in flight), then a fixed butterfly over the lanes
  for (int e = warp; e < p.ma * p.mb; e += kGramWarps) {
    const int r = e / p.mb, c = e % p.mb;
    double s = 0.0;
#pragma unroll 4
    for (unsigned bk = lane; bk < gridDim.x; bk += 32)
      s += __ldcg(p.partials + (size_t)bk * kBlkMax * kBlkMax + r * kBlkMax + c);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) p.out[e] = s * p.inv_n;
  }
  if (threadIdx.x == 0) *p.ticket = 0u;
}

// The coefficients travel in the kernel parameters (6.3 KB), so a
// combination needs no host-to-device copy (and no stream synchronisation
// for one) before its launch.
struct CombP {
  const void *X[kBlkMax + 8];
  void *Y[kBlkMax];
  int nin, nout;
  size_t n;
  double C[(kBlkMax + 8) * kBlkMax];  // nin x nout, row-major: Y_q += C[p*nout + q] X_p
  double d[kBlkMax];                  // nout constants (zeros when none)
  int accumulate;                     // Y_q = (accumulate ? Y_q : 0) + ...
  const int *flow;
};

// Y_q[i] = (accumulate ? Y_q[i] : 0) + sum_p C[p][q] X_p[i] + d[q]. A point's
// inputs (and, accumulating, its old outputs) are all loaded before any of its
// outputs is written, so Y may alias X and every load of a point is in flight
// at once. MI / MO bound nin / nout (registers); PTS consecutive points per
// thread, loaded as one vector when 2.
template <class T, int PTS> struct Pts;
template <class T> struct Pts<T, 1> {
  static __device__ __forceinline__ void ld(const void *b, size_t i, double (&v)[1]) {
    v[0] = (double)reinterpret_cast<const T *>(b)[i];
  }
  static __device__ __forceinline__ void st(void *b, size_t i, const double (&v)[1]) {
    reinterpret_cast<T *>(b)[i] = (T)v[0];
  }
};
template <class T> struct Pts<T, 2> {
  static __device__ __forceinline__ void ld(const void *b, size_t i, double (&v)[2]) {
    const c2<T> w = reinterpret_cast<const c2<T> *>(b)[i];
    v[0] = (double)w.x;
    v[1] = (double)w.y;
  }
  static __device__ __forceinline__ void st(void *b, size_t i, const double (&v)[2]) {
    reinterpret_cast<c2<T> *>(b)[i] = c2<T>{(T)v[0], (T)v[1]};
  }
};
template <class T, int MI, int MO, int PTS>
__global__ void __launch_bounds__(256) combine_kernel(const __grid_constant__ CombP p) {
  __shared__ double sc[(kBlkMax + 8) * kBlkMax + kBlkMax];
  if (p.flow && *((volatile const int *)p.flow) == 0) return;
  for (int e = threadIdx.x; e < p.nin * p.nout; e += blockDim.x) sc[e] = p.C[e];
  for (int e = threadIdx.x; e < p.nout; e += blockDim.x) sc[(kBlkMax + 8) * kBlkMax + e] = p.d[e];
  __syncthreads();
  const double *dd = sc + (kBlkMax + 8) * kBlkMax;
  const size_t nv = p.n / PTS;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += (size_t)gridDim.x * blockDim.x) {
    double x[MI][PTS], y[MO][PTS];
#pragma unroll
    for (int q = 0; q < MI; q++) {
      if (q < p.nin) Pts<T, PTS>::ld(p.X[q], i, x[q]);
      else
#pragma unroll
        for (int e = 0; e < PTS; e++) x[q][e] = 0.0;
    }
#pragma unroll
    for (int q = 0; q < MO; q++) {
      if (q < p.nout && p.accumulate) Pts<T, PTS>::ld(p.Y[q], i, y[q]);
      else
#pragma unroll
        for (int e = 0; e < PTS; e++) y[q][e] = 0.0;
    }
#pragma unroll
    for (int q = 0; q < MO; q++) {
      if (q < p.nout) {
        double o[PTS];
#pragma unroll
        for (int e = 0; e < PTS; e++) {
          double s = y[q][e];
#pragma unroll
          for (int r = 0; r < MI; r++)
            if (r < p.nin) s += sc[r * p.nout + q] * x[r][e];
          o[e] = s + dd[q];
        }
        Pts<T, PTS>::st(p.Y[q], i, o);
      }
    }
  }
}

// Start block of hiosd_lobpcg_initialization (LOBPCG.cpp:31-42) with
// Eigen's MatrixXd::Random(k, N^3) replaced by a SplitMix64 stream:
// V[i][j] = -1 + 2 u(seed, j*k + i) (the matrix is column-major).
template <class T>
__global__ void lobpcg_random_kernel(T *V, int k, size_t n, unsigned long long seed) {
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (size_t)gridDim.x * blockDim.x)
    for (int i = 0; i < k; i++) {
      unsigned long long z = seed + ((unsigned long long)(j * k + i) + 1ull) * 0x9E3779B97F4A7C15ull;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      z = z ^ (z >> 31);
      const double u = (double)(z >> 11) * 1.1102230246251565404e-16;  // 2^-53
      V[(size_t)i * n + j] = (T)(-1.0 + 2.0 * u);
    }
}

// The two spring updates of Spring_Pairing (SPM.cpp:203-216), in the
// reference's sequential order: phi1 sees the updated phi0.
template <class T>
__global__ void spring_kernel(T *phi0, T *phi1, size_t n, double dt, double ks, const int *flow) {
  if (flow && *((volatile const int *)flow) == 0) return;
  const T k = (T)ks, t = (T)dt;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    T p0 = phi0[i], p1 = phi1[i];
    T fs = k * p1 + (-k) * p0;
    p0 = (T)1 * p0 + t * fs;
    fs = k * p0 + (-k) * p1;
    p1 = (T)1 * p1 + t * fs;
    phi0[i] = p0;
    phi1[i] = p1;
  }
}

// End of one Spring_Pairing iteration (SPM.cpp:220-256): res = max_i ||grad F(Phi_i)||
// from the two ngrad norms, record it and disarm the chain when res <= tol.
__global__ void spm_check_kernel(double *scal, int *flow, double *stats, double tol, int cap) {
  if (flow[FW_GO] == 0) return;
  const double r0 = sqrt(scal[0 * kScal + SC_GN2]), r1 = sqrt(scal[1 * kScal + SC_GN2]);
  const double res = r0 > r1 ? r0 : r1;
  const int it = flow[FW_ITER];
  if (stats && it < cap) stats[it] = res;
  flow[FW_ITER] = it + 1;
  if (!(res > tol)) flow[FW_GO] = 0;
}

}  // namespace spm
