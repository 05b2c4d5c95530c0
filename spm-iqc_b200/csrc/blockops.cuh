// Block kernels of the LOBPCG and SPM solvers: the tall-skinny Gram on FP64
// tensor cores, the block combination Y = X C + d, the seeded start block, and
// the SPM spring update / stop check.
#pragma once

#include "fft_core.cuh"

namespace spm {

constexpr int kBlkMax = 24;      // vectors per block operand (3k with k <= 8)
constexpr int kGramBlocks = 296; // 2 CTAs per SM
constexpr int kGramWarps = 8;

constexpr int kStageBlocks = 148;  // staged Gram: one CTA per SM of a B200 (a fixed grid: fixed partial sums)
constexpr int kStageWarps = 16;    // its consumer warps (plus one producer warp)

struct GramP {
  const void *X[kBlkMax];
  const void *Y[kBlkMax];
  int ma, mb;
  size_t n;          // points per vector (multiple of 8)
  double inv_n;      // normalisation of <.,.> (1/N^3)
  double *partials;  // [kGramBlocks][kBlkMax * kBlkMax]
  unsigned *ticket;
  double *out;       // ma x mb, row-major (the staged kernel adds out[ma*mb]: its error flag)
  const int *flow;   // optional gate
  // staged kernel only: the distinct fields of X and Y, each staged once
  const void *F[2 * kBlkMax];
  unsigned char xf[kBlkMax], yf[kBlkMax];  // X_a = F[xf[a]], Y_b = F[yf[b]]
  int nf;
  int chunk_bytes;   // bytes of one field per chunk (a multiple of 128 dividing the field)
  int stages;
  int *err;          // the context's error word (bounded waits)
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

// The same Gram with the fields staged through shared memory. Each CTA streams
// its chunks (chunk c: points [c CH, (c+1) CH) of every distinct field, CH =
// chunk_bytes / sizeof(T); CTA b takes chunks b, b + grid, ...) through a ring
// of `stages` buffers. A producer warp issues one bulk copy per field and
// chunk (lane f copies field f), completing on the buffer's "full" mbarrier,
// and refills a buffer once the 16 consumer warps have arrived on its "empty"
// mbarrier, so the consumers never wait for one another and a whole chunk of
// every field is in flight per buffer without registers or per-thread loads.
// The consumers read the fragments from shared memory (rows padded by 16
// bytes: the 8 rows x 4 lanes of a fragment load fall in distinct bank
// groups) and issue the same DMMA m8n8k4 pairs as gram_kernel. A field that
// is both an X and a Y operand (the aliased Grams of the block
// orthogonalisations) is read from HBM once. Sums are in a fixed order: a
// warp's k-steps in chunk order, then the warps, then the CTAs.
// TA / TB: 8-vector tiles of X / Y (ma <= 8 TA, mb <= 8 TB).
template <class T, int TA, int TB>
__global__ void __launch_bounds__((kStageWarps + 1) * 32, 1) gram_staged_kernel(const __grid_constant__ GramP p) {
  constexpr int NW = kStageWarps + 1;  // warps: consumers 0..15, producer 16
  extern __shared__ __align__(128) unsigned char gsm_raw[];
  __shared__ int s_err, s_last, s_issued;
  if (p.flow && *((volatile const int *)p.flow) == 0) return;
  unsigned char *st = smem_base128(gsm_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gid = lane >> 2, tig = lane & 3;
  const int nf = p.nf, CB = p.chunk_bytes, RS = CB + 16, ST = p.stages;
  const int CH = CB / (int)sizeof(T);
  uint64_t *full = reinterpret_cast<uint64_t *>(st + (size_t)ST * nf * RS);
  uint64_t *empty = full + ST;
  using V2 = c2<T>;
  const size_t nch = p.n / (size_t)CH;
  const int mine = nch > blockIdx.x ? (int)((nch - 1 - blockIdx.x) / gridDim.x + 1) : 0;
  if (tid == 0) {
    for (int s = 0; s < ST; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kStageWarps);
    }
    s_err = 0;
    s_issued = 0;
    fence_barrier_init();
  }
  __syncthreads();
  double acc[TA][TB][2];
#pragma unroll
  for (int i = 0; i < TA; i++)
#pragma unroll
    for (int j = 0; j < TB; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
  if (warp == kStageWarps) {
    // producer: chunk i into buffer i % ST once chunk i - ST is consumed
    for (int i = 0; i < mine; i++) {
      const int s = i % ST;
      const bool ok = i < ST || mbar_wait(&empty[s], (unsigned)((i / ST - 1) & 1), &s_err);
      if (!__all_sync(0xffffffffu, ok)) break;  // the warp leaves together
      const size_t c = blockIdx.x + (size_t)i * gridDim.x;
      if (lane == 0) mbar_expect_tx(&full[s], (unsigned)(nf * CB));
      __syncwarp();
      unsigned char *dst = st + (size_t)s * nf * RS;
      for (int f = lane; f < nf; f += 32)
        bulk_g2s(dst + (size_t)f * RS, reinterpret_cast<const unsigned char *>(p.F[f]) + c * CB, (unsigned)CB,
                 &full[s]);
      if (lane == 0) s_issued = i + 1;
    }
  } else {
    // this lane's fragment rows (byte offsets within a buffer; -1: beyond ma / mb)
    int ra[TA], rb[TB];
#pragma unroll
    for (int t = 0; t < TA; t++) ra[t] = (8 * t + gid < p.ma) ? (int)p.xf[8 * t + gid] * RS : -1;
#pragma unroll
    for (int t = 0; t < TB; t++) rb[t] = (8 * t + gid < p.mb) ? (int)p.yf[8 * t + gid] * RS : -1;
    for (int i = 0; i < mine; i++) {
      const int s = i % ST;
      const bool ok = mbar_wait(&full[s], (unsigned)((i / ST) & 1), &s_err);
      if (!__all_sync(0xffffffffu, ok)) break;  // the warp leaves together
      const unsigned char *buf = st + (size_t)s * nf * RS;
      // 8-point groups g of the chunk: lane (gid, tig) takes points 8g + 2 tig, +1
      for (int g = warp; g < CH / 8; g += kStageWarps) {
        V2 a[TA], b[TB];
#pragma unroll
        for (int t = 0; t < TA; t++)
          a[t] = ra[t] >= 0 ? reinterpret_cast<const V2 *>(buf + ra[t])[4 * g + tig] : V2{0, 0};
#pragma unroll
        for (int t = 0; t < TB; t++)
          b[t] = rb[t] >= 0 ? reinterpret_cast<const V2 *>(buf + rb[t])[4 * g + tig] : V2{0, 0};
#pragma unroll
        for (int ii = 0; ii < TA; ii++)
#pragma unroll
          for (int j = 0; j < TB; j++) {
            dmma_8x8x4(acc[ii][j][0], acc[ii][j][1], (double)a[ii].x, (double)b[j].x);
            dmma_8x8x4(acc[ii][j][0], acc[ii][j][1], (double)a[ii].y, (double)b[j].y);
          }
      }
      // this warp is done reading buffer s: order its reads before the
      // producer's next bulk copy into it
      fence_proxy_async();
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
  }
  __syncthreads();
  if (tid == 0) {
    if (s_err) {
      // a wait gave up: let the copies still in flight land (bounded) before
      // the buffers are reused below or the CTA exits
      const int issued = s_issued;
      for (int i = issued > ST ? issued - ST : 0; i < issued; i++)
        for (long k = 0; k < kSpinLimit && !mbar_try_wait(&full[i % ST], (unsigned)((i / ST) & 1)); k++)
          __nanosleep(256);
    }
    for (int s = 0; s < ST; s++) {
      mbar_inval(&full[s]);
      mbar_inval(&empty[s]);
    }
  }
  __syncthreads();
  // CTA total in a fixed warp order (the ring's bytes hold the per-warp tiles)
  double *tile = reinterpret_cast<double *>(st);
  constexpr int RA = 8 * TA, RB = 8 * TB;
  if (warp < kStageWarps) {
#pragma unroll
    for (int i = 0; i < TA; i++)
#pragma unroll
      for (int j = 0; j < TB; j++) {
        const int r = i * 8 + gid, c = j * 8 + 2 * tig;
        tile[(warp * RA + r) * RB + c] = acc[i][j][0];
        tile[(warp * RA + r) * RB + c + 1] = acc[i][j][1];
      }
  }
  __syncthreads();
  double *part = p.partials + (size_t)blockIdx.x * kBlkMax * kBlkMax;
  for (int e = tid; e < RA * RB; e += NW * 32) {
    double s = 0.0;
    for (int w = 0; w < kStageWarps; w++) s += tile[w * RA * RB + e];
    part[(e / RB) * kBlkMax + e % RB] = s;
  }
  if (tid == 0 && s_err) atomicExch(p.err, 1);
  __threadfence();
  __syncthreads();
  if (tid == 0) s_last = (atomicAdd(p.ticket, 1u) == gridDim.x - 1u);
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // grid total of every entry in a fixed order (as gram_kernel)
  for (int e = warp; e < p.ma * p.mb; e += NW) {
    const int r = e / p.mb, c = e % p.mb;
    double s = 0.0;
#pragma unroll 4
    for (unsigned bk = lane; bk < gridDim.x; bk += 32)
      s += __ldcg(p.partials + (size_t)bk * kBlkMax * kBlkMax + r * kBlkMax + c);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) p.out[e] = s * p.inv_n;
  }
  if (tid == 0) {
    p.out[p.ma * p.mb] = (double)*((volatile int *)p.err);
    *p.ticket = 0u;
  }
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
  // staged kernel only (no accumulation; C packed with row stride kBlkMax:
  // C[p * kBlkMax + q]): the distinct inputs, each staged once
  const void *F[kBlkMax + 8];
  unsigned char xf[kBlkMax + 8];      // X_p = F[xf[p]]
  int nf;
  int chunk_bytes;                    // as GramP
  int stages;
  int *err;
  // optional (staged kernel): norms[q] = inv_n sum_i Y_q[i]^2 of the outputs,
  // summed in a fixed order through partials [grid][kBlkMax] and a ticket;
  // norms[nout] receives the error word
  double *norms;
  double *partials;
  unsigned *ticket;
  double inv_n;
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

// The same combination (without accumulation, nout <= NO) with the inputs
// staged through shared memory by a producer warp, as gram_staged_kernel
// does: chunk c of every distinct input lands in a ring buffer, and one of two
// groups of 8 consumer warps (alternate chunks, so two chunks are worked on at
// once) computes the chunk's outputs point by point (thread j of the
// chunk: Y_q[j] = sum_p C[p][q] X_p[j] + d[q], the coefficients read from the
// kernel parameters at fixed offsets) and stores them. Same operations in the
// same order as combine_kernel, so the results are the same bits. A chunk's
// inputs are all in shared memory before any of its outputs is stored, and
// chunks are disjoint, so Y may alias X. With p.norms the kernel also returns
// the outputs' squared norms (LOBPCG's residual norms of W = H V - alpha V).
constexpr int kCombWarps = 16;  // consumer warps: two groups of 8, taking alternate chunks
constexpr int kCombGroupWarps = 8;
template <class T, int NI, int NO>
__global__ void __launch_bounds__((kCombWarps + 1) * 32, 1) combine_staged_kernel(const __grid_constant__ CombP p) {
  extern __shared__ __align__(128) unsigned char csm_raw[];
  __shared__ int s_err, s_issued;
  if (p.flow && *((volatile const int *)p.flow) == 0) return;
  unsigned char *st = smem_base128(csm_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nf = p.nf, CB = p.chunk_bytes, RS = CB + 16, ST = p.stages;
  const int CH = CB / (int)sizeof(T);
  uint64_t *full = reinterpret_cast<uint64_t *>(st + (size_t)ST * nf * RS);
  uint64_t *empty = full + ST;
  const size_t nch = p.n / (size_t)CH;
  const int mine = nch > blockIdx.x ? (int)((nch - 1 - blockIdx.x) / gridDim.x + 1) : 0;
  if (tid == 0) {
    for (int s = 0; s < ST; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kCombGroupWarps);
    }
    s_err = 0;
    s_issued = 0;
    fence_barrier_init();
  }
  __syncthreads();
  if (warp == kCombWarps) {
    for (int i = 0; i < mine; i++) {
      const int s = i % ST;
      const bool ok = i < ST || mbar_wait(&empty[s], (unsigned)((i / ST - 1) & 1), &s_err);
      if (!__all_sync(0xffffffffu, ok)) break;
      const size_t c = blockIdx.x + (size_t)i * gridDim.x;
      if (lane == 0) mbar_expect_tx(&full[s], (unsigned)(nf * CB));
      __syncwarp();
      unsigned char *dst = st + (size_t)s * nf * RS;
      for (int f = lane; f < nf; f += 32)
        bulk_g2s(dst + (size_t)f * RS, reinterpret_cast<const unsigned char *>(p.F[f]) + c * CB, (unsigned)CB,
                 &full[s]);
      if (lane == 0) s_issued = i + 1;
    }
  }
  double nsq[NO];  // squared norms of this thread's outputs
#pragma unroll
  for (int q = 0; q < NO; q++) nsq[q] = 0.0;
  if (warp < kCombWarps) {
    const int grp = warp / kCombGroupWarps, gt = tid - grp * kCombGroupWarps * 32;
    for (int i = grp; i < mine; i += kCombWarps / kCombGroupWarps) {
      const int s = i % ST;
      const bool ok = mbar_wait(&full[s], (unsigned)((i / ST) & 1), &s_err);
      if (!__all_sync(0xffffffffu, ok)) break;
      const unsigned char *buf = st + (size_t)s * nf * RS;
      const size_t base = (blockIdx.x + (size_t)i * gridDim.x) * (size_t)CH;
      for (int j = gt; j < CH; j += kCombGroupWarps * 32) {
        double o[NO];
#pragma unroll
        for (int q = 0; q < NO; q++) o[q] = 0.0;
#pragma unroll
        for (int r = 0; r < NI; r++) {
          if (r < p.nin) {
            const double x = (double)reinterpret_cast<const T *>(buf + (size_t)p.xf[r] * RS)[j];
#pragma unroll
            for (int q = 0; q < NO; q++) o[q] = __fma_rn(p.C[r * kBlkMax + q], x, o[q]);
          }
        }
#pragma unroll
        for (int q = 0; q < NO; q++)
          if (q < p.nout) {
            const T y = (T)(o[q] + p.d[q]);
            reinterpret_cast<T *>(p.Y[q])[base + j] = y;
            nsq[q] += (double)y * (double)y;
          }
      }
      fence_proxy_async();
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
  }
  __syncthreads();
  if (tid == 0) {
    if (s_err) {
      // a wait gave up: let the copies still in flight land (bounded)
      const int issued = s_issued;
      for (int i = issued > ST ? issued - ST : 0; i < issued; i++)
        for (long k = 0; k < kSpinLimit && !mbar_try_wait(&full[i % ST], (unsigned)((i / ST) & 1)); k++)
          __nanosleep(256);
      atomicExch(p.err, 1);
    }
    for (int s = 0; s < ST; s++) {
      mbar_inval(&full[s]);
      mbar_inval(&empty[s]);
    }
  }
  if (!p.norms) return;
  // the outputs' squared norms: per CTA in a fixed thread order, then over
  // the CTAs in a fixed order by the last CTA
  __syncthreads();
  double *red = reinterpret_cast<double *>(st);  // [threads][NO], over the idle ring
  const int nthr = (kCombWarps + 1) * 32;
#pragma unroll
  for (int q = 0; q < NO; q++) red[(size_t)tid * NO + q] = nsq[q];
  __syncthreads();
  __shared__ int s_last;
  if (tid < NO) {
    double t = 0.0;
    for (int u = 0; u < nthr; u++) t += red[(size_t)u * NO + tid];
    p.partials[(size_t)blockIdx.x * kBlkMax + tid] = t;
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) s_last = (atomicAdd(p.ticket, 1u) == gridDim.x - 1u);
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (tid < NO && tid < p.nout) {
    double t = 0.0;
    for (unsigned bk = 0; bk < gridDim.x; bk++) t += __ldcg(p.partials + (size_t)bk * kBlkMax + tid);
    p.norms[tid] = t * p.inv_n;
  }
  if (tid == 0) {
    p.norms[p.nout] = (double)*((volatile int *)p.err);
    *p.ticket = 0u;
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
// reference's sequential order: phi1 sees the updated phi0. dd2 (optional):
// the pair's squared distance, for a spring of rest length `rest` (the
// reference's spring_d and kd = ks (dd - spring_d), SPM.cpp:179, 206-212,
// which it computes but does not apply): the force ks (dd - rest) along the
// unit vector (phi1 - phi0) / dd, i.e. the coefficient ks (dd - rest) / dd.
template <class T>
__global__ void spring_kernel(T *phi0, T *phi1, size_t n, double dt, double ks, const int *flow,
                              const double *dd2 = nullptr, double rest = 0.0) {
  if (flow && *((volatile const int *)flow) == 0) return;
  double kc = ks;
  if (dd2) {
    const double dd = sqrt(*dd2);
    kc = dd > 0.0 ? ks * ((dd - rest) / dd) : 0.0;
  }
  const T k = (T)kc, t = (T)dt;
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
