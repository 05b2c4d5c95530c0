// The three streaming passes of a fused pseudo-spectral step on an N^3 grid.
//
//   plane_fwd : thread-block clusters of CL = N/32 CTAs, each cluster looping
//               over x-planes. Each CTA takes 32 z-rows of the real field,
//               applies a pointwise prologue (the nonlinear term, an energy
//               density, ...), does the R2C z-transform of its rows; the
//               cluster then exchanges columns through distributed shared
//               memory and each CTA does the y-transform of 16 spectral columns.
//   pencil    : CTAs looping over tiles of 16 x-pencils (two ky rows
//               {ky, -ky} x 8 columns): forward x-transform, a per-spectral-point
//               operator (gradient step, G multiply, preconditioner, SPM force
//               update, ...) with reductions, inverse x-transform.
//   plane_inv : inverse of plane_fwd (y, then C2R z) with a pointwise epilogue.
//
// All three kernels are persistent: the input of the next tile is fetched
// with bulk asynchronous copies into a shared-memory stage (completion on an
// mbarrier) while the current tile is transformed. Line transforms are
// two-level: each thread holds R1 elements of a line in registers (radix-R1
// DFT), one shared-memory exchange, then an 8- or 16-point DFT.
//
// Every kernel first checks the optional "go" word so that a chain of steps
// enqueued ahead stops exactly where the reference's loop would (LPsrc.cpp:52).
#pragma once

#include "fft_core.cuh"

namespace spm {

template <int N> struct Geo {
  static_assert(N % 32 == 0 && N >= 32 && N <= 256, "grid size must be a multiple of 32 in [32, 256]");
  static constexpr int M = N / 2;           // complex points per packed z-line
  static constexpr int CL = N / kRows;      // CTAs per cluster = per x-plane
  static constexpr int N1 = M / 8;          // z stage-1 radix (z stage-2 radix is 8)
  static constexpr int M1 = N / 16;         // y/x stage-1 radix (stage-2 radix is 16)
  static constexpr int PLANE_UNITS = kRows * M;  // = 16 N: 32 rows, or 16 columns x N
  static constexpr int PENCIL_UNITS = M1 * 16 * 16;   // = 16 N
  static constexpr int STAGE_UNITS = 16 * N;          // one staged tile (plane rows / columns / pencils)
  static constexpr int PTILES = (N / 2) * (M / 8);    // pencil tiles per field
};

// Shared-memory layout (complex units): twiddles N | z-twiddles N/2 | work | stage | mbarriers | reduction
// (+128 bytes to align the base for the tensor copies)
template <int N, class T, int CPS, int RW = kRows> constexpr size_t plane_smem() {
  return sizeof(c2<T>) * (N + N / 2 + RW * (N / 2) + (CPS == 1 ? Geo<N>::STAGE_UNITS : 0)) + 16 +
         sizeof(double) * 32 * kRedMax + 128;
}
// Pencil tiles: the rows {ky, -ky} x TC spectral columns (TC = 8, or 4 for
// the narrow variant), 2 TC x-pencils of N points, one CTA of 16 x 2 TC threads.
template <int N, int TC = 8> struct PencilGeo {
  static_assert(TC == 8 || TC == 4, "pencil tiles are 8 or 4 columns wide");
  static constexpr int NP = 2 * TC;                   // pencils per tile
  static constexpr int TH = 16 * NP;                  // threads per CTA
  static constexpr int UNITS = Geo<N>::M1 * 16 * NP;  // x-transform exchange
  static constexpr int STAGE = 2 * N * TC;            // one staged tile
  static constexpr int NCH = (N / 2) / TC;            // column chunks per ky row
  static constexpr int PTILES = (N / 2) * NCH;        // tiles per field
  static constexpr int SYMN = (TC + 1) * (N / 2 + 1); // symbol entries per tile
};
// Pencil symbol table (per tile): TC + 1 kz rows (the tile's columns and
// kz = N/2) x |Kx| = 0..N/2, one double2 half of the K^2 symbols each.
template <int N, int TC = 8> constexpr int pencil_sym_entries() { return PencilGeo<N, TC>::SYMN; }
template <int N, class T, int TC = 8> constexpr size_t pencil_smem_n(int stages, int symbufs) {
  using PG = PencilGeo<N, TC>;
  return sizeof(c2<T>) * (N + PG::UNITS + (size_t)stages * PG::STAGE) + 16 + sizeof(double) * 32 * kRedMax +
         sizeof(double2) * PG::SYMN * symbufs + 128;
}
// CTAs of `smem` bytes that one SM holds (228 KB per SM, 1 KB reserved per CTA,
// at most 227 KB per CTA).
constexpr int smem_ctas_per_sm(size_t smem) { return smem > 232448 ? 0 : (int)(233472 / (smem + 1024)); }
// Symbol buffers of the pencil: two (the next tile's copies start a whole
// tile ahead) where the second one costs no resident CTA, else one.
template <int N, class T, int TC = 8> constexpr int pencil_sym_bufs(int stages, bool sym) {
  return !sym ? 0
         : smem_ctas_per_sm(pencil_smem_n<N, T, TC>(stages, 2)) == smem_ctas_per_sm(pencil_smem_n<N, T, TC>(stages, 1))
             ? 2
             : 1;
}
// Resident pencil CTAs per SM the registers are budgeted for. 8-column tiles:
// two for FP32 pencils whose shared memory (one symbol buffer) lets two CTAs
// of 256 threads share an SM, which bounds them to 128 registers a thread;
// else one. (At 256^3 FP32 the gradient pencil does not fit twice: one CTA
// with two symbol buffers beat two CTAs with one buffer each.) 4-column tiles
// (128 threads): as many as their shared memory allows, at most four.
template <int N, class T, int TC = 8> constexpr int pencil_min_ctas(int stages, bool sym) {
  if constexpr (TC == 4) {
    const int k = smem_ctas_per_sm(pencil_smem_n<N, T, TC>(stages, pencil_sym_bufs<N, T, TC>(stages, sym)));
    return k < 1 ? 1 : (k > 4 ? 4 : k);
  } else {
    return sizeof(T) == 4 && smem_ctas_per_sm(pencil_smem_n<N, T>(stages, sym ? 1 : 0)) >= 2 ? 2 : 1;
  }
}
template <int N, class T, int TC = 8> constexpr size_t pencil_smem(int stages, bool sym) {
  return pencil_smem_n<N, T, TC>(stages, pencil_sym_bufs<N, T, TC>(stages, sym));
}

__device__ __forceinline__ unsigned char *smem_base128(unsigned char *raw) {
  return raw + ((128u - (smem_u32(raw) & 127u)) & 127u);
}

__device__ __forceinline__ bool flow_stopped(const KParams &p, int b) {
  const int *f = flow_of(p, b);
  return f != nullptr && *((volatile const int *)f + FW_GO) == 0;
}
// The step's stop is armed (FW_PENDING, set by its pencil pass before launch).
__device__ __forceinline__ bool flow_pending(const KParams &p, int b) {
  const int *f = flow_of(p, b);
  return f != nullptr && *((volatile const int *)f + FW_PENDING) != 0;
}

// This CTA's global exchange area in region e (e = 0: inverse exchange, 1:
// forward; the software-pipelined fused pass also uses 2 and 3, a second
// area of each) and that of rank 0 of its cluster (the cluster's CTAs are
// consecutive in x). Each region holds xg_cap areas of 16 N complex values
// (32-row CTAs), or twice as many of 8 N (16-row CTAs).
template <int N, class T, int RW = kRows, int R = 2> struct XgAreas {
  c2<T> *own[R] = {};
  const c2<T> *first[R] = {};
  __device__ XgAreas(const KParams &p, int rank) {
    if (p.xg == nullptr) return;
    constexpr size_t U = (size_t)RW * (N / 2);
    const size_t region = (size_t)p.xg_cap * Geo<N>::PLANE_UNITS;
    c2<T> *xg = reinterpret_cast<c2<T> *>(p.xg);
    for (int e = 0; e < R; e++) {
      own[e] = xg + e * region + (size_t)blockIdx.x * U;
      first[e] = xg + e * region + (size_t)(blockIdx.x - rank) * U;
    }
  }
};

__device__ __forceinline__ void report_error(const KParams &p, int s_err) {
  if (s_err && p.err && threadIdx.x == 0) atomicExch(p.err, 1);
}

// --------------------------------------------------------------- plane phases
// The line-transform phases of the plane passes, shared by plane_fwd,
// plane_inv and the fused plane_inv_fwd. A CTA of a cluster owns RW z-rows
// (real space; 32, or 16 in the variant with four CTAs per SM) and CW = RW/2
// packed spectral columns of the current x-plane, with 8 RW threads; `buf` is
// its exchange area, which the other CTAs of the cluster read through
// distributed shared memory (or global areas, XG).
template <int N, class T, int RW = kRows> struct Plane {
  using G = Geo<N>;
  using T2 = c2<T>;
  static constexpr int M = G::M, N1 = G::N1, M1 = G::M1;
  static constexpr int CW = RW / 2;     // spectral columns per CTA
  static constexpr int TH = 8 * RW;     // threads per CTA
  static constexpr int CL = N / RW;     // CTAs per cluster = per x-plane
  static constexpr int UNITS = RW * M;  // exchange units per CTA (= CW columns x N)
  static constexpr int XS = 16 * CW;    // y-stage exchange stride per stage-1 output index
  // The z phases of a row stay inside one warp: warp w owns rows
  // RPW*w .. RPW*w + RPW - 1 in every z phase, and the z exchange of row r
  // lies inside row r's own M units, so those phases need only warp barriers.
  static constexpr int RPW = RW / (TH / 32);
  static_assert(RPW * 8 == 32, "8 threads per row in the row-parallel z stages");

  // z-exchange slot of stage-1 output (j2, k1) of row r, rotated by j2 so the
  // 8 threads of a row (and the 8 values a stage-2 task reads) fall in
  // distinct bank groups.
  __device__ static int zslot(int r, int j2, int k1) { return r * M + j2 * N1 + (k1 + j2) % N1; }

  // forward z, stage 1 of task (row r, j2): v = row elements j = j1*8 + j2
  // (after the prologue); radix-N1 DFT, twiddle, store into the z exchange.
  __device__ static void zf1_store(T2 *buf, const T2 *ztw, T2 (&v)[N1], int r, int j2) {
    Dft<-1, N1, T2>::run(v);
    sfor<0, N1>([&](auto K1) {
      constexpr int k1 = SPM_CI(K1);
      buf[zslot(r, j2, k1)] = (k1 == 0) ? v[k1] : cmul(v[k1], ztw[k1 * 8 + j2]);
    });
  }

  // forward z, stage 2 (8-point DFTs over j2 -> k = k1 + N1*k2) and the
  // real-to-complex post-processing of the packed lines (pairs q, M-q), each
  // warp on its own rows. Ends with a cluster barrier: the rows [r][M] are
  // then ready for remote reads, in buf or (XG) in the CTA's global exchange
  // area gx.
  template <bool XG = false, bool SYNC = true>
  __device__ static void zf2_post(T2 *buf, const T2 *tw, int tid, cg::cluster_group &cluster, T2 *gx = nullptr) {
    const int warp = tid >> 5, lane = tid & 31;
    {
      constexpr int NT = RPW * N1;  // tasks (r, k1) of this warp
      constexpr int TPT = (NT + 31) / 32;
      T2 u[TPT][8];
#pragma unroll
      for (int t = 0; t < TPT; t++) {
        const int q = lane + 32 * t;
        if (q < NT) {
          const int r = RPW * warp + q / N1, k1 = q % N1;
#pragma unroll
          for (int j2 = 0; j2 < 8; j2++) u[t][j2] = buf[zslot(r, j2, k1)];
        }
      }
      __syncwarp();
#pragma unroll
      for (int t = 0; t < TPT; t++) {
        const int q = lane + 32 * t;
        if (q < NT) {
          const int r = RPW * warp + q / N1, k1 = q % N1;
          Dft<-1, 8, T2>::run(u[t]);
#pragma unroll
          for (int k2 = 0; k2 < 8; k2++) buf[r * M + k1 + N1 * k2] = u[t][k2];
        }
      }
    }
    __syncwarp();
    {
      constexpr int NT = RPW * (M / 2);
      const uint64_t pol = XG ? l2_keep_policy() : 0;
      for (int task = lane; task < NT; task += 32) {
        const int r = RPW * warp + task / (M / 2), q = task % (M / 2);
        const T2 *Z = buf + r * M;
        T2 *O = (XG ? gx : buf) + r * M;
        auto put = [&](int i, T2 v) {
          if constexpr (XG) st_keep(O + i, v, pol);
          else O[i] = v;
        };
        if (q == 0) {
          const T2 z0 = Z[0];
          const T2 a = Z[M / 2];
          const T2 e = {a.x, (T)0};            // (a + conj a)/2
          const T2 o = {a.y, (T)0};            // (a - conj a)/(2i)
          put(0, T2{z0.x + z0.y, z0.x - z0.y});  // X_0 + i X_{N/2}
          put(M / 2, cadd(e, cmul(tw[M / 2], o)));
        } else {
          const T2 a = Z[q], c = Z[M - q];
          const T2 e1 = {(T)0.5 * (a.x + c.x), (T)0.5 * (a.y - c.y)};  // (Z_q + conj Z_{M-q})/2
          const T2 o1 = {(T)0.5 * (a.y + c.y), (T)0.5 * (c.x - a.x)};  // (Z_q - conj Z_{M-q})/(2i)
          const T2 e2 = {e1.x, -e1.y};
          const T2 o2 = {o1.x, -o1.y};
          put(q, cadd(e1, cmul(tw[q], o1)));
          put(M - q, cadd(e2, cmul(tw[M - q], o2)));
        }
      }
    }
    if constexpr (SYNC) cluster.sync();
  }

  // forward y over this CTA's 16 columns: gather element y = 16*j1 + j2 of
  // column c from the CTA holding row y, radix-M1 DFT, exchange, radix-16
  // DFT, store the spectral column into dst[plane][ky][M]. With XG the rows
  // come from the global exchange areas of the cluster's CTAs (gp = the area
  // of rank 0; rank k's at gp + k * UNITS), which stay untouched until
  // every CTA has passed the next plane's first cluster barrier, so no
  // "done reading" barrier is needed.
  template <bool XG = false>
  __device__ static void yf(T2 *buf, const T2 *tw, int tid, int rank, cg::cluster_group &cluster, T2 *dst,
                            int plane, const T2 *gp = nullptr) {
    {
      const int c = tid % CW, j2 = tid / CW;
      const int col = rank * CW + c;
      const uint64_t pol = XG ? l2_keep_policy() : 0;
      T2 v[M1];
      sfor<0, M1>([&](auto J1) {
        constexpr int j1 = SPM_CI(J1);
        const int y = 16 * j1 + j2;
        if constexpr (XG) {
          v[j1] = ld_keep(gp + (size_t)(y / RW) * UNITS + (y % RW) * M + col, pol);
        } else {
          const T2 *rem = cluster.map_shared_rank(buf, (unsigned)(y / RW));
          v[j1] = rem[(y % RW) * M + col];
        }
      });
      Dft<-1, M1, T2>::run(v);  // consumes every gathered value
      // done reading the other CTAs' rows: they may overwrite them after the
      // wait, which comes after the twiddles
      if constexpr (!XG) cluster_arrive_relaxed();
      sfor<1, M1>([&](auto K1) {
        constexpr int k1 = SPM_CI(K1);
        v[k1] = cmul(v[k1], tw[j2 * k1]);
      });
      if constexpr (!XG) cluster_wait();
      sfor<0, M1>([&](auto K1) {
        constexpr int k1 = SPM_CI(K1);
        buf[k1 * XS + j2 * CW + c] = v[k1];
      });
    }
    __syncthreads();
    if (tid < CW * M1) {
      const int c = tid % CW, k1 = tid / CW;
      const int col = rank * CW + c;
      const uint64_t spol = l2_stream_policy();
      T2 u[16];
#pragma unroll
      for (int j2 = 0; j2 < 16; j2++) u[j2] = buf[k1 * XS + j2 * CW + c];
      Dft<-1, 16, T2>::run(u);
#pragma unroll
      for (int k2 = 0; k2 < 16; k2++) {
        const int ky = k1 + M1 * k2;
        st_stream(dst + ((size_t)plane * N + ky) * M + col, u[k2], spol);
      }
    }
  }

  // Position of (y, column c) in the inverse-y output: stage 2 of task
  // (c, k1) writes its outputs y = k1 + M1*k2 back to the slots it read.
  __device__ static int ycol(int y, int c) { return (y % M1) * XS + (y / M1) * CW + c; }

  // inverse y over this CTA's 16 columns; ld(ky, c) returns the input value.
  // Leaves y-line values at ycol(y, c) in buf (or, XG, in the CTA's global
  // exchange area gx) and ends with a cluster barrier.
  template <bool XG = false, class LD, bool SYNC = true>
  __device__ static void yi(T2 *buf, const T2 *tw, int tid, cg::cluster_group &cluster, LD ld, T2 *gx = nullptr) {
    {
      const int c = tid % CW, j2 = tid / CW;
      T2 v[M1];
      sfor<0, M1>([&](auto J1) {
        constexpr int j1 = SPM_CI(J1);
        v[j1] = ld(16 * j1 + j2, c);
      });
      Dft<+1, M1, T2>::run(v);
      sfor<0, M1>([&](auto K1) {
        constexpr int k1 = SPM_CI(K1);
        buf[k1 * XS + j2 * CW + c] = (k1 == 0) ? v[k1] : cmulc(v[k1], tw[j2 * k1]);
      });
    }
    __syncthreads();
    if (tid < CW * M1) {
      T2 u[16];
      const int c = tid % CW, k1 = tid / CW;
#pragma unroll
      for (int j2 = 0; j2 < 16; j2++) u[j2] = buf[k1 * XS + j2 * CW + c];
      Dft<+1, 16, T2>::run(u);
#pragma unroll
      for (int k2 = 0; k2 < 16; k2++) {  // to ycol(k1 + M1*k2, c)
        if constexpr (XG) st_keep(gx + k1 * XS + k2 * CW + c, u[k2], l2_keep_policy());
        else buf[k1 * XS + k2 * CW + c] = u[k2];
      }
    }
    if constexpr (SYNC) cluster.sync();
  }

  // Complex-to-real pre-processing fused with stage 1 of the inverse z
  // transform. Thread (r, j2) (j2 = tid & 7, r = tid >> 3) transforms Z_q of
  // row r for q = 8 j1 + j2. Z_q and Z_{M-q} come from the same two gathered
  // values X_q, X_{M-q} (column owners, through distributed shared memory), and
  // M - q = 8 (N1-1-j1) + (8-j2), so lanes j2 and (8-j2) & 7 of a row each
  // build half of the pairs and swap the partner halves with shuffles (lane 0
  // pairs q = 0 with M/2; lanes 0 and 4 are their own partners). The "done
  // reading" arrive follows the last use of a gathered value and its wait
  // comes only before the stores into the row, so the radix-N1 DFT runs in
  // between. Ends with the z exchange of each row written (same warp). With
  // XG the columns come from the global exchange areas of the cluster's CTAs
  // (gp as in yf) and buf is free at once.
  template <bool XG = false>
  __device__ static void c2r_zi1(T2 *buf, const T2 *tw, const T2 *ztw, int tid, int rank,
                                 cg::cluster_group &cluster, const T2 *gp = nullptr) {
    constexpr int H = N1 / 2;
    static_assert(N1 % 2 == 0, "pairs");
    const int j2 = tid & 7, r = tid >> 3, lane = tid & 31;
    const int y = rank * RW + r;
    const uint64_t pol = XG ? l2_keep_policy() : 0;
    auto col = [&](int q) -> T2 {  // X_q of row y from its column owner
      if constexpr (XG) return ld_keep(gp + (size_t)(q / CW) * UNITS + ycol(y, q % CW), pol);
      else return cluster.map_shared_rank(buf, (unsigned)(q / CW))[ycol(y, q % CW)];
    };
    T2 v[N1], w[H];
#pragma unroll
    for (int j = 0; j < H; j++) {
      const int q = 8 * j + j2;
      if (q == 0) {
        const T2 P = col(0);
        const T2 a = col(M / 2);
        // Z_0 = (X0 + XM) + i (X0 - XM) from the packed value P = X0 + i XM
        v[0] = T2{P.x + P.y, P.x - P.y};
        // Z_{M/2} = (a + conj a) + i w^{-M/2} (a - conj a)
        const T2 e = {a.x + a.x, (T)0};
        const T2 o = {(T)0, a.y + a.y};
        w[0] = cadd(e, mul_di<+1>(cmulc(o, tw[M / 2])));
      } else {
        const T2 a = col(q);
        const T2 c = col(M - q);
        // Z_q = (X_q + conj X_{M-q}) + i w^{-q} (X_q - conj X_{M-q})
        const T2 e1 = {a.x + c.x, a.y - c.y}, d1 = {a.x - c.x, a.y + c.y};
        const T2 e2 = {c.x + a.x, c.y - a.y}, d2 = {c.x - a.x, c.y + a.y};
        v[j] = cadd(e1, mul_di<+1>(cmulc(d1, tw[q])));
        w[j] = cadd(e2, mul_di<+1>(cmulc(d2, tw[M - q])));
      }
    }
    // every gathered value is consumed: done reading the column owners
    if constexpr (!XG) cluster_arrive_relaxed();
    const int src = (lane & ~7) | ((8 - j2) & 7);
#pragma unroll
    for (int j = 0; j < H; j++) {
      // the partner's w[j] is Z at j1 = N1-1-j of this lane; lane 0 (its own
      // partner) holds Z_{M/2} in w[0], so it sends its pairs rotated by one
      const T2 snd = (j2 == 0) ? w[(j + 1) % H] : w[j];
      v[N1 - 1 - j] = T2{__shfl_sync(0xffffffffu, snd.x, src), __shfl_sync(0xffffffffu, snd.y, src)};
    }
    Dft<+1, N1, T2>::run(v);
    sfor<1, N1>([&](auto K1) {
      constexpr int k1 = SPM_CI(K1);
      v[k1] = cmulc(v[k1], ztw[k1 * 8 + j2]);
    });
    if constexpr (!XG) cluster_wait();  // the other CTAs are done reading this CTA's columns
    sfor<0, N1>([&](auto K1) {
      constexpr int k1 = SPM_CI(K1);
      buf[zslot(r, j2, k1)] = v[k1];
    });
    __syncwarp();
  }

  // inverse z, stage 2 of task (r, k1) of this warp's rows: 8-point DFTs;
  // sink(r, j, z_j) gets z_j = y_{2j} + i y_{2j+1}, j = k1 + N1*k2. With
  // TO_SMEM the sink may overwrite the warp's rows in buf: every task is read
  // first, then a warp barrier, then the sinks.
  template <bool TO_SMEM, class SINK> __device__ static void zi2(T2 *buf, int tid, SINK sink) {
    const int warp = tid >> 5, lane = tid & 31;
    constexpr int NT = RPW * N1;
    constexpr int TPT = (NT + 31) / 32;
    if constexpr (!TO_SMEM) {
#pragma unroll
      for (int t2 = 0; t2 < TPT; t2++) {
        const int q = lane + 32 * t2;
        if (q < NT) {
          const int r = RPW * warp + q / N1, k1 = q % N1;
          T2 u[8];
#pragma unroll
          for (int j2 = 0; j2 < 8; j2++) u[j2] = buf[zslot(r, j2, k1)];
          Dft<+1, 8, T2>::run(u);
#pragma unroll
          for (int k2 = 0; k2 < 8; k2++) sink(r, k1 + N1 * k2, u[k2]);
        }
      }
    } else {
      T2 u[TPT][8];
#pragma unroll
      for (int t2 = 0; t2 < TPT; t2++) {
        const int q = lane + 32 * t2;
        if (q < NT) {
          const int r = RPW * warp + q / N1, k1 = q % N1;
#pragma unroll
          for (int j2 = 0; j2 < 8; j2++) u[t2][j2] = buf[zslot(r, j2, k1)];
          Dft<+1, 8, T2>::run(u[t2]);
        }
      }
      __syncwarp();
#pragma unroll
      for (int t2 = 0; t2 < TPT; t2++) {
        const int q = lane + 32 * t2;
        if (q < NT) {
          const int r = RPW * warp + q / N1, k1 = q % N1;
#pragma unroll
          for (int k2 = 0; k2 < 8; k2++) sink(r, k1 + N1 * k2, u[t2][k2]);
        }
      }
    }
  }
};

// Loads the twiddles into shared memory: tw[j] = exp(-2 pi i j/N) and the
// z-stage table ztw[k1*8 + j2] = w^{2 j2 k1}.
template <int N, class T> __device__ __forceinline__ void plane_twiddles(const KParams &p, c2<T> *tw, c2<T> *ztw) {
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = reinterpret_cast<const c2<T> *>(p.tw)[i];
  __syncthreads();
  for (int i = threadIdx.x; i < N / 2; i += blockDim.x) ztw[i] = tw[(2 * (i & 7) * (i >> 3)) % N];
}

// --------------------------------------------------------------- plane_fwd
// Pro: static constexpr int NR; static constexpr unsigned MAXM;
//      __device__ static T2 pro(const KParams&, int b, size_t idx, T2 x, double (&acc)[NR]);
//        (x = reals idx, idx+1 of the input field; returns the values to transform)
//      __device__ static void fin(const KParams&, int b, const double (&tot)[NR]);
// CPS = CTAs per SM the variant is built for: 1 stages the next plane's rows
// in shared memory with a bulk copy; 2 has no stage (half the shared memory,
// so two CTAs share an SM) and loads its rows straight from global memory.
template <int N, class T, class Pro, int CPS, int XG = 0, int RW = kRows>
__global__ void __launch_bounds__(8 * RW, CPS) plane_fwd_kernel(const __grid_constant__ KParams p) {
  using G = Geo<N>;
  using T2 = c2<T>;
  using P = Plane<N, T, RW>;
  constexpr int N1 = G::N1;
  constexpr bool STAGED = (CPS == 1);
  static_assert(!STAGED || RW == kRows, "the staged variant has 32-row CTAs");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T2 *tw = reinterpret_cast<T2 *>(smem_base128(smem_raw));
  T2 *ztw = tw + N;                  // ztw[k1*8 + j2] = w^{2 j2 k1}
  T2 *buf = ztw + N / 2;
  T2 *stage = buf + P::UNITS;  // 32 rows of N reals
  uint64_t *bar = reinterpret_cast<uint64_t *>(stage + (STAGED ? G::STAGE_UNITS : 0));
  double *red = reinterpret_cast<double *>(bar + 2);
  __shared__ int s_err;
  grid_dep_sync();
  if (flow_stopped(p, blockIdx.y)) return;

  cg::cluster_group cluster = cg::this_cluster();
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int b = blockIdx.y;
  const int rank = (int)cluster.block_rank();
  const XgAreas<N, T, RW> xa(p, rank);
  const uint64_t spol = l2_stream_policy();  // streamed field data
  const int cid = blockIdx.x / P::CL, ncl = gridDim.x / P::CL;
  const T *src = reinterpret_cast<const T *>(p.in[b]);
  T2 *dst = reinterpret_cast<T2 *>(p.out[b]);
  auto issue = [&](int plane) {  // warp 0: one bulk copy per row of this CTA
    if (lane == 0) mbar_expect_tx(bar, (unsigned)(RW * N * sizeof(T)));
    __syncwarp();
    bulk_g2s(stage + lane * (N / 2), src + ((size_t)plane * N + rank * RW + lane) * N, N * sizeof(T), bar);
  };
  if (tid == 0) {
    mbar_init(bar, 1);
    s_err = 0;
    fence_barrier_init();
  }
  plane_twiddles<N, T>(p, tw, ztw);
  double acc[Pro::NR > 0 ? Pro::NR : 1];
#pragma unroll
  for (int r = 0; r < (Pro::NR > 0 ? Pro::NR : 1); r++) acc[r] = ((Pro::MAXM >> r) & 1u) ? -1.0e308 : 0.0;
  int plane = cid;
  if (STAGED && warp == 0 && plane < N) issue(plane);
  __syncthreads();

  for (int it = 0; plane < N; plane += ncl, it++) {
    const int next = plane + ncl;
    if (STAGED) mbar_wait(bar, it & 1, &s_err);
    // next plane's rows towards L2 while this one is transformed
    if (!STAGED && next < N && tid < RW)
      prefetch_l2(src + ((size_t)next * N + rank * RW + tid) * N, N * sizeof(T));
    {
      const int j2 = tid & 7, r = tid >> 3;
      const size_t rowoff = ((size_t)plane * N + (size_t)(rank * RW + r)) * N;
      const T2 *row = STAGED ? stage + r * (N / 2) : reinterpret_cast<const T2 *>(src + rowoff);
      T2 v[N1];
      auto prologue = [&](auto &a) {
        sfor<0, N1>([&](auto J1) {
          constexpr int j1 = SPM_CI(J1);
          const int j = j1 * 8 + j2;
          v[j1] = Pro::pro(p, b, rowoff + 2 * j, STAGED ? row[j] : ld_stream(row + j, spol), a);
        });
      };
      if constexpr (use_facc<T, Pro>()) {
        float fa[Pro::NR];
        facc_init<Pro::NR, Pro::MAXM>(fa);
        prologue(fa);
        facc_fold<Pro::NR, Pro::MAXM>(acc, fa);
      } else {
        prologue(acc);
      }
      P::zf1_store(buf, ztw, v, r, j2);
    }
    if (STAGED) __syncthreads();  // every row of the stage is read
    else __syncwarp();
    if (STAGED && warp == 0 && next < N) {
      fence_proxy_async();
      issue(next);
    }
    // one cluster barrier per plane here: the two areas alternate, so a CTA
    // rewrites an area only after every CTA has passed the barrier that
    // follows the last reads of it
    P::template zf2_post<(XG & kXgFwd) != 0>(buf, tw, tid, cluster, xa.own[it & 1]);
    P::template yf<(XG & kXgFwd) != 0>(buf, tw, tid, rank, cluster, dst, plane, xa.first[it & 1]);
    __syncthreads();
  }
  report_error(p, s_err);
  if constexpr (Pro::NR > 0) {
    double tot[Pro::NR];
    if (grid_reduce<Pro::NR, Pro::MAXM>(acc, red, p.partials + (size_t)b * kPartStride * kRedMax,
                                        p.tickets + b, gridDim.x, blockIdx.x, tot))
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
// Stages: [A (if FI)][S (if SI)], each 2 rows x N x 8 columns, [row][x][cc].
template <int N, class T, class Op, int TC = 8>
__global__ void __launch_bounds__(PencilGeo<N, TC>::TH,
                                  pencil_min_ctas<N, T, TC>((Op::FI ? 1 : 0) + (Op::SI ? 1 : 0), Op::SYM >= 0))
    pencil_kernel(const __grid_constant__ KParams p) {
  using G = Geo<N>;
  using PG = PencilGeo<N, TC>;
  using T2 = c2<T>;
  constexpr int M = G::M, M1 = G::M1;
  constexpr int NP = PG::NP, TH = PG::TH, XU = 16 * NP;  // pencils, threads, exchange stride
  constexpr int NST = (Op::FI ? 1 : 0) + (Op::SI ? 1 : 0);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T2 *tw = reinterpret_cast<T2 *>(smem_base128(smem_raw));
  T2 *ex = tw + N;
  T2 *sA = ex + PG::UNITS;
  T2 *sS = sA + (Op::FI ? PG::STAGE : 0);
  uint64_t *bars = reinterpret_cast<uint64_t *>(ex + PG::UNITS + NST * PG::STAGE);
  double *red = reinterpret_cast<double *>(bars + 2);
  double2 *stab = reinterpret_cast<double2 *>(red + 32 * kRedMax);  // symbol buffers (one or two tiles)
  __shared__ int s_err;
  grid_dep_sync();
  if (flow_stopped(p, blockIdx.y)) return;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int b = blockIdx.y;
  const int pen = tid % NP, rowsel = pen / TC, cc = pen % TC;
  const uint64_t spol = l2_stream_policy();  // outputs: evict first
  const bool has2 = (tid / NP) < M1;  // owns a stage-2 task (pencil, k1)
  const int k1 = tid / NP;
  // Tiles run columns-fastest, so concurrently resident CTAs read adjacent
  // TC-column segments of the same ky rows.
  constexpr int NCH = PG::NCH;
  // Symbols: a tile's points have |Ky| = t (rows t and N - t, t > 0), Kz in
  // its TC columns (or N/2 for the packed c = 0 column) and any Kx, so the
  // (TC + 1) x (N/2 + 1) entries it needs are staged in shared memory (the table
  // lookups of every point would otherwise wait on L2). The copies are
  // asynchronous, awaited just before the tile's point operator; with two
  // buffers they start at the top of the previous tile, with one once the
  // previous tile's point operator is done. Tiles with t = 0 (rows 0 and
  // N/2) read the table.
  constexpr bool USE_SYM = Op::SYM >= 0;
  constexpr int KXS = N / 2 + 1, SYMN = PG::SYMN;
  constexpr int SYMB = pencil_sym_bufs<N, T, TC>(NST, USE_SYM);
  auto sym_stage = [&](int tl, double2 *dst) {
    const int tt = tl / NCH, cz = (tl % NCH) * TC;
    const double2 *g = reinterpret_cast<const double2 *>(gtab_of(p, b)) + (USE_SYM ? Op::SYM : 0);
    for (int e = tid; e < SYMN; e += TH) {
      const int row = e / KXS, a = e - row * KXS;
      const int kz = row < TC ? cz + row : N / 2;
      cp_async16(dst + e, g + 2 * (a * a + tt * tt + kz * kz));
    }
  };
  // this tile's copies complete (with two buffers the next tile's may not)
  auto sym_wait = [&]() {
    if constexpr (SYMB == 2)
      cp_async_wait_all_but_last();
    else
      cp_async_wait_all();
  };
  // thread 0: two tensor boxes (TC columns x all x) for rows ky0, ky1 of a tile
  auto issue = [&](const CUtensorMap *map, T2 *dst, uint64_t *bar, int tile) {
    const int t = tile / NCH, c0 = (tile % NCH) * TC;
    const int ky0 = t, ky1 = (t == 0) ? N / 2 : N - t;
    mbar_expect_tx(bar, (unsigned)(2 * N * TC * sizeof(T2)));
    tma_load_3d(dst, map, 2 * c0, ky0, 0, bar);
    tma_load_3d(dst + N * TC, map, 2 * c0, ky1, 0, bar);
  };
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    s_err = 0;
    fence_barrier_init();
  }
  for (int i = tid; i < N; i += TH) tw[i] = reinterpret_cast<const T2 *>(p.tw)[i];
  double acc[Op::NR > 0 ? Op::NR : 1];
#pragma unroll
  for (int r = 0; r < (Op::NR > 0 ? Op::NR : 1); r++) acc[r] = ((Op::MAXM >> r) & 1u) ? -1.0e308 : 0.0;
  __syncthreads();
  int tile = blockIdx.x;
  if (tid == 0 && tile < PG::PTILES) {
    if (Op::FI) issue(&p.tmi[b], sA, &bars[0], tile);
    if (Op::SI) issue(&p.tms[b], sS, &bars[1], tile);
  }
  if constexpr (USE_SYM) {
    if (tile < PG::PTILES && tile / NCH != 0) sym_stage(tile, stab);
    if constexpr (SYMB == 2) cp_async_commit();
  }

  for (int it = 0; tile < PG::PTILES; tile += gridDim.x, it++) {
    const int next = tile + gridDim.x;
    const int t = tile / NCH;
    const int c0 = (tile % NCH) * TC;
    const int ky0 = t, ky1 = (t == 0) ? N / 2 : N - t;
    const int ky = rowsel ? ky1 : ky0;
    const int col = c0 + cc;
    const bool dc = (c0 == 0);
    double2 *const sym_cur = stab + (SYMB == 2 ? (it & 1) * SYMN : 0);
    if constexpr (SYMB == 2) {
      // the other buffer's tile (two back) finished its point operator
      if (next < PG::PTILES && next / NCH != 0) sym_stage(next, stab + ((it + 1) & 1) * SYMN);
      cp_async_commit();
    }
    if constexpr (USE_SYM && !Op::FI) {
      sym_wait();
      __syncthreads();
    }
    // symbols of (Kx, Ky, Kz) for kz row `row` of the tile (TC: kz = N/2)
    auto sym_at = [&](int Kx, int Ky, int Kz, int row) -> double2 {
      if constexpr (!USE_SYM) {
        return double2{0.0, 0.0};
      } else {
        if (t != 0) return sym_cur[row * KXS + (Kx < 0 ? -Kx : Kx)];
        return symbols_half(p, Kx * Kx + Ky * Ky + Kz * Kz, Op::SYM, b);
      }
    };

    T2 F[16];
    if constexpr (Op::FI) {
      mbar_wait(&bars[0], it & 1, &s_err);
      {  // stage 1: task (pencil, j2 = tid/NP): x = 16*j1 + j2
        const int j2 = tid / NP;
        T2 v[M1];
        sfor<0, M1>([&](auto J1) {
          constexpr int j1 = SPM_CI(J1);
          v[j1] = sA[(rowsel * N + 16 * j1 + j2) * TC + cc];
        });
        Dft<-1, M1, T2>::run(v);
        sfor<0, M1>([&](auto K1) {
          constexpr int kk = SPM_CI(K1);
          ex[kk * XU + j2 * NP + pen] = (kk == 0) ? v[kk] : cmul(v[kk], tw[j2 * kk]);
        });
      }
      if constexpr (USE_SYM) sym_wait();  // this tile's symbols, seen after the barrier
      __syncthreads();
      if (tid == 0 && next < PG::PTILES) {
        fence_proxy_async();
        issue(&p.tmi[b], sA, &bars[0], next);
      }
      if (has2) {
#pragma unroll
        for (int j2 = 0; j2 < 16; j2++) F[j2] = ex[k1 * XU + j2 * NP + pen];
        Dft<-1, 16, T2>::run(F);  // F[k2] at kx = k1 + M1*k2
      }
    }
    if constexpr (Op::SI) mbar_wait(&bars[1], it & 1, &s_err);
    // partner values at (-kx, -ky) for the packed c = 0 pencils, through ex
    if constexpr (!Op::LIN) {
      if (dc) {
        __syncthreads();
        T2 *D = ex;  // [quantity][rowsel][kx]
        if (has2 && cc == 0) {
#pragma unroll
          for (int k2 = 0; k2 < 16; k2++) {
            const int kx = k1 + M1 * k2;
            if constexpr (Op::FI) D[(0 * 2 + rowsel) * N + kx] = F[k2];
            if constexpr (Op::SI) D[(1 * 2 + rowsel) * N + kx] = sS[(rowsel * N + kx) * TC];
          }
        }
        __syncthreads();
      }
    }
    // the per-point operator
    auto point_ops = [&](auto &acc) {
      T2 *so = Op::SO ? reinterpret_cast<T2 *>(p.sto[b]) : nullptr;
      const int Ky = wave(ky, N);
      const int pr = (t == 0) ? rowsel : 1 - rowsel;
#pragma unroll
      for (int k2 = 0; k2 < 16; k2++) {
        const int kx = k1 + M1 * k2;
        const int Kx = wave(kx, N);
        const T2 f = Op::FI ? F[k2] : T2{0, 0};
        const T2 s = Op::SI ? sS[(rowsel * N + kx) * TC + cc] : T2{0, 0};
        T2 o_st = {0, 0}, o_inv = {0, 0};
        if (!Op::LIN && dc && cc == 0) {
          // unpack X(., ., 0) and X(., ., N/2), apply, repack
          const int nk = kx ? N - kx : 0;
          T2 f0 = {0, 0}, fM = {0, 0}, s0 = {0, 0}, sM = {0, 0};
          if constexpr (Op::FI) {
            const T2 q = ex[(0 * 2 + pr) * N + nk];
            f0 = T2{(T)0.5 * (f.x + q.x), (T)0.5 * (f.y - q.y)};
            fM = T2{(T)0.5 * (f.y + q.y), (T)0.5 * (q.x - f.x)};
          }
          if constexpr (Op::SI) {
            const T2 q = ex[(1 * 2 + pr) * N + nk];
            s0 = T2{(T)0.5 * (s.x + q.x), (T)0.5 * (s.y - q.y)};
            sM = T2{(T)0.5 * (s.y + q.y), (T)0.5 * (q.x - s.x)};
          }
          T2 so0, inv0, soM, invM;
          Op::point(p, b, Kx, Ky, 0, sym_at(Kx, Ky, 0, 0), f0, s0, so0, inv0, acc, 1.0);
          Op::point(p, b, Kx, Ky, -N / 2, sym_at(Kx, Ky, N / 2, TC), fM, sM, soM, invM, acc, 1.0);
          o_st = T2{so0.x - soM.y, so0.y + soM.x};
          o_inv = T2{inv0.x - invM.y, inv0.y + invM.x};
        } else {
          Op::point(p, b, Kx, Ky, col, sym_at(Kx, Ky, col, cc), f, s, o_st, o_inv, acc, dc && cc == 0 ? 1.0 : 2.0);
        }
        if constexpr (Op::SO) st_stream(so + ((size_t)kx * N + ky) * M + col, o_st, spol);
        F[k2] = o_inv;
      }
    };
    if (has2) {
      if constexpr (use_facc<T, Op>()) {
        float fa[Op::NR];
        facc_init<Op::NR, Op::MAXM>(fa);
        point_ops(fa);
        facc_fold<Op::NR, Op::MAXM>(acc, fa);
      } else {
        point_ops(acc);
      }
    }
    __syncthreads();  // sS, stab and ex reads done
    if constexpr (Op::SI) {
      if (tid == 0 && next < PG::PTILES) {
        fence_proxy_async();
        issue(&p.tms[b], sS, &bars[1], next);
      }
    }
    if constexpr (SYMB == 1)
      if (next < PG::PTILES && next / NCH != 0) sym_stage(next, stab);
    if constexpr (Op::INV) {
      if (has2) {
        Dft<+1, 16, T2>::run(F);  // over k2 -> j2
#pragma unroll
        for (int j2 = 0; j2 < 16; j2++)
          ex[k1 * XU + j2 * NP + pen] = (j2 == 0 || k1 == 0) ? F[j2] : cmulc(F[j2], tw[j2 * k1]);
      }
      __syncthreads();
      {
        const int j2 = tid / NP;
        T2 v[M1];
        sfor<0, M1>([&](auto K1) { v[SPM_CI(K1)] = ex[SPM_CI(K1) * XU + j2 * NP + pen]; });
        Dft<+1, M1, T2>::run(v);
        T2 *dst = reinterpret_cast<T2 *>(p.out[b]);
        sfor<0, M1>([&](auto J1) {
          constexpr int j1 = SPM_CI(J1);
          const int x = 16 * j1 + j2;
          st_stream(dst + ((size_t)x * N + ky) * M + col, v[j1], spol);
        });
      }
      __syncthreads();
    }
  }
  report_error(p, s_err);
  if constexpr (Op::NR > 0) {
    double tot[Op::NR];
    if (grid_reduce<Op::NR, Op::MAXM>(acc, red, p.partials + (size_t)b * kPartStride * kRedMax,
                                      p.tickets + b, gridDim.x, blockIdx.x, tot))
      Op::fin(p, b, tot);
  }
}

// --------------------------------------------------------------- plane_inv
// Epi: static constexpr int NR; static constexpr unsigned MAXM;
//      __device__ static T2 epi(const KParams&, int b, size_t idx, T2 y, double (&acc)[NR]);
//        (y = unnormalised inverse transform at reals idx, idx+1; returns values to store)
//      __device__ static void fin(const KParams&, int b, const double (&tot)[NR]);
// CPS as for plane_fwd: 1 stages the next plane's columns with a tensor copy,
// 2 loads them straight from global memory (two CTAs per SM).
template <int N, class T, class Epi, int CPS, int XG = 0, int RW = kRows>
__global__ void __launch_bounds__(8 * RW, CPS) plane_inv_kernel(const __grid_constant__ KParams p) {
  using G = Geo<N>;
  using T2 = c2<T>;
  using P = Plane<N, T, RW>;
  constexpr int M = G::M;
  constexpr bool STAGED = (CPS == 1);
  static_assert(!STAGED || RW == kRows, "the staged variant has 32-row CTAs");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T2 *tw = reinterpret_cast<T2 *>(smem_base128(smem_raw));
  T2 *ztw = tw + N;
  T2 *buf = ztw + N / 2;
  T2 *stage = buf + P::UNITS;  // [ky][16 columns]
  uint64_t *bar = reinterpret_cast<uint64_t *>(stage + (STAGED ? G::STAGE_UNITS : 0));
  double *red = reinterpret_cast<double *>(bar + 2);
  __shared__ int s_err;
  grid_dep_sync();
  if (flow_stopped(p, blockIdx.y)) return;

  cg::cluster_group cluster = cg::this_cluster();
  const int tid = threadIdx.x;
  const int b = blockIdx.y;
  const int rank = (int)cluster.block_rank();
  const XgAreas<N, T, RW> xa(p, rank);
  const uint64_t spol = l2_stream_policy();  // streamed field data
  const int cid = blockIdx.x / P::CL, ncl = gridDim.x / P::CL;
  auto issue = [&](int plane) {  // thread 0: one tensor box (this CTA's 16 columns x all ky)
    mbar_expect_tx(bar, (unsigned)(N * 16 * sizeof(T2)));
    tma_load_3d(stage, &p.tmi[b], 2 * rank * P::CW, 0, plane, bar);
  };
  if (tid == 0) {
    mbar_init(bar, 1);
    s_err = 0;
    fence_barrier_init();
  }
  plane_twiddles<N, T>(p, tw, ztw);
  double acc[Epi::NR > 0 ? Epi::NR : 1];
#pragma unroll
  for (int r = 0; r < (Epi::NR > 0 ? Epi::NR : 1); r++) acc[r] = ((Epi::MAXM >> r) & 1u) ? -1.0e308 : 0.0;
  int plane = cid;
  if (STAGED && tid == 0 && plane < N) issue(plane);
  __syncthreads();
  const T2 *gsrc = reinterpret_cast<const T2 *>(p.in[b]);
  T *outb = reinterpret_cast<T *>(p.out[b]);  // null: reductions only

  for (int it = 0; plane < N; plane += ncl, it++) {
    const int next = plane + ncl;
    if (STAGED) mbar_wait(bar, it & 1, &s_err);
    // next plane's columns towards L2 while this one is transformed
    if (!STAGED && next < N)
      for (int i = tid; i < N; i += P::TH)
        prefetch_l2(gsrc + ((size_t)next * N + i) * M + rank * P::CW, P::CW * sizeof(T2));
    P::template yi<(XG & kXgInv) != 0>(
        buf, tw, tid, cluster,
        [&](int ky, int c) -> T2 {
          return STAGED ? stage[ky * 16 + c]
                        : ld_stream(gsrc + ((size_t)plane * N + ky) * M + rank * P::CW + c, spol);
        },
        xa.own[it & 1]);  // alternating areas, as in plane_fwd
    if (STAGED && tid == 0 && next < N) {
      fence_proxy_async();
      issue(next);
    }
    P::template c2r_zi1<(XG & kXgInv) != 0>(buf, tw, ztw, tid, rank, cluster, xa.first[it & 1]);
    auto epilogue = [&](auto &a) {
      P::template zi2<false>(buf, tid, [&](int r, int j, T2 z) {
        const size_t rowoff = ((size_t)plane * N + (size_t)(rank * RW + r)) * N;
        const T2 val = Epi::epi(p, b, rowoff + 2 * j, z, a);
        if (outb) reinterpret_cast<T2 *>(outb + rowoff)[j] = val;
      });
    };
    if constexpr (use_facc<T, Epi>()) {
      float fa[Epi::NR];
      facc_init<Epi::NR, Epi::MAXM>(fa);
      epilogue(fa);
      facc_fold<Epi::NR, Epi::MAXM>(acc, fa);
    } else {
      epilogue(acc);
    }
    __syncthreads();
  }
  report_error(p, s_err);
  if constexpr (Epi::NR > 0) {
    double tot[Epi::NR];
    if (grid_reduce<Epi::NR, Epi::MAXM>(acc, red, p.partials + (size_t)b * kPartStride * kRedMax,
                                        p.tickets + b, gridDim.x, blockIdx.x, tot))
      Epi::fin(p, b, tot);
  }
}

// --------------------------------------------------------------- plane_inv_fwd
// One x-plane pass that joins a step's inverse plane transform with the next
// step's forward one: B (p.in, the spectrum of the pencil pass) -> inverse y,
// C2R z -> epilogue -> phi rows kept in shared memory -> prologue -> R2C z,
// y -> A (p.out). phi itself goes to memory (p.sto) only on the step where the
// flow stops (the pencil pass armed FW_PENDING): the forward half is then
// skipped. A chain of K steps is plane_fwd, K pencils, K-1 of these and one
// plane_inv, so the real field crosses HBM once per chain instead of twice per
// step. Direct loads; CPS (2, 3 or 4) CTAs per SM, the layout of plane_fwd's
// direct variant.
template <int N, class T, class Epi, class Pro, int CPS, int XG = 0, int RW = kRows>
__global__ void __launch_bounds__(8 * RW, CPS) plane_inv_fwd_kernel(const __grid_constant__ KParams p) {
  using G = Geo<N>;
  using T2 = c2<T>;
  using P = Plane<N, T, RW>;
  constexpr int M = G::M, N1 = G::N1;
  constexpr int NE = Epi::NR, NP = Pro::NR, NA = (NE + NP > 0) ? NE + NP : 1;
  static_assert(NA <= kRedMax, "reduction count");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T2 *tw = reinterpret_cast<T2 *>(smem_base128(smem_raw));
  T2 *ztw = tw + N;
  T2 *buf = ztw + N / 2;
  uint64_t *bar = reinterpret_cast<uint64_t *>(buf + P::UNITS);
  double *red = reinterpret_cast<double *>(bar + 2);
  grid_dep_sync();
  if (flow_stopped(p, blockIdx.y)) return;
  // uniform over the grid: set by the pencil pass of this step, before launch
  const bool stop = flow_pending(p, blockIdx.y);

  cg::cluster_group cluster = cg::this_cluster();
  const int tid = threadIdx.x;
  const int b = blockIdx.y;
  const int rank = (int)cluster.block_rank();
  const XgAreas<N, T, RW> xa(p, rank);
  const uint64_t spol = l2_stream_policy();  // streamed field data
  const int cid = blockIdx.x / P::CL, ncl = gridDim.x / P::CL;
  plane_twiddles<N, T>(p, tw, ztw);
  double acc_e[NE > 0 ? NE : 1], acc_p[NP > 0 ? NP : 1];
#pragma unroll
  for (int r = 0; r < (NE > 0 ? NE : 1); r++) acc_e[r] = ((Epi::MAXM >> r) & 1u) ? -1.0e308 : 0.0;
#pragma unroll
  for (int r = 0; r < (NP > 0 ? NP : 1); r++) acc_p[r] = ((Pro::MAXM >> r) & 1u) ? -1.0e308 : 0.0;
  __syncthreads();
  const T2 *gsrc = reinterpret_cast<const T2 *>(p.in[b]);
  T2 *dst = reinterpret_cast<T2 *>(p.out[b]);
  T *phi = reinterpret_cast<T *>(p.sto[b]);

  for (int plane = cid; plane < N; plane += ncl) {
    // next plane's columns towards L2 while this one is transformed
    if (plane + ncl < N)
      for (int i = tid; i < N; i += P::TH)
        prefetch_l2(gsrc + ((size_t)(plane + ncl) * N + i) * M + rank * P::CW, P::CW * sizeof(T2));
    P::template yi<(XG & kXgInv) != 0>(
        buf, tw, tid, cluster,
        [&](int ky, int c) -> T2 { return ld_stream(gsrc + ((size_t)plane * N + ky) * M + rank * P::CW + c, spol); },
        xa.own[0]);
    P::template c2r_zi1<(XG & kXgInv) != 0>(buf, tw, ztw, tid, rank, cluster, xa.first[0]);
    if (stop) {
      P::template zi2<false>(buf, tid, [&](int r, int j, T2 z) {
        const size_t rowoff = ((size_t)plane * N + (size_t)(rank * RW + r)) * N;
        reinterpret_cast<T2 *>(phi + rowoff)[j] = Epi::epi(p, b, rowoff + 2 * j, z, acc_e);
      });
      // no forward exchange on this path: its barrier keeps the inverse areas
      // of this plane from being rewritten while a peer still reads them
      if constexpr ((XG & kXgInv) != 0) cluster.sync();
    } else {
      // phi rows [r][M] in buf (each warp writes and then reads its own rows)
      P::template zi2<true>(buf, tid, [&](int r, int j, T2 z) {
        const size_t rowoff = ((size_t)plane * N + (size_t)(rank * RW + r)) * N;
        buf[r * M + j] = Epi::epi(p, b, rowoff + 2 * j, z, acc_e);
      });
      __syncwarp();
      {
        const int j2 = tid & 7, r = tid >> 3;
        const size_t rowoff = ((size_t)plane * N + (size_t)(rank * RW + r)) * N;
        T2 v[N1];
        auto prologue = [&](auto &a) {
          sfor<0, N1>([&](auto J1) {
            constexpr int j1 = SPM_CI(J1);
            const int j = j1 * 8 + j2;
            v[j1] = Pro::pro(p, b, rowoff + 2 * j, buf[r * M + j], a);
          });
        };
        if constexpr (use_facc<T, Pro>()) {
          float fa[Pro::NR];
          facc_init<Pro::NR, Pro::MAXM>(fa);
          prologue(fa);
          facc_fold<Pro::NR, Pro::MAXM>(acc_p, fa);
        } else {
          prologue(acc_p);
        }
        __syncwarp();  // the warp's rows are read before its z exchange overwrites them
        P::zf1_store(buf, ztw, v, r, j2);
      }
      __syncwarp();
      P::template zf2_post<(XG & kXgFwd) != 0>(buf, tw, tid, cluster, xa.own[1]);
      P::template yf<(XG & kXgFwd) != 0>(buf, tw, tid, rank, cluster, dst, plane, xa.first[1]);
    }
    __syncthreads();
  }
  double all[NA], tot[NA];
#pragma unroll
  for (int r = 0; r < NE; r++) all[r] = acc_e[r];
#pragma unroll
  for (int r = 0; r < NP; r++) all[NE + r] = acc_p[r];
  if constexpr (NE + NP == 0) all[0] = 0.0;
  if (grid_reduce<NA, (Epi::MAXM | (Pro::MAXM << NE))>(all, red, p.partials + (size_t)b * kPartStride * kRedMax,
                                                        p.tickets + b, gridDim.x, blockIdx.x, tot)) {
    double te[NE > 0 ? NE : 1], tp[NP > 0 ? NP : 1];
#pragma unroll
    for (int r = 0; r < NE; r++) te[r] = tot[r];
#pragma unroll
    for (int r = 0; r < NP; r++) tp[r] = tot[NE + r];
    Epi::fin(p, b, te);
    if (!stop) Pro::fin(p, b, tp);
  }
}


// --------------------------------------------------------------- plane_inv_fwd, pipelined
// plane_inv_fwd with both exchanges through the L2 areas, software-pipelined
// over the cluster's x-planes. A plane is three phases:
//   A(p): inverse y of this CTA's columns (loads B), into its inverse area;
//   Z(p): C2R z from every CTA's inverse area, epilogue, prologue, R2C z,
//         into its forward area;
//   Y(p): forward y from every CTA's forward area, stores A.
// Each exchange needs a cluster barrier between the writes of one phase and
// the reads of the next. Here the barrier is split into its arrive (release)
// and its wait (acquire), with independent work of a neighbouring plane in
// between, so the CTA computes while the slowest CTA of its cluster catches up:
//   step i = 0 .. n: A(p_i), Y(p_i-1), Z(p_i) (the phases that exist)
// with the forward barrier of p_i-1 spanning A(p_i) and the inverse barrier of
// p_i spanning Y(p_i-1). Planes alternate between two inverse and two forward
// areas (regions 0/2 and 1/3): an area is rewritten two planes later, after a
// barrier every reader passed after its last read. The arithmetic is that of
// plane_inv_fwd, so results are identical. The stopping step (FW_PENDING)
// runs the inverse half only, as plane_inv_fwd does.
template <int N, class T, class Epi, class Pro, int CPS, int RW>
__global__ void __launch_bounds__(8 * RW, CPS) plane_inv_fwd_pipe_kernel(const __grid_constant__ KParams p) {
  using G = Geo<N>;
  using T2 = c2<T>;
  using P = Plane<N, T, RW>;
  constexpr int M = G::M, N1 = G::N1;
  constexpr int NE = Epi::NR, NP = Pro::NR, NA = (NE + NP > 0) ? NE + NP : 1;
  static_assert(NA <= kRedMax, "reduction count");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T2 *tw = reinterpret_cast<T2 *>(smem_base128(smem_raw));
  T2 *ztw = tw + N;
  T2 *buf = ztw + N / 2;
  uint64_t *bar = reinterpret_cast<uint64_t *>(buf + P::UNITS);
  double *red = reinterpret_cast<double *>(bar + 2);
  grid_dep_sync();
  if (flow_stopped(p, blockIdx.y)) return;
  const bool stop = flow_pending(p, blockIdx.y);

  cg::cluster_group cluster = cg::this_cluster();
  const int tid = threadIdx.x;
  const int b = blockIdx.y;
  const int rank = (int)cluster.block_rank();
  const XgAreas<N, T, RW, 4> xa(p, rank);
  const uint64_t spol = l2_stream_policy();
  const int cid = blockIdx.x / P::CL, ncl = gridDim.x / P::CL;
  plane_twiddles<N, T>(p, tw, ztw);
  double acc_e[NE > 0 ? NE : 1], acc_p[NP > 0 ? NP : 1];
#pragma unroll
  for (int r = 0; r < (NE > 0 ? NE : 1); r++) acc_e[r] = ((Epi::MAXM >> r) & 1u) ? -1.0e308 : 0.0;
#pragma unroll
  for (int r = 0; r < (NP > 0 ? NP : 1); r++) acc_p[r] = ((Pro::MAXM >> r) & 1u) ? -1.0e308 : 0.0;
  __syncthreads();
  const T2 *gsrc = reinterpret_cast<const T2 *>(p.in[b]);
  T2 *dst = reinterpret_cast<T2 *>(p.out[b]);
  T *phi = reinterpret_cast<T *>(p.sto[b]);

  // A(plane) into inverse area `slot` (no barrier)
  auto phase_a = [&](int plane, int slot) {
    if (plane + ncl < N)
      for (int i = tid; i < N; i += P::TH)
        prefetch_l2(gsrc + ((size_t)(plane + ncl) * N + i) * M + rank * P::CW, P::CW * sizeof(T2));
    auto ld = [&](int ky, int c) -> T2 {
      return ld_stream(gsrc + ((size_t)plane * N + ky) * M + rank * P::CW + c, spol);
    };
    P::template yi<true, decltype(ld), false>(buf, tw, tid, cluster, ld, slot ? xa.own[2] : xa.own[0]);
  };
  // Z(plane) from the inverse areas `slot` into forward area `slot` (no barrier)
  auto phase_z = [&](int plane, int slot) {
    P::template c2r_zi1<true>(buf, tw, ztw, tid, rank, cluster, slot ? xa.first[2] : xa.first[0]);
    P::template zi2<true>(buf, tid, [&](int r, int j, T2 z) {
      const size_t rowoff = ((size_t)plane * N + (size_t)(rank * RW + r)) * N;
      buf[r * M + j] = Epi::epi(p, b, rowoff + 2 * j, z, acc_e);
    });
    __syncwarp();
    {
      const int j2 = tid & 7, r = tid >> 3;
      const size_t rowoff = ((size_t)plane * N + (size_t)(rank * RW + r)) * N;
      T2 v[N1];
      auto prologue = [&](auto &a) {
        sfor<0, N1>([&](auto J1) {
          constexpr int j1 = SPM_CI(J1);
          const int j = j1 * 8 + j2;
          v[j1] = Pro::pro(p, b, rowoff + 2 * j, buf[r * M + j], a);
        });
      };
      if constexpr (use_facc<T, Pro>()) {
        float fa[Pro::NR];
        facc_init<Pro::NR, Pro::MAXM>(fa);
        prologue(fa);
        facc_fold<Pro::NR, Pro::MAXM>(acc_p, fa);
      } else {
        prologue(acc_p);
      }
      __syncwarp();
      P::zf1_store(buf, ztw, v, r, j2);
    }
    __syncwarp();
    P::template zf2_post<true, false>(buf, tw, tid, cluster, slot ? xa.own[3] : xa.own[1]);
  };
  // Y(plane) from the forward areas `slot`, stores A
  auto phase_y = [&](int plane, int slot) {
    P::template yf<true>(buf, tw, tid, rank, cluster, dst, plane, slot ? xa.first[3] : xa.first[1]);
  };

  if (stop) {
    for (int plane = cid; plane < N; plane += ncl) {
      P::template yi<true>(
          buf, tw, tid, cluster,
          [&](int ky, int c) -> T2 { return ld_stream(gsrc + ((size_t)plane * N + ky) * M + rank * P::CW + c, spol); },
          xa.own[0]);
      P::template c2r_zi1<true>(buf, tw, ztw, tid, rank, cluster, xa.first[0]);
      P::template zi2<false>(buf, tid, [&](int r, int j, T2 z) {
        const size_t rowoff = ((size_t)plane * N + (size_t)(rank * RW + r)) * N;
        reinterpret_cast<T2 *>(phi + rowoff)[j] = Epi::epi(p, b, rowoff + 2 * j, z, acc_e);
      });
      // keeps the inverse areas of this plane from being rewritten while a peer still reads them
      cluster.sync();
    }
  } else {
    // planes cid + i * ncl, i < n (the same n on every CTA of the cluster);
    // step i runs A(p_i), Y(p_i-1), Z(p_i), each phase written once
    const int n = cid < N ? (N - cid + ncl - 1) / ncl : 0;
    for (int i = 0; i <= n; i++) {
      const int plane = cid + i * ncl;
      if (i < n) {
        __syncthreads();
        phase_a(plane, i & 1);
      }
      if (i > 0) cluster_wait();    // forward areas of p_i-1 complete
      if (i < n) cluster_arrive();  // inverse areas of p_i written
      if (i > 0) {
        __syncthreads();
        phase_y(plane - ncl, (i - 1) & 1);
      }
      if (i < n) {
        cluster_wait();  // inverse areas of p_i complete
        __syncthreads();
        phase_z(plane, i & 1);
        cluster_arrive();  // forward areas of p_i written
      }
    }
  }
  __syncthreads();
  double all[NA], tot[NA];
#pragma unroll
  for (int r = 0; r < NE; r++) all[r] = acc_e[r];
#pragma unroll
  for (int r = 0; r < NP; r++) all[NE + r] = acc_p[r];
  if constexpr (NE + NP == 0) all[0] = 0.0;
  if (grid_reduce<NA, (Epi::MAXM | (Pro::MAXM << NE))>(all, red, p.partials + (size_t)b * kPartStride * kRedMax,
                                                        p.tickets + b, gridDim.x, blockIdx.x, tot)) {
    double te[NE > 0 ? NE : 1], tp[NP > 0 ? NP : 1];
#pragma unroll
    for (int r = 0; r < NE; r++) te[r] = tot[r];
#pragma unroll
    for (int r = 0; r < NP; r++) tp[r] = tot[NE + r];
    Epi::fin(p, b, te);
    if (!stop) Pro::fin(p, b, tp);
  }
}

}  // namespace spm
