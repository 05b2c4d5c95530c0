// Runtime behind the oracle's shim headers (fftw3-mpi.h, mpi.h, eigen3/Eigen/Dense).
// TEST INFRASTRUCTURE ONLY: linked with the reference's own src/*.cpp so they run
// unchanged as the CPU oracle. Nothing in the product links this file.
//
//  * FFT: FFTW's published DFT definition (unnormalised, sign -1 forward / +1
//    backward, row-major 3D, in place). Mixed-radix recursive Cooley-Tukey with
//    radix-4/2 butterflies and a generic radix for 3/5/other primes. Twiddles
//    exp(sign*2*pi*i*j/n) are evaluated per index in long double (no
//    recurrence), then rounded to double. Lines along the two strided axes are
//    gathered in blocks; lines are distributed over std::threads when
//    spm_shim_fft_set_threads(n>1) is called.
//  * MPI: one rank; collectives copy send to receive buffers.
//  * Eigen's MatrixXd::Random: SplitMix64 stream, uniform in [-1,1).
#include "fftw3-mpi.h"
#include "mpi.h"

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <sys/time.h>
#include <thread>
#include <vector>

typedef std::complex<double> cd;

namespace {

int g_threads = 1;

struct Line {
  int n = 0;
  int sign = -1;
  std::vector<int> fac;  // radices, product n
  std::vector<cd> tw;    // tw[j] = exp(sign*2*pi*i*j/n)
};

void make_line(Line &l, int n, int sign) {
  l.n = n;
  l.sign = sign;
  l.fac.clear();
  int m = n;
  while (m % 4 == 0) { l.fac.push_back(4); m /= 4; }
  while (m % 2 == 0) { l.fac.push_back(2); m /= 2; }
  for (int p = 3; m > 1; p += 2)
    while (m % p == 0) { l.fac.push_back(p); m /= p; }
  l.tw.resize(n);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int j = 0; j < n; j++) {
    long double a = 2.0L * pi * (long double)j / (long double)n;
    l.tw[j] = cd((double)cosl(a), (double)(sign * sinl(a)));
  }
}

// out[0..n) = DFT_n(in[0], in[s], ..., in[(n-1)s]); tw is the table of the
// top-level length N; w_n^e = tw[e * (N/n)].
void fft_rec(const cd *in, long s, cd *out, int n, const int *fac, const Line &L, int tstride) {
  if (n == 1) { out[0] = in[0]; return; }
  const int p = fac[0];
  const int m = n / p;
  for (int q = 0; q < p; q++) fft_rec(in + q * s, s * p, out + (long)q * m, m, fac + 1, L, tstride * p);
  const int N = L.n;
  if (p == 2) {
    for (int k = 0; k < m; k++) {
      cd a = out[k], b = out[m + k] * L.tw[(long)k * tstride % N];
      out[k] = a + b;
      out[m + k] = a - b;
    }
  } else if (p == 4) {
    const cd jj(0.0, (double)L.sign);  // w_4 = exp(sign*i*pi/2)
    for (int k = 0; k < m; k++) {
      cd a0 = out[k];
      cd a1 = out[m + k] * L.tw[(long)k * tstride % N];
      cd a2 = out[2 * m + k] * L.tw[(long)2 * k * tstride % N];
      cd a3 = out[3 * m + k] * L.tw[(long)3 * k * tstride % N];
      cd t0 = a0 + a2, t1 = a0 - a2, t2 = a1 + a3, t3 = (a1 - a3) * jj;
      out[k] = t0 + t2;
      out[m + k] = t1 + t3;
      out[2 * m + k] = t0 - t2;
      out[3 * m + k] = t1 - t3;
    }
  } else {
    std::vector<cd> t(p);
    const long tp = N / p;  // w_p^e = tw[e * N/p]
    for (int k = 0; k < m; k++) {
      for (int q = 0; q < p; q++) t[q] = out[(long)q * m + k] * L.tw[(long)q * k * tstride % N];
      for (int r = 0; r < p; r++) {
        cd acc = 0.0;
        for (int q = 0; q < p; q++) acc += t[q] * L.tw[((long)q * r % p) * tp];
        out[(long)r * m + k] = acc;
      }
    }
  }
}

void line_fft(const Line &L, cd *x, cd *tmp) {
  fft_rec(x, 1, tmp, L.n, L.fac.data(), L, 1);
  std::memcpy(x, tmp, sizeof(cd) * L.n);
}

// Runs body(lo, hi) over [0, n) split into g_threads contiguous ranges.
template <typename F>
void par_for(long n, F body) {
  int t = g_threads;
  if (t <= 1 || n < 2 * t) { body(0L, n); return; }
  std::vector<std::thread> th;
  for (int i = 0; i < t; i++) {
    long lo = n * i / t, hi = n * (i + 1) / t;
    th.emplace_back([=]() { body(lo, hi); });
  }
  for (auto &x : th) x.join();
}


}  // namespace

struct spm_shim_plan {
  long n0, n1, n2;
  cd *buf;
  int sign;
  Line l0, l1, l2;
};

extern "C" {

void spm_shim_fft_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
int spm_shim_fft_get_threads(void) { return g_threads; }

void *fftw_malloc(size_t n) { return std::malloc(n); }
fftw_complex *fftw_alloc_complex(size_t n) { return (fftw_complex *)std::malloc(n * sizeof(fftw_complex)); }
void fftw_free(void *p) { std::free(p); }

void fftw_mpi_init(void) {}

ptrdiff_t fftw_mpi_local_size_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm,
                                 ptrdiff_t *local_n0, ptrdiff_t *local_0_start) {
  *local_n0 = n0;
  *local_0_start = 0;
  return n0 * n1 * n2;
}

fftw_plan fftw_mpi_plan_dft_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, fftw_complex *in,
                               fftw_complex *out, MPI_Comm, int sign, unsigned) {
  if (in != out) return nullptr;  // the reference only plans in place (My_FFT.cpp:99-115)
  spm_shim_plan *p = new spm_shim_plan;
  p->n0 = n0; p->n1 = n1; p->n2 = n2;
  p->buf = reinterpret_cast<cd *>(in);
  p->sign = sign;
  make_line(p->l0, (int)n0, sign);
  make_line(p->l1, (int)n1, sign);
  make_line(p->l2, (int)n2, sign);
  return p;
}

void fftw_destroy_plan(fftw_plan p) { delete p; }
void fftw_mpi_broadcast_wisdom(MPI_Comm) {}
int fftw_import_wisdom_from_filename(const char *) { return 0; }
int fftw_export_wisdom_to_filename(const char *) { return 1; }

void fftw_execute(const fftw_plan p) {
  const long n0 = p->n0, n1 = p->n1, n2 = p->n2;
  cd *a = p->buf;
  const long B = 8;  // lines gathered per block on the strided axes
  const long nmax = std::max(n0, std::max(n1, n2));
  const long nb2 = (n2 + B - 1) / B;
  // axis 2: contiguous lines
  par_for(n0 * n1, [&](long lo, long hi) {
    std::vector<cd> tmp(nmax);
    for (long l = lo; l < hi; l++) line_fft(p->l2, a + l * n2, tmp.data());
  });
  // axis 1 (stride n2) and axis 0 (stride n1*n2): gather B lines, transform, scatter
  par_for(n0 * nb2, [&](long lo, long hi) {
    std::vector<cd> tmp(nmax * (B + 1));
    cd *g = tmp.data() + nmax;
    for (long blk = lo; blk < hi; blk++) {
      long i0 = blk / nb2, i2b = (blk % nb2) * B;
      long nb = std::min(B, n2 - i2b);
      for (long i1 = 0; i1 < n1; i1++)
        for (long b = 0; b < nb; b++) g[b * n1 + i1] = a[(i0 * n1 + i1) * n2 + i2b + b];
      for (long b = 0; b < nb; b++) line_fft(p->l1, g + b * n1, tmp.data());
      for (long i1 = 0; i1 < n1; i1++)
        for (long b = 0; b < nb; b++) a[(i0 * n1 + i1) * n2 + i2b + b] = g[b * n1 + i1];
    }
  });
  par_for(n1 * nb2, [&](long lo, long hi) {
    std::vector<cd> tmp(nmax * (B + 1));
    cd *g = tmp.data() + nmax;
    for (long blk = lo; blk < hi; blk++) {
      long i1 = blk / nb2, i2b = (blk % nb2) * B;
      long nb = std::min(B, n2 - i2b);
      for (long i0 = 0; i0 < n0; i0++)
        for (long b = 0; b < nb; b++) g[b * n0 + i0] = a[(i0 * n1 + i1) * n2 + i2b + b];
      for (long b = 0; b < nb; b++) line_fft(p->l0, g + b * n0, tmp.data());
      for (long i0 = 0; i0 < n0; i0++)
        for (long b = 0; b < nb; b++) a[(i0 * n1 + i1) * n2 + i2b + b] = g[b * n0 + i0];
    }
  });
}

// ---------------------------------------------------------------- MPI, 1 rank
int MPI_Init(int *, char ***) { return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return 0; }
int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return 0; }
int MPI_Barrier(MPI_Comm) { return 0; }
double MPI_Wtime(void) {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
int MPI_Reduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (s != MPI_IN_PLACE) std::memmove(r, s, (size_t)count * (size_t)t);
  return 0;
}
int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (s != MPI_IN_PLACE) std::memmove(r, s, (size_t)count * (size_t)t);
  return 0;
}
int MPI_Scatter(const void *s, int sc, MPI_Datatype st, void *r, int, MPI_Datatype, int, MPI_Comm) {
  if (s != r) std::memmove(r, s, (size_t)sc * (size_t)st);
  return 0;
}
int MPI_Gather(const void *s, int sc, MPI_Datatype st, void *r, int, MPI_Datatype, int, MPI_Comm) {
  if (s != r) std::memmove(r, s, (size_t)sc * (size_t)st);
  return 0;
}

// ------------------------------------------------------ Eigen Random stream
static uint64_t g_seed = 0, g_counter = 0;
void spm_shim_eigen_seed(uint64_t seed) { g_seed = seed; g_counter = 0; }
// n-th SplitMix64 output of the stream seeded with g_seed, mapped to [-1, 1).
double spm_shim_eigen_next_uniform(void) {
  uint64_t z = g_seed + (g_counter + 1) * 0x9E3779B97F4A7C15ULL;
  g_counter++;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return -1.0 + 2.0 * ((double)(z >> 11) * std::ldexp(1.0, -53));
}

}  // extern "C"
