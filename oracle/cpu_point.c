/* Pointwise passes of the FFTW-class CPU baseline (oracle/cpu_mkl.py): the
 * real-space and spectral work of one semi-implicit gradient step of SPM-IQC
 * (src/LPsrc.cpp:8-117) around two library transforms, each fused into one
 * OpenMP pass over the data so the baseline is bound by its transforms, not by
 * temporaries.
 *
 * TEST INFRASTRUCTURE ONLY (a timed CPU baseline); the product never links it.
 *
 * Layouts: real fields are N^3 doubles, row-major; spectra are the R2C half
 * spectrum N x N x (N/2 + 1) complex (re, im interleaved), as torch.fft.rfftn
 * returns it. gtab[K2] holds G at K^2 = Kx^2 + Ky^2 + Kz^2 (integer wave
 * numbers, Initialization.cpp:95-166), 3 (N/2)^2 + 1 entries.
 */
#include <math.h>
#include <stddef.h>

/* f = Tau phi + Gamma phi^2 - phi^3 (LPsrc.cpp:58-62); returns
 * sum(-Tau/2 phi^2 - Gamma/3 phi^3 + phi^4/4) (LPsrc.cpp:10-24). */
double spm_cpu_real_pass(const double *phi, double *f, long n, double tau, double gam) {
  double e = 0.0;
  const double mt2 = -0.5 * tau, mg3 = -gam / 3.0;
#pragma omp parallel for reduction(+ : e) schedule(static)
  for (long i = 0; i < n; i++) {
    const double u = phi[i];
    e += u * u * (mt2 + u * (mg3 + 0.25 * u));
    f[i] = u * (tau + u * (gam - u));
  }
  return e;
}

/* One spectral pass (LPsrc.cpp:27-35, 64-84 and the spectral form of
 * nrmp(ngrad_cam)^2, LPsrc.cpp:119-173): fh = FFT(f) unnormalised in, u the
 * current spectrum (normalised), u1 = (dt fh/N^3 + u)/(1 + dt G), u1_0 = 0.
 * out[0] = 1/2 sum G |u|^2, out[1] = max |Re(u1 - u)|, out[2] = sum_{k != 0}
 * |G u - fh/N^3|^2, each over the full spectrum (weights 2 off the kz = 0,
 * N/2 planes). */
void spm_cpu_spec_pass(const double *u, const double *fh, double *u1, const double *gtab, int N, double dt,
                       double inv_n3, double *out) {
  const int H = N / 2 + 1;
  double e1 = 0.0, g2 = 0.0, res = 0.0;
#pragma omp parallel for reduction(+ : e1, g2) reduction(max : res) schedule(static)
  for (long row = 0; row < (long)N * N; row++) {
    const int ix = (int)(row / N), iy = (int)(row % N);
    const int kx = ix < N / 2 ? ix : ix - N, ky = iy < N / 2 ? iy : iy - N;
    const int k2xy = kx * kx + ky * ky;
    const size_t base = (size_t)row * H * 2;
    for (int kz = 0; kz < H; kz++) {
      const size_t o = base + 2 * (size_t)kz;
      const double G = gtab[k2xy + kz * kz];
      const double w = (kz == 0 || kz == N / 2) ? 1.0 : 2.0;
      const double ur = u[o], ui = u[o + 1];
      const double fr = fh[o] * inv_n3, fi = fh[o + 1] * inv_n3;
      e1 += w * 0.5 * G * (ur * ur + ui * ui);
      double vr = (dt * fr + ur) / (1.0 + dt * G), vi = (dt * fi + ui) / (1.0 + dt * G);
      if (row == 0 && kz == 0) {
        vr = vi = 0.0;
      } else {
        const double gr = G * ur - fr, gi = G * ui - fi;
        g2 += w * (gr * gr + gi * gi);
      }
      const double d = fabs(vr - ur);
      if (d > res) res = d;
      u1[o] = vr;
      u1[o + 1] = vi;
    }
  }
  out[0] = e1;
  out[1] = res;
  out[2] = g2;
}
