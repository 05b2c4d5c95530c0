// Pointwise policies that specialise the three transform passes into the
// reference's hot-path routines. Each policy cites the SPM-IQC code it follows.
#pragma once

#include "fft_kernels.cuh"

namespace spm {

template <class T> __device__ __forceinline__ const T *fld(const void *p) { return reinterpret_cast<const T *>(p); }
__device__ __forceinline__ double *scal_of(const KParams &p, int b) { return p.scal + (size_t)b * kScal; }

// ===================================================================== prologues
// Transform the field as it is; no reduction.
template <class T> struct ProIdent {
  static constexpr int NR = 0;
  static constexpr unsigned MAXM = 0;
  __device__ static c2<T> pro(const KParams &, int, size_t, c2<T> x, double (&)[1]) { return x; }
  __device__ static void fin(const KParams &, int, const double (&)[1]) {}
};

// Local polynomials of the model in Horner form (a few ulp from the
// reference's term-by-term order, LPsrc.cpp:10-24, 58-62):
//   nonlinear force  f(u) = Tau u + Gamma u^2 - u^3 = u (Tau + u (Gamma - u))
//   energy density   e(u) = -Tau/2 u^2 - Gamma/3 u^3 + u^4/4
//                         = u^2 (-Tau/2 + u (-Gamma/3 + u/4))
// (The outer products are rounded explicitly so that no kernel contracts them
// into the sums that follow.)
template <class T> __device__ __forceinline__ T poly_force(T u, T tau, T gam) {
  return mul_rn(u, fma_rn(u, gam - u, tau));
}
template <class T> __device__ __forceinline__ T poly_energy(T u, T mtau2, T mgam3) {
  return mul_rn(mul_rn(u, u), fma_rn(u, fma_rn((T)0.25, u, mgam3), mtau2));
}

// Gradient step (LPsrc.cpp:44-75): transform f(u) and sum the energy density.
// FACC: in FP32 the energy density is summed in FP32 over a row's points of
// one thread before it joins the FP64 total.
template <class T> struct ProGrad {
  static constexpr int NR = 1;
  static constexpr unsigned MAXM = 0;
  static constexpr bool FACC = true;
  template <class A> __device__ static c2<T> pro(const KParams &p, int b, size_t, c2<T> x, A (&acc)[1]) {
    const ModelC &m = model(p, b);
    const T tau = (T)m.Tau, gam = (T)m.Gamma;
    const T mtau2 = (T)(-0.5 * m.Tau), mgam3 = (T)(-m.Gamma / 3.0);
    acc[0] += (A)poly_energy(x.x, mtau2, mgam3) + (A)poly_energy(x.y, mtau2, mgam3);
    return c2<T>{poly_force(x.x, tau, gam), poly_force(x.y, tau, gam)};
  }
  __device__ static void fin(const KParams &p, int b, const double (&tot)[1]) {
    scal_of(p, b)[SC_E2] = tot[0] * model(p, b).inv_n3;
  }
};

// Hessian-vector product (LOBPCG.cpp:113-166): transform v; accumulate sum(v)
// and sum((-Tau - 2 Gamma phi + 3 phi^2) v) so the epilogue can remove the mean
// mu = G(0) mean(v) + mean(c(phi) v) without a second pass (aux0 = phi).
template <class T> struct ProHv {
  static constexpr int NR = 2;
  static constexpr unsigned MAXM = 0;
  __device__ static c2<T> pro(const KParams &p, int b, size_t idx, c2<T> x, double (&acc)[2]) {
    const c2<T> ph = __ldg(reinterpret_cast<const c2<T> *>(fld<T>(p.aux0[b]) + idx));
    const T tau = (T)p.m.Tau, gam = (T)p.m.Gamma;
    acc[0] += (double)x.x + (double)x.y;
    acc[1] += (double)((-tau - (T)2 * gam * ph.x + (T)3 * ph.x * ph.x) * x.x);
    acc[1] += (double)((-tau - (T)2 * gam * ph.y + (T)3 * ph.y * ph.y) * x.y);
    return x;
  }
  __device__ static void fin(const KParams &p, int b, const double (&tot)[2]) {
    scal_of(p, b)[SC_MU] = p.m.G0 * (tot[0] * p.m.inv_n3) + tot[1] * p.m.inv_n3;
  }
};

// Negative gradient (LPsrc.cpp:119-173): transform phi; accumulate sum(f),
// f = Tau phi + Gamma phi^2 - phi^3, whose mean is the mean the reference
// subtracts (the G-term has zero mean because its k = 0 mode is removed).
template <class T> struct ProNgrad {
  static constexpr int NR = 1;
  static constexpr unsigned MAXM = 0;
  __device__ static c2<T> pro(const KParams &p, int, size_t, c2<T> x, double (&acc)[1]) {
    const T tau = (T)p.m.Tau, gam = (T)p.m.Gamma;
    acc[0] += (double)poly_force(x.x, tau, gam) + (double)poly_force(x.y, tau, gam);
    return x;
  }
  __device__ static void fin(const KParams &p, int b, const double (&tot)[1]) {
    scal_of(p, b)[SC_MU] = tot[0] * p.m.inv_n3;
  }
};

// Preconditioner (LOBPCG.cpp:168-199): transform w; the epilogue removes the
// mean ikt2(0) * mean(w).
template <class T> struct ProPrecond {
  static constexpr int NR = 1;
  static constexpr unsigned MAXM = 0;
  __device__ static c2<T> pro(const KParams &, int, size_t, c2<T> x, double (&acc)[1]) {
    acc[0] += (double)x.x + (double)x.y;
    return x;
  }
  __device__ static void fin(const KParams &p, int b, const double (&tot)[1]) {
    scal_of(p, b)[SC_MU] = p.m.ikt0 * (tot[0] * p.m.inv_n3);
  }
};

// SPM force step (SPM.cpp:34-99, 103-168) with beta = 1. Transforms
// T = x + N(x), N = Tau x + Gamma x^2 - x^3 (its mean only touches the k = 0
// mode, which the step zeroes), and accumulates the projection
//   <f, v> = -<x, Gv> + <N, v> - mean(N) mean(v),  f = ngrad(x),
// where Gv = IFFT(G FFT(v), k = 0 removed) is prepared once per tangent.
// aux0 = v, aux1 = Gv.
// FACC: in FP32 the four sums run in FP32 over a row's points of one thread
// before they join the FP64 totals.
template <class T> struct ProForce {
  static constexpr int NR = 4;
  static constexpr unsigned MAXM = 0;
  static constexpr bool FACC = true;
  template <class A> __device__ static c2<T> pro(const KParams &p, int b, size_t idx, c2<T> x, A (&acc)[4]) {
    const c2<T> v = __ldg(reinterpret_cast<const c2<T> *>(fld<T>(p.aux0[b]) + idx));
    const c2<T> gv = __ldg(reinterpret_cast<const c2<T> *>(fld<T>(p.aux1[b]) + idx));
    const T tau = (T)p.m.Tau, gam = (T)p.m.Gamma;
    const T n0 = poly_force(x.x, tau, gam);
    const T n1 = poly_force(x.y, tau, gam);
    acc[0] += (A)x.x * (A)gv.x + (A)x.y * (A)gv.y;
    acc[1] += (A)n0 * (A)v.x + (A)n1 * (A)v.y;
    acc[2] += (A)n0 + (A)n1;
    acc[3] += (A)v.x + (A)v.y;
    return c2<T>{x.x + n0, x.y + n1};
  }
  __device__ static void fin(const KParams &p, int b, const double (&tot)[4]) {
    const double s = -tot[0] * p.m.inv_n3 + tot[1] * p.m.inv_n3 -
                     (tot[2] * p.m.inv_n3) * (tot[3] * p.m.inv_n3);
    scal_of(p, b)[SC_S] = p.m.factor * s;
  }
};

// SPM tangent (SPM.cpp:15-32): transform d = Phi1 - Phi0 (in = Phi1, aux0 =
// Phi0) and accumulate |d|^2; the pencil scales by 1/||d||.
template <class T> struct ProTangent {
  static constexpr int NR = 1;
  static constexpr unsigned MAXM = 0;
  static constexpr bool FACC = true;
  template <class A> __device__ static c2<T> pro(const KParams &p, int b, size_t idx, c2<T> x, A (&acc)[1]) {
    const c2<T> a = p.aux0[b] ? __ldg(reinterpret_cast<const c2<T> *>(fld<T>(p.aux0[b]) + idx)) : c2<T>{0, 0};
    const c2<T> d = {x.x - a.x, x.y - a.y};
    acc[0] += (A)d.x * (A)d.x + (A)d.y * (A)d.y;
    return d;
  }
  __device__ static void fin(const KParams &p, int b, const double (&tot)[1]) {
    scal_of(p, b)[SC_NRM2] = tot[0] * p.m.inv_n3;
  }
};

// HiSD position step (HISD.cpp:200-256): transforms y = x + beta (N(x) - T)
// with N = Tau x + Gamma x^2 - x^3 (its mean only reaches the k = 0 mode,
// which the step zeroes) and T = 2 PV(f) (aux0); beta in m.factor.
template <class T> struct ProHisd {
  static constexpr int NR = 0;
  static constexpr unsigned MAXM = 0;
  __device__ static c2<T> pro(const KParams &p, int b, size_t idx, c2<T> x, double (&)[1]) {
    const c2<T> t = __ldg(reinterpret_cast<const c2<T> *>(fld<T>(p.aux0[b]) + idx));
    const T tau = (T)p.m.Tau, gam = (T)p.m.Gamma, beta = (T)p.m.factor;
    return c2<T>{x.x + beta * (poly_force(x.x, tau, gam) - t.x), x.y + beta * (poly_force(x.y, tau, gam) - t.y)};
  }
  __device__ static void fin(const KParams &, int, const double (&)[1]) {}
};

// ===================================================================== pencil ops
// Forward transform with the reference's 1/N^3 (My_FFT.cpp:9-13): store only.
template <class T> struct OpFwd {
  static constexpr bool FI = true, SI = false, SO = true, INV = false, LIN = true;
  static constexpr int SYM = -1;
  static constexpr int NR = 0;
  static constexpr unsigned MAXM = 0;
  __device__ static void point(const KParams &p, int, int, int, int, double2, c2<T> f, c2<T>, c2<T> &so,
                               c2<T> &, double (&)[1], double) {
    so = cscale(f, (T)p.m.inv_n3);
  }
  __device__ static void fin(const KParams &, int, const double (&)[1]) {}
};

// Backward transform of a stored spectrum (My_FFT.cpp:15-21): inverse only.
template <class T> struct OpInv {
  static constexpr bool FI = false, SI = true, SO = false, INV = true, LIN = true;
  static constexpr int SYM = -1;
  static constexpr int NR = 0;
  static constexpr unsigned MAXM = 0;
  __device__ static void point(const KParams &, int, int, int, int, double2, c2<T>, c2<T> s, c2<T> &, c2<T> &inv,
                               double (&)[1], double) {
    inv = s;
  }
  __device__ static void fin(const KParams &, int, const double (&)[1]) {}
};

// One semi-implicit gradient step (LPsrc.cpp:64-84) with the energy and
// ||grad F|| of the incoming state:
//   u' = (dt f^ + u) / (1 + dt G), u'_0 = 0,  res = max |Re(u' - u)|,
//   E1 = 1/2 sum G |u|^2,  ||grad F||^2 = sum_{k != 0} |G u - f^|^2.
// FACC: in FP32 the three reductions run in FP32 over a thread's 16 points of
// a tile (the differences G u - f^ and u' - u of FP32 values, which carry
// FP32 rounding already), then join the FP64 totals.
template <class T> struct OpGrad {
  static constexpr bool FI = true, SI = true, SO = true, INV = true, LIN = false;
  static constexpr int SYM = 0;  // {G, 1/(1 + dt G)}
  static constexpr int NR = 3;
  static constexpr unsigned MAXM = 0x2;
  static constexpr bool FACC = true;
  template <class A>
  __device__ static void point(const KParams &p, int b, int Kx, int Ky, int Kz, double2 sy, c2<T> f, c2<T> s,
                               c2<T> &so, c2<T> &inv, A (&acc)[3], double w) {
    const A G = (A)sy.x;
    const T dt = (T)model(p, b).dt;
    const c2<T> fh = cscale(f, (T)model(p, b).inv_n3);
    const T iden = (T)sy.y;  // 1 / (1 + dt G)
    c2<T> u1 = {(dt * fh.x + s.x) * iden, (dt * fh.y + s.y) * iden};
    const bool k0 = (Kx == 0 && Ky == 0 && Kz == 0);
    if (k0) u1 = c2<T>{0, 0};
    const A wa = (A)w;
    acc[0] += wa * (A)0.5 * G * ((A)s.x * (A)s.x + (A)s.y * (A)s.y);
    acc[1] = fmax(acc[1], fabs((A)u1.x - (A)s.x));
    if (!k0) {
      const A gx = G * (A)s.x - (A)fh.x, gy = G * (A)s.y - (A)fh.y;
      acc[2] += wa * (gx * gx + gy * gy);
    }
    so = u1;
    inv = u1;
  }
  // Record (E, res, ||grad F||) of this step; arm the stop when the reference's
  // criterion res <= 1e-16 (LPsrc.cpp:52) or ||grad F|| <= tol_grad holds.
  __device__ static void fin(const KParams &p, int b, const double (&tot)[3]) {
    double *sc = scal_of(p, b);
    const double E = tot[0] + sc[SC_E2];
    const double gn = sqrt(tot[2]);
    sc[SC_E1] = tot[0];
    sc[SC_RES] = tot[1];
    sc[SC_GN2] = tot[2];
    int *flow = flow_of(p, b);
    if (flow) {
      const ModelC &m = model(p, b);
      double *stats = stats_of(p, b);
      const int it = flow[FW_ITER];
      if (stats) {
        stats[4 * it + 0] = E;
        stats[4 * it + 1] = tot[1];
        stats[4 * it + 2] = gn;
        stats[4 * it + 3] = tot[0];
      }
      flow[FW_ITER] = it + 1;
      if (!(tot[1] > 1e-16) || (m.tol_grad > 0 && gn <= m.tol_grad) || (m.max_steps > 0 && it + 1 >= m.max_steps))
        flow[FW_PENDING] = 1;
    }
  }
};

// G multiply for the Hessian-vector product (LOBPCG.cpp:126-134; the k = 0
// mode is kept) or, with ZERO_DC, for ngrad_cam (LPsrc.cpp:133-142).
template <class T, bool ZERO_DC> struct OpGmul {
  static constexpr bool FI = true, SI = false, SO = false, INV = true, LIN = false;
  static constexpr int SYM = 0;
  static constexpr int NR = 0;
  static constexpr unsigned MAXM = 0;
  __device__ static void point(const KParams &p, int, int Kx, int Ky, int Kz, double2 sy, c2<T> f, c2<T>, c2<T> &,
                               c2<T> &inv, double (&)[1], double) {
    const T g = (T)sy.x;
    inv = cscale(cscale(f, (T)p.m.inv_n3), g);
    if (ZERO_DC && Kx == 0 && Ky == 0 && Kz == 0) inv = c2<T>{0, 0};
  }
  __device__ static void fin(const KParams &, int, const double (&)[1]) {}
};

// Preconditioner symbol 1/(G + |Tau| + 0.02) (Initialization.cpp:123-129, LOBPCG.cpp:175-179).
template <class T> struct OpPrecond {
  static constexpr bool FI = true, SI = false, SO = false, INV = true, LIN = false;
  static constexpr int SYM = 1;  // {1/(G + |Tau| + 0.02), 1/(1 + G)}
  static constexpr int NR = 0;
  static constexpr unsigned MAXM = 0;
  __device__ static void point(const KParams &p, int, int Kx, int Ky, int Kz, double2 sy, c2<T> f, c2<T>, c2<T> &,
                               c2<T> &inv, double (&)[1], double) {
    const T ik = (T)sy.x;  // 1 / (G + |Tau| + 0.02)
    inv = cscale(cscale(f, (T)p.m.inv_n3), ik);
  }
  __device__ static void fin(const KParams &, int, const double (&)[1]) {}
};

// SPM force update (SPM.cpp:82-91): x'^ = (x^ + N^ - s v^) / (1 + G), x'^_0 = 0,
// with s = factor * <ngrad(x), v> from the prologue and v^ (st) the stored
// spectrum of the tangent.
template <class T> struct OpForce {
  static constexpr bool FI = true, SI = true, SO = false, INV = true, LIN = false;
  static constexpr int SYM = 1;
  static constexpr int NR = 0;
  static constexpr unsigned MAXM = 0;
  __device__ static void point(const KParams &p, int b, int Kx, int Ky, int Kz, double2 sy, c2<T> f, c2<T> s, c2<T> &,
                               c2<T> &inv, double (&)[1], double) {
    const T iden = (T)sy.y;  // 1 / (1 + G)
    const T sc = (T)scal_of(p, b)[SC_S];
    const c2<T> fh = cscale(f, (T)p.m.inv_n3);
    inv = c2<T>{(fh.x - sc * s.x) * iden, (fh.y - sc * s.y) * iden};
    if (Kx == 0 && Ky == 0 && Kz == 0) inv = c2<T>{0, 0};
  }
  __device__ static void fin(const KParams &, int, const double (&)[1]) {}
};

// Tangent spectrum v^ = FFT(d) / (N^3 ||d||) (stored) and the G-weighted
// field Gv = IFFT(G v^, k = 0 removed) (inverse output). With NORM false the
// field is taken as given (||d|| := 1), for force steps along a caller's v.
template <class T, bool NORM = true> struct OpTangent {
  static constexpr bool FI = true, SI = false, SO = true, INV = true, LIN = false;
  static constexpr int SYM = 0;
  static constexpr int NR = 0;
  static constexpr unsigned MAXM = 0;
  __device__ static void point(const KParams &p, int b, int Kx, int Ky, int Kz, double2 sy, c2<T> f, c2<T>, c2<T> &so,
                               c2<T> &inv, double (&)[1], double) {
    const T inrm = NORM ? (T)(1.0 / sqrt(scal_of(p, b)[SC_NRM2])) : (T)1;
    const c2<T> v = cscale(cscale(f, (T)p.m.inv_n3), inrm);
    so = v;
    const T g = (T)sy.x;
    inv = (Kx == 0 && Ky == 0 && Kz == 0) ? c2<T>{0, 0} : cscale(v, g);
  }
  __device__ static void fin(const KParams &, int, const double (&)[1]) {}
};

// HiSD spectral update (HISD.cpp:246-256): x'^ = Re(y^ / (1 + beta G)) with
// the imaginary part set to 0, as the reference does, and x'^_0 = 0.
template <class T> struct OpHisd {
  static constexpr bool FI = true, SI = false, SO = false, INV = true, LIN = false;
  static constexpr int SYM = 0;
  static constexpr int NR = 0;
  static constexpr unsigned MAXM = 0;
  __device__ static void point(const KParams &p, int, int Kx, int Ky, int Kz, double2 sy, c2<T> f, c2<T>, c2<T> &,
                               c2<T> &inv, double (&)[1], double) {
    const T beta = (T)p.m.factor;
    const T den = (T)1 + beta * (T)sy.x;
    inv = c2<T>{f.x * (T)p.m.inv_n3 / den, (T)0};
    if (Kx == 0 && Ky == 0 && Kz == 0) inv = c2<T>{0, 0};
  }
  __device__ static void fin(const KParams &, int, const double (&)[1]) {}
};

// E1 = 1/2 sum_k G |u_k|^2 of a stored spectrum (LPsrc.cpp:27-35): reduction only.
template <class T> struct OpE1 {
  static constexpr bool FI = false, SI = true, SO = false, INV = false, LIN = false;
  static constexpr int SYM = 0;
  static constexpr int NR = 1;
  static constexpr unsigned MAXM = 0;
  __device__ static void point(const KParams &p, int, int Kx, int Ky, int Kz, double2 sy, c2<T>, c2<T> s, c2<T> &, c2<T> &,
                               double (&acc)[1], double w) {
    const double G = sy.x;
    acc[0] += w * 0.5 * G * ((double)s.x * (double)s.x + (double)s.y * (double)s.y);
  }
  __device__ static void fin(const KParams &p, int b, const double (&tot)[1]) {
    scal_of(p, b)[SC_E1] = tot[0];
  }
};

// ===================================================================== epilogues
template <class T> struct EpiStore {
  static constexpr int NR = 0;
  static constexpr unsigned MAXM = 0;
  __device__ static c2<T> epi(const KParams &, int, size_t, c2<T> y, double (&)[1]) { return y; }
  __device__ static void fin(const KParams &, int, const double (&)[1]) {}
};

// Store phi' of a gradient step; the last CTA disarms the chain when the
// step's pencil pass armed the stop (LPsrc.cpp:52 loop exit).
template <class T> struct EpiFlow {
  static constexpr int NR = 1;
  static constexpr unsigned MAXM = 0;
  __device__ static c2<T> epi(const KParams &, int, size_t, c2<T> y, double (&)[1]) { return y; }
  __device__ static void fin(const KParams &p, int b, const double (&)[1]) {
    int *flow = flow_of(p, b);
    if (flow && flow[FW_PENDING]) flow[FW_GO] = 0;
  }
};

// ngrad_cam epilogue (LPsrc.cpp:151-172): g = y - Tau phi - Gamma phi^2 + phi^3,
// minus its mean (= -mean f), negated. Also sums the result squared
// (nrmp, BasicOperators.cpp:158-164). aux0 = phi.
template <class T> struct EpiNgrad {
  static constexpr int NR = 1;
  static constexpr unsigned MAXM = 0;
  static constexpr bool FACC = true;
  template <class A> __device__ static c2<T> epi(const KParams &p, int b, size_t idx, c2<T> y, A (&acc)[1]) {
    const c2<T> ph = __ldg(reinterpret_cast<const c2<T> *>(fld<T>(p.aux0[b]) + idx));
    const T tau = (T)p.m.Tau, gam = (T)p.m.Gamma;
    const T mg = -(T)scal_of(p, b)[SC_MU];
    c2<T> o;
    o.x = -((y.x - tau * ph.x - gam * (ph.x * ph.x) + ph.x * ph.x * ph.x) - mg);
    o.y = -((y.y - tau * ph.y - gam * (ph.y * ph.y) + ph.y * ph.y * ph.y) - mg);
    acc[0] += (A)o.x * (A)o.x + (A)o.y * (A)o.y;
    return o;
  }
  __device__ static void fin(const KParams &p, int b, const double (&tot)[1]) {
    scal_of(p, b)[SC_GN2] = tot[0] * p.m.inv_n3;
  }
};

// hv_cam epilogue (LOBPCG.cpp:136-156): y + (-Tau - 2 Gamma phi + 3 phi^2) v - mu.
// aux0 = phi, aux1 = v.
// The Hessian product before its mean removal, for LOBPCG's block: o = y +
// (-Tau - 2 Gamma phi + 3 phi^2) v, whose mean is the mu that hv_cam subtracts
// (LOBPCG.cpp:136-156). Sums scal[SC_MU] = mean(o), scal[SC_SUM1] = <v, o>,
// scal[SC_SUM2] = mean(v), so the caller can apply the projection where it uses
// the product (no pass over phi before the transform). aux0 = phi, aux1 = v.
template <class T> struct EpiHvRaw {
  static constexpr int NR = 3;
  static constexpr unsigned MAXM = 0;
  __device__ static c2<T> epi(const KParams &p, int b, size_t idx, c2<T> y, double (&acc)[3]) {
    const c2<T> ph = __ldg(reinterpret_cast<const c2<T> *>(fld<T>(p.aux0[b]) + idx));
    const c2<T> v = __ldg(reinterpret_cast<const c2<T> *>(fld<T>(p.aux1[b]) + idx));
    const T tau = (T)p.m.Tau, gam = (T)p.m.Gamma;
    const c2<T> o = {y.x + (-tau - (T)2 * gam * ph.x + (T)3 * ph.x * ph.x) * v.x,
                     y.y + (-tau - (T)2 * gam * ph.y + (T)3 * ph.y * ph.y) * v.y};
    acc[0] += (double)o.x + (double)o.y;
    acc[1] += (double)v.x * (double)o.x + (double)v.y * (double)o.y;
    acc[2] += (double)v.x + (double)v.y;
    return o;
  }
  __device__ static void fin(const KParams &p, int b, const double (&tot)[3]) {
    double *sc = scal_of(p, b);
    sc[SC_MU] = tot[0] * p.m.inv_n3;
    sc[SC_SUM1] = tot[1] * p.m.inv_n3;
    sc[SC_SUM2] = tot[2] * p.m.inv_n3;
  }
};

template <class T> struct EpiHv {
  static constexpr int NR = 0;
  static constexpr unsigned MAXM = 0;
  __device__ static c2<T> epi(const KParams &p, int b, size_t idx, c2<T> y, double (&)[1]) {
    const c2<T> ph = __ldg(reinterpret_cast<const c2<T> *>(fld<T>(p.aux0[b]) + idx));
    const c2<T> v = __ldg(reinterpret_cast<const c2<T> *>(fld<T>(p.aux1[b]) + idx));
    const T tau = (T)p.m.Tau, gam = (T)p.m.Gamma, mu = (T)scal_of(p, b)[SC_MU];
    return c2<T>{y.x + (-tau - (T)2 * gam * ph.x + (T)3 * ph.x * ph.x) * v.x - mu,
                 y.y + (-tau - (T)2 * gam * ph.y + (T)3 * ph.y * ph.y) * v.y - mu};
  }
  __device__ static void fin(const KParams &, int, const double (&)[1]) {}
};

// Tangent epilogue: returns Gv and, when p.sto[b] is set, also writes the
// real-space tangent v = (Phi1 - Phi0) / ||Phi1 - Phi0|| (SPM.cpp:21-31) there
// (aux0 = Phi0, aux1 = Phi1).
template <class T> struct EpiTangent {
  static constexpr int NR = 0;
  static constexpr unsigned MAXM = 0;
  __device__ static c2<T> epi(const KParams &p, int b, size_t idx, c2<T> y, double (&)[1]) {
    if (p.sto[b]) {
      const c2<T> a = __ldg(reinterpret_cast<const c2<T> *>(fld<T>(p.aux0[b]) + idx));
      const c2<T> c = __ldg(reinterpret_cast<const c2<T> *>(fld<T>(p.aux1[b]) + idx));
      const T d = (T)sqrt(scal_of(p, b)[SC_NRM2]);
      *reinterpret_cast<c2<T> *>(reinterpret_cast<T *>(p.sto[b]) + idx) = c2<T>{(c.x - a.x) / d, (c.y - a.y) / d};
    }
    return y;
  }
  __device__ static void fin(const KParams &, int, const double (&)[1]) {}
};

// HiSD epilogue: stores x' and Dx = x' - x (p.sto) where x is the field being
// overwritten (p.aux1; each value is read by the thread that writes it).
template <class T> struct EpiHisd {
  static constexpr int NR = 0;
  static constexpr unsigned MAXM = 0;
  __device__ static c2<T> epi(const KParams &p, int b, size_t idx, c2<T> y, double (&)[1]) {
    const c2<T> x = *reinterpret_cast<const c2<T> *>(fld<T>(p.aux1[b]) + idx);
    *reinterpret_cast<c2<T> *>(reinterpret_cast<T *>(p.sto[b]) + idx) = c2<T>{y.x - x.x, y.y - x.y};
    return y;
  }
  __device__ static void fin(const KParams &, int, const double (&)[1]) {}
};

// precond_camnew epilogue (LOBPCG.cpp:187-197): y - mu.
template <class T> struct EpiPrecond {
  static constexpr int NR = 0;
  static constexpr unsigned MAXM = 0;
  __device__ static c2<T> epi(const KParams &p, int b, size_t, c2<T> y, double (&)[1]) {
    const T mu = (T)scal_of(p, b)[SC_MU];
    return c2<T>{y.x - mu, y.y - mu};
  }
  __device__ static void fin(const KParams &, int, const double (&)[1]) {}
};

}  // namespace spm
