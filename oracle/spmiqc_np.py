"""CPU restatement (NumPy, FP64) of SPM-IQC's pseudo-spectral hot path.

TEST INFRASTRUCTURE ONLY. This module is the oracle: tests, the smoke check and
bench.py's CPU-baseline leg use it as the checker. The product path never
imports it and has no CPU fallback.

Every function follows one reference routine, cited as file:line within the
SPM-IQC project, and keeps the reference's data conventions: real fields are
real float64 arrays of shape (N, N, N) (row-major i*N*N + j*N + k); spectra are
full complex N^3 arrays from the forward transform normalised by 1/N^3
(src/My_FFT.cpp:4-13); the backward transform is unnormalised
(src/My_FFT.cpp:15-21). FFTW's DFT (sign -1 forward) is computed with
numpy.fft (pocketfft), which implements the same definition.

This restatement is pinned against the reference's own sources, compiled
unchanged with single-rank shims (oracle/Makefile, oracle/refbind.py), by
tests/test_oracle.py.
"""
from __future__ import annotations

import numpy as np

# src/Initialization.cpp:152-153
GK_PH = 0.568809
GK_D = (1.969182919080340, -14.949858723012090, 37.445683882581790,
        -38.839451762550148, 13.999261011773505)

SPLITMIX_GAMMA = np.uint64(0x9E3779B97F4A7C15)


# ----------------------------------------------------------------- generators
def splitmix64(seed: int, idx: np.ndarray) -> np.ndarray:
    """n-th output of the SplitMix64 stream seeded with `seed` (0-based n)."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (idx.astype(np.uint64) + np.uint64(1)) * SPLITMIX_GAMMA
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform_pm1(seed: int, idx: np.ndarray) -> np.ndarray:
    """SplitMix64 outputs mapped to [-1, 1): -1 + 2 * (z >> 11) * 2^-53."""
    z = splitmix64(seed, idx)
    return -1.0 + 2.0 * ((z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53)


# ----------------------------------------------------------------- the model
def wave_index(N: int) -> np.ndarray:
    """Integer wave numbers K[i] = i for i < N/2 else i - N (Initialization.cpp:97-107)."""
    i = np.arange(N)
    return np.where(i < N // 2, i, i - N)


def ksquare(N: int, L: float) -> np.ndarray:
    """k^2 = ((PK_0^2 + PK_1^2) + PK_2^2), PK_i = (1/L) K_i (Initialization.cpp:132-148)."""
    pk = (1.0 / L) * wave_index(N).astype(np.float64)
    p2 = pk * pk
    return (p2[:, None, None] + p2[None, :, None]) + p2[None, None, :]


def get_GK(k2):
    """Pair kernel G(k^2) (Initialization.cpp:150-166)."""
    d0, d2, d4, d6, d8 = GK_D
    s2 = GK_PH * GK_PH
    k4 = k2 * k2
    k6 = k4 * k2
    k8 = k6 * k2
    return np.exp(-0.5 * k2 / s2) * (d0 + d2 * k2 + d4 * k4 + d6 * k6 + d8 * k8) + 0.08


class Model:
    """Parameters and k-space tables of one grid (Initialization.cpp:7-42, 123-174)."""

    def __init__(self, N: int, L: float = 26.0, Tau: float = -0.0061,
                 Gamma: float = 0.30, dt: float = 0.3):
        self.N, self.L, self.Tau, self.Gamma, self.dt = int(N), float(L), float(Tau), float(Gamma), float(dt)
        self.n3 = self.N ** 3
        self.k2 = ksquare(self.N, self.L)
        self.G = get_GK(self.k2)                                   # epmckt2_local
        self.ikt2 = 1.0 / (self.G + abs(self.Tau) + 0.02)          # Initialization.cpp:123-129

    # src/My_FFT.cpp:4-13 (forward, normalised) and :15-21 (backward)
    def my_fft(self, x):
        return np.fft.fftn(x) / self.n3

    def my_ifft(self, X):
        return np.fft.ifftn(X) * self.n3

    # src/BasicOperators.cpp:132-172
    def inpfp(self, p, q) -> float:
        return float(np.sum(p * q) / self.n3)

    def nrmp(self, p) -> float:
        return float(np.sqrt(self.inpfp(p, p)))

    # src/LPsrc.cpp:8-38
    def energy(self, phi, uF) -> float:
        u2 = phi * phi
        u3 = u2 * phi
        u4 = u3 * phi
        nln = -0.5 * self.Tau * u2 - self.Gamma * u3 / 3 + 0.25 * u4
        E2 = float(np.sum(nln) / self.n3)
        E1 = 0.5 * float(np.sum((uF.real * uF.real + uF.imag * uF.imag) * self.G))
        return E1 + E2

    # src/LPsrc.cpp:40-117, one loop iteration
    def grad_step(self, phi, uF):
        """Returns (phi', uF', E, res); E is get_Ene at the incoming state."""
        E = self.energy(phi, uF)
        u2 = phi * phi
        u3 = u2 * phi
        f = self.Tau * phi + self.Gamma * u2 - u3
        fF = self.my_fft(f)
        uF1 = (self.dt * fF + uF) / (1 + self.dt * self.G)
        uF1[0, 0, 0] = 0.0
        res = float(np.max(np.abs(uF1.real - uF.real)))
        phi1 = self.my_ifft(uF1).real
        return phi1, uF1, E, res

    # src/LPsrc.cpp:119-173
    def ngrad(self, phi):
        phif = self.my_fft(phi)
        phif[0, 0, 0] = 0.0
        g = self.my_ifft(self.G * phif).real
        u2 = phi * phi
        u3 = u2 * phi
        g = g - self.Tau * phi - self.Gamma * u2 + u3
        g = g - np.sum(g) / self.n3
        return -1.0 * g

    def grad_norm(self, phi) -> float:
        """||grad F|| = nrmp(ngrad_cam(phi)), the residual of SPM.cpp:224-229."""
        return self.nrmp(self.ngrad(phi))

    # src/LOBPCG.cpp:113-166
    def hv(self, phi, v):
        vf = self.my_fft(v)
        h = self.my_ifft(self.G * vf).real
        h = h + (-self.Tau - 2 * self.Gamma * phi + 3 * phi * phi) * v
        return h - np.sum(h) / self.n3

    # src/LOBPCG.cpp:168-199
    def precond(self, w):
        wf = self.my_fft(w) * self.ikt2
        w = self.my_ifft(wf).real
        return w - np.sum(w) / self.n3

    # src/BasicOperators.cpp:229-255 (modified Gram-Schmidt, in place)
    def orth_v2V(self, v, V, k):
        for i in range(k):
            t = self.inpfp(v, V[i])
            v -= t * V[i]

    def orth_Vi(self, V, k):
        for i in range(k):
            t = self.inpfp(V[i], V[k])
            V[k] -= t * V[i]

    # src/LOBPCG.cpp:10-109 with MatrixXd::Random = SplitMix64 stream (col-major)
    def lobpcg_init(self, k: int, seed: int):
        n3 = self.n3
        idx = np.arange(k * n3, dtype=np.uint64)
        R = uniform_pm1(seed, idx).reshape(n3, k).T.copy()        # R[i, j] = u(j*k + i)
        V = R.reshape(k, self.N, self.N, self.N)
        for i in range(k):
            V[i] -= np.sum(V[i]) / n3
        for i in range(k):
            for j in range(i):
                t = self.inpfp(V[i], V[j])
                V[i] -= t * V[j]
            V[i] *= 1.0 / self.nrmp(V[i])
        return V

    # src/LOBPCG.cpp:207-487 (one call, `maxiter` iterations)
    def lobpcg_inip(self, x, V, maxiter: int = 21):
        k = V.shape[0]
        shape = V.shape
        V = V.copy()
        U = np.zeros(shape)
        W = np.zeros(shape)
        Y = np.zeros(shape)
        Vp = np.zeros(shape)
        Up = np.zeros(shape)
        for i in range(k):
            self.orth_Vi(V, i)
            V[i] *= 1.0 / self.nrmp(V[i])
        ritz = None
        for _ in range(maxiter):
            emp = np.ones(3 * k, dtype=bool)
            for i in range(k):
                U[i] = self.hv(x, V[i])
                a = self.inpfp(V[i], U[i])
                W[i] = 1 * U[i] + (-a) * V[i]
                W[i] = self.precond(W[i])
                self.orth_v2V(W[i], V, k)
                self.orth_Vi(W, i)
                nw = self.nrmp(W[i])
                if nw > 1e-8:
                    W[i] *= 1.0 / nw
                    Y[i] = self.hv(x, W[i])
                else:
                    W[i] = 0.0
                    Y[i] = 0.0
                    emp[k + i] = False
            for i in range(k):
                self.orth_v2V(Vp[i], V, k)
                self.orth_v2V(Vp[i], W, k)
                self.orth_Vi(Vp, i)
                nv = self.nrmp(Vp[i])
                if nv > 1e-8:
                    Vp[i] *= 1.0 / nv
                    Up[i] = self.hv(x, Vp[i])
                else:
                    Vp[i] = 0.0
                    Up[i] = 0.0
                    emp[2 * k + i] = False
            UU = np.concatenate([V, W, Vp]).reshape(3 * k, -1)[emp]
            YY = np.concatenate([U, Y, Up]).reshape(3 * k, -1)[emp]
            P = UU @ YY.T
            P = (P.T + P) * 0.5
            P = P / self.n3
            vals, vecs = np.linalg.eigh(P)
            ritz = vals[:k].copy()
            Vp[:] = V
            Up[:] = U
            V = (vecs[:, :k].T @ UU).reshape(shape)
            for i in range(k):
                V[i] -= np.sum(V[i]) / self.n3
            for i in range(k):
                self.orth_v2V(V[i], V, i)
                V[i] *= 1.0 / self.nrmp(V[i])
        return V, ritz

    def _lob_step(self, x, V, U, W, Y, Vp, Up, V0=None):
        """One iteration body of src/HISD.cpp:258-444 (the LOBPCG update of V
        at position x, with the previous V as the P block); returns the new V.
        With V0 (src/GOSD.cpp:298-326) W, Vp and V are also kept orthogonal to V0."""
        k = V.shape[0]
        shape = V.shape
        emp = np.ones(3 * k, dtype=bool)
        for i in range(k):
            U[i] = self.hv(x, V[i])
            a = self.inpfp(V[i], U[i])
            W[i] = 1 * U[i] + (-a) * V[i]
            W[i] = self.precond(W[i])
            self.orth_v2V(W[i], V, k)
            if V0 is not None:
                self.orth_v2V(W[i], V0, V0.shape[0])
            self.orth_Vi(W, i)
            nw = self.nrmp(W[i])
            if nw > 1e-8:
                W[i] *= 1.0 / nw
                Y[i] = self.hv(x, W[i])
            else:
                W[i] = 0.0
                Y[i] = 0.0
                emp[k + i] = False
        for i in range(k):
            self.orth_v2V(Vp[i], V, k)
            self.orth_v2V(Vp[i], W, k)
            if V0 is not None:
                self.orth_v2V(Vp[i], V0, V0.shape[0])
            self.orth_Vi(Vp, i)
            nv = self.nrmp(Vp[i])
            if nv > 1e-8:
                Vp[i] *= 1.0 / nv
                Up[i] = self.hv(x, Vp[i])
            else:
                Vp[i] = 0.0
                Up[i] = 0.0
                emp[2 * k + i] = False
        UU = np.concatenate([V, W, Vp]).reshape(3 * k, -1)[emp]
        YY = np.concatenate([U, Y, Up]).reshape(3 * k, -1)[emp]
        P = UU @ YY.T
        P = (P.T + P) * 0.5 / self.n3
        vals, vecs = np.linalg.eigh(P)
        Vp[:] = V
        Up[:] = U
        V = (vecs[:, :k].T @ UU).reshape(shape)
        for i in range(k):
            V[i] -= np.sum(V[i]) / self.n3
        for i in range(k):
            self.orth_v2V(V[i], V, i)
            if V0 is not None:
                self.orth_v2V(V[i], V0, V0.shape[0])
            V[i] *= 1.0 / self.nrmp(V[i])
        return V

    # src/HISD.cpp:86-485 (hiosd_lobpcg_sieh); with V0, src/GOSD.cpp:123-531
    # (hiosd_lobpcg_sieh_V0)
    def hisd(self, x, V, dt=0.8, betat=8.0, betau=0.02, epsf=1e-7, maxiter=10000, V0=None):
        """Returns (x, V, residual history)."""
        k = V.shape[0]
        x = x.copy()
        V = V.copy()
        shape = V.shape
        U, W, Y, Vp, Up = (np.zeros(shape) for _ in range(5))
        for i in range(k):
            self.orth_Vi(V, i)
            V[i] *= 1.0 / self.nrmp(V[i])
        pv = lambda f: sum(self.inpfp(f, V[i]) * V[i] for i in range(k))  # PV_Cplx
        f = self.ngrad(x)
        gp = np.zeros_like(x)
        Dx = f - 2.0 * pv(f) + dt  # FuncRealAddAConst (HISD.cpp:180)
        hist = []
        for _ in range(maxiter):
            tm = 2.0 * pv(f)
            g = f - tm
            Dg = g - gp
            gp = g
            bta = abs(self.inpfp(Dx, Dg) / self.inpfp(Dg, Dg))
            bta = max(min(bta, betat * dt), betau * dt)
            xp = x
            nln = self.Tau * x + self.Gamma * x * x - x * x * x
            nln = nln - np.sum(nln) / self.n3
            rho = (self.my_fft(x) + bta * self.my_fft(nln) - bta * self.my_fft(tm)) / (1 + bta * self.G)
            rho = rho.real + 0j          # the reference keeps the real part only (HISD.cpp:249-252)
            rho[0, 0, 0] = 0.0
            x = self.my_ifft(rho).real
            Dx = x - xp
            V = self._lob_step(x, V, U, W, Y, Vp, Up, V0)
            f = self.ngrad(x)
            res = self.nrmp(f)
            hist.append(res)
            if res < epsf:
                break
        return x, V, np.array(hist)

    def rayleigh(self, x, v) -> float:
        """src/BasicOperators.cpp:174-185."""
        return self.inpfp(v, self.hv(x, v)) / self.inpfp(v, v)

    # src/SPM.cpp:15-32
    def tangent(self, phi0, phi1):
        v = phi1 - phi0
        return v / self.nrmp(v)

    # src/SPM.cpp:34-99 (factor 1) and :103-168 (factor 2); beta = 1
    def force_step(self, x, v, factor: float = 1.0):
        f = self.ngrad(x)
        tmpp = self.inpfp(f, v) * v
        if factor != 1.0:
            tmpp = factor * tmpp
        u2 = x * x
        u3 = u2 * x
        rho = self.my_fft(x)
        nln = self.Tau * x + self.Gamma * u2 - u3
        nln = nln - np.sum(nln) / self.n3
        tF = self.my_fft(tmpp)
        nF = self.my_fft(nln)
        bta = 1.0
        rho = (rho + bta * nF - bta * tF) / (1 + bta * self.G)
        rho[0, 0, 0] = 0.0
        return self.my_ifft(rho).real

    def natural_forces(self, x, v):
        return self.force_step(x, v, 1.0)

    def minmax_forces(self, x, v):
        return self.force_step(x, v, 2.0)

    # src/SPM.cpp:170-263
    def spring_pairing(self, phi0, phi1, maxiter, tol, rest: float = 0.0):
        """Returns (phi0, phi1, iterations, last residual). rest > 0: a spring of
        that rest length, the reference's unused kd = ks (dd - spring_d)
        (SPM.cpp:199-212) applied along (phi1 - phi0) / dd, with dd measured
        once per iteration after the natural-force step."""
        dt, ks = 0.001, 1.0
        P = [phi0.copy(), phi1.copy()]
        res, it = 1e-6, 0
        while res > tol and it < maxiter:
            it += 1
            v = self.tangent(P[0], P[1])
            for i in range(2):
                P[i] = self.natural_forces(P[i], v)
            if rest > 0:
                dd = self.nrmp(P[1] - P[0])
                ks = 1.0 * ((dd - rest) / dd) if dd > 0 else 0.0
            for i in range(2):
                Fs = ks * P[1] + (-ks) * P[0] if i == 0 else ks * P[0] + (-ks) * P[1]
                P[i] = 1 * P[i] + dt * Fs
            v = self.tangent(P[0], P[1])
            res = 0.0
            for i in range(2):
                P[i] = self.minmax_forces(P[i], v)
                res = max(res, self.grad_norm(P[i]))
            for i in range(2):
                Fs = ks * P[1] + (-ks) * P[0] if i == 0 else ks * P[0] + (-ks) * P[1]
                P[i] = 1 * P[i] + dt * Fs
        return P[0], P[1], it, res


# ------------------------------------------------------------ synthetic inputs
def uniform_field(N: int, seed: int, amp: float = 0.1):
    """phi0 ~ U[-amp, amp) from the SplitMix64 stream (index = flat grid index), mean removed."""
    u = uniform_pm1(seed, np.arange(N ** 3, dtype=np.uint64)).reshape(N, N, N) * amp
    return u - np.sum(u) / N ** 3
