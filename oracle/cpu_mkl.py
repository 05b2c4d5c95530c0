"""FFTW-class CPU baseline: the semi-implicit gradient step of SPM-IQC
(src/LPsrc.cpp:40-117) over torch's CPU FFT (Intel MKL) on all host threads,
with the pointwise work in two fused OpenMP passes (oracle/cpu_point.c).

TEST INFRASTRUCTURE ONLY (a timed CPU baseline beside the reference itself):
bench.py's CPU-baseline leg times it and tests/test_oracle.py pins it against
the reference's golden vectors; the product path never imports it.

Why it exists: the reference plans its transforms with FFTW_PATIENT
(src/My_FFT.cpp:70-85). FFTW is not installed here, so the compiled reference
runs over a project-written FFT shim; this restatement gives the same step on
a vendor-tuned FFT library of FFTW's class, so the GPU/CPU ratio can be read
against both.

One step does what one get_min_u_F iteration does, and also what the GPU step
reports, so the work per step matches the GPU's:
  E   = mean(-Tau/2 phi^2 - Gamma/3 phi^3 + phi^4/4) + 1/2 sum_k G |u_k|^2
        (LPsrc.cpp:8-38, at the incoming state),
  f   = Tau phi + Gamma phi^2 - phi^3, f^ = FFT(f)/N^3 (LPsrc.cpp:58-62),
  u'  = (dt f^ + u)/(1 + dt G), u'_0 = 0 (LPsrc.cpp:64-75),
  res = max |Re(u' - u)| (LPsrc.cpp:77-84),
  ||grad F||^2 = sum_{k != 0} |G u - f^|^2 (the spectral form of
        nrmp(ngrad_cam(phi))^2, LPsrc.cpp:119-173, by Parseval),
  phi' = IFFT(u') * N^3 (LPsrc.cpp:108).
Transforms are real-to-complex (rfftn / irfftn), which for real data equals the
reference's full C2C transform; u is kept as the half spectrum.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from . import spmiqc_np as npo

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cpu_point.c")
LIB = os.path.join(HERE, "_ref", "libcpupoint.so")
_lib = None


def build() -> str:
    """Compiles cpu_point.c (gcc, OpenMP) into oracle/_ref/ when it is missing or older."""
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    out = subprocess.run(["gcc", "-O3", "-march=x86-64-v2", "-fopenmp", "-fPIC", "-shared", SRC, "-o", LIB, "-lm"],
                         capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("cpu_point.c build failed:\n" + out.stderr)
    return LIB


def _load():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(build())
        dp = ctypes.c_void_p
        L.spm_cpu_real_pass.restype = ctypes.c_double
        L.spm_cpu_real_pass.argtypes = [dp, dp, ctypes.c_long, ctypes.c_double, ctypes.c_double]
        L.spm_cpu_spec_pass.restype = None
        L.spm_cpu_spec_pass.argtypes = [dp, dp, dp, dp, ctypes.c_int, ctypes.c_double, ctypes.c_double, dp]
        _lib = L
    return _lib


class MklFlow:
    def __init__(self, N: int, L: float = 26.0, Tau: float = -0.0061, Gamma: float = 0.30, dt: float = 0.3,
                 threads: int | None = None):
        import torch
        self.torch = torch
        if threads:
            torch.set_num_threads(int(threads))
            os.environ["OMP_NUM_THREADS"] = str(int(threads))
        self.threads = torch.get_num_threads()
        self.lib = _load()
        self.N, self.Tau, self.Gamma, self.dt = int(N), float(Tau), float(Gamma), float(dt)
        self.n3 = float(N) ** 3
        h = N // 2
        self.gtab = np.ascontiguousarray(npo.get_GK(np.arange(3 * h * h + 1, dtype=np.float64) / (L * L)))
        self.f = torch.empty((N, N, N), dtype=torch.float64)
        self.fh = torch.empty((N, N, h + 1), dtype=torch.complex128)
        self.sums = np.zeros(3)

    def spectrum(self, phi):
        """u = FFT(phi)/N^3 as the half spectrum (My_FFT.cpp:4-13)."""
        return self.torch.fft.rfftn(phi) / self.n3

    def step(self, phi, u):
        """One gradient step; returns (phi', u', E, res, ||grad F||). phi and u
        are replaced (new tensors are returned; the old ones are reused as
        the next step's buffers by the caller's rebinding)."""
        t, L = self.torch, self.lib
        E2 = L.spm_cpu_real_pass(phi.data_ptr(), self.f.data_ptr(), phi.numel(), self.Tau, self.Gamma) / self.n3
        t.fft.rfftn(self.f, out=self.fh)
        u1 = t.empty_like(u)
        L.spm_cpu_spec_pass(u.data_ptr(), self.fh.data_ptr(), u1.data_ptr(), self.gtab.ctypes.data, self.N, self.dt,
                            1.0 / self.n3, self.sums.ctypes.data)
        e1, res, g2 = (float(x) for x in self.sums)
        phi1 = t.fft.irfftn(u1, s=phi.shape, out=phi)
        phi1.mul_(self.n3)
        return phi1, u1, E2 + e1, res, float(np.sqrt(g2))
