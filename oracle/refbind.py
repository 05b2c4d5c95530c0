"""ctypes binding of the compiled reference (oracle/_ref/libspmref.so).

TEST INFRASTRUCTURE ONLY: the reference's own src/*.cpp built unchanged against
the shims in oracle/shim (see oracle/Makefile and oracle/ref_harness.cpp).
Tests, __graft_entry__.smoke() and bench.py's CPU baseline / reference arm use
it as the checker or the timed CPU reference; the product never loads it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libspmref.so")
# the same harness with the hot-path routines resolved to the GPU compat layer
COMPAT_LIB = os.path.join(HERE, "_ref", "libspmref_compat.so")
# The reference checkout: $SPMIQC_REFERENCE, else a directory named
# "reference" beside this repository.
REFDIR_DEFAULT = os.environ.get("SPMIQC_REFERENCE") or os.path.join(os.path.dirname(os.path.dirname(HERE)),
                                                                    "reference")

_dp = ctypes.POINTER(ctypes.c_double)
_libs = {}


def build(refdir: str = REFDIR_DEFAULT, quiet: bool = True) -> bool:
    """Compile the oracle with its Makefile when the reference tree is present."""
    if not os.path.isdir(os.path.join(refdir, "src")):
        return os.path.exists(LIB)
    out = subprocess.run(["make", "-C", HERE, f"REFDIR={refdir}"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    return True


def build_compat(refdir: str = REFDIR_DEFAULT) -> bool:
    """Compile the drop-in check library (needs the CUDA library built)."""
    if not os.path.isdir(os.path.join(refdir, "src")):
        return os.path.exists(COMPAT_LIB)
    out = subprocess.run(["make", "-C", HERE, f"REFDIR={refdir}", "compat"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("compat harness build failed:\n" + out.stdout + out.stderr)
    return True


def available(path: str = LIB) -> bool:
    return os.path.exists(path)


def lib(path: str = LIB):
    if path not in _libs:
        if not available(path):
            raise FileNotFoundError(path)
        L = ctypes.CDLL(path)
        L.ref_setup.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.ref_get_Ene.restype = ctypes.c_double
        L.ref_inpfp.restype = ctypes.c_double
        L.ref_rayleighq.restype = ctypes.c_double
        L.ref_get_GK.restype = ctypes.c_double
        L.ref_get_GK.argtypes = [ctypes.c_double]
        L.ref_lobpcg_init.argtypes = [ctypes.c_int, ctypes.c_uint64, _dp]
        L.ref_lobpcg_inip.argtypes = [_dp, ctypes.c_int, ctypes.c_int, _dp]
        L.ref_spring_pairing.argtypes = [_dp, _dp, ctypes.c_double, ctypes.c_double]
        L.ref_save_phi.argtypes = [_dp, ctypes.c_char_p]
        L.ref_load_phi.argtypes = [ctypes.c_char_p, _dp]
        L.ref_save_option_v.argtypes = [ctypes.c_int, _dp, ctypes.c_char_p]
        L.ref_load_option_v.argtypes = [ctypes.c_int, ctypes.c_char_p, _dp]
        L.ref_initial_value.argtypes = [ctypes.c_int, ctypes.c_char_p, _dp]
        L.ref_hisd.argtypes = [_dp, ctypes.c_int, _dp] + [ctypes.c_double] * 4 + [ctypes.c_int]
        L.ref_gosd.argtypes = [_dp, ctypes.c_int, _dp, ctypes.c_int, _dp] + [ctypes.c_double] * 4 + [ctypes.c_int]
        _libs[path] = L
    return _libs[path]


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


class Ref:
    """One configured reference instance (the reference keeps its state in globals)."""

    def __init__(self, N, L=26.0, Tau=-0.0061, Gamma=0.30, dt=0.3, threads=1, path=LIB):
        self.N, self.n3 = N, N ** 3
        self.L = lib(path)
        self.L.ref_set_threads(int(threads))
        if self.L.ref_setup(N, L, Tau, Gamma, dt) != 0:
            raise ValueError("ref_setup failed")

    def set_threads(self, n):
        """Host threads of the shim FFT (1: serial)."""
        self.L.ref_set_threads(int(n))

    def _z(self, k=1):
        return np.zeros((k, self.N, self.N, self.N)) if k > 1 else np.zeros((self.N,) * 3)

    def tables(self):
        G, ik = self._z(), self._z()
        self.L.ref_get_tables(_p(G), _p(ik))
        return G, ik

    def set_state(self, phi, uF=None):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        if uF is None:
            self.L.ref_set_state(_p(phi))
        else:
            uFi = np.ascontiguousarray(np.stack([uF.real, uF.imag], axis=-1))
            self.L.ref_set_state2(_p(phi), _p(uFi))

    def get_state(self):
        phi = self._z()
        uFi = np.zeros((self.N, self.N, self.N, 2))
        self.L.ref_get_state(_p(phi), _p(uFi))
        return phi, uFi[..., 0] + 1j * uFi[..., 1]

    def energy(self):
        return self.L.ref_get_Ene()

    def grad_steps(self, n):
        E, res, g = np.zeros(n), np.zeros(n), np.zeros(n)
        self.L.ref_grad_steps(n, _p(E), _p(res), _p(g))
        return E, res, g

    def get_min_u_F(self, maxit):
        self.L.ref_get_min_u_F(int(maxit))

    def ngrad(self, phi):
        out = self._z()
        self.L.ref_ngrad(_p(np.ascontiguousarray(phi)), _p(out))
        return out

    def hv(self, phi, v):
        out = self._z()
        self.L.ref_hv(_p(np.ascontiguousarray(phi)), _p(np.ascontiguousarray(v)), _p(out))
        return out

    def precond(self, w):
        w = np.array(w, dtype=np.float64, order="C")
        self.L.ref_precond(_p(w))
        return w

    def inpfp(self, p, q):
        return self.L.ref_inpfp(_p(np.ascontiguousarray(p)), _p(np.ascontiguousarray(q)))

    def rayleigh(self, phi, v):
        return self.L.ref_rayleighq(_p(np.ascontiguousarray(phi)), _p(np.ascontiguousarray(v)))

    def lobpcg_init(self, k, seed):
        V = self._z(k) if k > 1 else np.zeros((1, self.N, self.N, self.N))
        self.L.ref_lobpcg_init(k, seed, _p(V))
        return V

    def lobpcg_inip(self, phi, V, maxiter=21):
        V = np.array(V, dtype=np.float64, order="C")
        self.L.ref_lobpcg_inip(_p(np.ascontiguousarray(phi)), V.shape[0], int(maxiter), _p(V))
        return V

    def tangent(self, phi0, phi1):
        out = self._z()
        self.L.ref_get_Tv(_p(np.ascontiguousarray(phi0)), _p(np.ascontiguousarray(phi1)), _p(out))
        return out

    def natural_forces(self, x, v):
        x = np.array(x, dtype=np.float64, order="C")
        self.L.ref_natural_forces(_p(x), _p(np.ascontiguousarray(v)))
        return x

    def minmax_forces(self, x, v):
        x = np.array(x, dtype=np.float64, order="C")
        self.L.ref_minmax_forces(_p(x), _p(np.ascontiguousarray(v)))
        return x

    def spring_pairing(self, phi0, phi1, maxiter, tol):
        a = np.array(phi0, dtype=np.float64, order="C")
        b = np.array(phi1, dtype=np.float64, order="C")
        self.L.ref_spring_pairing(_p(a), _p(b), float(maxiter), float(tol))
        return a, b

    def hisd(self, x, V, dt=0.8, betat=8.0, betau=0.02, epsf=1e-7, maxiter=10000):
        """hiosd_lobpcg_sieh on copies of (x, V); returns the updated pair."""
        x = np.array(x, dtype=np.float64, order="C")
        V = np.array(V, dtype=np.float64, order="C")
        self.L.ref_hisd(_p(x), V.shape[0], _p(V), dt, betat, betau, epsf, int(maxiter))
        return x, V

    def gosd(self, x, V, V0, dt=0.8, betat=8.0, betau=1.3, epsf=1e-9, maxiter=40000):
        """hiosd_lobpcg_sieh_V0 on copies of (x, V) with the fixed fields V0."""
        x = np.array(x, dtype=np.float64, order="C")
        V = np.array(V, dtype=np.float64, order="C")
        V0 = np.ascontiguousarray(V0, dtype=np.float64)
        self.L.ref_gosd(_p(x), V.shape[0], _p(V), V0.shape[0], _p(V0), dt, betat, betau, epsf, int(maxiter))
        return x, V

    # File_Op.cpp: the reference's field files
    def save_phi(self, phi, path):
        self.L.ref_save_phi(_p(np.ascontiguousarray(phi, dtype=np.float64)), path.encode())

    def load_phi(self, path):
        phi = self._z()
        self.L.ref_load_phi(path.encode(), _p(phi))
        return phi

    def save_option_v(self, V, path):
        V = np.ascontiguousarray(V, dtype=np.float64)
        self.L.ref_save_option_v(V.shape[0], _p(V), path.encode())

    def load_option_v(self, k, path):
        V = self._z(k) if k > 1 else self._z()[None]
        V = np.ascontiguousarray(V.reshape(k, self.N, self.N, self.N))
        self.L.ref_load_option_v(k, path.encode(), _p(V))
        return V

    def initial_value(self, choice, root):
        """get_initial_value: u_F of phase `choice` read from root/initData."""
        u = np.zeros((self.N, self.N, self.N, 2))
        if self.L.ref_initial_value(int(choice), root.encode(), _p(u)) != 0:
            raise OSError("initial value: cannot enter " + root)
        return u[..., 0] + 1j * u[..., 1]

    def close(self):
        self.L.ref_teardown()
