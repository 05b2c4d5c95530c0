"""Python mirror of the C ABI of libspmiqc_cuda.so (include/spmiqc.h).

Method names follow the SPM-IQC routines they replace (get_Ene, get_min_u_F,
ngrad_cam, hv_cam, precond_camnew, my_fft, my_ifft, inpfp, ...). Device memory
comes from torch tensors (plumbing only): real fields are contiguous CUDA
tensors of shape (N, N, N) in the context's precision, packed spectra are
complex tensors of shape (N, N, N // 2).

There is no CPU fallback: if the library is missing or no GPU is visible the
constructor raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libspmiqc_cuda.so")

SPM_FP64, SPM_FP32, SPM_MIXED = 0, 1, 2
SPM_JOB_RELAX, SPM_JOB_LOBPCG, SPM_JOB_SPM = 0, 1, 2
SPM_ERR_ARG, SPM_ERR_CUDA, SPM_ERR_NOMEM, SPM_ERR_STATE, SPM_ERR_CANCELLED = 1, 2, 3, 6, 7
_vp = ctypes.c_void_p
_lib = None


class SpmError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"spmiqc status {status}: {msg}")
        self.status = status


class StepStats(ctypes.Structure):
    _fields_ = [("energy", ctypes.c_double), ("res", ctypes.c_double),
                ("grad_norm", ctypes.c_double), ("e1", ctypes.c_double)]


class JobDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("N", ctypes.c_int), ("precision", ctypes.c_int), ("k", ctypes.c_int),
                ("max_steps", ctypes.c_int), ("guard", ctypes.c_int), ("L", ctypes.c_double),
                ("Tau", ctypes.c_double), ("Gamma", ctypes.c_double), ("dt", ctypes.c_double),
                ("tol", ctypes.c_double), ("switch_tol", ctypes.c_double), ("seed", ctypes.c_uint64)]


class JobResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("steps", ctypes.c_int), ("energy", ctypes.c_double),
                ("residual", ctypes.c_double), ("evals", ctypes.c_double * 8), ("t_submit", ctypes.c_double),
                ("t_start", ctypes.c_double), ("t_end", ctypes.c_double), ("message", ctypes.c_char * 128)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("budget_bytes", ctypes.c_size_t), ("max_slots", ctypes.c_int), ("fake_device", ctypes.c_int),
                ("fake_ms_per_munit", ctypes.c_double), ("fake_device_bytes", ctypes.c_size_t),
                ("max_bypass", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_int64), ("failed", ctypes.c_int64), ("cancelled", ctypes.c_int64),
                ("pending", ctypes.c_int64), ("running", ctypes.c_int), ("peak_running", ctypes.c_int),
                ("peak_bytes", ctypes.c_size_t), ("budget_bytes", ctypes.c_size_t), ("p50_s", ctypes.c_double),
                ("p99_s", ctypes.c_double), ("elapsed_s", ctypes.c_double)]


def lib():
    """Loads libspmiqc_cuda.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is not built; run `python spm-iqc_b200/build.py`")
        L = ctypes.CDLL(LIB_PATH)
        sig = {
            "spm_ctx_create": [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                               ctypes.c_int, _vp, ctypes.POINTER(_vp)],
            "spm_ctx_destroy": [_vp],
            "spm_set_stream": [_vp, _vp],
            "spm_sync": [_vp],
            "spm_fft": [_vp, _vp, _vp],
            "spm_ifft": [_vp, _vp, _vp],
            "spm_spectrum_to_full": [_vp, _vp, _vp],
            "spm_spectrum_from_full": [_vp, _vp, _vp],
            "spm_energy": [_vp, _vp, _vp, ctypes.POINTER(ctypes.c_double)],
            "spm_grad_flow": [_vp, _vp, _vp, ctypes.c_int, ctypes.c_double, ctypes.POINTER(StepStats),
                              ctypes.POINTER(ctypes.c_int)],
            "spm_ngrad": [_vp, _vp, _vp, ctypes.POINTER(ctypes.c_double)],
            "spm_hv": [_vp, _vp, _vp, _vp, ctypes.c_int],
            "spm_precond": [_vp, _vp, ctypes.c_int],
            "spm_inpfp": [_vp, _vp, _vp, ctypes.POINTER(ctypes.c_double)],
            "spm_block_gram": [_vp, ctypes.POINTER(_vp), ctypes.c_int, ctypes.POINTER(_vp), ctypes.c_int,
                               ctypes.POINTER(ctypes.c_double)],
            "spm_block_combine": [_vp, ctypes.POINTER(_vp), ctypes.c_int, ctypes.POINTER(_vp), ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)],
            "spm_supported_size": [ctypes.c_int],
            "spm_lobpcg_init": [_vp, _vp, ctypes.c_int, ctypes.c_uint64],
            "spm_lobpcg": [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                           ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                           ctypes.POINTER(ctypes.c_int)],
            "spm_get_tv": [_vp, _vp, _vp, _vp],
            "spm_natural_forces": [_vp, _vp, _vp],
            "spm_minmax_forces": [_vp, _vp, _vp],
            "spm_spring_pairing": [_vp, _vp, _vp, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_int)],
            "spm_spring_pairing_mixed": [_vp, _vp, _vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_int)],
            "spm_server_create": [ctypes.POINTER(ServerConfig), ctypes.POINTER(_vp)],
            "spm_server_submit": [_vp, ctypes.POINTER(JobDesc), _vp, _vp, ctypes.POINTER(ctypes.c_int64)],
            "spm_server_cancel": [_vp, ctypes.c_int64],
            "spm_server_wait": [_vp, ctypes.c_int64, ctypes.c_int, ctypes.POINTER(JobResult), _vp],
            "spm_server_release": [_vp, ctypes.c_int64],
            "spm_server_get_stats": [_vp, ctypes.POINTER(ServerStats)],
            "spm_server_destroy": [_vp],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        L.spm_last_error.restype = ctypes.c_char_p
        L.spm_status_str.restype = ctypes.c_char_p
        L.spm_status_str.argtypes = [ctypes.c_int]
        L.spm_field_bytes.restype = ctypes.c_size_t
        L.spm_field_bytes.argtypes = [_vp]
        L.spm_job_footprint.restype = ctypes.c_size_t
        L.spm_job_footprint.argtypes = [ctypes.POINTER(JobDesc)]
        L.spm_launch_count.restype = ctypes.c_uint64
        L.spm_launch_count.argtypes = [_vp]
        _lib = L
    return _lib


def check(status: int):
    if status != 0:
        raise SpmError(status, lib().spm_last_error().decode())


def _ptr(t) -> int:
    return t.data_ptr()


class SpmContext:
    """One grid + model parameters on one CUDA device (the reference's globals)."""

    def __init__(self, N: int, L: float = 26.0, Tau: float = -0.0061, Gamma: float = 0.30, dt: float = 0.3,
                 precision: str = "fp64", stream=None):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("spmiqc needs a CUDA device (no CPU path)")
        self.torch = torch
        self.N = int(N)
        self.L, self.Tau, self.Gamma, self.dt = float(L), float(Tau), float(Gamma), float(dt)
        self.precision = precision
        self.prec = SPM_FP64 if precision == "fp64" else SPM_FP32
        self.rdtype = torch.float64 if self.prec == SPM_FP64 else torch.float32
        self.cdtype = torch.complex128 if self.prec == SPM_FP64 else torch.complex64
        h = _vp()
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        check(lib().spm_ctx_create(self.N, self.L, self.Tau, self.Gamma, self.dt, self.prec, _vp(s),
                                   ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().spm_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- buffers
    def field(self, nb: int | None = None):
        shape = (self.N,) * 3 if nb is None else (nb,) + (self.N,) * 3
        return self.torch.zeros(shape, dtype=self.rdtype, device="cuda")

    def spectrum(self):
        return self.torch.zeros((self.N, self.N, self.N // 2), dtype=self.cdtype, device="cuda")

    def launches(self) -> int:
        return int(lib().spm_launch_count(self.h))

    def sync(self):
        check(lib().spm_sync(self.h))

    # ---- My_FFT.cpp
    def my_fft(self, x, xhat=None):
        xhat = self.spectrum() if xhat is None else xhat
        check(lib().spm_fft(self.h, _ptr(x), _ptr(xhat)))
        return xhat

    def my_ifft(self, xhat, x=None):
        x = self.field() if x is None else x
        check(lib().spm_ifft(self.h, _ptr(xhat), _ptr(x)))
        return x

    def to_full(self, xhat):
        full = self.torch.zeros((self.N,) * 3, dtype=self.torch.complex128, device="cuda")
        check(lib().spm_spectrum_to_full(self.h, _ptr(xhat), _ptr(full)))
        return full

    def from_full(self, full):
        xhat = self.spectrum()
        full = full.to(self.torch.complex128).contiguous()
        check(lib().spm_spectrum_from_full(self.h, _ptr(full), _ptr(xhat)))
        return xhat

    # ---- LPsrc.cpp
    def get_Ene(self, phi, uhat) -> float:
        e = ctypes.c_double()
        check(lib().spm_energy(self.h, _ptr(phi), _ptr(uhat), ctypes.byref(e)))
        return e.value

    def get_min_u_F(self, phi, uhat, max_steps: int, tol_grad: float = 0.0):
        """Runs up to max_steps gradient steps in place; returns an (n, 4) array
        of per-step (energy, res, ||grad F||, E1)."""
        st = (StepStats * max(1, max_steps))()
        n = ctypes.c_int()
        check(lib().spm_grad_flow(self.h, _ptr(phi), _ptr(uhat), int(max_steps), float(tol_grad), st,
                                  ctypes.byref(n)))
        return np.array([[s.energy, s.res, s.grad_norm, s.e1] for s in st[:n.value]]).reshape(-1, 4)

    def get_min_u_F_mixed(self, phi, uhat, max_steps: int, tol_grad: float, switch_tol: float = 0.0):
        """FP32 flow to switch_tol (0: as far as FP32 goes), then FP64 polish to tol_grad (FP64 context).
        Returns (stats (n, 4), steps_fp32, steps_fp64)."""
        st = (StepStats * max(1, max_steps))()
        a, b = ctypes.c_int(), ctypes.c_int()
        f = lib().spm_grad_flow_mixed
        f.argtypes = [_vp, _vp, _vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.POINTER(StepStats),
                      ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        check(f(self.h, _ptr(phi), _ptr(uhat), int(max_steps), float(tol_grad), float(switch_tol), st,
                ctypes.byref(a), ctypes.byref(b)))
        n = a.value + b.value
        return np.array([[s.energy, s.res, s.grad_norm, s.e1] for s in st[:n]]).reshape(-1, 4), a.value, b.value

    def tune(self, knob: str, value: int):
        f = lib().spm_tune
        f.argtypes = [_vp, ctypes.c_char_p, ctypes.c_int]
        check(f(self.h, knob.encode(), int(value)))

    def autotune(self, steps: int = 20):
        """spm_autotune: times the candidate schedules, keeps the fastest; returns (plane_cps, fuse_planes)."""
        f = lib().spm_autotune
        f.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        a, b = ctypes.c_int(), ctypes.c_int()
        check(f(self.h, int(steps), ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def tuning(self) -> dict:
        """The current values of the tuning knobs (spm_tune_get)."""
        f = lib().spm_tune_get
        f.argtypes = [_vp, ctypes.c_char_p]
        return {k: int(f(self.h, k.encode())) for k in ("plane_cps", "fuse_planes", "plane_xg", "pencil_tc", "pdl")}

    def ngrad_cam(self, phi, grad=None):
        grad = self.field() if grad is None else grad
        nrm = ctypes.c_double()
        check(lib().spm_ngrad(self.h, _ptr(phi), _ptr(grad), ctypes.byref(nrm)))
        return grad, nrm.value

    # ---- LOBPCG.cpp
    def hv_cam(self, phi, v, hv=None):
        """v: (N,N,N) or (nb,N,N,N); returns H v with the same shape."""
        hv = self.torch.empty_like(v) if hv is None else hv
        nb = 1 if v.dim() == 3 else v.shape[0]
        check(lib().spm_hv(self.h, _ptr(phi), _ptr(v), _ptr(hv), nb))
        return hv

    def precond_camnew(self, w):
        nb = 1 if w.dim() == 3 else w.shape[0]
        check(lib().spm_precond(self.h, _ptr(w), nb))
        return w

    def hiosd_lobpcg_initialization(self, k: int, seed: int = 0):
        """Random mean-free orthonormal start block, shape (k, N, N, N)."""
        V = self.field(k)
        check(lib().spm_lobpcg_init(self.h, _ptr(V), int(k), ctypes.c_uint64(seed)))
        return V

    def hiosd_lobpcg_inip(self, phi, V, maxiter: int = 21, tol: float = 0.0):
        """maxiter LOBPCG iterations on V (k, N, N, N) in place; returns
        (evals, residuals, iterations)."""
        k = V.shape[0]
        ev = (ctypes.c_double * k)()
        rs = (ctypes.c_double * k)()
        it = ctypes.c_int()
        check(lib().spm_lobpcg(self.h, _ptr(phi), _ptr(V), int(k), int(maxiter), float(tol), ev, rs,
                               ctypes.byref(it)))
        return np.array(ev[:]), np.array(rs[:]), it.value

    def lobpcg_guarded(self, phi, V, k: int, maxiter: int = 400, tol: float = 1e-8):
        """LOBPCG on the whole block V (k + guard fields) stopping when the first
        k residuals are <= tol; returns (evals, residuals, iterations) of the
        whole block."""
        kb = V.shape[0]
        ev = (ctypes.c_double * kb)()
        rs = (ctypes.c_double * kb)()
        it = ctypes.c_int()
        f = lib().spm_lobpcg_guarded
        f.argtypes = [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                      ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
        check(f(self.h, _ptr(phi), _ptr(V), int(k), int(kb - k), int(maxiter), float(tol), ev, rs, ctypes.byref(it)))
        return np.array(ev[:]), np.array(rs[:]), it.value

    # ---- SPM.cpp
    def hiosd_lobpcg_sieh(self, x, V, dt: float = 0.8, betat: float = 8.0, betau: float = 0.02,
                          epsf: float = 1e-7, maxiter: int = 10000):
        """HiSD (HISD.cpp:86-485) on (x, V) in place; returns the ||grad F|| history."""
        f = lib().spm_hisd
        f.argtypes = [_vp, _vp, _vp, ctypes.c_int] + [ctypes.c_double] * 4 + \
            [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
        hist = (ctypes.c_double * max(1, maxiter))()
        it = ctypes.c_int()
        k = V.shape[0] if V.dim() == 4 else 1
        check(f(self.h, _ptr(x), _ptr(V), k, float(dt), float(betat), float(betau), float(epsf), int(maxiter),
                hist, ctypes.byref(it)))
        return np.array(hist[:it.value])

    def hiosd_lobpcg_sieh_V0(self, x, V, V0, dt: float = 0.8, betat: float = 8.0, betau: float = 1.3,
                             epsf: float = 1e-9, maxiter: int = 40000):
        """GOSD (GOSD.cpp:123-531): HiSD with V kept orthogonal to the fixed fields V0; returns the history."""
        f = lib().spm_gosd
        f.argtypes = [_vp, _vp, _vp, ctypes.c_int, _vp, ctypes.c_int] + [ctypes.c_double] * 4 + \
            [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
        hist = (ctypes.c_double * max(1, maxiter))()
        it = ctypes.c_int()
        k = V.shape[0] if V.dim() == 4 else 1
        k0 = V0.shape[0] if V0.dim() == 4 else 1
        check(f(self.h, _ptr(x), _ptr(V), k, _ptr(V0), k0, float(dt), float(betat), float(betau), float(epsf),
                int(maxiter), hist, ctypes.byref(it)))
        return np.array(hist[:it.value])

    def get_Tv(self, phi0, phi1, v=None):
        v = self.field() if v is None else v
        check(lib().spm_get_tv(self.h, _ptr(phi0), _ptr(phi1), _ptr(v)))
        return v

    def Natural_Forces(self, x, v):
        check(lib().spm_natural_forces(self.h, _ptr(x), _ptr(v)))
        return x

    def MinMax_Forces(self, x, v):
        check(lib().spm_minmax_forces(self.h, _ptr(x), _ptr(v)))
        return x

    def set_spring_length(self, rest: float):
        """Rest length of the SPM spring (0: the reference's zero-length spring)."""
        f = lib().spm_set_spring_length
        f.argtypes = [_vp, ctypes.c_double]
        check(f(self.h, float(rest)))

    def Spring_Pairing(self, phi0, phi1, maxiter: int, tol: float):
        """Runs the spring pair iteration in place; returns the residual history."""
        hist = (ctypes.c_double * max(1, maxiter))()
        it = ctypes.c_int()
        check(lib().spm_spring_pairing(self.h, _ptr(phi0), _ptr(phi1), int(maxiter), float(tol), hist,
                                       ctypes.byref(it)))
        return np.array(hist[:it.value])

    def Spring_Pairing_mixed(self, phi0, phi1, maxiter: int, tol: float, switch_tol: float = 0.0):
        """FP32 iterations to switch_tol, then FP64 to tol; returns (history, fp32 iterations, fp64 iterations)."""
        hist = (ctypes.c_double * max(1, maxiter))()
        a, b = ctypes.c_int(), ctypes.c_int()
        check(lib().spm_spring_pairing_mixed(self.h, _ptr(phi0), _ptr(phi1), int(maxiter), float(tol),
                                             float(switch_tol), hist, ctypes.byref(a), ctypes.byref(b)))
        return np.array(hist[:a.value + b.value]), a.value, b.value

    def initial_field(self, path: str, l: float, phi=None):
        """get_initial_value of an initData file (shell scale l): phi = Re(my_ifft(u_F))."""
        phi = self.field() if phi is None else phi
        f = lib().spm_initial_field
        f.argtypes = [_vp, ctypes.c_char_p, ctypes.c_double, _vp]
        check(f(self.h, path.encode(), float(l), _ptr(phi)))
        return phi

    # ---- BasicOperators.cpp
    def inpfp(self, p, q) -> float:
        out = ctypes.c_double()
        check(lib().spm_inpfp(self.h, _ptr(p), _ptr(q), ctypes.byref(out)))
        return out.value

    def nrmp(self, p) -> float:
        return float(np.sqrt(self.inpfp(p, p)))

    def block_gram(self, X, Y) -> np.ndarray:
        """G[a, b] = inpfp(X[a], Y[b]) for sequences of fields X, Y (at most 24 each;
        fields may repeat and be shared between X and Y), the LOBPCG Gram."""
        X, Y = list(X), list(Y)
        xa = (_vp * len(X))(*[_ptr(f) for f in X])
        ya = (_vp * len(Y))(*[_ptr(f) for f in Y])
        G = np.zeros((len(X), len(Y)), dtype=np.float64)
        check(lib().spm_block_gram(self.h, xa, len(X), ya, len(Y),
                                   G.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return G

    def block_combine(self, X, Y, C, d=None):
        """Y[q] = sum_p C[p, q] X[p] + d[q] in place on the fields Y (which may be
        fields of X), the LOBPCG block update; C is len(X) x len(Y)."""
        X, Y = list(X), list(Y)
        C = np.ascontiguousarray(C, dtype=np.float64)
        assert C.shape == (len(X), len(Y))
        xa = (_vp * len(X))(*[_ptr(f) for f in X])
        ya = (_vp * len(Y))(*[_ptr(f) for f in Y])
        dp = None
        if d is not None:
            d = np.ascontiguousarray(d, dtype=np.float64)
            dp = d.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        check(lib().spm_block_combine(self.h, xa, len(X), ya, len(Y),
                                      C.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), dp))


_KINDS = {"relax": SPM_JOB_RELAX, "lobpcg": SPM_JOB_LOBPCG, "spm": SPM_JOB_SPM}
_PRECS = {"fp64": SPM_FP64, "fp32": SPM_FP32, "mixed": SPM_MIXED}


def job_desc(kind: str, N: int, precision: str = "fp64", k: int = 4, max_steps: int = 1000, L: float = 26.0,
             Tau: float = -0.0061, Gamma: float = 0.30, dt: float = 0.3, tol: float = 1e-8,
             switch_tol: float = 0.0, seed: int = 0, guard: int = 0) -> JobDesc:
    """guard: LOBPCG guard vectors (k + guard <= 8), see lobpcg_guarded."""
    return JobDesc(_KINDS[kind], int(N), _PRECS[precision], int(k), int(max_steps), int(guard), float(L),
                   float(Tau), float(Gamma), float(dt), float(tol), float(switch_tol), int(seed))


def job_footprint(desc: JobDesc) -> int:
    return int(lib().spm_job_footprint(ctypes.byref(desc)))


class JobServer:
    """The library's job server (spm_server_*): jobs of mixed kinds and grid
    sizes admitted by device-memory footprint into max_slots concurrent slots.
    fake_device=True runs the scheduler without a GPU (jobs sleep
    fake_ms_per_munit ms per million grid points per step)."""

    def __init__(self, budget_bytes: int = 0, max_slots: int = 4, fake_device: bool = False,
                 fake_ms_per_munit: float = 0.0, fake_device_bytes: int = 0, max_bypass: int = 0):
        if not fake_device:
            import torch
            if not torch.cuda.is_available():
                raise RuntimeError("spmiqc needs a CUDA device (no CPU path)")
        cfg = ServerConfig(int(budget_bytes), int(max_slots), int(bool(fake_device)), float(fake_ms_per_munit),
                           int(fake_device_bytes), int(max_bypass))
        h = _vp()
        check(lib().spm_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self.sizes = {}

    def submit(self, desc: JobDesc, phi0: np.ndarray, phi1: np.ndarray | None = None) -> int:
        p0 = np.ascontiguousarray(phi0, dtype=np.float64)
        p1 = None if phi1 is None else np.ascontiguousarray(phi1, dtype=np.float64)
        jid = ctypes.c_int64()
        check(lib().spm_server_submit(self.h, ctypes.byref(desc), p0.ctypes.data,
                                      None if p1 is None else p1.ctypes.data, ctypes.byref(jid)))
        n = desc.N ** 3
        self.sizes[jid.value] = (desc.k * n if desc.kind == SPM_JOB_LOBPCG else n, desc.N)
        return jid.value

    def cancel(self, jid: int):
        check(lib().spm_server_cancel(self.h, int(jid)))

    def wait(self, jid: int, block: bool = True, field: bool = True):
        """Returns (JobResult, field or None), or None if the job is unfinished (block=False)."""
        res = JobResult()
        cnt, N = self.sizes[jid]
        out = np.empty(cnt, dtype=np.float64) if field else None
        st = lib().spm_server_wait(self.h, int(jid), int(block), ctypes.byref(res),
                                   None if out is None else out.ctypes.data)
        if st == SPM_ERR_STATE and not block:
            return None
        check(st)
        if out is not None and res.status == 0:
            out = out.reshape((-1, N, N, N)) if cnt != N ** 3 else out.reshape((N, N, N))
        elif out is not None:
            out = None
        return res, out

    def release(self, jid: int):
        check(lib().spm_server_release(self.h, int(jid)))
        self.sizes.pop(jid, None)

    def stats(self) -> ServerStats:
        s = ServerStats()
        check(lib().spm_server_get_stats(self.h, ctypes.byref(s)))
        return s

    def close(self):
        if getattr(self, "h", None):
            lib().spm_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- field files
def save_field_txt(path: str, x) -> None:
    """Save_phi / Save_Option_V format ("%.16e \\n" per value) from a host array."""
    a = np.ascontiguousarray(x, dtype=np.float64)
    f = lib().spm_save_field_txt
    f.argtypes = [ctypes.c_char_p, _vp, ctypes.c_size_t]
    check(f(path.encode(), a.ctypes.data, a.size))


def load_field_txt(path: str, count: int) -> np.ndarray:
    out = np.empty(int(count), dtype=np.float64)
    f = lib().spm_load_field_txt
    f.argtypes = [ctypes.c_char_p, _vp, ctypes.c_size_t]
    check(f(path.encode(), out.ctypes.data, out.size))
    return out


class CheckpointInfo(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int), ("nfields", ctypes.c_int), ("precision", ctypes.c_int),
                ("L", ctypes.c_double), ("Tau", ctypes.c_double), ("Gamma", ctypes.c_double),
                ("dt", ctypes.c_double), ("step", ctypes.c_int64)]


def save_checkpoint(path: str, fields, L: float, Tau: float, Gamma: float, dt: float, step: int = 0,
                    precision: int = SPM_FP64) -> None:
    a = np.ascontiguousarray(fields, dtype=np.float64)
    N = a.shape[-1]
    info = CheckpointInfo(N, a.size // N ** 3, precision, L, Tau, Gamma, dt, step)
    f = lib().spm_checkpoint_save
    f.argtypes = [ctypes.c_char_p, _vp, _vp]
    check(f(path.encode(), ctypes.byref(info), a.ctypes.data))


def load_checkpoint(path: str):
    """Returns (info, fields of shape (nfields, N, N, N))."""
    info = CheckpointInfo()
    f = lib().spm_checkpoint_load
    f.argtypes = [ctypes.c_char_p, _vp, _vp, ctypes.c_size_t]
    check(f(path.encode(), ctypes.byref(info), None, 0))
    out = np.empty((info.nfields, info.N, info.N, info.N))
    check(f(path.encode(), ctypes.byref(info), out.ctypes.data, out.size))
    return info, out


def batch_grad_flow(ctxs, phis, uhats, max_steps: int, tol_grad: float, switch_tol: float = 0.0,
                    steps_per_launch: int = 16):
    """spm_batch_grad_flow: all instances advanced by one captured graph per launch; returns the steps per instance."""
    n = len(ctxs)
    f = lib().spm_batch_grad_flow
    arr = ctypes.c_void_p * n
    f.argtypes = [arr, arr, arr, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                  ctypes.POINTER(ctypes.c_int)]
    done = (ctypes.c_int * n)()
    check(f(arr(*[c.h.value for c in ctxs]), arr(*[_ptr(p) for p in phis]), arr(*[_ptr(u) for u in uhats]), n,
            int(max_steps), float(tol_grad), float(switch_tol), int(steps_per_launch), done))
    return list(done)
