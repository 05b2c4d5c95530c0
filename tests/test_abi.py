"""The C ABI library loads and exports every function its headers declare (no
GPU calls), and the host-side helpers behave (no GPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "spm-iqc_b200", "lib")


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(spm_\w+)\s*\(", text)))


def test_cuda_library_exports_every_declared_symbol():
    lib = os.path.join(LIBDIR, "libspmiqc_cuda.so")
    if not os.path.exists(lib):
        pytest.skip("library not built")
    L = ctypes.CDLL(lib)
    names = declared("spmiqc.h")
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    L.spm_status_str.restype = ctypes.c_char_p
    assert L.spm_status_str(0) == b"ok"
    assert L.spm_supported_size(256) == 1 and L.spm_supported_size(100) == 0


COMPAT_SIGNATURES = {
    "my_fft(double (*) [2], double (*) [2])", "my_ifft(double (*) [2], double (*) [2])", "My_mpi_fft_set_up()",
    "get_Ene()", "get_min_u_F()", "ngrad_cam(double (*) [2], double (*) [2])",
    "hv_cam(double (*) [2], double (*) [2], double (*) [2])", "precond_camnew(double (*) [2])",
    "hiosd_lobpcg_initialization(Option*, int)", "hiosd_lobpcg_inip(double (*) [2], Option*)",
    "copy_option_V(Option*, Option*, int)", "copy_option_V(double (**) [2], Option*, int)",
    "copy_option_V(double (*) [2], Option*, int)",
    "get_Tv(double (**) [2], double (*) [2])", "Natural_Forces(double (*) [2], double (*) [2])",
    "MinMax_Forces(double (*) [2], double (*) [2])", "Spring_Pairing(double (**) [2], double, double)",
    "Gs_gri_nuc(double (*) [2], double (*) [2])",
}


def test_compat_library_exports_the_reference_signatures():
    """Every C++ function of the reference's My_FFT / LPsrc / LOBPCG / SPM
    objects is defined, with the same mangled name, by the drop-in."""
    import shutil
    import subprocess
    lib = os.path.join(LIBDIR, "libspmiqc_compat.so")
    if not os.path.exists(lib) or not shutil.which("nm"):
        pytest.skip("compat library or nm missing")
    out = subprocess.run(["nm", "-D", "-C", "--defined-only", lib], capture_output=True, text=True).stdout
    have = {line.split(" ", 2)[2].strip() for line in out.splitlines() if " T " in line}
    missing = COMPAT_SIGNATURES - have
    assert not missing, missing


def test_context_rejects_bad_arguments_without_gpu_work():
    lib = os.path.join(LIBDIR, "libspmiqc_cuda.so")
    if not os.path.exists(lib):
        pytest.skip("library not built")
    L = ctypes.CDLL(lib)
    L.spm_ctx_create.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    h = ctypes.c_void_p()
    assert L.spm_ctx_create(100, 26.0, -0.0061, 0.3, 0.3, 0, None, ctypes.byref(h)) == 5  # unsupported size
    assert L.spm_ctx_create(64, -1.0, -0.0061, 0.3, 0.3, 0, None, ctypes.byref(h)) == 1   # bad L
    assert L.spm_ctx_create(64, 26.0, -0.0061, 0.3, 0.3, 7, None, ctypes.byref(h)) == 5   # bad precision


def test_icosahedral_shell():
    import inputs
    s = inputs.icosahedral_shell()
    assert s.shape == (30, 3)
    norms = np.linalg.norm(s, axis=1)
    assert np.all(np.abs(norms - 26.0) < 0.05)
    assert len({tuple(x) for x in s}) == 30
    assert len({tuple(x) for x in inputs.bcc_shell(26.0)}) == 12
    assert len({tuple(x) for x in inputs.fcc_shell(26.0)}) == 8


def test_generators_are_deterministic():
    import inputs
    a = inputs.cosine_shell(16, inputs.icosahedral_shell(), seed=3)
    b = inputs.cosine_shell(16, inputs.icosahedral_shell(), seed=3)
    assert np.array_equal(a, b)
    u = inputs.uniform(16, 4)
    assert abs(u.mean()) < 1e-15 and u.max() <= 0.1 + 1e-3 and u.min() >= -0.1 - 1e-3
