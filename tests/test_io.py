"""Field files, checkpoints and initData (CPU, no GPU): the library's writers
and readers against the reference's own File_Op.cpp and get_initial_value
(compiled in the oracle), byte for byte where the format is text."""
import ctypes
import os

import numpy as np
import pytest

from oracle import refbind
from oracle import spmiqc_np as npo

REFROOT = refbind.REFDIR_DEFAULT


@pytest.fixture(scope="module")
def lib():
    import spmiqc
    L = spmiqc.lib()
    L.spm_save_field_txt.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t]
    L.spm_load_field_txt.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t]
    L.spm_checkpoint_save.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p]
    L.spm_checkpoint_load.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]
    L.spm_initdata_spectrum.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_void_p]
    return L


class CkInfo(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int), ("nfields", ctypes.c_int), ("precision", ctypes.c_int),
                ("L", ctypes.c_double), ("Tau", ctypes.c_double), ("Gamma", ctypes.c_double),
                ("dt", ctypes.c_double), ("step", ctypes.c_int64)]


def _ref(N):
    if not refbind.available():
        pytest.skip("compiled reference not built")
    return refbind.Ref(N)


def test_field_file_matches_reference_bytes(lib, tmp_path):
    N = 16
    phi = npo.uniform_field(N, 3) * 1e3  # a range of exponents
    phi.flat[5] = 0.0
    phi.flat[6] = -1e-300
    ours, theirs = str(tmp_path / "ours.txt"), str(tmp_path / "ref.txt")
    assert lib.spm_save_field_txt(ours.encode(), phi.ctypes.data, phi.size) == 0
    r = _ref(N)
    r.save_phi(phi, theirs)
    assert open(ours, "rb").read() == open(theirs, "rb").read()
    # each reads the other's file exactly
    back = np.empty_like(phi)
    assert lib.spm_load_field_txt(theirs.encode(), back.ctypes.data, back.size) == 0
    assert np.array_equal(back, phi)
    assert np.array_equal(r.load_phi(ours), phi)
    # too short a file is an error
    assert lib.spm_load_field_txt(ours.encode(), back.ctypes.data, back.size + 1) != 0
    r.close()


def test_eigenvector_block_file_matches_reference(lib, tmp_path):
    N, k = 16, 3
    V = np.stack([npo.uniform_field(N, 10 + i) for i in range(k)])
    ours, theirs = str(tmp_path / "V_ours.txt"), str(tmp_path / "V_ref.txt")
    assert lib.spm_save_field_txt(ours.encode(), V.ctypes.data, V.size) == 0
    r = _ref(N)
    r.save_option_v(V, theirs)
    assert open(ours, "rb").read() == open(theirs, "rb").read()
    assert np.array_equal(r.load_option_v(k, ours), V)
    r.close()


def test_checkpoint_round_trip_and_corruption(lib, tmp_path):
    N = 16
    f = np.stack([npo.uniform_field(N, 1), npo.uniform_field(N, 2)])
    info = CkInfo(N, 2, 0, 26.0, -0.0061, 0.30, 0.3, 1234)
    path = str(tmp_path / "ck.bin")
    assert lib.spm_checkpoint_save(path.encode(), ctypes.byref(info), f.ctypes.data) == 0
    assert not os.path.exists(path + ".tmp")
    got = CkInfo()
    assert lib.spm_checkpoint_load(path.encode(), ctypes.byref(got), None, 0) == 0  # header only
    assert (got.N, got.nfields, got.step, got.L, got.Tau) == (N, 2, 1234, 26.0, -0.0061)
    out = np.zeros_like(f)
    assert lib.spm_checkpoint_load(path.encode(), ctypes.byref(got), out.ctypes.data, 1) != 0  # too small
    assert lib.spm_checkpoint_load(path.encode(), ctypes.byref(got), out.ctypes.data, out.size) == 0
    assert np.array_equal(out, f)
    data = bytearray(open(path, "rb").read())
    data[-100] ^= 0x10
    bad = str(tmp_path / "bad.bin")
    open(bad, "wb").write(bytes(data))
    assert lib.spm_checkpoint_load(bad.encode(), ctypes.byref(got), out.ctypes.data, out.size) != 0
    open(bad, "wb").write(bytes(data[:1000]))
    assert lib.spm_checkpoint_load(bad.encode(), ctypes.byref(got), out.ctypes.data, out.size) != 0
    open(bad, "wb").write(b"not a checkpoint" * 10)
    assert lib.spm_checkpoint_load(bad.encode(), ctypes.byref(got), None, 0) != 0


# get_initial_value pairs each phase with its shell scale l (Initialization.cpp:251-296)
PHASES = [(0, "DIS", 1.0), (1, "BCC", np.sqrt(2.0)), (2, "FCC", np.sqrt(3.0)), (3, "HPC", np.sqrt(2.0)),
          (5, "DG", np.sqrt(6.0))]


@pytest.mark.parametrize("choice,name,l", PHASES)
def test_initdata_reader_matches_reference(lib, choice, name, l):
    path = os.path.join(REFROOT, "initData", name)
    if not os.path.exists(path):
        pytest.skip("reference initData not present")
    N, L = 64, 26.0
    # the reference indexes u_F without a bounds check: only compare files that fit the grid
    toks = open(path).read().split()
    n = int(toks[0])
    recs = np.array([int(t) for t in toks[1:1 + 4 * n]] + [0] * max(0, 4 * n - (len(toks) - 1))).reshape(n, 4)
    ks = np.round(recs[:, :3] / l * L)
    if n and np.max(np.abs(ks)) >= N // 2:
        pytest.skip("modes beyond the grid")
    ours = np.zeros((N, N, N, 2))
    assert lib.spm_initdata_spectrum(path.encode(), N, L, float(l), ours.ctypes.data) == 0
    r = _ref(N)
    theirs = r.initial_value(choice, REFROOT)
    r.close()
    assert np.array_equal(ours[..., 0] + 1j * ours[..., 1], theirs)


def test_initdata_reader_rejects_modes_outside_the_grid(lib, tmp_path):
    p = tmp_path / "big"
    p.write_text("1\n 5 0 0 1\n")
    out = np.zeros((16, 16, 16, 2))
    assert lib.spm_initdata_spectrum(str(p).encode(), 16, 26.0, 1.0, out.ctypes.data) != 0
