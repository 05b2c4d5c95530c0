"""CPU checks of the oracle (no GPU).

1. The NumPy restatement reproduces the golden vectors that the reference's
   own sources produced (tests/golden/ref_golden.npz, see make_golden.py).
2. When oracle/_ref is built here, the compiled reference and the NumPy
   restatement agree routine by routine on fresh seeded inputs.
3. Known-answer identities that pin the transform and the model without any
   reference output: phi = 0, a single cosine mode, the Hessian at phi = 0,
   Parseval, Hv as the derivative of -grad F, the FFTW sign convention.
"""
import os

import numpy as np
import pytest

from conftest import rel
from oracle import refbind
from oracle import spmiqc_np as npo

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_golden.npz"))


def sig(a):
    idx = np.array([0, 1, 7, 100, 333, 1000, 2047, 4095, 5000, 9999, 12345, 16383, 20000, 22222, 30000,
                    32767, 3, 17, 64, 255, 511, 777, 1024, 1500, 2500, 7000, 11111, 15000, 18000, 25000,
                    28000, 31000])
    a = np.asarray(a).ravel()
    return np.concatenate([[a.sum(), (a * a).sum()], a[idx % a.size]])


@pytest.mark.parametrize("N,steps", [(16, 20), (32, 10)])
def test_numpy_oracle_matches_reference_golden(N, steps):
    m = npo.Model(N)
    phi = npo.uniform_field(N, 7)
    v = npo.uniform_field(N, 11, amp=1.0)
    p, u = phi.copy(), m.my_fft(phi)
    for s in range(steps):
        g = m.grad_norm(p)
        p, u, e, r = m.grad_step(p, u)
        assert abs(e - GOLD[f"N{N}_E"][s]) <= 1e-12 * abs(e)
        assert abs(r - GOLD[f"N{N}_res"][s]) <= 1e-10 * abs(r)
        assert abs(g - GOLD[f"N{N}_gnorm"][s]) <= 1e-12 * abs(g)
    tv = m.tangent(phi, phi + 0.01 * v)
    a, b, _, _ = m.spring_pairing(phi, phi + 0.001 * tv, 3, 1e-9)
    fields = {"phi_end": p, "ngrad": m.ngrad(phi), "hv": m.hv(phi, v), "precond": m.precond(v), "tangent": tv,
              "nf": m.natural_forces(phi, tv), "mm": m.minmax_forces(phi, tv), "spm0": a, "spm1": b}
    for k, val in fields.items():
        ref = GOLD[f"N{N}_{k}"] if N == 16 else GOLD[f"N{N}_{k}_sig"]
        got = val if N == 16 else sig(val)
        assert rel(got, ref) < 1e-12, k
    V0 = m.lobpcg_init(3, 5)
    assert rel(sig(V0), GOLD[f"N{N}_V0"]) < 1e-12
    V1, _ = m.lobpcg_inip(phi, V0, 6)
    ritz = np.array([m.rayleigh(phi, V1[i]) for i in range(3)])
    assert rel(ritz, GOLD[f"N{N}_ritz"]) < 1e-11


@pytest.mark.parametrize("N,steps", [(16, 20), (32, 10)])
def test_mkl_cpu_baseline_matches_reference_golden(N, steps):
    """The FFTW-class CPU baseline (torch/MKL restatement of the gradient step)
    reproduces the compiled reference's per-step energy, res and ||grad F||."""
    import torch
    from oracle import cpu_mkl
    f = cpu_mkl.MklFlow(N, threads=2)
    p = torch.from_numpy(npo.uniform_field(N, 7))
    u = f.spectrum(p)
    for s in range(steps):
        p, u, e, r, g = f.step(p, u)
        assert abs(e - GOLD[f"N{N}_E"][s]) <= 1e-12 * abs(e)
        assert abs(r - GOLD[f"N{N}_res"][s]) <= 1e-10 * abs(r)
        assert abs(g - GOLD[f"N{N}_gnorm"][s]) <= 1e-12 * abs(g)
    ref = GOLD[f"N{N}_phi_end"] if N == 16 else GOLD[f"N{N}_phi_end_sig"]
    got = p.numpy() if N == 16 else sig(p.numpy())
    assert rel(got, ref) < 1e-12


@pytest.mark.skipif(not refbind.available(), reason="oracle/_ref not built")
def test_compiled_reference_matches_numpy():
    N = 16
    m = npo.Model(N)
    r = refbind.Ref(N, L=21.0, Tau=-0.012, Gamma=0.25, dt=0.2)
    m = npo.Model(N, L=21.0, Tau=-0.012, Gamma=0.25, dt=0.2)
    G, ik = r.tables()
    assert rel(G, m.G) < 1e-14 and rel(ik, m.ikt2) < 1e-14
    phi = npo.uniform_field(N, 31)
    v = npo.uniform_field(N, 32, amp=1.0)
    r.set_state(phi)
    E, res, g = r.grad_steps(4)
    p, u = phi.copy(), m.my_fft(phi)
    for s in range(4):
        gg = m.grad_norm(p)
        p, u, e, rr = m.grad_step(p, u)
        assert abs(E[s] - e) <= 1e-13 * abs(e) and abs(g[s] - gg) <= 1e-12 * gg
    assert rel(r.hv(phi, v), m.hv(phi, v)) < 1e-13
    assert rel(r.precond(v), m.precond(v)) < 1e-13
    assert rel(r.ngrad(phi), m.ngrad(phi)) < 1e-13
    r.close()


# ------------------------------------------------------------ known answers
def test_zero_field():
    m = npo.Model(16)
    z = np.zeros((16,) * 3)
    assert m.energy(z, m.my_fft(z)) == 0.0
    assert np.all(m.ngrad(z) == 0.0)
    p, u, e, r = m.grad_step(z, m.my_fft(z))
    assert e == 0.0 and r == 0.0 and np.all(p == 0)


def test_single_cosine_mode_energy():
    N, L, A = 32, 26.0, 0.05
    m = npo.Model(N, L=L)
    n = np.array([3, 1, 2])
    i = np.arange(N)
    phi = A * np.cos(2 * np.pi * ((n[0] * i)[:, None, None] + (n[1] * i)[None, :, None] +
                                  (n[2] * i)[None, None, :]) / N)
    k2 = float(np.sum((n / L) ** 2))
    E1 = 0.5 * npo.get_GK(k2) * A * A / 2
    # local density means of cos^2 = 1/2, cos^3 = 0, cos^4 = 3/8
    E2 = -0.5 * m.Tau * A * A / 2 + 0.25 * A ** 4 * 3 / 8
    assert abs(m.energy(phi, m.my_fft(phi)) - (E1 + E2)) < 1e-15


def test_hessian_at_zero_is_diagonal():
    N = 16
    m = npo.Model(N)
    z = np.zeros((N,) * 3)
    for n in ([1, 0, 0], [2, 3, 1], [5, 5, 5]):
        i = np.arange(N)
        e = np.cos(2 * np.pi * ((n[0] * i)[:, None, None] + (n[1] * i)[None, :, None] + (n[2] * i)[None, None, :]) / N)
        lam = npo.get_GK(float(np.sum((np.array(n) / m.L) ** 2))) - m.Tau
        assert rel(m.hv(z, e), lam * e) < 1e-13


def test_hv_is_derivative_of_minus_ngrad():
    N = 16
    m = npo.Model(N)
    phi = npo.uniform_field(N, 3)
    v = npo.uniform_field(N, 4, amp=1.0)
    v = v - v.mean()
    h = 1e-5
    fd = -(m.ngrad(phi + h * v) - m.ngrad(phi - h * v)) / (2 * h)
    assert rel(m.hv(phi, v), fd) < 1e-8


def test_parseval_and_fftw_sign():
    N = 16
    m = npo.Model(N)
    x = npo.uniform_field(N, 9)
    X = m.my_fft(x)
    assert abs(m.inpfp(x, x) - float(np.sum(np.abs(X) ** 2))) < 1e-15
    # FFTW_FORWARD = exp(-2 pi i jk/n): a shifted delta has phase exp(-2 pi i k / N)
    d = np.zeros((N,) * 3)
    d[0, 0, 1] = 1.0
    D = m.my_fft(d) * N ** 3
    assert abs(D[0, 0, 1] - np.exp(-2j * np.pi / N)) < 1e-15


def test_splitmix_uniform_matches_shim_stream():
    # the oracle's MatrixXd::Random replacement and the input generators share one stream definition
    import inputs
    idx = np.arange(10, dtype=np.uint64)
    assert np.array_equal(npo.uniform_pm1(5, idx), -1.0 + 2.0 * inputs.unit(5, idx))


def test_hisd_restatement_matches_reference():
    """hiosd_lobpcg_sieh (HISD.cpp:86-485): the NumPy restatement against the
    reference compiled in place, 1 and 8 iterations, k = 1 and 2."""
    if not refbind.available():
        pytest.skip("compiled reference not built")
    N = 16
    m = npo.Model(N, L=10.0, Tau=-0.05)
    x = npo.uniform_field(N, 3) + 0.05 * np.cos(2 * np.pi * np.arange(N) / N)[:, None, None]
    r = refbind.Ref(N, L=10.0, Tau=-0.05)
    for k, its in ((1, 1), (1, 8), (2, 8)):
        V = m.lobpcg_init(k, 5)
        xr, Vr = r.hisd(x, V, maxiter=its, epsf=1e-30)
        xo, Vo, _ = m.hisd(x, V, maxiter=its, epsf=1e-30)
        assert np.max(np.abs(xr - xo)) <= 1e-12 * np.max(np.abs(xo))
        for i in range(k):  # eigenvectors up to sign
            d = min(np.max(np.abs(Vr[i] - Vo[i])), np.max(np.abs(Vr[i] + Vo[i])))
            assert d <= 1e-9, (k, its, i, d)
    r.close()


def test_gosd_restatement_matches_reference():
    """hiosd_lobpcg_sieh_V0 (GOSD.cpp:123-531): HiSD with the directions kept
    orthogonal to a fixed subspace V0 (here the two lowest Hessian modes at
    the start), NumPy restatement against the compiled reference."""
    if not refbind.available():
        pytest.skip("compiled reference not built")
    N = 16
    m = npo.Model(N, L=10.0, Tau=-0.05)
    x = npo.uniform_field(N, 3) + 0.05 * np.cos(2 * np.pi * np.arange(N) / N)[:, None, None]
    V0, _ = m.lobpcg_inip(x, m.lobpcg_init(2, 9), 6)
    V = m.lobpcg_init(1, 5)
    r = refbind.Ref(N, L=10.0, Tau=-0.05)
    xr, Vr = r.gosd(x, V, V0, betau=0.02, maxiter=6, epsf=1e-30)
    xo, Vo, _ = m.hisd(x, V, betau=0.02, maxiter=6, epsf=1e-30, V0=V0)
    r.close()
    assert np.max(np.abs(xr - xo)) <= 1e-12 * np.max(np.abs(xo))
    assert min(np.max(np.abs(Vr[0] - Vo[0])), np.max(np.abs(Vr[0] + Vo[0]))) <= 1e-9
    assert abs(m.inpfp(Vo[0], V0[0])) < 1e-12 and abs(m.inpfp(Vo[0], V0[1])) < 1e-12
