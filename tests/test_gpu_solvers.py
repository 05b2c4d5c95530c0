"""CUDA LOBPCG and Spring Pair Method vs the FP64 oracle (1e-11 relative for
fields and eigenvalues; eigenvectors compared as subspaces)."""
import numpy as np
import pytest

from conftest import rel
from oracle import spmiqc_np as npo

pytestmark = pytest.mark.gpu
TOL = 1e-11


@pytest.fixture(scope="module")
def spm(cuda):
    import spmiqc
    return spmiqc


def t(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a)).cuda()


def subspace_ritz(m, phi, V):
    """Eigenvalues of V^T H V / N^3 for an orthonormal block (rotation invariant)."""
    k = V.shape[0]
    HV = np.stack([m.hv(phi, V[i]) for i in range(k)])
    M = np.array([[m.inpfp(V[i], HV[j]) for j in range(k)] for i in range(k)])
    return np.linalg.eigvalsh(0.5 * (M + M.T))


@pytest.mark.parametrize("N,k", [(32, 3), (64, 2)])
def test_lobpcg_init_matches_oracle(spm, cuda, N, k):
    m = npo.Model(N)
    ctx = spm.SpmContext(N)
    V = ctx.hiosd_lobpcg_initialization(k, seed=5).cpu().numpy()
    ref = m.lobpcg_init(k, 5)
    assert rel(V, ref) < TOL


@pytest.mark.parametrize("N,k,iters", [(32, 3, 6), (64, 4, 8)])
def test_lobpcg_matches_oracle(spm, cuda, N, k, iters):
    m = npo.Model(N)
    ctx = spm.SpmContext(N)
    phi = npo.uniform_field(N, 7)
    V0 = m.lobpcg_init(k, 5)
    Vd = t(cuda, V0)
    ev, rs, it = ctx.hiosd_lobpcg_inip(t(cuda, phi), Vd, iters)
    assert it == iters
    Vg = Vd.cpu().numpy()
    Vr, _ = m.lobpcg_inip(phi, V0, iters)
    # eigenvalues of the block (rotation invariant) and per-vector Rayleigh quotients
    rg, rr = subspace_ritz(m, phi, Vg), subspace_ritz(m, phi, Vr)
    assert np.max(np.abs(rg - rr)) <= TOL * np.max(np.abs(rr))
    assert np.max(np.abs(np.sort(ev) - rr)) <= 1e-9 * np.max(np.abs(rr))
    # the two blocks span the same subspace (principal angles)
    s = np.linalg.svd(Vg.reshape(k, -1) @ Vr.reshape(k, -1).T / N ** 3, compute_uv=False)
    assert np.min(s) > 1 - 1e-9
    # orthonormal and mean free
    G = Vg.reshape(k, -1) @ Vg.reshape(k, -1).T / N ** 3
    assert np.max(np.abs(G - np.eye(k))) < 1e-12
    assert np.max(np.abs(Vg.reshape(k, -1).mean(1))) < 1e-14


@pytest.mark.parametrize("k", [8, 3])
def test_lobpcg_direct_block_kernels_agree(spm, cuda, k):
    """The block kernels staged through shared memory (default) and the direct
    ones (knob block_stage 0: Grams by gram_kernel, the residual norms from a
    Gram of W instead of the combination) give the same LOBPCG iterates to
    rounding; k = 3 runs the residual combination on the direct kernel even
    when staged (six inputs)."""
    N = 64
    m = npo.Model(N)
    phi = t(cuda, npo.uniform_field(N, 7))
    V0 = m.lobpcg_init(k, 5)
    out = []
    for stage in (1, 0):
        ctx = spm.SpmContext(N)
        ctx.tune("block_stage", stage)
        Vd = t(cuda, V0)
        ev, rs, it = ctx.hiosd_lobpcg_inip(phi, Vd, 10)
        out.append((ev, rs, Vd.cpu().numpy()))
    (e1, r1, V1), (e0, r0, V0b) = out
    assert np.max(np.abs(e1 - e0)) <= 1e-12 * np.max(np.abs(e0))
    assert np.max(np.abs(r1 - r0)) <= 1e-9 * np.max(r0)
    s = np.linalg.svd(V1.reshape(k, -1) @ V0b.reshape(k, -1).T / N ** 3, compute_uv=False)
    assert np.min(s) > 1 - 1e-10


def test_lobpcg_at_zero_field_finds_lowest_kernel_modes(spm, cuda):
    """Known answer: H(0) is diagonal in k with eigenvalues G(k) - Tau. With
    L = 5 on a 32^3 grid the |n| = 5 shell (30 modes, k^2 = 1, G = min) is an
    exactly degenerate lowest cluster with a clear gap above it."""
    N, L = 32, 5.0
    m = npo.Model(N, L=L)
    ctx = spm.SpmContext(N, L=L)
    phi = cuda.zeros((N,) * 3, dtype=cuda.float64, device="cuda")
    V = ctx.hiosd_lobpcg_initialization(2, seed=1)
    ev, rs, it = ctx.hiosd_lobpcg_inip(phi, V, 100, tol=1e-8)
    k2 = m.k2.ravel()  # the k = 0 mode is excluded: the block is kept mean free
    exact = np.sort((m.G - m.Tau).ravel()[k2 > 0])[:2]
    assert it < 100 and np.max(rs) <= 1e-8
    # eigenvalue error ~ residual^2 / gap ~ 1e-13 absolute
    assert np.allclose(np.sort(ev), exact, rtol=1e-9, atol=0)


@pytest.mark.parametrize("N", [32, 64])
def test_tangent_and_force_steps(spm, cuda, N):
    m = npo.Model(N)
    ctx = spm.SpmContext(N)
    phi = npo.uniform_field(N, 3)
    d = npo.uniform_field(N, 4, amp=1.0)
    v = ctx.get_Tv(t(cuda, phi), t(cuda, phi + 0.01 * d)).cpu().numpy()
    vr = m.tangent(phi, phi + 0.01 * d)
    assert rel(v, vr) < TOL
    x = t(cuda, phi)
    ctx.Natural_Forces(x, t(cuda, vr))
    assert rel(x.cpu().numpy(), m.natural_forces(phi, vr)) < TOL
    x = t(cuda, phi)
    ctx.MinMax_Forces(x, t(cuda, vr))
    assert rel(x.cpu().numpy(), m.minmax_forces(phi, vr)) < TOL


@pytest.mark.parametrize("N", [32, 64])
def test_spring_pairing(spm, cuda, N):
    m = npo.Model(N)
    ctx = spm.SpmContext(N)
    phi = npo.uniform_field(N, 9)
    d = npo.uniform_field(N, 10, amp=1.0)
    vr = m.tangent(phi, phi + d)
    p0, p1 = t(cuda, phi), t(cuda, phi + 0.001 * vr)
    hist = ctx.Spring_Pairing(p0, p1, 4, 1e-9)
    a, b, it, res = m.spring_pairing(phi, phi + 0.001 * vr, 4, 1e-9)
    assert len(hist) == it == 4
    assert abs(hist[-1] - res) <= 1e-9 * res
    assert rel(p0.cpu().numpy(), a) < TOL and rel(p1.cpu().numpy(), b) < TOL


@pytest.mark.parametrize("N", [32, 64])
def test_spring_pairing_with_rest_length(spm, cuda, N):
    """The opt-in spring rest length (spm_set_spring_length) against the
    oracle's restatement: 4 iterations from replicas 0.05 apart with rest
    length 0.1 (the spring pushes them apart), and 0 restores the reference's
    spring bit for bit."""
    m = npo.Model(N)
    phi = npo.uniform_field(N, 9)
    vr = m.tangent(phi, phi + npo.uniform_field(N, 10, amp=1.0))
    out = {}
    for rest in (0.1, 0.0):
        ctx = spm.SpmContext(N)
        ctx.set_spring_length(rest)
        p0, p1 = t(cuda, phi), t(cuda, phi + 0.05 * vr)
        hist = ctx.Spring_Pairing(p0, p1, 4, 1e-9)
        a, b, it, res = m.spring_pairing(phi, phi + 0.05 * vr, 4, 1e-9, rest=rest)
        assert len(hist) == it == 4
        assert abs(hist[-1] - res) <= 1e-9 * res
        assert rel(p0.cpu().numpy(), a) < TOL and rel(p1.cpu().numpy(), b) < TOL
        out[rest] = (p0.cpu().numpy(), p1.cpu().numpy(), m.nrmp(b - a))
    assert out[0.1][2] > out[0.0][2]  # the rest length keeps the pair further apart
    ctx = spm.SpmContext(N)
    p0, p1 = t(cuda, phi), t(cuda, phi + 0.05 * vr)
    ctx.Spring_Pairing(p0, p1, 4, 1e-9)
    assert np.array_equal(p0.cpu().numpy(), out[0.0][0]) and np.array_equal(p1.cpu().numpy(), out[0.0][1])
    with pytest.raises(spm.SpmError):
        ctx.set_spring_length(-1.0)


def test_spring_pairing_stops_at_tolerance(spm, cuda):
    N = 32
    m = npo.Model(N)
    ctx = spm.SpmContext(N)
    phi = npo.uniform_field(N, 9)
    vr = m.tangent(phi, phi + npo.uniform_field(N, 10, amp=1.0))
    p0, p1 = t(cuda, phi), t(cuda, phi + 0.001 * vr)
    hist = ctx.Spring_Pairing(p0, p1, 50, 1e3)  # the first residual is below the tolerance
    assert len(hist) == 1


@pytest.mark.parametrize("k", [1, 2])
def test_hisd_matches_oracle(spm, cuda, k):
    """HiSD (hiosd_lobpcg_sieh, HISD.cpp:86-485) on the device against the FP64
    oracle: positions, unstable directions (up to sign) and the ||grad F||
    history after 8 iterations."""
    N = 32
    m = npo.Model(N, L=10.0, Tau=-0.05)
    x0 = npo.uniform_field(N, 3) + 0.05 * np.cos(2 * np.pi * np.arange(N) / N)[:, None, None]
    V0 = m.lobpcg_init(k, 5)
    xo, Vo, ho = m.hisd(x0, V0, maxiter=8, epsf=1e-30)
    ctx = spm.SpmContext(N, L=10.0, Tau=-0.05)
    x = cuda.from_numpy(x0.copy()).cuda()
    V = cuda.from_numpy(V0.copy()).cuda()
    h = ctx.hiosd_lobpcg_sieh(x, V, maxiter=8, epsf=1e-30)
    assert len(h) == 8
    assert np.max(np.abs(h - ho) / ho) < 1e-9
    assert rel(x.cpu().numpy(), xo) < 1e-10
    Vg = V.cpu().numpy()
    for i in range(k):
        assert min(rel(Vg[i], Vo[i]), rel(-Vg[i], Vo[i])) < 1e-8, i


def test_gosd_matches_oracle(spm, cuda):
    """GOSD (hiosd_lobpcg_sieh_V0, GOSD.cpp:123-531) on the device against the
    FP64 oracle, with two fixed directions V0; V stays orthogonal to V0."""
    N = 32
    m = npo.Model(N, L=10.0, Tau=-0.05)
    x0 = npo.uniform_field(N, 3) + 0.05 * np.cos(2 * np.pi * np.arange(N) / N)[:, None, None]
    V00, _ = m.lobpcg_inip(x0, m.lobpcg_init(2, 9), 6)
    Vs = m.lobpcg_init(1, 5)
    xo, Vo, ho = m.hisd(x0, Vs, betau=0.02, maxiter=6, epsf=1e-30, V0=V00)
    ctx = spm.SpmContext(N, L=10.0, Tau=-0.05)
    x = cuda.from_numpy(x0.copy()).cuda()
    V = cuda.from_numpy(Vs.copy()).cuda()
    V0 = cuda.from_numpy(np.ascontiguousarray(V00)).cuda()
    h = ctx.hiosd_lobpcg_sieh_V0(x, V, V0, betau=0.02, maxiter=6, epsf=1e-30)
    assert len(h) == 6 and np.max(np.abs(h - ho) / ho) < 1e-9
    assert rel(x.cpu().numpy(), xo) < 1e-10
    Vg = V.cpu().numpy()
    assert min(rel(Vg[0], Vo[0]), rel(-Vg[0], Vo[0])) < 1e-8
    assert max(abs(m.inpfp(Vg[0], V00[i])) for i in range(2)) < 1e-12


def test_lobpcg_guard_vectors_converge_a_close_pair(spm, cuda):
    """A k = 4 solve whose 4th eigenvalue has a close neighbour (a cosine-shell
    field of the serving stream, N = 64): the block of 4 stalls far above 1e-8
    within 400 iterations, the block of 8 with the stop test on the first 4
    (spm_lobpcg_guarded) reaches it. The returned pairs are checked directly,
    ||H v_i - lambda_i v_i|| through the Hessian product, and the converged
    eigenvalues agree between the two runs; guard = 0 is spm_lobpcg."""
    import workloads
    spec = next(s for s in workloads.serving_stream(seed=2024, n_jobs=32) if s.kind == "lobpcg" and s.N == 64)
    ctx = spm.SpmContext(64, L=spec.L, Tau=spec.Tau)
    phi = t(cuda, workloads.field(spec))
    V4 = ctx.hiosd_lobpcg_initialization(4, seed=spec.seed)
    ev4, rs4, it4 = ctx.hiosd_lobpcg_inip(phi, V4, maxiter=400, tol=1e-8)
    assert it4 == 400 and rs4[3] > 1e-6
    V8 = ctx.hiosd_lobpcg_initialization(8, seed=spec.seed)
    ev8, rs8, it8 = ctx.lobpcg_guarded(phi, V8, 4, maxiter=400, tol=1e-8)
    assert it8 < 400 and max(rs8[:4]) <= 1e-8
    HV = ctx.hv_cam(phi, V8[:4].contiguous())
    for i in range(4):
        r = HV[i] - float(ev8[i]) * V8[i]
        assert ctx.nrmp(r) <= 2e-8 * max(1.0, abs(ev8[i]))
        assert abs(ctx.nrmp(V8[i]) - 1.0) < 1e-12
    # the pairs the block of 4 did converge are the same eigenvalues
    assert np.max(np.abs(ev8[:3] - ev4[:3]) / np.abs(ev4[:3])) < 1e-10
    # no guards: the same iteration as spm_lobpcg
    Va = ctx.hiosd_lobpcg_initialization(3, seed=1)
    Vb = Va.clone()
    a = ctx.hiosd_lobpcg_inip(phi, Va, maxiter=5)
    b = ctx.lobpcg_guarded(phi, Vb, 3, maxiter=5, tol=0.0)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
    assert cuda.equal(Va, Vb)
