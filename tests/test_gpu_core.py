"""CUDA path vs the FP64 oracle: transforms, energy, gradient flow, ngrad, Hv,
preconditioner, inner products. Tolerance: the FP64 parity bar, 1e-11
relative (scale-relative max difference for fields)."""
import numpy as np
import pytest

from conftest import rel
from oracle import spmiqc_np as npo

pytestmark = pytest.mark.gpu

SIZES = [32, 64, 96, 128, 160, 192]
TOL = 1e-11


@pytest.fixture(scope="module")
def spm(cuda):
    import spmiqc
    return spmiqc


def t(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("N", SIZES + [256])
def test_fft_matches_dft(spm, cuda, N):
    ctx = spm.SpmContext(N)
    x = npo.uniform_field(N, 100 + N)
    xd = t(cuda, x)
    xh = ctx.my_fft(xd)
    full = ctx.to_full(xh).cpu().numpy()
    ref = np.fft.fftn(x) / N ** 3
    assert rel(full, ref) < 1e-13
    back = ctx.my_ifft(xh).cpu().numpy()
    assert rel(back, x) < 1e-13
    # from_full is the inverse of to_full on Hermitian data
    xh2 = ctx.from_full(cuda.from_numpy(ref).cuda())
    assert rel(xh2.cpu().numpy(), xh.cpu().numpy()) < 1e-13


@pytest.mark.parametrize("N", [32, 64, 96])
def test_energy(spm, cuda, N):
    m = npo.Model(N)
    ctx = spm.SpmContext(N)
    phi = npo.uniform_field(N, 7)
    uF = m.my_fft(phi)
    pd = t(cuda, phi)
    uh = ctx.my_fft(pd)
    E = ctx.get_Ene(pd, uh)
    assert abs(E - m.energy(phi, uF)) <= TOL * abs(m.energy(phi, uF))


@pytest.mark.parametrize("N", [32, 64, 96, 160])
def test_grad_flow_steps(spm, cuda, N):
    m = npo.Model(N)
    ctx = spm.SpmContext(N)
    phi = npo.uniform_field(N, 11)
    pd = t(cuda, phi)
    uh = ctx.my_fft(pd)
    st = ctx.get_min_u_F(pd, uh, 12)
    assert st.shape == (12, 4)
    p, u = phi.copy(), m.my_fft(phi)
    for s in range(12):
        g = m.grad_norm(p)
        p, u, e, r = m.grad_step(p, u)
        assert abs(st[s, 0] - e) <= TOL * abs(e), s
        assert abs(st[s, 1] - r) <= 1e-9 * abs(r), s
        assert abs(st[s, 2] - g) <= 1e-9 * abs(g), s
    assert rel(pd.cpu().numpy(), p) < TOL
    assert rel(ctx.to_full(uh).cpu().numpy(), u) < TOL


@pytest.mark.parametrize("N", [32, 64, 96])
def test_ngrad(spm, cuda, N):
    m = npo.Model(N)
    ctx = spm.SpmContext(N)
    phi = npo.uniform_field(N, 3)
    g, nrm = ctx.ngrad_cam(t(cuda, phi))
    ref = m.ngrad(phi)
    assert rel(g.cpu().numpy(), ref) < TOL
    assert abs(nrm - m.nrmp(ref)) <= TOL * m.nrmp(ref)


@pytest.mark.parametrize("N", [32, 64, 128])
def test_hv_batch(spm, cuda, N):
    m = npo.Model(N)
    ctx = spm.SpmContext(N)
    phi = npo.uniform_field(N, 5)
    V = np.stack([npo.uniform_field(N, 20 + i, amp=1.0) for i in range(3)])
    H = ctx.hv_cam(t(cuda, phi), t(cuda, V)).cpu().numpy()
    for i in range(3):
        assert rel(H[i], m.hv(phi, V[i])) < TOL


@pytest.mark.parametrize("N", [32, 64])
def test_precond_batch(spm, cuda, N):
    m = npo.Model(N)
    ctx = spm.SpmContext(N)
    W = np.stack([npo.uniform_field(N, 40 + i, amp=1.0) for i in range(2)])
    Wd = t(cuda, W)
    ctx.precond_camnew(Wd)
    out = Wd.cpu().numpy()
    for i in range(2):
        assert rel(out[i], m.precond(W[i])) < TOL


def test_inpfp(spm, cuda):
    N = 64
    m = npo.Model(N)
    ctx = spm.SpmContext(N)
    a, b = npo.uniform_field(N, 1), npo.uniform_field(N, 2)
    assert abs(ctx.inpfp(t(cuda, a), t(cuda, b)) - m.inpfp(a, b)) <= 1e-12 * abs(m.inpfp(a, b))


# block shapes of the LOBPCG Grams (as index lists into one pool of fields):
# V^T U, V^T V, [V W]^T W, [V W P]^T P, S^T HS, ragged tiles, repeats, a shifted alias
GRAM_SHAPES = {
    "8x8": (list(range(8)), list(range(8, 16))),
    "self8": (list(range(8)), list(range(8))),
    "qx16": (list(range(16)), list(range(8, 16))),
    "qx24": (list(range(24)), list(range(16, 24))),
    "rr24": (list(range(24)), list(range(24, 48))),
    "ragged": (list(range(5)), list(range(30, 43))),
    "repeat": ([0, 0, 1, 2, 1], [2, 0]),
    "shift": (list(range(17)), [2, 3, 4]),
}


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("N", [32, 96])
@pytest.mark.parametrize("shape", sorted(GRAM_SHAPES))
def test_block_gram(spm, cuda, N, prec, shape):
    """spm_block_gram against NumPy (the Gram of LOBPCG.cpp:336-358), with the
    fields staged through shared memory (default) and read directly: within
    1e-13 of sqrt(G_aa G_bb) (the FP32 fields' products are exact in the FP64
    sums), and the same bits on a second call."""
    xs, ys = GRAM_SHAPES[shape]
    nfld = max(xs + ys) + 1
    rng = np.random.default_rng(7 * N + nfld)
    pool = rng.uniform(-1.0, 1.0, (nfld,) + (N,) * 3) + 0.3 * rng.standard_normal((nfld, 1, 1, 1))
    if prec == "fp32":
        pool = pool.astype(np.float32)
    pd = t(cuda, pool)
    flat = pool.reshape(nfld, -1).astype(np.float64)
    ref = flat[xs] @ flat[ys].T / N ** 3
    nrm = np.sqrt(np.einsum("ij,ij->i", flat, flat) / N ** 3)
    scale = np.outer(nrm[xs], nrm[ys])
    ctx = spm.SpmContext(N, precision=prec)
    for stage in (1, 0):
        ctx.tune("block_stage", stage)
        G = ctx.block_gram([pd[i] for i in xs], [pd[j] for j in ys])
        assert G.shape == ref.shape
        assert np.max(np.abs(G - ref) / scale) < 1e-13, (stage, np.max(np.abs(G - ref) / scale))
        G2 = ctx.block_gram([pd[i] for i in xs], [pd[j] for j in ys])
        assert np.array_equal(G, G2)


# (inputs, outputs) as index lists into one pool of fields; outputs that are
# also inputs are updated in place
COMB_SHAPES = {
    "w16": (list(range(16)), list(range(16, 24))),
    "p24_inplace": (list(range(24)), list(range(16, 24))),
    "v8_inplace_d": (list(range(8)), list(range(8))),
    "max32": (list(range(32)), list(range(32, 40))),
    "ragged": (list(range(5)), [7, 8, 9]),
    "wide12": (list(range(10)), list(range(10, 22))),
    "repeat": ([0, 1, 0, 2], [3]),
    "repeat9": ([0, 1, 2, 0, 1, 2, 3, 3, 4], [5, 6]),
}


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("N", [32, 96])
@pytest.mark.parametrize("shape", sorted(COMB_SHAPES))
def test_block_combine(spm, cuda, N, prec, shape):
    """spm_block_combine (the Ritz update of LOBPCG.cpp:403-418) against NumPy
    within 1e-13 of sum_p |C_pq| |X_p| (FP32: the FP32 rounding of the FP64
    result), in place where outputs are inputs; the inputs staged through
    shared memory (default) give the same bits as the direct kernel."""
    xs, ys = COMB_SHAPES[shape]
    nfld = max(xs + ys) + 1
    rng = np.random.default_rng(11 * N + nfld)
    pool = rng.uniform(-1.0, 1.0, (nfld,) + (N,) * 3)
    if prec == "fp32":
        pool = pool.astype(np.float32)
    C = rng.standard_normal((len(xs), len(ys)))
    d = rng.standard_normal(len(ys)) if shape.endswith("_d") else None
    flat = pool.reshape(nfld, -1).astype(np.float64)
    ref = C.T @ flat[xs] + (0.0 if d is None else d[:, None])
    scale = np.abs(C).T @ np.abs(flat[xs]) + 1e-300
    tol = 1e-13 if prec == "fp64" else 2 ** -23
    ctx = spm.SpmContext(N, precision=prec)
    outs = []
    for stage in (1, 0):
        ctx.tune("block_stage", stage)
        pd = t(cuda, pool)
        ctx.block_combine([pd[i] for i in xs], [pd[j] for j in ys], C, d)
        got = pd.cpu().numpy().reshape(nfld, -1)[ys].astype(np.float64)
        assert np.max(np.abs(got - ref) / np.maximum(scale, np.abs(ref))) < tol, stage
        # fields that are not outputs are untouched
        others = [i for i in range(nfld) if i not in ys]
        assert np.array_equal(pd.cpu().numpy()[others], pool[others])
        outs.append(got)
    assert np.array_equal(outs[0], outs[1])


def test_block_entry_points_reject_bad_blocks(spm, cuda):
    """spm_block_gram / spm_block_combine refuse blocks beyond their limits and
    an output field listed twice."""
    ctx = spm.SpmContext(32)
    f = ctx.field(3)
    with pytest.raises(spm.SpmError):
        ctx.block_gram([f[0]] * 25, [f[1]])
    with pytest.raises(spm.SpmError):
        ctx.block_combine([f[0], f[1]], [f[2], f[2]], np.ones((2, 2)))
    with pytest.raises(spm.SpmError):
        ctx.block_combine([f[0]] * 33, [f[1]], np.ones((33, 1)))


@pytest.mark.parametrize("N", [32, 64, 128, 160, 192])
def test_fused_plane_chain_is_bit_identical(spm, cuda, N):
    """Chains of steps with the fused inverse -> forward plane pass give the
    same bits (records, phi, u) as three passes per step, also when the flow
    stops inside a chain (tol_grad reached mid-chunk)."""
    phi = npo.uniform_field(N, 31)
    out = []
    for fuse in (0, 1):
        ctx = spm.SpmContext(N, Tau=-0.02)
        ctx.tune("fuse_planes", fuse)
        pd = t(cuda, phi)
        uh = ctx.my_fft(pd)
        a = ctx.get_min_u_F(pd, uh, 37)
        b = ctx.get_min_u_F(pd, uh, 3000, tol_grad=float(a[-1, 2]) * 0.3)
        out.append((a, b, pd.cpu().numpy(), uh.cpu().numpy()))
    (a0, b0, p0, u0), (a1, b1, p1, u1) = out
    assert len(b0) < 3000 and len(b0) == len(b1)
    assert np.array_equal(a0, a1) and np.array_equal(b0, b1)
    assert np.array_equal(p0, p1) and np.array_equal(u0, u1)


@pytest.mark.parametrize("N,prec", [(64, "fp64"), (96, "fp64"), (256, "fp64"), (128, "fp32"), (192, "fp32")])
def test_exchange_routes_are_bit_identical(spm, cuda, N, prec):
    """Gradient chains whose plane kernels exchange through global areas in L2
    (plane_xg 1, 2, 3; plane_cps 2, 3, 5 (16-row CTAs), 6 (the same, pipelined over planes) and, in
    FP32, 4) give the same fields as exchanges
    through distributed shared memory, and records equal to rounding."""
    phi = npo.uniform_field(N, 12)
    dt = np.float64 if prec == "fp64" else np.float32
    out = []
    combos = ((2, 0), (2, 1), (2, 2), (2, 3), (3, 3), (5, 3), (6, 3)) + (((4, 3), (4, 0)) if prec == "fp32" else ())
    for cps, xg in combos:
        e = spm.SpmContext(N, Tau=-0.02, precision=prec)
        e.tune("plane_cps", cps)
        e.tune("plane_xg", xg)
        assert e.tuning()["plane_xg"] == xg
        p = t(cuda, phi.astype(dt))
        u = e.my_fft(p)
        st = e.get_min_u_F(p, u, 23)
        mid = (p.cpu().numpy(), u.cpu().numpy())
        # then a flow that stops inside a chain (the fused pass's stopping path)
        st2 = e.get_min_u_F(p, u, 3000, tol_grad=float(st[-1, 2]) * 0.5)
        out.append((st, mid, len(st2), p.cpu().numpy(), u.cpu().numpy()))
    for st, mid, n2, p, u in out[1:]:
        assert np.array_equal(mid[0], out[0][1][0]) and np.array_equal(mid[1], out[0][1][1])
        assert n2 == out[0][2] < 3000
        assert np.array_equal(p, out[0][3]) and np.array_equal(u, out[0][4])
        assert rel(st, out[0][0]) < 1e-12


def test_autotune_picks_a_schedule_and_keeps_results(spm, cuda):
    """The autotuner returns one of its candidates, remembers it for the next
    context of the same kind, and every schedule gives the same fields (the
    transforms' arithmetic does not depend on the schedule) with records equal
    to rounding (the reduction grids differ)."""
    N = 64
    c = spm.SpmContext(N)
    cps, fuse = c.autotune(10)
    assert cps in (1, 2, 3) and fuse in (0, 1)
    d = spm.SpmContext(N)
    assert d.autotune(10) == (cps, fuse)
    assert d.tuning() == c.tuning() and c.tuning()["plane_xg"] in (0, 1, 2, 3)
    phi = npo.uniform_field(N, 8)
    out = []
    for k_cps, k_fuse in ((1, 1), (2, 1), (3, 1), (2, 0)):
        e = spm.SpmContext(N)
        e.tune("plane_cps", k_cps)
        e.tune("fuse_planes", k_fuse)
        p = t(cuda, phi)
        u = e.my_fft(p)
        st = e.get_min_u_F(p, u, 20)
        out.append((st, p.cpu().numpy()))
    for st, p in out[1:]:
        assert np.array_equal(p, out[0][1])
        assert rel(st, out[0][0]) < 1e-13


@pytest.mark.parametrize("N,prec", [(32, "fp64"), (64, "fp64"), (256, "fp64"), (96, "fp32"), (256, "fp32")])
def test_narrow_pencil_tiles_are_bit_identical(spm, cuda, N, prec):
    """Pencil passes with 4-column tiles (knob pencil_tc 4: 8 pencils and 128
    threads per CTA, several CTAs per SM) give the same fields as 8-column
    tiles, for gradient steps, a Hessian-vector block and the preconditioner;
    reductions (step records) agree to rounding (their summation order
    follows the tiling)."""
    phi = npo.uniform_field(N, 19)
    V = np.stack([npo.uniform_field(N, 50 + i, amp=1.0) for i in range(2)])
    dt = np.float64 if prec == "fp64" else np.float32
    out = []
    for tc in (8, 4):
        e = spm.SpmContext(N, Tau=-0.02, precision=prec)
        e.tune("pencil_tc", tc)
        p = t(cuda, phi.astype(dt))
        u = e.my_fft(p)
        st = e.get_min_u_F(p, u, 17)
        H = e.hv_cam(p, t(cuda, V.astype(dt)))
        W = t(cuda, V.astype(dt))
        e.precond_camnew(W)
        out.append((st, p.cpu().numpy(), u.cpu().numpy(), H.cpu().numpy(), W.cpu().numpy()))
        e.close()
    (s8, p8, u8, h8, w8), (s4, p4, u4, h4, w4) = out
    assert np.array_equal(p8, p4) and np.array_equal(u8, u4)
    assert np.array_equal(h8, h4) and np.array_equal(w8, w4)
    assert rel(s4, s8) < (1e-12 if prec == "fp64" else 1e-5)


@pytest.mark.parametrize("N,prec,cps", [(64, "fp64", 2), (256, "fp64", 5), (256, "fp64", 6), (256, "fp32", 4)])
def test_dependent_launches_are_bit_identical(spm, cuda, N, prec, cps):
    """Plane and pencil kernels launched as programmatic dependents (knob pdl
    1, the autotuner's choice at 256^3: a launch is set up while the previous
    kernel of the stream completes, and the kernel waits on the device for it
    before its first memory access) give the same bits as plain stream order
    (pdl 0): a gradient chain with the 16-row and pipelined schedules, one that
    stops inside a chain, a Hessian-vector block (several waves of clusters)
    and the preconditioner. The grids are the same either way, so the step
    records are equal too."""
    phi = npo.uniform_field(N, 23)
    V = np.stack([npo.uniform_field(N, 60 + i, amp=1.0) for i in range(3)])
    dt = np.float64 if prec == "fp64" else np.float32
    out = []
    for pdl in (0, 1):
        e = spm.SpmContext(N, Tau=-0.02, precision=prec)
        e.tune("plane_cps", cps)
        e.tune("plane_xg", 3)
        e.tune("pdl", pdl)
        assert e.tuning()["pdl"] == pdl
        with pytest.raises(spm.SpmError):
            e.tune("pdl", 2)
        p = t(cuda, phi.astype(dt))
        u = e.my_fft(p)
        st = e.get_min_u_F(p, u, 19)
        st2 = e.get_min_u_F(p, u, 3000, tol_grad=float(st[-1, 2]) * 0.5)
        H = e.hv_cam(p, t(cuda, V.astype(dt)))
        W = t(cuda, V.astype(dt))
        e.precond_camnew(W)
        out.append((st, st2, p.cpu().numpy(), u.cpu().numpy(), H.cpu().numpy(), W.cpu().numpy()))
        e.close()
    a, b = out
    assert len(a[1]) == len(b[1]) < 3000
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
