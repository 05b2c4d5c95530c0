"""FP32 bulk arithmetic and the mixed-precision flow, with errors stated
against FP64: an FP32 gradient step is within 1e-5 (scale-relative) of the
FP64 oracle; the mixed flow (FP32 to a switch threshold, FP64 polish) reaches
||grad F|| <= 1e-8 with the energy within 1e-10 relative of the all-FP64 GPU
flow (the mixed-precision acceptance bar)."""
import numpy as np
import pytest

from conftest import rel
from oracle import spmiqc_np as npo

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [32, 64, 96])
def test_fp32_step_error_vs_fp64_oracle(cuda, N):
    import spmiqc
    m = npo.Model(N)
    ctx = spmiqc.SpmContext(N, precision="fp32")
    phi = npo.uniform_field(N, 11)
    pd = cuda.from_numpy(phi.astype(np.float32)).cuda()
    uh = ctx.my_fft(pd)
    st = ctx.get_min_u_F(pd, uh, 5)
    p, u = phi.copy(), m.my_fft(phi)
    for s in range(5):
        g = m.grad_norm(p)
        p, u, e, r = m.grad_step(p, u)
        assert abs(st[s, 0] - e) <= 1e-5 * abs(e)
        assert abs(st[s, 2] - g) <= 1e-4 * abs(g)
    assert rel(pd.cpu().double().numpy(), p) < 1e-5


def test_mixed_flow_matches_fp64_minimum(cuda):
    """A relaxation that provably converges: a random field (U[-0.1, 0.1]) at
    Tau < 0 relaxes to the disordered minimum, the slowest mode contracting by
    1 - dt |Tau| / (1 + dt G_min) per step. Energies are compared on the scale of
    the initial energy (the minimum's energy is itself ~ ||grad F||^2 / |Tau|)."""
    import spmiqc
    N = 64
    phi0 = npo.uniform_field(N, 21)
    ctx = spmiqc.SpmContext(N)
    a = cuda.from_numpy(phi0).cuda()
    ua = ctx.my_fft(a)
    E0 = ctx.get_Ene(a, ua)
    sa = ctx.get_min_u_F(a, ua, 60000, tol_grad=1e-8)
    b = cuda.from_numpy(phi0).cuda()
    ub = ctx.my_fft(b)
    sb, n32, n64 = ctx.get_min_u_F_mixed(b, ub, 60000, tol_grad=1e-8, switch_tol=1e-6)
    assert sa[-1, 2] <= 1e-8 and sb[-1, 2] <= 1e-8, (len(sa), n32, n64, sa[-1], sb[-1])
    assert n32 > 0 and n64 > 0
    Ea = ctx.get_Ene(a, ua)
    Eb = ctx.get_Ene(b, ub)
    assert abs(Ea - Eb) <= 1e-10 * abs(E0), (Ea, Eb, E0)
    assert rel(b.cpu().numpy(), a.cpu().numpy()) < 1e-4  # both within ||grad F|| / |Tau| of the minimum


@pytest.mark.parametrize("group,pdl", [(1, 0), (0, 0), (1, 1), (0, 1)])
def test_batched_flows_match_single_flows(cuda, group, pdl):
    """spm_batch_grad_flow over instances of different N and parameters gives,
    per instance, exactly the steps and state of a single flow (deterministic
    reductions: identical bits alone and in the batch), both when instances of
    one size share every launch (batch_group 1: three 32^3 instances with
    different L and Tau in one launch per pass, two 64^3 ones in another) and
    when each instance has its own launches (batch_group 0); with pdl 1 the
    captured graph's plane and pencil kernels are joined by programmatic edges
    and the single flows run as dependent launches."""
    import ctypes
    import spmiqc
    lib = spmiqc.lib()
    f = lib.spm_batch_grad_flow
    f.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                  ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                  ctypes.POINTER(ctypes.c_int)]
    specs = [(32, 26.0, -0.0061, 1), (64, 20.0, -0.01, 2), (96, 28.0, -0.015, 3), (32, 18.0, -0.02, 4),
             (64, 29.0, -0.004, 5), (32, 22.5, -0.012, 6)]
    ctxs, phis, uhs, singles = [], [], [], []
    for N, L, tau, seed in specs:
        c = spmiqc.SpmContext(N, L=L, Tau=tau)
        c.tune("batch_group", group)
        c.tune("pdl", pdl)
        p0 = npo.uniform_field(N, seed)
        p = cuda.from_numpy(p0).cuda()
        ctxs.append(c), phis.append(p), uhs.append(c.my_fft(p))
        q = cuda.from_numpy(p0).cuda()
        uq = c.my_fft(q)
        st = c.get_min_u_F(q, uq, 3000, tol_grad=1e-7)
        singles.append((len(st), q))
    cuda.cuda.synchronize()
    n = len(specs)
    arr = lambda xs: (ctypes.c_void_p * n)(*[ctypes.c_void_p(x) for x in xs])
    done = (ctypes.c_int * n)()
    spmiqc.check(f(arr([c.h.value for c in ctxs]), arr([p.data_ptr() for p in phis]),
                   arr([u.data_ptr() for u in uhs]), n, 3000, 1e-7, 0.0, 16, done))
    for i in range(n):
        assert done[i] == singles[i][0], (i, done[i], singles[i][0])
        assert cuda.equal(phis[i], singles[i][1]), i


def test_mixed_flow_fp32_as_far_as_it_goes(cuda):
    """switch_tol = 0: the FP32 phase runs to the tolerance or to its rounding
    floor; the FP64 polish then needs few steps, and the minimum matches the
    all-FP64 one on the initial-energy scale."""
    import spmiqc
    N = 64
    phi0 = npo.uniform_field(N, 22)
    ctx = spmiqc.SpmContext(N)
    a = cuda.from_numpy(phi0).cuda()
    ua = ctx.my_fft(a)
    E0 = ctx.get_Ene(a, ua)
    sa = ctx.get_min_u_F(a, ua, 60000, tol_grad=1e-8)
    b = cuda.from_numpy(phi0).cuda()
    ub = ctx.my_fft(b)
    sb, n32, n64 = ctx.get_min_u_F_mixed(b, ub, 60000, tol_grad=1e-8, switch_tol=0.0)
    assert sa[-1, 2] <= 1e-8 and sb[-1, 2] <= 1e-8
    assert n32 > 0.8 * len(sa) and n64 < 0.2 * len(sa), (n32, n64, len(sa))
    assert abs(ctx.get_Ene(a, ua) - ctx.get_Ene(b, ub)) <= 1e-10 * abs(E0)


def test_spring_pairing_fp32_phase_tracks_fp64(cuda):
    """The FP32 phase of the mixed Spring_Pairing follows the FP64 iteration to
    FP32 accuracy (20 iterations, no switch)."""
    import spmiqc
    N = 32
    p0 = npo.uniform_field(N, 40)
    p1 = p0 + 0.01 * npo.uniform_field(N, 41)
    ctx = spmiqc.SpmContext(N)
    a0, a1 = cuda.from_numpy(p0).cuda(), cuda.from_numpy(p1).cuda()
    ha = ctx.Spring_Pairing(a0, a1, 20, 1e-30)
    b0, b1 = cuda.from_numpy(p0).cuda(), cuda.from_numpy(p1).cuda()
    hb, i32, i64 = ctx.Spring_Pairing_mixed(b0, b1, 20, 1e-30, switch_tol=0.0)
    assert i32 == 20 and i64 == 0 and len(hb) == len(ha) == 20
    assert np.max(np.abs(hb - ha) / ha) < 1e-4
    assert rel(b0.cpu().numpy(), a0.cpu().numpy()) < 1e-5 and rel(b1.cpu().numpy(), a1.cpu().numpy()) < 1e-5


def test_batched_mixed_flows_reach_tolerance(cuda):
    """spm_batch_grad_flow with an FP32 phase (switch 1e-7, stagnation stop)
    and FP64 polish: every instance reaches ||grad F|| <= 1e-8 with the energy
    of its all-FP64 single flow to 1e-10 of the initial energy."""
    import spmiqc
    specs = [(32, 26.0, -0.02, 1), (64, 20.0, -0.015, 2), (32, 18.0, -0.01, 3)]
    ctxs, phis, uhs, ref = [], [], [], []
    for N, L, tau, seed in specs:
        c = spmiqc.SpmContext(N, L=L, Tau=tau)
        p0 = npo.uniform_field(N, seed)
        p = cuda.from_numpy(p0).cuda()
        ctxs.append(c), phis.append(p), uhs.append(c.my_fft(p))
        q = cuda.from_numpy(p0).cuda()
        uq = c.my_fft(q)
        E0 = c.get_Ene(q, uq)
        c.get_min_u_F(q, uq, 60000, tol_grad=1e-8)
        ref.append((E0, c.get_Ene(q, uq)))
    spmiqc.batch_grad_flow(ctxs, phis, uhs, 60000, 1e-8, switch_tol=1e-7, steps_per_launch=32)
    for c, p, u, (E0, E) in zip(ctxs, phis, uhs, ref):
        assert c.ngrad_cam(p)[1] <= 1e-8 * 1.01
        assert abs(c.get_Ene(p, u) - E) <= 1e-10 * abs(E0)
