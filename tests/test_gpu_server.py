"""Job server on the GPU: a mix of relaxation, eigenmode and saddle jobs of
different grid sizes and precisions runs concurrently, and every job's result
(field, energy, residual, eigenvalues, step count) is bit-identical to the
same job run alone on an idle server, and to the direct API call. A running
job cancelled from the host stops at its next check."""
import time

import numpy as np
import pytest

from oracle import spmiqc_np as npo

pytestmark = pytest.mark.gpu


def _jobs():
    import spmiqc
    jd = spmiqc.job_desc
    a = npo.uniform_field(64, 5)
    b = npo.uniform_field(32, 6)
    c = npo.uniform_field(32, 7)
    d0 = npo.uniform_field(32, 8)
    d1 = d0 + 0.01 * npo.uniform_field(32, 9)
    e = npo.uniform_field(96, 10)
    return [
        (jd("relax", 64, max_steps=400, tol=1e-9, L=20.0, Tau=-0.01), a, None),
        (jd("relax", 32, "mixed", max_steps=3000, tol=1e-8, switch_tol=1e-6, Tau=-0.02), b, None),
        (jd("lobpcg", 32, k=4, max_steps=15, tol=0.0, seed=11), c, None),
        (jd("spm", 32, max_steps=40, tol=1e-12), d0, d1),
        (jd("relax", 96, "fp32", max_steps=200, tol=1e-7, Tau=-0.015), e, None),
        (jd("spm", 32, "mixed", max_steps=200, tol=1e-9, switch_tol=1e-5), d1, d0),
    ]


def _run(jobs, slots):
    import spmiqc
    out = []
    with spmiqc.JobServer(max_slots=slots) as srv:
        ids = [srv.submit(d, p0, p1) for d, p0, p1 in jobs]
        for i in ids:
            out.append(srv.wait(i))
        st = srv.stats()
    return out, st


def test_results_identical_alone_and_in_the_mix(cuda):
    jobs = _jobs()
    mix, st = _run(jobs, slots=len(jobs))
    assert st.completed == len(jobs) and st.failed == 0
    assert st.peak_running >= 2
    for i, job in enumerate(jobs):
        alone, _ = _run([job], slots=1)
        ra, fa = alone[0]
        rm, fm = mix[i]
        assert ra.status == 0 and rm.status == 0, (i, ra.status, rm.status)
        assert ra.steps == rm.steps, i
        assert ra.energy == rm.energy and ra.residual == rm.residual, i
        assert list(ra.evals) == list(rm.evals), i
        assert np.array_equal(fa, fm), i


def test_relax_job_matches_direct_api(cuda):
    import spmiqc
    N = 64
    p0 = npo.uniform_field(N, 5)
    ctx = spmiqc.SpmContext(N, L=20.0, Tau=-0.01)
    p = cuda.from_numpy(p0).cuda()
    u = ctx.my_fft(p)
    stats = ctx.get_min_u_F(p, u, 400, tol_grad=1e-9)
    E = ctx.get_Ene(p, u)
    with spmiqc.JobServer(max_slots=2) as srv:
        r, f = srv.wait(srv.submit(spmiqc.job_desc("relax", N, max_steps=400, tol=1e-9, L=20.0, Tau=-0.01), p0))
    assert r.steps == len(stats)
    assert r.energy == E
    assert np.array_equal(f, p.cpu().numpy())


def test_cancel_running_job_on_gpu(cuda):
    import spmiqc
    N = 256  # ~0.4 ms per step: far from converged after 1 s
    with spmiqc.JobServer(max_slots=2) as srv:
        jid = srv.submit(spmiqc.job_desc("relax", N, max_steps=200000, tol=1e-300), npo.uniform_field(N, 3))
        time.sleep(1.0)
        srv.cancel(jid)
        r, f = srv.wait(jid)
        ok = srv.submit(spmiqc.job_desc("relax", 32, max_steps=10, tol=1e-9), npo.uniform_field(32, 4))
        r2, _ = srv.wait(ok)
    assert r.status == spmiqc.SPM_ERR_CANCELLED and f is None
    assert r.t_end - r.t_start < 5.0
    assert r2.status == 0
