"""Scheduler of the job server (spm_server_*) on a fake device, no GPU:
admission by device-memory footprint and slots, continuous admission of jobs
that arrive while others run, first-fit with a bypass limit, cancellation of
waiting and running jobs, allocation refusal on the device, latency
percentiles. The fake device sleeps in proportion to N^3 x steps."""
import time

import numpy as np
import pytest

import spmiqc
from spmiqc import JobServer, job_desc, job_footprint


def _phi(N, v=0.0):
    return np.full((N, N, N), v)


def _wait_all(srv, ids):
    return {j: srv.wait(j)[0] for j in ids}


def test_footprint_grows_with_size_and_kind():
    fr = [job_footprint(job_desc("relax", N)) for N in (64, 128, 192, 256)]
    assert fr == sorted(fr) and fr[-1] > 8 * fr[1] * 0.9
    assert job_footprint(job_desc("relax", 128, "fp32")) < job_footprint(job_desc("relax", 128))
    assert job_footprint(job_desc("relax", 128, "mixed")) > job_footprint(job_desc("relax", 128))
    lob = job_footprint(job_desc("lobpcg", 128, k=4))
    assert lob > job_footprint(job_desc("spm", 128)) > job_footprint(job_desc("relax", 128))
    # the field arrays of the job itself are a lower bound
    assert job_footprint(job_desc("lobpcg", 256, k=8)) > (1 + 7 * 8) * 256 ** 3 * 8


def test_admission_respects_budget_and_slots():
    d = job_desc("relax", 64, max_steps=100)
    fp = job_footprint(d)
    with JobServer(budget_bytes=int(2.5 * fp), max_slots=4, fake_device=True, fake_ms_per_munit=1.0) as srv:
        ids = [srv.submit(d, _phi(64, i)) for i in range(6)]
        res = _wait_all(srv, ids)
        st = srv.stats()
    assert all(r.status == 0 for r in res.values())
    assert st.completed == 6 and st.failed == 0
    assert st.peak_bytes <= st.budget_bytes and st.peak_running == 2
    # never more than two jobs in flight at any time
    ev = sorted([(r.t_start, 1) for r in res.values()] + [(r.t_end, -1) for r in res.values()])
    live = 0
    for _, s in ev:
        live += s
        assert live <= 2


def test_slots_limit_and_concurrency():
    d = job_desc("relax", 64, max_steps=200)
    with JobServer(budget_bytes=1 << 40, max_slots=3, fake_device=True, fake_ms_per_munit=1.0) as srv:
        ids = [srv.submit(d, _phi(64)) for _ in range(7)]
        res = _wait_all(srv, ids)
        st = srv.stats()
    assert st.peak_running == 3
    # three overlapped: the makespan is well below the serial sum
    span = max(r.t_end for r in res.values()) - min(r.t_start for r in res.values())
    serial = sum(r.t_end - r.t_start for r in res.values())
    assert span < 0.6 * serial


def test_late_arrival_joins_running_jobs():
    """Continuous batching: a job submitted while another runs starts before
    the running one ends."""
    with JobServer(budget_bytes=1 << 40, max_slots=4, fake_device=True, fake_ms_per_munit=2.0) as srv:
        a = srv.submit(job_desc("relax", 128, max_steps=150), _phi(128))  # ~0.6 s
        time.sleep(0.1)
        b = srv.submit(job_desc("relax", 64, max_steps=50), _phi(64))
        ra, rb = srv.wait(a)[0], srv.wait(b)[0]
    assert rb.t_start < ra.t_end and rb.t_end < ra.t_end
    assert rb.t_start - rb.t_submit < 0.05


def test_first_fit_with_bypass_limit():
    big = job_desc("relax", 128, max_steps=60)
    small = job_desc("relax", 64, max_steps=40)
    fb, fs = job_footprint(big), job_footprint(small)
    budget = fb + 2 * fs + 1
    with JobServer(budget_bytes=budget, max_slots=8, fake_device=True, fake_ms_per_munit=2.0,
                   max_bypass=2) as srv:
        b1 = srv.submit(big, _phi(128))
        time.sleep(0.02)
        b2 = srv.submit(big, _phi(128))      # does not fit while b1 runs
        s = [srv.submit(small, _phi(64)) for _ in range(4)]
        r = _wait_all(srv, [b1, b2] + s)
    # s[0], s[1] pass b2 (two bypasses); s[2], s[3] wait until b2 has started
    assert r[s[0]].t_start < r[b2].t_start and r[s[1]].t_start < r[b2].t_start
    assert r[s[2]].t_start >= r[b2].t_start and r[s[3]].t_start >= r[b2].t_start
    assert r[b2].t_start >= r[b1].t_end - 1e-3


def test_cancel_waiting_and_running_jobs():
    d = job_desc("relax", 128, max_steps=500)  # ~2 s at 2 ms per Munit-step
    with JobServer(budget_bytes=1 << 40, max_slots=1, fake_device=True, fake_ms_per_munit=2.0) as srv:
        a = srv.submit(d, _phi(128))
        b = srv.submit(d, _phi(128))
        time.sleep(0.1)
        srv.cancel(b)               # waiting
        srv.cancel(a)               # running: stops at its next check
        ra, rb = srv.wait(a)[0], srv.wait(b)[0]
        st = srv.stats()
        c = srv.submit(job_desc("relax", 64, max_steps=10), _phi(64, 0.5))
        rc, fc = srv.wait(c)
    assert ra.status == spmiqc.SPM_ERR_CANCELLED and rb.status == spmiqc.SPM_ERR_CANCELLED
    assert ra.t_end - ra.t_start < 1.0
    assert st.cancelled == 2 and st.completed == 0
    assert rc.status == 0 and np.all(fc == 0.5)


def test_allocation_refused_fails_job_and_server_continues():
    """The device refuses an allocation that the admission estimate allowed
    (memory held by someone else): that job fails with SPM_ERR_NOMEM, the
    reservation is returned and later jobs run."""
    d = job_desc("relax", 64, max_steps=100)
    fp = job_footprint(d)
    with JobServer(budget_bytes=4 * fp, max_slots=4, fake_device=True, fake_ms_per_munit=2.0,
                   fake_device_bytes=int(1.5 * fp)) as srv:
        ids = [srv.submit(d, _phi(64)) for _ in range(3)]
        res = _wait_all(srv, ids)
        late = srv.submit(d, _phi(64))
        rl = srv.wait(late)[0]
        st = srv.stats()
    codes = sorted(r.status for r in res.values())
    assert codes.count(0) >= 1 and codes.count(spmiqc.SPM_ERR_NOMEM) >= 1
    assert rl.status == 0
    assert st.failed == codes.count(spmiqc.SPM_ERR_NOMEM)


def test_job_larger_than_budget_is_refused_at_submission():
    d = job_desc("lobpcg", 256, k=8)
    with JobServer(budget_bytes=1 << 30, max_slots=2, fake_device=True) as srv:
        with pytest.raises(spmiqc.SpmError) as e:
            srv.submit(d, _phi(256))
        assert e.value.status == spmiqc.SPM_ERR_NOMEM
        with pytest.raises(spmiqc.SpmError):
            srv.submit(job_desc("relax", 100), _phi(100))  # size not built
        with pytest.raises(spmiqc.SpmError):
            srv.submit(job_desc("spm", 64), _phi(64))      # needs two replicas


def test_lobpcg_guard_vectors_are_checked_and_counted():
    """A LOBPCG job's guard vectors add to its footprint; k + guard above 8,
    a negative guard, or a guard on another kind of job is refused; the job
    returns its k vectors."""
    fp4 = job_footprint(job_desc("lobpcg", 128, k=4))
    fp8 = job_footprint(job_desc("lobpcg", 128, k=8))
    assert job_footprint(job_desc("lobpcg", 128, k=4, guard=4)) == fp8 > fp4
    with JobServer(budget_bytes=1 << 40, max_slots=2, fake_device=True, fake_ms_per_munit=0.01) as srv:
        for bad in (job_desc("lobpcg", 64, k=6, guard=3), job_desc("lobpcg", 64, k=4, guard=-1),
                    job_desc("relax", 64, guard=2)):
            with pytest.raises(spmiqc.SpmError) as e:
                srv.submit(bad, _phi(64))
            assert e.value.status == spmiqc.SPM_ERR_ARG
        j = srv.submit(job_desc("lobpcg", 32, k=3, guard=2, max_steps=5), _phi(32, 0.5))
        r, V = srv.wait(j)
    assert r.status == 0 and V.shape == (3, 32, 32, 32)


def test_latency_percentiles_and_results():
    rng = np.random.default_rng(3)
    with JobServer(budget_bytes=1 << 40, max_slots=2, fake_device=True, fake_ms_per_munit=1.0) as srv:
        ids = []
        for i in range(12):
            N = int(rng.choice([64, 128]))
            kind = ["relax", "lobpcg", "spm"][i % 3]
            p = _phi(N, float(i))
            ids.append((srv.submit(job_desc(kind, N, max_steps=20, k=2), p, p + 1 if kind == "spm" else None),
                        kind, i))
        lat = []
        for jid, kind, i in ids:
            r, f = srv.wait(jid)
            assert r.status == 0
            lat.append(r.t_end - r.t_submit)
            want = float(i) + (1 if kind == "spm" else 0)
            assert f is not None and np.all(f == want)
            srv.release(jid)
        st = srv.stats()
    lat = np.sort(lat)
    assert st.completed == 12
    assert abs(st.p50_s - lat[5]) < 1e-3 and abs(st.p99_s - lat[-1]) < 1e-3


def test_serving_stream_is_seeded_and_mixed():
    import workloads
    a = workloads.serving_stream(7, 400)
    b = workloads.serving_stream(7, 400)
    assert a == b
    kinds = [s.kind for s in a]
    assert 0.6 < kinds.count("relax") / 400 < 0.8 and 0.12 < kinds.count("lobpcg") / 400 < 0.28
    assert 0.04 < kinds.count("spm") / 400 < 0.16
    assert {s.N for s in a} == {64, 128, 192, 256}
    gaps = np.diff([0.0] + [s.t_arrival for s in a])
    assert 0.2 < gaps.mean() < 0.3          # mean 4 jobs/s
    assert all(18 <= s.L <= 30 and -0.02 <= s.Tau <= 0 and 0.1 <= s.amp <= 0.2 for s in a)
    s = a[0]
    f = workloads.field(s, N=32)
    assert f.shape == (32, 32, 32) and np.isfinite(f).all()
    p0, p1 = workloads.replicas(s, f)
    assert 0.005 < np.max(np.abs(p1 - p0)) <= 0.01 + 1e-12
