"""Headline benchmark: semi-implicit gradient-flow steps/s on a 256^3 grid, FP64.

Workload (one "step" = one get_min_u_F iteration, LPsrc.cpp:52-110, with its
energy, res and ||grad F|| reductions): N = 256, L = 26, Tau = -0.0061,
Gamma = 0.30, dt = 0.3, phi0 = 0.15 * sum over the 30 icosahedral shell vectors
of cos(2 pi n.x/N + theta) + N(0, 1e-3^2) noise (seeded). Fields stay in HBM;
each step moves 0.81 GB (6 fields) through HBM, well above the 126 MB L2, so no
L2 flush is needed.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun): every rank runs an independent 256^3 flow (replicas:
the path needs no exchange between GPUs); value = steps of all ranks / max
rank time. Extra keys report Hv/s (batch of 8), FP32 steps/s, per-step p50/p99,
the per-kernel roofline and the CPU baseline.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "spm-iqc_b200"))

N = 256
L, TAU, GAMMA, DT = 26.0, -0.0061, 0.30, 0.3
METRIC = "N=256^3 grad-flow steps/s (FP64)"
WORKLOAD = ("grad-flow 256^3 FP64, L=26, Tau=-0.0061, Gamma=0.30, dt=0.3, phi0 = icosahedral "
            "30-vector cosine shell (amp 0.15) + N(0,1e-3) noise")


def kernel_traffic(schedule=None):
    """DRAM bytes per launch of the step kernels at 256^3 FP64, from the ncu
    captures summarised in profiles/kernel_traffic_256_fp64.md (lines
    `traffic <kernel> <bytes> <plane_cps,fuse_planes,plane_xg>`): those of the
    given schedule, else of the first schedule listed."""
    out, first = {}, {}
    want = None if schedule is None else f"{schedule['plane_cps']},{schedule['fuse_planes']},{schedule['plane_xg']}"
    try:
        with open(os.path.join(ROOT, "profiles", "kernel_traffic_256_fp64.md")) as f:
            for line in f:
                parts = line.split()
                if len(parts) == 4 and parts[0] == "traffic":
                    first.setdefault(parts[1], int(parts[2]))
                    if parts[3] == want:
                        out[parts[1]] = int(parts[2])
    except OSError:
        pass
    return out or first


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "100", "-i", str(self.idx)], stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for i, n in enumerate(names):
                    if "Active" in r[5 + i] and "Not" not in r[5 + i]:
                        reasons.add(n)
            except Exception:
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    """One process per GPU (torchrun env). NCCL with a GPU; gloo on a CPU-only
    host (the multi-rank logic is tested that way)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if not dist.is_initialized():
            if torch.cuda.is_available():
                torch.cuda.set_device(local)
                dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
            else:
                dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    return rank, world, local


def _dev():
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def gather_over_ranks(items: list, world: int) -> list:
    """Concatenation of every rank's list (same order of ranks on all ranks)."""
    if world == 1:
        return list(items)
    import torch.distributed as dist
    out = [None] * world
    dist.all_gather_object(out, list(items))
    return [x for part in out for x in part]


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_dev())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def initial_field(seed: int):
    import inputs
    return inputs.cosine_shell(N, inputs.icosahedral_shell(), amp=0.15, seed=seed, noise=1e-3)


def cpu_reference_steps(phi, budget_s: float, max_steps: int, warm: int = 1):
    """Times the reference's own get_min_u_F loop (compiled in place, shimmed
    FFT on all host threads), one iteration per call, until budget_s elapses."""
    from oracle import refbind
    threads = os.cpu_count() or 1
    r = refbind.Ref(N, L, TAU, GAMMA, DT, threads=threads)
    r.set_state(phi)
    for _ in range(warm):
        r.get_min_u_F(1)
    t0 = time.perf_counter()
    n = 0
    while n < max_steps and (time.perf_counter() - t0) < budget_s:
        r.get_min_u_F(1)
        n += 1
    dt = time.perf_counter() - t0
    r.close()
    return n / dt, threads, n, dt


def cpu_legs(ctx, phi_h, budget_s: float = 20.0, n_parity: int = 3, max_timed: int = 10):
    """The CPU side of the benchmark, on the same 256^3 workload and phi0:

    * parity: the reference's own get_min_u_F (compiled here, one rank) runs
      n_parity steps that record E, res and ||grad F|| per step, then up to
      max_timed plain iterations (timed: cpu_baseline); the GPU context the
      benchmark times (its autotuned schedule) runs the same number of steps
      from the same phi0, and the records, the final phi and u, and the final
      energy and ||grad F|| are compared (the FP64 bar is 1e-11 relative);
    * the same reference on one host thread (a bounded sample);
    * an FFTW-class arm: the step restated over torch's CPU FFT (MKL) on all
      host threads (oracle/cpu_mkl.py), the reference planning FFTW with
      FFTW_PATIENT (My_FFT.cpp:70-85) where this image has no FFTW.
    Returns (cpu_baseline, parity, serial, mkl)."""
    import numpy as np
    import torch
    from oracle import refbind
    threads = os.cpu_count() or 1
    r = refbind.Ref(N, L, TAU, GAMMA, DT, threads=threads)
    r.set_state(phi_h)
    E, res, g = r.grad_steps(n_parity)
    t0 = time.perf_counter()
    n = 0
    while n < max_timed and (time.perf_counter() - t0) < budget_s:
        r.get_min_u_F(1)
        n += 1
    dt = time.perf_counter() - t0
    cpu = {"value": n / dt, "unit": "steps/s", "cores": threads, "kind": "reference",
           "sample": f"{n} full 256^3 steps in {dt:.1f} s after {n_parity} recorded steps (reference src/*.cpp "
                     f"compiled unchanged, project FFT shim on {threads} threads)"}
    p_ref, u_ref = r.get_state()
    E_end = r.energy()
    g_end = float(np.sqrt(np.mean(r.ngrad(p_ref) ** 2)))
    # one host thread: a bounded sample of the same loop
    r.set_threads(1)
    t0 = time.perf_counter()
    ns = 0
    while ns < 3 and (ns == 0 or (time.perf_counter() - t0) < 0.5 * budget_s):
        r.get_min_u_F(1)
        ns += 1
    dts = time.perf_counter() - t0
    r.close()
    serial = {"value": ns / dts, "unit": "steps/s", "cores": 1, "kind": "reference",
              "sample": f"{ns} full 256^3 steps in {dts:.1f} s, shim FFT on one thread"}
    total = n_parity + n
    phi = torch.from_numpy(phi_h.copy()).cuda()
    uh = ctx.my_fft(phi)
    st = ctx.get_min_u_F(phi, uh, total)
    E_gpu, g_gpu = ctx.get_Ene(phi, uh), ctx.ngrad_cam(phi)[1]
    pg, ug = phi.cpu().numpy(), ctx.to_full(uh).cpu().numpy()

    def srel(a, b):
        return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
    parity = {"steps": total, "schedule": ctx.tuning(),
              "per_step_max_rel_dE": float(np.max(np.abs(st[:n_parity, 0] - E) / np.abs(E))),
              "per_step_max_rel_dgrad": float(np.max(np.abs(st[:n_parity, 2] - g) / np.abs(g))),
              "per_step_max_rel_dres": float(np.max(np.abs(st[:n_parity, 1] - res) / np.abs(res))),
              "final_rel_dE": abs(E_gpu - E_end) / abs(E_end), "final_rel_dgrad": abs(g_gpu - g_end) / g_end,
              "phi_scale_rel_diff": srel(pg, p_ref), "u_scale_rel_diff": srel(ug, u_ref), "bar": 1e-11}
    parity["pass"] = all(parity[k] <= 1e-11 for k in ("per_step_max_rel_dE", "per_step_max_rel_dgrad",
                                                          "final_rel_dE", "final_rel_dgrad", "phi_scale_rel_diff",
                                                          "u_scale_rel_diff"))
    del phi, uh
    mkl = mkl_arm(phi_h, budget_s=0.5 * budget_s, max_steps=20, threads=threads)
    return cpu, parity, serial, mkl


def mkl_arm(phi_h, budget_s: float, max_steps: int, threads: int):
    """The gradient step over torch's CPU FFT (MKL): one warm-up step, then
    timed steps until budget_s or max_steps."""
    import torch
    from oracle import cpu_mkl
    f = cpu_mkl.MklFlow(N, L, TAU, GAMMA, DT, threads=threads)
    p = torch.from_numpy(phi_h.copy())
    u = f.spectrum(p)
    p, u, *_ = f.step(p, u)
    t0 = time.perf_counter()
    n = 0
    while n < max_steps and (time.perf_counter() - t0) < budget_s:
        p, u, *_ = f.step(p, u)
        n += 1
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "steps/s", "cores": f.threads, "kind": "port",
            "sample": f"{n} full 256^3 steps in {dt:.1f} s: the step (E, res, ||grad F||, one R2C and one C2R "
                      f"transform) restated over torch.fft on the CPU (Intel MKL), {f.threads} threads"}


def reference_arm(args, rank, world):
    if rank != 0:
        return 0
    import numpy as np
    from oracle import refbind
    if not refbind.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libspmref.so not built"}))
        return 0
    phi = initial_field(1)
    warm = min(args.warmup, 1)
    v, cores, n, dt = cpu_reference_steps(phi, budget_s=90.0, max_steps=args.steps, warm=warm)
    sample = (f"{n} of the requested {args.steps} steps (each step the full 256^3 workload), "
              f"{dt:.1f} s, after {warm} warm-up step(s); reference src/*.cpp compiled unchanged with the "
              f"project FFT shim on {cores} threads")
    try:  # the same step over an FFTW-class library FFT, beside the shimmed reference
        mkl = mkl_arm(phi, budget_s=15.0, max_steps=max(args.steps, 1), threads=cores)
    except Exception as ex:
        mkl = {"value": None, "sample": f"unavailable: {ex}"}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": world,
            "steps": n, "warmup": warm, "ms_per_step": 1000.0 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "N": N},
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": cores, "kind": "reference", "sample": sample},
            "cpu_baseline_mkl": mkl,
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# Step caps of the serving jobs: each job runs to ||grad F|| (LOBPCG: the
# block residual) <= 1e-8 and stops there; the cap only bounds jobs whose
# stationary point keeps the flow above the tolerance (a saddle, or a minimum
# whose rounding floor of ||grad F|| lies near 1e-8, as the SPM saddle search's
# index-1 point at 256^3 does with a floor of about 1.08e-8).
SERVE_CAPS = {"relax": 20000, "lobpcg": 400, "spm": 3000}
# LOBPCG jobs (k = 4) iterate a block of 8 and stop on the first 4 residuals:
# the stream's cosine-shell fields have close eigenvalue pairs around the 4th,
# where a block of 4 stalls above 1e-8 within the cap
SERVE_LOBPCG_GUARD = 4


def _serve_run(specs, fields, precision_of, slots, tol, fake=False, t0=None):
    """Replays the arrival stream into a job server; returns per-job results and
    server stats. fake: the server's fake device (scheduler only, no GPU)."""
    import spmiqc
    srv = (spmiqc.JobServer(budget_bytes=64 << 30, max_slots=slots, fake_device=True, fake_ms_per_munit=0.5)
           if fake else spmiqc.JobServer(max_slots=slots))
    ids = []
    t0 = time.perf_counter() if t0 is None else t0
    for s, (p0, p1) in zip(specs, fields):
        delay = s.t_arrival - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        prec = precision_of(s.kind)
        d = spmiqc.job_desc(s.kind, s.N, prec, k=4, max_steps=SERVE_CAPS[s.kind], L=s.L, Tau=s.Tau, tol=tol,
                            switch_tol=0.0, seed=s.seed, guard=SERVE_LOBPCG_GUARD if s.kind == "lobpcg" else 0)
        ids.append(srv.submit(d, p0, p1))
    res = [srv.wait(i, field=False)[0] for i in ids]
    st = srv.stats()
    srv.close()
    return res, st


def serve_ranks(specs, make_fields, rank, world, slots, precision_of, tol, fake=False):
    """Runs this rank's share of the stream (jobs partitioned over the ranks by
    device-memory footprint, arrival times kept) and returns the whole-job
    aggregate on every rank: completed jobs of all ranks / the longest makespan,
    latency percentiles over all jobs."""
    import numpy as np
    import workloads
    mine = workloads.partition_jobs(specs, world)[rank]
    sub = [specs[i] for i in mine]
    fields = [make_fields(s) for s in sub]
    barrier(world)
    res, st = _serve_run(sub, fields, precision_of, slots, tol, fake=fake)
    ok = [r for r in res if r.status == 0]
    span = (max(r.t_end for r in res) - min(r.t_submit for r in res)) if res else 0.0
    lat = gather_over_ranks([r.t_end - r.t_submit for r in ok], world)
    fails = gather_over_ranks([f"{s.kind} N={s.N}: {r.message.decode()}" for s, r in zip(sub, res) if r.status != 0],
                              world)
    conv = {k: int(sum(1 for s, r in zip(sub, res) if s.kind == k and r.status == 0 and r.residual <= tol))
            for k in SERVE_CAPS}
    conv = {k: sum(c[k] for c in gather_over_ranks([conv], world)) for k in SERVE_CAPS}
    completed = len(lat)
    span = max_over_ranks(span, world)
    # rank 0's server peaks, the same on every rank
    peak_run0, peak_gb0 = gather_over_ranks([(int(st.peak_running), st.peak_bytes / 1e9)], world)[0]
    lat = np.array(lat) if lat else np.zeros(1)
    return {"failures": fails, "jobs_per_s": completed / span if span > 0 else 0.0,
            "p50_s": float(np.percentile(lat, 50, method="inverted_cdf")),
            "p99_s": float(np.percentile(lat, 99, method="inverted_cdf")), "completed": completed,
            "failed": len(fails), "peak_running_rank0": int(peak_run0),
            "peak_reserved_gb_rank0": peak_gb0, "makespan_s": span, "reached_tol": conv,
            "jobs_per_rank": [len(p) for p in workloads.partition_jobs(specs, world)]}


def batch_core(n_inst, cap, branches, rank=0, world=1):
    """Batched relaxations: n_inst instances of uneven sizes (N in {64, ...,
    256}, L ~ U[18, 30], Tau ~ U[-0.02, 0], BCC / FCC / icosahedral cosine
    fields) relaxed together by spm_batch_grad_flow (one captured graph per
    launch; instances of one size share every launch; FP32 bulk, then FP64
    polish) to ||grad F|| <= 1e-8 or the step cap, next to the same instances
    relaxed one after another in FP64 with spm_grad_flow (the reference's one
    flow per program); with `branches` also the batched run with one branch and
    launch per instance. Whole-batch time with the fields resident on the
    device. Returns the summary (rank 0's view)."""
    import torch
    import spmiqc
    import workloads
    specs = workloads.batch_instances(seed=7 + rank, n=n_inst)
    fields = [workloads.field(s, device="cuda") for s in specs]
    tol = 1e-8
    out = {}
    arms = ("batched_mixed", "batched_mixed_branches", "serial_fp64") if branches else ("batched_mixed", "serial_fp64")
    for name in arms:
        ctxs = [spmiqc.SpmContext(s.N, L=s.L, Tau=s.Tau) for s in specs]
        for c, s in zip(ctxs, specs):
            c.autotune(20)
            # batched_mixed: instances of one size share every launch; _branches: one branch per instance
            c.tune("batch_group", 0 if name == "batched_mixed_branches" else 1)
        phis = [torch.from_numpy(f.copy()).cuda() for f in fields]
        uhs = [c.my_fft(p) for c, p in zip(ctxs, phis)]
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        if name.startswith("batched_mixed"):
            steps = spmiqc.batch_grad_flow(ctxs, phis, uhs, cap, tol, switch_tol=1e-7, steps_per_launch=32)
        else:
            steps = [len(c.get_min_u_F(p, u, cap, tol_grad=tol)) for c, p, u in zip(ctxs, phis, uhs)]
        torch.cuda.synchronize()
        dt = max_over_ranks(time.perf_counter() - t0, world)
        gn = [c.ngrad_cam(p)[1] for c, p in zip(ctxs, phis)]
        E = [c.get_Ene(p, u) for c, p, u in zip(ctxs, phis, uhs)]
        out[name] = {"seconds": dt, "instances_per_s": world * len(specs) / dt, "steps": steps,
                     "reached_tol": int(sum(g <= tol for g in gn)), "grad_norm": gn, "energy": E}
        for c in ctxs:
            c.close()
        del phis, uhs
        torch.cuda.empty_cache()
    a, b = out["batched_mixed"], out["serial_fp64"]
    both = [i for i in range(len(specs)) if a["grad_norm"][i] <= tol and b["grad_norm"][i] <= tol]
    # energies of converged flows: absolute difference, and relative to max(|E|, 1e-6) (a field that
    # decays to the disordered state has E ~ 0, where a plain relative difference says nothing)
    eabs = max((abs(a["energy"][i] - b["energy"][i]) for i in both), default=None)
    ediff = max((abs(a["energy"][i] - b["energy"][i]) / max(abs(b["energy"][i]), 1e-6) for i in both), default=None)
    keys = ("seconds", "instances_per_s", "steps", "reached_tol")
    return {"instances_per_s": a["instances_per_s"], "speedup_vs_serial_fp64": b["seconds"] / a["seconds"],
            "batched_mixed": {k: a[k] for k in keys}, "serial_fp64": {k: b[k] for k in keys},
            "batched_mixed_branches": ({k: out["batched_mixed_branches"][k] for k in keys}
                                       if "batched_mixed_branches" in out else None),
            "not_converged": [[s.N, round(s.L, 3), round(s.Tau, 5), s.shell, float(g)]
                              for s, g in zip(specs, b["grad_norm"]) if g > tol],
            "max_abs_energy_diff_where_both_converged": eabs, "max_rel_energy_diff_where_both_converged": ediff,
            "energy_range": [min(b["energy"]), max(b["energy"])],
            "config": {"workload": "batched relaxations", "instances": [[s.N, round(s.L, 3), round(s.Tau, 5), s.shell]
                                                                     for s in specs],
                       "step_cap": cap, "tol": tol, "switch_tol": 1e-7, "steps_per_launch": 32}}


def batch_bench(args):
    """The batched-relaxation workload as its own JSON line (batch_core)."""
    import torch
    rank, world, local = dist_setup()
    torch.cuda.set_device(local)
    r = batch_core(args.batch_n, args.batch_steps, args.batch_branches, rank, world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": f"batched relaxations: instances/s to ||grad F|| <= 1e-8 ({args.batch_n} uneven instances)",
            "value": r["instances_per_s"], "unit": "instances/s", "n_gpus": world, "higher_is_better": True,
            "scaling": "weak", "data": "synthetic", "dtype": "f32+f64"}
    line.update({k: v for k, v in r.items() if k != "instances_per_s"})
    print(json.dumps(line))
    return 0


def serve_core(n_jobs, slots, rank=0, world=1):
    """Serving workload: a seeded Poisson stream (mean 4 jobs/s) of 70%
    relaxations (FP32 + FP64 polish), 20% k=4 LOBPCG (FP64) and 10% SPM saddle
    searches (FP32 + FP64 polish), N in {64, 128, 192, 256}, every job to
    tolerance 1e-8 within its step cap (SERVE_CAPS), run through the job server
    with concurrent slots, next to the same stream executed serially in FP64
    (one job at a time, as the reference's one-job-per-program drivers do)."""
    import torch
    import workloads
    specs = workloads.serving_stream(seed=2024, n_jobs=n_jobs, rate=4.0 * world)

    def make_fields(s):
        p = workloads.field(s, device="cuda")
        return workloads.replicas(s, p) if s.kind == "spm" else (p, None)

    tol = 1e-8
    out = {}
    for name, nsl, prec in (("served", slots, lambda k: "fp64" if k == "lobpcg" else "mixed"),
                            ("serial_fp64", 1, lambda k: "fp64")):
        out[name] = serve_ranks(specs, make_fields, rank, world, nsl, prec, tol)
        torch.cuda.empty_cache()
    kinds = {k: sum(1 for s in specs if s.kind == k) for k in SERVE_CAPS}
    sizes = {str(n): sum(1 for s in specs if s.N == n) for n in (64, 128, 192, 256)}
    return {"jobs_per_s": out["served"]["jobs_per_s"], "p50_s": out["served"]["p50_s"], "p99_s": out["served"]["p99_s"],
            "speedup_vs_serial_fp64": (out["served"]["jobs_per_s"] / out["serial_fp64"]["jobs_per_s"]
                                       if out["serial_fp64"]["jobs_per_s"] else None),
            "served": out["served"], "serial_fp64": out["serial_fp64"],
            "config": {"workload": "serving stream", "jobs": len(specs), "kinds": kinds, "sizes": sizes,
                       "caps": SERVE_CAPS, "lobpcg_guard": SERVE_LOBPCG_GUARD, "tol": tol, "slots": slots, "seed": 2024, "rate_per_s": 4.0 * world,
                       "parallelism": f"jobs partitioned by footprint over {world} GPU(s)"}}


def serve_bench(args):
    """The serving workload as its own JSON line (serve_core)."""
    import torch
    rank, world, local = dist_setup()
    torch.cuda.set_device(local)
    r = serve_core(args.serve_jobs, args.serve_slots, rank, world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": "serving jobs/s (Poisson 4/s, 70% relax / 20% LOBPCG k=4 / 10% SPM)",
            "value": r["jobs_per_s"], "unit": "jobs/s", "n_gpus": world, "higher_is_better": True,
            "scaling": "weak", "data": "synthetic"}
    line.update({k: v for k, v in r.items() if k != "jobs_per_s"})
    print(json.dumps(line))
    return 0


def config_legs(ctx, phi_h):
    """The two 256^3 FP64 workloads beyond the timed flow (their own keys on the
    benchmark line), from the same icosahedral phi0:

    config2: semi-implicit gradient flow (LPsrc.cpp:40-117) to ||grad F|| <= 1e-8
      in FP64 and in FP32 + FP64 polish, then LOBPCG k = 8 (LOBPCG.cpp:207-487)
      to a residual <= 1e-8 at the end state. The stationary point this field
      relaxes to has one negative Hessian eigenvalue and three near-zero
      (translation) ones, so ||grad F|| bottoms out just above 1e-8: the flows
      run to a step cap with tol 1e-8 (floor reported), and the FP64 / mixed
      time comparison is made at tol_reached, the lowest tolerance both reach.
    config3: Spring_Pairing (SPM.cpp:170-263) from that stationary point +- delta v1
      (v1 the unstable eigenmode, nrmp(v1) = 1; delta = 0.001, the reference's
      own separation, main_SPM.cpp:109-119) in FP64 and in FP32 + FP64 polish,
      with the saddle energy and the unstable eigenvalue (LOBPCG k = 1 with 3
      guard vectors at the saddle) of the mixed run against the all-FP64 run."""
    import numpy as np
    import torch
    out = {"config2": {}, "config3": {}}
    c2 = out["config2"]
    tol, tol_r, cap, sw = 1e-8, 1.2e-8, 40000, 2e-8

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return r, time.perf_counter() - t0

    runs = {}
    for mode in ("fp64", "mixed"):
        a = torch.from_numpy(phi_h.copy()).cuda()
        ua = ctx.my_fft(a)
        if mode == "fp64":
            st, sec = timed(lambda: ctx.get_min_u_F(a, ua, cap, tol_grad=tol_r))
            n32, n64 = 0, len(st)
        else:
            (st, n32, n64), sec = timed(lambda: ctx.get_min_u_F_mixed(a, ua, cap, tol_grad=tol_r, switch_tol=sw))
        runs[mode] = (a, ua)
        c2[mode] = {"tol": tol_r, "seconds": sec, "fp32_steps": n32, "fp64_steps": n64,
                    "grad_norm": float(st[-1, 2]), "reached": bool(st[-1, 2] <= tol_r),
                    "energy": ctx.get_Ene(a, ua)}
    c2["mixed"]["switch_tol"] = sw
    c2["speedup_mixed_vs_fp64"] = c2["fp64"]["seconds"] / c2["mixed"]["seconds"]
    c2["energy_rel_diff_mixed_vs_fp64"] = abs(c2["mixed"]["energy"] - c2["fp64"]["energy"]) / abs(c2["fp64"]["energy"])
    # the FP64 state continues toward 1e-8: where ||grad F|| bottoms out
    a, ua = runs["fp64"]
    del runs["mixed"]
    st = ctx.get_min_u_F(a, ua, cap - c2["fp64"]["fp64_steps"], tol_grad=tol)
    c2["toward_1e-8"] = {"tol": tol, "steps_total": c2["fp64"]["fp64_steps"] + len(st),
                         "min_grad_norm": float(st[:, 2].min()), "reached": bool(st[:, 2].min() <= tol),
                         "energy": ctx.get_Ene(a, ua)}
    V = ctx.hiosd_lobpcg_initialization(8, seed=3)
    (ev, rs, its), sec = timed(lambda: ctx.hiosd_lobpcg_inip(a, V, maxiter=800, tol=1e-8))
    c2["lobpcg_k8"] = {"tol": 1e-8, "iterations": its, "seconds": sec, "iterations_per_s": its / sec,
                       "evals": [float(x) for x in ev], "max_residual": float(max(rs)),
                       "reached": bool(max(rs) <= 1e-8)}
    v1 = V[0].clone()
    del V
    torch.cuda.empty_cache()
    c3 = out["config3"]
    delta, tol3, cap3, sw3 = 0.001, 1.1e-8, 3000, 3e-8
    c3.update({"delta": delta, "tol": tol3, "cap": cap3})
    for mode in ("fp64", "mixed"):
        p0 = (a - delta * v1).contiguous()
        p1 = (a + delta * v1).contiguous()
        if mode == "fp64":
            h, sec = timed(lambda: ctx.Spring_Pairing(p0, p1, cap3, tol3))
            n32, n64 = 0, len(h)
        else:
            (h, n32, n64), sec = timed(lambda: ctx.Spring_Pairing_mixed(p0, p1, cap3, tol3, switch_tol=sw3))
        mid = (0.5 * (p0 + p1)).contiguous()
        um = ctx.my_fft(mid)
        # the unstable mode: LOBPCG k = 1 with 3 guard vectors (the translation
        # modes, eigenvalues ~1e-8, sit close above it)
        W = ctx.hiosd_lobpcg_initialization(4, seed=9)
        ev, rs, lits = ctx.lobpcg_guarded(mid, W, 1, maxiter=800, tol=1e-8)
        c3[mode] = {"seconds": sec, "fp32_iterations": n32, "fp64_iterations": n64, "residual": float(h[-1]),
                    "reached": bool(h[-1] <= tol3), "saddle_energy": ctx.get_Ene(mid, um),
                    "unstable_eigenvalue": float(ev[0]), "lobpcg_k": 1, "lobpcg_guard": 3,
                    "lobpcg_iterations": lits, "lobpcg_residual": float(rs[0])}
        del p0, p1, mid, um, W
        torch.cuda.empty_cache()
    c3["mixed"]["switch_tol"] = sw3
    c3["speedup_mixed_vs_fp64"] = c3["fp64"]["seconds"] / c3["mixed"]["seconds"]
    c3["saddle_energy_rel_err"] = abs(c3["mixed"]["saddle_energy"] - c3["fp64"]["saddle_energy"]) / abs(
        c3["fp64"]["saddle_energy"])
    c3["unstable_eigenvalue_rel_err"] = abs(c3["mixed"]["unstable_eigenvalue"] - c3["fp64"]["unstable_eigenvalue"]) / abs(
        c3["fp64"]["unstable_eigenvalue"])
    del a, ua, v1
    torch.cuda.empty_cache()
    return out


def solver_legs(ctx, phi):
    """LOBPCG (k = 8, the reference's 21 iterations per call) and 50 SPM
    spring-pair iterations (replicas phi and phi + 0.001 v1) on the field phi,
    one timed call each after a warm-up call."""
    import torch
    solvers = {}
    try:
        # the building blocks: my_fft, my_ifft, ngrad_cam (one call each, 20 times)
        uh = ctx.my_fft(phi)
        back = torch.empty_like(phi)
        grad = torch.empty_like(phi)
        ctx.my_ifft(uh, back)
        ctx.ngrad_cam(phi, grad)
        for name, fn in (("my_fft", lambda: ctx.my_fft(phi, uh)), ("my_ifft", lambda: ctx.my_ifft(uh, back)),
                         ("ngrad_cam", lambda: ctx.ngrad_cam(phi, grad))):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(20):
                fn()
            torch.cuda.synchronize()
            solvers[name + "_per_s"] = 20 / (time.perf_counter() - t0)
        del uh, back, grad
        Vb = ctx.hiosd_lobpcg_initialization(8, seed=3)
        ctx.hiosd_lobpcg_inip(phi, Vb, maxiter=2)
        Vb = ctx.hiosd_lobpcg_initialization(8, seed=3)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ev, rs, its = ctx.hiosd_lobpcg_inip(phi, Vb, maxiter=21)
        torch.cuda.synchronize()
        dt_l = time.perf_counter() - t0
        solvers["lobpcg_k8"] = {"seconds_per_call": dt_l, "iterations": its, "iterations_per_s": its / dt_l,
                                "max_residual": float(max(rs))}
        v1 = Vb[0].clone()
        del Vb
        p0 = phi.clone()
        p1 = phi + 0.001 * v1
        ctx.Spring_Pairing(p0, p1, 2, 0.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hist = ctx.Spring_Pairing(p0, p1, 50, 0.0)
        torch.cuda.synchronize()
        dt_s = time.perf_counter() - t0
        solvers["spm"] = {"iterations": len(hist), "iterations_per_s": len(hist) / dt_s,
                          "last_residual": float(hist[-1])}
        del p0, p1, v1
    except Exception as ex:  # a solver leg that fails is reported, not fatal
        solvers["error"] = str(ex)[:200]
    torch.cuda.empty_cache()
    return solvers


def solvers_bench(args):
    """LOBPCG and SPM iterations at 256^3 FP64 on the bench field after 100
    gradient steps (one JSON line; also the command of their ncu captures)."""
    import torch
    import spmiqc
    rank, world, local = dist_setup()
    torch.cuda.set_device(local)
    n = args.solvers_n
    ctx = spmiqc.SpmContext(n, L, TAU, GAMMA, DT, "fp64")
    import inputs
    phi = torch.from_numpy(inputs.cosine_shell(n, inputs.icosahedral_shell(), amp=0.15, seed=1 + rank,
                                               noise=1e-3)).cuda()
    uh = ctx.my_fft(phi)
    ctx.get_min_u_F(phi, uh, 100)
    out = solver_legs(ctx, phi)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"metric": f"LOBPCG k=8 iterations/s and SPM iterations/s ({n}^3 FP64)",
                          f"solvers_{n}_fp64": out, "n_gpus": world, "data": "synthetic",
                          "config": {"workload": "bench field after 100 gradient steps", "N": n}}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--flow-precision", default="fp64", choices=["fp64", "fp32"],
                    help="precision of the --only-flow run")
    ap.add_argument("--only-flow", action="store_true",
                    help="run only the warm-up and timed gradient steps (used for ncu captures)")
    ap.add_argument("--no-precision", action="store_true", help="skip the FP64 vs mixed time-to-tolerance leg")
    ap.add_argument("--no-configs", action="store_true", help="skip the config2 / config3 legs")
    ap.add_argument("--schedule", default=None,
                    help="plane_cps,fuse_planes,plane_xg for the FP64 context instead of the autotuner's choice "
                         "(fixed kernel variants for ncu captures)")
    ap.add_argument("--tune", action="append", default=[], metavar="KNOB=V",
                    help="set a tuning knob (spm_tune) of the flow contexts before the autotuner runs, e.g. pdl=0")
    ap.add_argument("--serve", action="store_true", help="run the serving workload instead (one JSON line)")
    ap.add_argument("--serve-jobs", type=int, default=40)
    ap.add_argument("--serve-jobs-default", type=int, default=32,
                    help="jobs of the serving leg on the default benchmark line")
    ap.add_argument("--serve-slots", type=int, default=6)
    ap.add_argument("--batch", action="store_true", help="run the batched-relaxation workload instead (one JSON line)")
    ap.add_argument("--batch-n", type=int, default=24)
    ap.add_argument("--solvers", action="store_true", help="run only the LOBPCG and SPM legs (one JSON line)")
    ap.add_argument("--batch-steps", type=int, default=4000)
    ap.add_argument("--batch-branches", action="store_true",
                    help="--batch: also time the instances on separate branches (no shared launches)")
    ap.add_argument("--solvers-n", type=int, default=N, help="grid size of --solvers (small cases for ncu captures)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.serve:
        return serve_bench(args)
    if args.batch:
        return batch_bench(args)
    if args.solvers:
        return solvers_bench(args)
    rank, world, local = dist_setup()
    if args.impl == "reference":
        rc = reference_arm(args, rank, world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return rc

    import numpy as np
    import torch
    import spmiqc

    torch.cuda.set_device(local)
    L_ = spmiqc.lib()
    stream = torch.cuda.current_stream()
    # --only-flow may time the flow in FP32 (for captures of the FP32 kernels)
    prec = args.flow_precision if args.only_flow else "fp64"
    ctx = spmiqc.SpmContext(N, L, TAU, GAMMA, DT, prec, stream=stream.cuda_stream)
    knobs = [(kv.split("=")[0], int(kv.split("=")[1])) for kv in args.tune]
    for knob, v in knobs:
        ctx.tune(knob, v)
    # schedule choice by the autotuner, outside the timed region (FP32 too, for
    # the FP32 leg and the FP32 twin of the mixed flow)
    if args.schedule:
        for knob, v in zip(("plane_cps", "fuse_planes", "plane_xg"), args.schedule.split(",")):
            ctx.tune(knob, int(v))
    else:
        ctx.autotune(60)
    sched64 = ctx.tuning()
    _c32 = spmiqc.SpmContext(N, L, TAU, GAMMA, DT, "fp32", stream=stream.cuda_stream)
    for knob, v in knobs:
        _c32.tune(knob, v)
    if not args.schedule:
        _c32.autotune(60)
    sched32 = _c32.tuning()
    _c32.close()
    phi_h = initial_field(1 + rank)
    phi = torch.from_numpy(phi_h.astype(np.float32) if prec == "fp32" else phi_h).cuda()
    uh = ctx.my_fft(phi)
    S = N ** 3 * 8

    def run_steps(k, phi_t, uh_t, c=ctx):
        spmiqc.check(L_.spm_grad_flow_enqueue(c.h, phi_t.data_ptr(), uh_t.data_ptr(), int(k), 0.0))

    def collect(c=ctx):
        n = ctypes.c_int()
        spmiqc.check(L_.spm_grad_flow_collect(c.h, None, 0, ctypes.byref(n)))
        return n.value

    L_.spm_grad_flow_enqueue.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_double]
    L_.spm_grad_flow_collect.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_int)]
    L_.spm_grad_step_profile.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_double)]
    L_.spm_grad_flow_host.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]

    # warm-up
    run_steps(args.warmup, phi, uh)
    assert collect() == args.warmup
    # timed region: exactly K gated steps (the stop rule never fires on this workload; checked below)
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    l0 = ctx.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run_steps(args.steps, phi, uh)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    launches = ctx.launches() - l0
    done = collect()
    if done != args.steps:
        raise RuntimeError(f"the flow stopped after {done} of {args.steps} steps; timing would be invalid")
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, world)
    value = world * args.steps / (ms_max / 1000.0)
    if args.only_flow:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "steps/s", "steps": args.steps,
                              "warmup": args.warmup, "gpu_launches": int(launches), "only_flow": True,
                              "precision": prec, "schedule": ctx.tuning()}))
        ctx.close()
        return 0

    # per-step latency distribution (event after each step)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(201)]
    evs[0].record(stream)
    for i in range(200):
        run_steps(1, phi, uh)
        evs[i + 1].record(stream)
    torch.cuda.synchronize()
    lat = sorted(evs[i].elapsed_time(evs[i + 1]) for i in range(200))
    p50, p99 = lat[100], lat[197]

    # per-kernel durations of the chain the timed region runs (one plane_fwd,
    # then per step pencil + fused plane pass, one plane_inv) -> roofline of
    # the dominant per-step kernel. Algorithmic bytes per launch: pencil reads
    # A and u, writes u' and B (4S); the fused plane pass reads B, writes A
    # (2S); plane_fwd reads phi, writes A; plane_inv reads B, writes phi (2S).
    kms = (ctypes.c_double * 4)()
    spmiqc.check(L_.spm_grad_step_profile(ctx.h, phi.data_ptr(), uh.data_ptr(), 50, kms))
    kms = list(kms)
    hbm, peak_kind = peaks()
    names = ["plane_fwd<ProGrad>", "pencil<OpGrad>", "plane_inv_fwd<EpiFlow,ProGrad>", "plane_inv<EpiFlow>"]
    kern_bytes = [2 * S, 4 * S, 2 * S, 2 * S]
    dom = 1 if kms[1] >= kms[2] else 2
    achieved = kern_bytes[dom] / (kms[dom] * 1e-3) / 1e9
    step_bytes = (6 * args.steps + 2) * S / args.steps  # per step of the timed chain
    traffic = kernel_traffic(sched64).get(names[dom])

    # Hessian-vector products, block of 8 (LOBPCG k = 8)
    V = torch.from_numpy(np.random.default_rng(5).standard_normal((8, N, N, N))).cuda()
    HV = torch.empty_like(V)
    ctx.hv_cam(phi, V, HV)
    torch.cuda.synchronize()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 10
    h0.record(stream)
    for _ in range(reps):
        ctx.hv_cam(phi, V, HV)
    h1.record(stream)
    torch.cuda.synchronize()
    hv_per_s = 8 * reps / (h0.elapsed_time(h1) / 1000.0)
    del V, HV

    solvers = solver_legs(ctx, phi)

    # FP32 bulk (same workload, FP32 transforms, FP64 reductions)
    ctx32 = spmiqc.SpmContext(N, L, TAU, GAMMA, DT, "fp32", stream=stream.cuda_stream)
    if not args.schedule:
        ctx32.autotune(60)  # the remembered FP32 choice
    phi32 = torch.from_numpy(phi_h.astype(np.float32)).cuda()
    uh32 = ctx32.my_fft(phi32)
    run_steps(args.warmup, phi32, uh32, ctx32)
    collect(ctx32)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    run_steps(args.steps, phi32, uh32, ctx32)
    f1.record(stream)
    torch.cuda.synchronize()
    fp32_value = args.steps / (f0.elapsed_time(f1) / 1000.0)
    ctx32.close()

    # time to ||grad F|| <= 1e-8: FP64 flow vs FP32 transforms + FP64 polish,
    # on the disordered relaxation (uniform [-0.1, 0.1] start) that provably
    # converges: its slowest mode contracts by 1 - dt |Tau| / (1 + dt G_min)
    precision = None
    if not args.no_precision:
        import inputs
        pu = inputs.uniform(N, 77)
        runs = {}
        for mode in ("fp64", "mixed"):
            best = None
            for rep in range(2):  # best of two runs of each
                a = torch.from_numpy(pu).cuda()
                ua = ctx.my_fft(a)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                if mode == "fp64":
                    st = ctx.get_min_u_F(a, ua, 30000, tol_grad=1e-8)
                    n32, n64 = 0, len(st)
                else:
                    st, n32, n64 = ctx.get_min_u_F_mixed(a, ua, 30000, tol_grad=1e-8, switch_tol=0.0)
                torch.cuda.synchronize()
                dt_s = time.perf_counter() - t0
                if best is None or dt_s < best[0]:
                    best = (dt_s, n32, n64, float(st[-1, 2]), ctx.get_Ene(a, ua), a)
            runs[mode] = best
        e64, emx = runs["fp64"][4], runs["mixed"][4]
        precision = {
            "workload": "256^3 relaxation from uniform [-0.1,0.1] (seed 77), L=26, Tau=-0.0061, to ||grad F|| <= 1e-8",
            "fp64_s": runs["fp64"][0], "mixed_s": runs["mixed"][0], "speedup": runs["fp64"][0] / runs["mixed"][0],
            "timing": "best of two runs of each",
            "fp64_steps": runs["fp64"][2], "mixed_fp32_steps": runs["mixed"][1], "mixed_fp64_steps": runs["mixed"][2],
            "switch": "FP32 to 1e-8 or its rounding floor, then FP64", "grad_norm_fp64": runs["fp64"][3], "grad_norm_mixed": runs["mixed"][3],
            "energy_fp64": e64, "energy_mixed": emx,
            "energy_diff_rel_to_initial": abs(e64 - emx) / abs(ctx.get_Ene(torch.from_numpy(pu).cuda(),
                                                                           ctx.my_fft(torch.from_numpy(pu).cuda()))),
            "field_max_abs_diff": float((runs["fp64"][5] - runs["mixed"][5]).abs().max()),
        }
        del runs

    configs = None
    if world == 1 and not args.no_configs:
        try:
            configs = config_legs(ctx, phi_h)
        except Exception as ex:  # reported, not fatal
            configs = {"error": str(ex)[:300]}
        for key, fn in (("config4", lambda: batch_core(24, 20000, False)),
                        ("config5", lambda: serve_core(args.serve_jobs_default, args.serve_slots))):
            try:
                configs[key] = fn()
            except Exception as ex:
                configs[key] = {"error": str(ex)[:300]}
            torch.cuda.empty_cache()

    # end to end through the C ABI with the field in pinned host memory: per
    # step, upload phi, transform, one step, download phi and the step record
    ph_host = torch.from_numpy(phi_h.copy()).pin_memory()
    rec = (spmiqc.StepStats * 1)()
    nd = ctypes.c_int()
    spmiqc.check(L_.spm_grad_flow_host(ctx.h, ph_host.data_ptr(), 1, 0.0, rec, ctypes.byref(nd)))
    e2e_steps = 20
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        spmiqc.check(L_.spm_grad_flow_host(ctx.h, ph_host.data_ptr(), 1, 0.0, rec, ctypes.byref(nd)))
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e_value = world * e2e_steps / e2e_s
    # the same through one call per K steps (the reference's get_min_u_F runs
    # its whole loop per call): upload phi, K steps, download phi and the K
    # step records
    K = args.steps
    recs = (spmiqc.StepStats * K)()
    barrier(world)
    t0 = time.perf_counter()
    spmiqc.check(L_.spm_grad_flow_host(ctx.h, ph_host.data_ptr(), K, 0.0, recs, ctypes.byref(nd)))
    call_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e_call = {"value": world * nd.value / call_s, "unit": "steps/s", "steps_per_call": nd.value,
                "h2d_bytes_per_step": S / K, "d2h_bytes_per_step": (S + 32 * K) / K}

    cpu = parity = cpu_serial = cpu_mkl = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu, parity, cpu_serial, cpu_mkl = cpu_legs(ctx, phi_h)
        except Exception as ex:  # oracle not built on this box
            cpu = {"value": None, "unit": "steps/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"unavailable: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "N": N, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (0.81 GB of fields through HBM per step)",
                       "schedule_fp64": sched64, "schedule_fp32": sched32},
            "p50_ms": p50, "p99_ms": p99,
            "hv_per_s": hv_per_s, "solvers_256_fp64": solvers, "fp32_steps_per_s": fp32_value, "precision": precision,
            "kernels_ms": dict(zip(names, kms)),
            "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
                         "algorithmic_bytes": kern_bytes[dom], "traffic": traffic,
                         "traffic_source": "profiles/kernel_traffic_256_fp64.md (ncu dram__bytes per launch)",
                         "step_frac": (step_bytes / (ms_max / args.steps * 1e-3) / 1e9) / hbm},
            "clocks": clk,
            "gpu_launches": int(launches),
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": S, "d2h_bytes_per_step": S + 32},
            "e2e_per_call": e2e_call,
            "cpu_baseline": cpu,
            "cpu_baseline_serial": cpu_serial,
            "cpu_baseline_mkl": cpu_mkl,
            "parity": parity,
            "config2": configs.get("config2") if configs else None,
            "config3": configs.get("config3") if configs else None,
            "config4": configs.get("config4") if configs else None,
            "config5": configs.get("config5") if configs else None,
        }
        if configs and "error" in configs:
            line["configs_error"] = configs["error"]
        print(json.dumps(line))
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
