"""Seeded job streams for the serving and batched-relaxation workloads.

Neither workload exists in the reference (its drivers run one job per MPI
program); the parameters follow the reference's model: L, Tau of the phase
diagram scans (main_SPM.cpp:25-27 takes L, Tau, Gamma from the command line),
initial fields as sums of cosines over BCC (12), FCC (8) or icosahedral (30)
shells (Initialization.cpp:150-166, 322-328).

serving_stream(seed, n_jobs, rate): Poisson arrivals (mean `rate` jobs/s);
70% relaxations, 20% k=4 LOBPCG eigenmode solves, 10% SPM saddle searches;
N from {64, 128, 192, 256}; L ~ U[18, 30], Tau ~ U[-0.02, 0], amplitude
~ U[0.1, 0.2], N(0, 1e-3) noise.

The amplitude is the rms of the cosine sum (each of the m cosines has
amplitude amp * sqrt(2/m)), so fields over 8, 12 or 30 vectors have the same
size. Taken per cosine instead, a 30-vector sum reaches |phi| ~ 3 and the
explicit cubic term makes the semi-implicit step at dt = 0.3 diverge.
"""
from __future__ import annotations

import dataclasses

import numpy as np

import inputs

SHELLS = ("bcc", "fcc", "ico")


@dataclasses.dataclass
class JobSpec:
    t_arrival: float
    kind: str
    N: int
    L: float
    Tau: float
    shell: str
    amp: float
    seed: int


def serving_stream(seed: int, n_jobs: int, rate: float = 4.0, sizes=(64, 128, 192, 256)):
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_jobs):
        t += rng.exponential(1.0 / rate)
        u = rng.random()
        kind = "relax" if u < 0.7 else ("lobpcg" if u < 0.9 else "spm")
        out.append(JobSpec(t, kind, int(rng.choice(sizes)), float(rng.uniform(18, 30)), float(rng.uniform(-0.02, 0)),
                           SHELLS[int(rng.integers(3))], float(rng.uniform(0.1, 0.2)), int(rng.integers(1 << 31))))
    return out


def batch_instances(seed: int, n: int = 24, sizes=(64, 96, 128, 160, 192, 256)):
    """Batched-relaxation instances: N from `sizes` (each at least once when n
    allows), L ~ U[18, 30], Tau ~ U[-0.02, 0], BCC / FCC / icosahedral shells,
    amplitude ~ U[0.1, 0.2]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        N = sizes[i % len(sizes)] if i < len(sizes) else int(rng.choice(sizes))
        out.append(JobSpec(0.0, "relax", N, float(rng.uniform(18, 30)), float(rng.uniform(-0.02, 0)),
                           SHELLS[int(rng.integers(3))], float(rng.uniform(0.1, 0.2)), int(rng.integers(1 << 31))))
    return out


def shell_vectors(shell: str, L: float) -> np.ndarray:
    if shell == "bcc":
        return inputs.bcc_shell(L)
    if shell == "fcc":
        return inputs.fcc_shell(L)
    # icosahedral: the L = 26 integer shell rescaled to |k| ~ 1 at this L
    v = inputs.icosahedral_shell().astype(float) * (L / 26.0)
    return np.unique(np.round(v).astype(np.int64), axis=0)


def field(spec: JobSpec, N: int | None = None, device: str | None = None) -> np.ndarray:
    """The job's initial phi (float64, host). With device="cuda" the cosine sum
    is evaluated by torch on the GPU (input generation only; the noise then
    comes from torch's seeded generator), else by NumPy."""
    N = N or spec.N
    vec = shell_vectors(spec.shell, spec.L)
    # a shell beyond the grid's Nyquist range (small N, large L) is halved until it fits
    while np.max(np.abs(vec)) >= N // 2:
        vec = np.unique(np.round(vec / 2.0).astype(np.int64), axis=0)
        vec = vec[np.any(vec != 0, axis=1)]
    amp = spec.amp * np.sqrt(2.0 / len(vec))
    if device is None:
        return inputs.cosine_shell(N, vec, amp=amp, seed=spec.seed, noise=1e-3)
    import torch
    theta = 2 * np.pi * inputs.unit(spec.seed, np.arange(len(vec), dtype=np.uint64))
    i = torch.arange(N, device=device, dtype=torch.float64) * (2 * np.pi / N)
    phi = torch.zeros((N, N, N), device=device, dtype=torch.float64)
    for n, th in zip(vec, theta):
        phi += torch.cos(float(n[0]) * i[:, None, None] + float(n[1]) * i[None, :, None]
                         + float(n[2]) * i[None, None, :] + float(th))
    phi *= amp
    g = torch.Generator(device=device)
    g.manual_seed(spec.seed)
    phi += 1e-3 * torch.randn((N, N, N), device=device, dtype=torch.float64, generator=g)
    return phi.cpu().numpy()


def replicas(spec: JobSpec, phi: np.ndarray):
    """SPM job replicas: phi and phi + 0.01 cos(2 pi m x / N), m in {1, 2, 3}
    seeded (a long-wavelength displacement along x)."""
    m = int(np.random.default_rng(spec.seed).integers(1, 4))
    n = phi.shape[0]
    d = np.cos(2 * np.pi * m * np.arange(n) / n)
    return phi, phi + 0.01 * d[:, None, None]


def job_bytes(spec: JobSpec) -> int:
    """Device-memory footprint of the job as the job server admits it."""
    import spmiqc
    prec = "fp64" if spec.kind == "lobpcg" else "mixed"
    return spmiqc.job_footprint(spmiqc.job_desc(spec.kind, spec.N, prec, k=4))


def partition_jobs(specs, world: int):
    """Jobs over `world` GPUs (no exchange between them): largest footprint
    first, each to the GPU with the least total footprint so far (ties to the
    lower rank). Deterministic, so every rank computes the same partition;
    each rank's list is in arrival order."""
    load = [0] * world
    parts = [[] for _ in range(world)]
    order = sorted(range(len(specs)), key=lambda i: (-job_bytes(specs[i]), i))
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += job_bytes(specs[i])
    return [sorted(p) for p in parts]
