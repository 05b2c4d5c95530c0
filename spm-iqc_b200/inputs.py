"""Seeded synthetic initial fields for the benchmark workloads (NumPy, host).

The reference ships no benchmark inputs (its only used initial datum,
initData/DIS, is phi = 0), so the workloads define their own generators:
  * uniform(N, seed, amp):     U[-amp, amp) from SplitMix64, mean removed
                               (the 64^3 / 500-step gradient-flow workload);
  * cosine_shell(N, L, shell, amp, seed, noise): amp * sum_j cos(2 pi n_j.x/N + theta_j)
                               + N(0, noise^2) over a shell of integer wave
                               vectors n_j (icosahedral, BCC or FCC), with
                               phases theta_j ~ U[0, 2 pi); the reciprocal
                               vectors are k_j = n_j / L, so |k| ~ 1 lies on
                               the minimum of G (Initialization.cpp:150-166).
Integer wave vectors of the BCC / FCC shells follow the reference's rounding
rule n = round(k_hat * L) (Initialization.cpp:322-328).
"""
from __future__ import annotations

import itertools

import numpy as np

GAMMA = np.uint64(0x9E3779B97F4A7C15)


def splitmix64(seed: int, idx: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (idx.astype(np.uint64) + np.uint64(1)) * GAMMA
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def unit(seed: int, idx: np.ndarray) -> np.ndarray:
    """Uniform [0, 1) doubles from the 53 high bits."""
    return (splitmix64(seed, idx) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def gauss(seed: int, n: int) -> np.ndarray:
    """Standard normals by Box-Muller over consecutive SplitMix64 pairs."""
    m = (n + 1) // 2
    u1 = unit(seed, np.arange(0, 2 * m, 2, dtype=np.uint64))
    u2 = unit(seed, np.arange(1, 2 * m, 2, dtype=np.uint64))
    r = np.sqrt(-2.0 * np.log1p(-u1))
    z = np.concatenate([r * np.cos(2 * np.pi * u2), r * np.sin(2 * np.pi * u2)])
    return z[:n]


def uniform(N: int, seed: int, amp: float = 0.1) -> np.ndarray:
    idx = np.arange(N ** 3, dtype=np.uint64)
    u = (-1.0 + 2.0 * unit(seed, idx)).reshape(N, N, N) * amp
    return u - np.sum(u) / N ** 3


def icosahedral_shell() -> np.ndarray:
    """30 integer vectors: (+-26, 0, 0) and permutations, and the even (cyclic)
    permutations of (+-8, +-13, +-21); |(8, 13, 21)| = 25.96 ~ 26, so at L = 26
    all have |k| ~ 1 and are commensurate with the periodic box."""
    v = []
    for ax in range(3):
        for s in (26, -26):
            e = [0, 0, 0]
            e[ax] = s
            v.append(e)
    base = (8, 13, 21)
    for shift in range(3):
        p = base[shift:] + base[:shift]
        for sg in itertools.product((1, -1), repeat=3):
            v.append([p[0] * sg[0], p[1] * sg[1], p[2] * sg[2]])
    return np.array(v, dtype=np.int64)


def bcc_shell(L: float) -> np.ndarray:
    """12 vectors: permutations of (+-1, +-1, 0)/sqrt(2), scaled by L and rounded."""
    v = set()
    for perm in set(itertools.permutations((1, 1, 0))):
        for sg in itertools.product((1, -1), repeat=3):
            k = np.array(perm, dtype=float) * np.array(sg) / np.sqrt(2.0)
            v.add(tuple(int(np.round(x * L)) for x in k))
    return np.array(sorted(v), dtype=np.int64)


def fcc_shell(L: float) -> np.ndarray:
    """8 vectors: (+-1, +-1, +-1)/sqrt(3), scaled by L and rounded."""
    v = [[int(np.round(s * L / np.sqrt(3.0))) for s in sg] for sg in itertools.product((1, -1), repeat=3)]
    return np.array(v, dtype=np.int64)


def cosine_shell(N: int, shell: np.ndarray, amp: float = 0.15, seed: int = 1, noise: float = 1e-3) -> np.ndarray:
    """amp * sum_j cos(2 pi (n_j . x)/N + theta_j) + noise * N(0, 1) on an N^3 grid."""
    theta = 2 * np.pi * unit(seed, np.arange(len(shell), dtype=np.uint64))
    i = np.arange(N, dtype=np.int64)
    phi = np.zeros((N, N, N))
    for n, th in zip(shell, theta):
        tab = np.cos(2 * np.pi * np.arange(N) / N + th)
        m = ((n[0] * i)[:, None, None] + (n[1] * i)[None, :, None] + (n[2] * i)[None, None, :]) % N
        phi += tab[m]
    phi *= amp
    if noise:
        phi += noise * gauss(seed ^ 0x5DEECE66D, N ** 3).reshape(N, N, N)
    return phi
