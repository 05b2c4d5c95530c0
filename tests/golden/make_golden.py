"""Generates tests/golden/ref_golden.npz from the reference itself.

The values come from SPM-IQC's own src/*.cpp compiled unchanged against the
single-rank shims (oracle/_ref/libspmref.so, built by `make -C oracle`), on
seeded inputs that the tests regenerate. Run from the repository root:

    python tests/golden/make_golden.py

Stored: per-step (E, res, ||grad F||) of 20 gradient steps at 16^3 and 10 at
32^3; full 16^3 outputs of ngrad_cam, hv_cam, precond_camnew, Natural_Forces,
MinMax_Forces, get_Tv and 3 Spring_Pairing iterations; LOBPCG Rayleigh
quotients (hiosd_lobpcg_initialization + hiosd_lobpcg_inip); and, at 32^3,
signatures (sum, sum of squares, 32 samples) of the same fields.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import refbind  # noqa: E402
from oracle import spmiqc_np as npo  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_golden.npz")
SAMPLE_IDX = np.array([0, 1, 7, 100, 333, 1000, 2047, 4095, 5000, 9999, 12345, 16383, 20000, 22222, 30000,
                       32767, 3, 17, 64, 255, 511, 777, 1024, 1500, 2500, 7000, 11111, 15000, 18000, 25000,
                       28000, 31000])


def sig(a):
    a = np.asarray(a).ravel()
    return np.concatenate([[a.sum(), (a * a).sum()], a[SAMPLE_IDX % a.size]])


def main():
    refbind.build()
    d = {}
    for N, steps in ((16, 20), (32, 10)):
        r = refbind.Ref(N)
        phi = npo.uniform_field(N, 7)
        v = npo.uniform_field(N, 11, amp=1.0)
        r.set_state(phi)
        E, res, g = r.grad_steps(steps)
        phi_end, _ = r.get_state()
        d[f"N{N}_E"], d[f"N{N}_res"], d[f"N{N}_gnorm"] = E, res, g
        ng = r.ngrad(phi)
        hv = r.hv(phi, v)
        pc = r.precond(v)
        tv = r.tangent(phi, phi + 0.01 * v)
        nf = r.natural_forces(phi, tv)
        mm = r.minmax_forces(phi, tv)
        a, b = r.spring_pairing(phi, phi + 0.001 * tv, 3, 1e-9)
        V0 = r.lobpcg_init(3, 5)
        V1 = r.lobpcg_inip(phi, V0, 6)
        d[f"N{N}_ritz"] = np.array([r.rayleigh(phi, V1[i]) for i in range(3)])
        d[f"N{N}_V0"] = sig(V0)
        fields = {"phi_end": phi_end, "ngrad": ng, "hv": hv, "precond": pc, "tangent": tv, "nf": nf, "mm": mm,
                  "spm0": a, "spm1": b}
        for k, val in fields.items():
            d[f"N{N}_{k}" if N == 16 else f"N{N}_{k}_sig"] = val if N == 16 else sig(val)
        r.close()
    np.savez_compressed(OUT, **d)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
