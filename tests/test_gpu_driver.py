"""The driver replay (spm-iqc_b200/bin/spmiqc_drive): stage 1 (main_SPM.cpp)
and stage 2 (grad.cpp) on a small grid, against the same sequence of
reference routines replayed with the FP64 oracle, plus the stage-2
resume-by-cache behaviour (V1_saddle.txt)."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel
from oracle import spmiqc_np as npo

pytestmark = pytest.mark.gpu

DRIVE = os.path.join(ROOT, "spm-iqc_b200", "bin", "spmiqc_drive")
N, L, TAU, L_SHELL = 32, 18.0, -0.01, np.sqrt(2.0)
MODES = [(1, 1, 0), (1, 0, 1), (0, 1, 1), (1, -1, 0), (1, 0, -1), (0, 1, -1)]


def _write_initdata(path):
    """A BCC-type initData file listing +k and -k (amplitude 2 -> 0.2 in u_F)."""
    recs = [(a, b, c, 2) for a, b, c in MODES] + [(-a, -b, -c, 2) for a, b, c in MODES]
    with open(path, "w") as f:
        f.write(f"{len(recs)}\n")
        for r in recs:
            f.write("\t".join(str(x) for x in r) + "\n")


def _energies(out, label):
    return [float(m) for m in re.findall(label + r"\s*[:：]\s*([-+0-9.eE]+)", out)]


def _run(args, cwd):
    r = subprocess.run([DRIVE] + args, cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def _oracle_stage1(phi0, sign):
    m = npo.Model(N, L=L, Tau=TAU)
    p, u = phi0.copy(), m.my_fft(phi0)
    for _ in range(200):
        p, u, _, res = m.grad_step(p, u)
        if res <= 1e-16:
            break
    E = m.energy(p, m.my_fft(p))
    V = m.lobpcg_init(2, 0)
    for _ in range(2):
        V, _ = m.lobpcg_inip(p, V, 10)
    a, b, _, _ = m.spring_pairing(p, p + sign * 0.001 * V[0], 10, 1e-12)
    return E, m.energy(b, m.my_fft(b)), b


def test_driver_stages_match_oracle_replay(cuda, tmp_path):
    if not os.path.exists(DRIVE):
        pytest.fail("spmiqc_drive is not built")
    init = str(tmp_path / "BCCpm")
    _write_initdata(init)
    res = tmp_path / "result"
    res.mkdir()
    common = ["--N", str(N), "--L", str(L), "--Tau", str(TAU), "--max-iter", "200", "--lobpcg-iters", "10",
              "--result", str(res)]
    out1 = _run(["stage1"] + common + ["--init", init, "--l", f"{float(L_SHELL):.17g}", "--lobpcg-calls", "2",
                                       "--spm-maxiter", "10", "--spm-tol", "1e-12"], str(tmp_path))
    E = _energies(out1, "Energy of metastable state")[0]
    Es = _energies(out1, "Energy of transition state")[0]
    S1 = np.loadtxt(res / "S1.txt").reshape(N, N, N)

    # the initial field: Re(my_ifft(u_F)) of the listed modes
    uF = np.zeros((N, N, N), complex)
    for a, b, c in MODES:
        for s in (1, -1):
            k = [int(round(s * x / L_SHELL * L)) % N for x in (a, b, c)]
            uF[k[0], k[1], k[2]] = 0.2
    phi0 = npo.Model(N, L=L, Tau=TAU).my_ifft(uF).real
    best = None
    for sign in (1, -1):  # the eigenvector's sign is a convention of the eigensolver
        E_o, Es_o, S1_o = _oracle_stage1(phi0, sign)
        d = rel(S1, S1_o)
        if best is None or d < best[0]:
            best = (d, E_o, Es_o)
    d, E_o, Es_o = best
    assert abs(E - E_o) <= 1e-10 * abs(E_o), (E, E_o)
    assert abs(Es - Es_o) <= 1e-9 * abs(Es_o), (Es, Es_o)
    assert d < 1e-8

    # stage 2: computes V1_saddle.txt, then a rerun reuses it
    args2 = ["stage2"] + common + ["--lobpcg-calls", "2", "--lobpcg-calls2", "1"]
    out2 = _run(args2, str(tmp_path))
    assert "File does not exist" in out2 and (res / "V1_saddle.txt").exists()
    Et = _energies(out2, "Energy of transition state")[0]
    m = npo.Model(N, L=L, Tau=TAU)
    assert abs(Et - m.energy(S1, m.my_fft(S1))) <= 1e-10 * abs(Et)
    Emin = _energies(out2, "Energy of relaxed minimum")[0]
    assert Emin <= Et
    V = np.loadtxt(res / "V1_saddle.txt")
    assert V.size == 3 * N ** 3
    min1 = open(res / "Min.txt").read()
    out3 = _run(args2, str(tmp_path))
    assert "File  exists. Skipping LOBPCG calculation." in out3
    assert open(res / "Min.txt").read() == min1
    assert (res / "V0_Min.txt").exists()
