"""Failure detection on the GPU without a GPU fault: a bounded device wait
that cannot complete (an mbarrier arrival expecting bytes that no copy
delivers) runs out after a short limit, the kernel returns, the host reads
the error word as SPM_ERR_CUDA "... bounded wait ... timed out", and the same
context then computes correct results (checked against the oracle at the
FP64 parity bar, 1e-11 relative)."""
import ctypes

import numpy as np
import pytest

from conftest import rel
from oracle import spmiqc_np as npo

pytestmark = pytest.mark.gpu


def test_bounded_wait_timeout_is_reported_and_context_recovers(cuda):
    import spmiqc
    lib = spmiqc.lib()
    f = lib.spm_selftest_bounded_wait
    f.argtypes = [ctypes.c_void_p, ctypes.c_int]
    f.restype = ctypes.c_int
    N = 32
    ctx = spmiqc.SpmContext(N)
    for _ in range(2):  # reported every time, not only once
        rc = f(ctx.h, 2000)
        assert rc == spmiqc.SPM_ERR_CUDA, rc
        assert b"bounded wait" in lib.spm_last_error() and b"timed out" in lib.spm_last_error()
        ctx.sync()  # the error word was cleared by the read
        m = npo.Model(N)
        phi0 = npo.uniform_field(N, 404)
        pd = cuda.from_numpy(phi0.copy()).cuda()
        uh = ctx.my_fft(pd)
        st = ctx.get_min_u_F(pd, uh, 4)
        p, u = phi0.copy(), m.my_fft(phi0)
        for s in range(4):
            p, u, e, _ = m.grad_step(p, u)
            assert abs(st[s, 0] - e) <= 1e-11 * abs(e)
        assert rel(pd.cpu().numpy(), p) < 1e-11
    # out-of-range limits are refused on the host, nothing is launched
    assert f(ctx.h, 0) == spmiqc.SPM_ERR_ARG
    ctx.close()
