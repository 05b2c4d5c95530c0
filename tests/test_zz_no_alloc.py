"""The allocation-free inner-product entry point (spm_inpfp_batch_noalloc).

It exists for callers that cannot allocate device memory at the moment they
need the result (their memory is fully reserved by their own pool allocator,
or a cudaMalloc's device-wide synchronisation would stall their streams).
This test calls it through the C ABI twice in a row -- the second call reuses
the scratch the first one left behind -- and checks each result against the
context-based spm_inpfp at 1e-12 relative. It also checks that a batch above
the stated limit is refused on the host. It lives in its own file, collected
last, and passes both alone and after the other tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_inner_products_match(cuda):
    import spmiqc
    from oracle import spmiqc_np as npo

    lib = spmiqc.lib()
    f = lib.spm_inpfp_batch_noalloc
    f.argtypes = [ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    N, nb = 64, 3
    n = N ** 3
    ctx = spmiqc.SpmContext(N)
    stream = cuda.cuda.current_stream().cuda_stream
    P = cuda.from_numpy(np.stack([npo.uniform_field(N, 500 + b, amp=1.0) for b in range(nb)])).cuda()
    Q = cuda.from_numpy(np.stack([npo.uniform_field(N, 600 + b, amp=1.0) for b in range(nb)])).cuda()
    ref = [ctx.inpfp(P[b], Q[b]) for b in range(nb)]
    for call in range(2):
        out = cuda.full((nb,), float("nan"), dtype=cuda.float64, device="cuda")
        spmiqc.check(f(n, nb, spmiqc.SPM_FP64, P.data_ptr(), Q.data_ptr(), out.data_ptr(), stream))
        got = out.cpu().numpy()
        for b in range(nb):
            assert abs(got[b] - ref[b]) <= 1e-12 * abs(ref[b]), (call, b, got[b], ref[b])
    # FP32 inputs against the same reduction of the rounded values
    P32, Q32 = P.float().contiguous(), Q.float().contiguous()
    out = cuda.zeros((nb,), dtype=cuda.float64, device="cuda")
    spmiqc.check(f(n, nb, spmiqc.SPM_FP32, P32.data_ptr(), Q32.data_ptr(), out.data_ptr(), stream))
    exp = (P32.double() * Q32.double()).reshape(nb, -1).sum(1).cpu().numpy() / n
    assert np.allclose(out.cpu().numpy(), exp, rtol=1e-12, atol=0)
    # ragged sizes (fewer blocks than the scratch holds, one partial per block)
    # with all 16 ticket slots in use, two calls enqueued back to back on one
    # stream with no host synchronisation between them: the second call relies
    # only on its own ticket clear, in stream order
    for n_small in (1, 255, 1000):
        A = cuda.from_numpy(np.stack([npo.uniform_field(16, 700 + b, amp=1.0).ravel()[:n_small]
                                      for b in range(16)])).cuda()
        B = cuda.from_numpy(np.stack([npo.uniform_field(16, 800 + b, amp=1.0).ravel()[:n_small]
                                      for b in range(16)])).cuda()
        o1 = cuda.full((16,), float("nan"), dtype=cuda.float64, device="cuda")
        o2 = cuda.full((16,), float("nan"), dtype=cuda.float64, device="cuda")
        spmiqc.check(f(n_small, 16, spmiqc.SPM_FP64, A.data_ptr(), B.data_ptr(), o1.data_ptr(), stream))
        spmiqc.check(f(n_small, 16, spmiqc.SPM_FP64, B.data_ptr(), B.data_ptr(), o2.data_ptr(), stream))
        a, bb = A.cpu().numpy(), B.cpu().numpy()
        e1 = (a * bb).sum(1) / n_small
        e2 = (bb * bb).sum(1) / n_small
        assert np.allclose(o1.cpu().numpy(), e1, rtol=1e-12, atol=1e-300), n_small
        assert np.allclose(o2.cpu().numpy(), e2, rtol=1e-12, atol=1e-300), n_small
    # above the stated maximum: refused on the host with SPM_ERR_ARG
    big = cuda.zeros((17, 2), dtype=cuda.float64, device="cuda")
    rc = f(2, 17, spmiqc.SPM_FP64, big.data_ptr(), big.data_ptr(), out.data_ptr(), stream)
    assert rc == 1 and b"16" in lib.spm_last_error()
    ctx.close()
