"""The N > 1 paths of bench.py on CPU ranks (gloo, world size 2): max-over-
ranks timing, gathering, the footprint partition of serving jobs, and the
whole serving path on the job server's fake device."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import sys
    sys.path[:0] = [ROOT, os.path.join(ROOT, "spm-iqc_b200")]
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        import bench
        import torch.distributed as dist
        import workloads
        r, w, _ = bench.dist_setup()
        assert (r, w) == (rank, world) and dist.get_backend() == "gloo"
        mx = bench.max_over_ranks(rank + 0.5, world)
        got = bench.gather_over_ranks([rank * 10, rank * 10 + 1], world)
        specs = workloads.serving_stream(5, 24, rate=50.0, sizes=(32, 64))
        parts = workloads.partition_jobs(specs, world)
        agg = bench.serve_ranks(specs, lambda s: (workloads.field(s), workloads.field(s) if s.kind == "spm" else None),
                                rank, world, 2, lambda k: "fp64", 1e-8, fake=True)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, mx, got, parts, agg))
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e), None, None))


def test_two_rank_paths_on_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        r, *rest = q.get(timeout=240)
        out[r] = rest
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        assert out[r][0] != "error", out[r][1]
        mx, got, parts, agg = out[r]
        assert mx == 1.5
        assert got == [0, 1, 10, 11]
        assert sorted(parts[0] + parts[1]) == list(range(24)) and not set(parts[0]) & set(parts[1])
        assert agg["completed"] == 24 and agg["failed"] == 0 and sum(agg["jobs_per_rank"]) == 24
        assert agg["p50_s"] <= agg["p99_s"] and agg["jobs_per_s"] > 0
    assert out[0][3] == out[1][3]  # every rank sees the same aggregate
    # the partition balances the footprint
    import sys
    sys.path[:0] = [ROOT, os.path.join(ROOT, "spm-iqc_b200")]
    import workloads
    specs = workloads.serving_stream(5, 24, rate=50.0, sizes=(32, 64))
    loads = [sum(workloads.job_bytes(specs[i]) for i in p) for p in out[0][2]]
    assert max(loads) <= 1.3 * min(loads)


def test_bench_reads_the_committed_traffic_profile():
    """bench.py's roofline.traffic comes from the committed ncu summary: every
    chain kernel of the gradient step has a per-launch byte count there for
    each captured schedule; with schedule 5 the fused plane pass and the pencil
    pass move no more than 10 % above their algorithmic bytes (no re-reads),
    and the pipelined schedule 6 is recorded with its own (larger) traffic."""
    import sys
    sys.path[:0] = [ROOT, os.path.join(ROOT, "spm-iqc_b200")]
    import bench
    S = 256 ** 3 * 8
    kernels = {"pencil<OpGrad>", "plane_inv_fwd<EpiFlow,ProGrad>", "plane_fwd<ProGrad>", "plane_inv<EpiFlow>"}
    tr = bench.kernel_traffic({"plane_cps": 5, "fuse_planes": 1, "plane_xg": 3})
    assert set(tr) == kernels
    assert 0 < tr["pencil<OpGrad>"] <= 1.1 * 4 * S
    assert 0 < tr["plane_inv_fwd<EpiFlow,ProGrad>"] <= 1.1 * 2 * S
    t6 = bench.kernel_traffic({"plane_cps": 6, "fuse_planes": 1, "plane_xg": 3})
    assert set(t6) == kernels and t6["plane_inv_fwd<EpiFlow,ProGrad>"] > tr["plane_inv_fwd<EpiFlow,ProGrad>"]
    assert bench.kernel_traffic() == tr  # no schedule given: the first one listed
