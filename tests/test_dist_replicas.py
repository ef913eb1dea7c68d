"""bench.py's multi-GPU path (one process per GPU under torchrun, each rank
a replica building its own table) checked as two gloo ranks on CPU: the job
time is the slowest rank's, the value counts every rank's units, and the
reference arm runs on rank 0 alone."""
import contextlib
import io
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank: int, world: int, port: int, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank), EGTB_DIST_BACKEND="gloo")
    sys.path.insert(0, ROOT)
    import bench

    w, r, _, pg = bench.dist_setup()
    slowest = bench.max_over_ranks(pg, 10.0 + 5.0 * r, "cpu")
    value = bench.replica_value(100.0, w, slowest)
    # the reference arm: rank 0 builds and prints, the others return at once
    bench.reference_build_seconds = lambda *a, **k: (2.0, 1000)
    out = io.StringIO()

    class Args:
        workload, steps, warmup, gpus = "442-512", 2, 0, w

    with contextlib.redirect_stdout(out):
        bench.run_reference_arm(Args, w, r, pg)
    pg.barrier()
    q.put((r, w, slowest, value, out.getvalue()))
    pg.destroy_process_group()


def test_two_gloo_ranks_replicas():
    import torch.multiprocessing as mp

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import reference as R

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted(q.get(timeout=180) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    assert [g[1] for g in got] == [2, 2]
    assert [g[2] for g in got] == [15.0, 15.0]          # max over ranks
    assert got[0][3] == pytest.approx(100.0 * 2 / 15.0)  # every rank's units / slowest time
    assert got[1][4] == ""                                # rank 1 prints nothing
    if R.available():
        line = __import__("json").loads(got[0][4])
        assert line["impl"] == "reference" and line["value"] == pytest.approx(1000 / 2.0)
