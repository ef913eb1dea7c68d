"""The batched build over several GPUs: the 64 tables split over the ranks by
table (no collective on the data path). Host logic here: the split, and
bench.py's sharded leg as two gloo ranks on CPU (slowest rank's time, every
rank's boards). The GPU test (test_gpu_batch.py) checks each rank's books
against the single-process batch."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _B():
    import importlib
    return importlib.import_module("2048endgametablebase_b200.batch")


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_every_table_goes_to_exactly_one_rank(world):
    B = _B()
    tables = B.random_tables(64)
    share = B.shard_tables(tables, world)
    assert len(share) == world
    flat = sorted(i for s in share for i in s)
    assert flat == list(range(64))
    assert all(s == sorted(s) for s in share)
    loads = [sum(B.table_weight(tables[i]) for i in s) for s in share]
    heaviest = max(B.table_weight(t) for t in tables)
    # greedy by weight: no rank exceeds the mean by more than one table
    assert max(loads) <= sum(loads) / world + heaviest
    assert B.shard_tables(tables, world) == share  # deterministic


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

    w, r, local, pg = bench.dist_setup()
    B = _B()
    tables = B.random_tables(64)
    mine = B.shard_tables(tables, w)[r]
    calls = []

    def fake_build():
        calls.append(1)
        return mine, [], {"raw_boards": 1000 * (r + 1)}

    def fake_timer(fn, k):
        out = None
        for _ in range(k):
            out = fn()
        return out, 10.0 * (r + 1)

    line = bench.batch_shard_leg(local, w, r, pg, steps=3, warmup=2, build_shard=fake_build, device_timer=fake_timer)
    q.put((r, len(calls), line))
    pg.destroy_process_group()


def test_sharded_leg_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted((q.get(timeout=180) for _ in procs), key=lambda x: x[0])
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    for r, calls, line in got:
        assert calls == 5                                     # 2 warm-up + 3 timed builds
        assert line["ms_per_step"] == 20.0                   # the slowest rank
        assert line["config"]["boards"] == 3000              # every rank's boards
        assert line["config"]["tables"] == 64
        assert line["value"] == pytest.approx(3000 / 0.020)
        assert line["scaling"] == "strong" and line["n_gpus"] == 2
