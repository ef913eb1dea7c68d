"""Batched build (egtb_build_batch): every table's books must be the books the
plain build (egtb_build, pinned to the reference's files by the golden tests)
writes for it, byte for byte, whatever the launch parameters, capacity
regrowth or graph replay; small tables are also checked against the oracle."""
import hashlib
import importlib
import os

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def _B():
    return importlib.import_module("2048endgametablebase_b200.batch")


def _batch_digests(tables):
    B = _B()
    return [[hashlib.sha256(B.batch_book(i, L)).hexdigest() for L in range(t.steps)] for i, t in enumerate(tables)]


def _plain_digests(table, dtype="float32"):
    B = _B()
    st = B.build_one_at_a_time([table], dtype)[0]
    return [hashlib.sha256(B.plain_book(L)).hexdigest() for L in range(table.steps)], st


@pytest.fixture(scope="module")
def small_tables():
    return _B().random_tables(12, seed=11, cells=(6, 8), targets=(6, 7))


def test_batch_books_equal_plain_books(small_tables):
    B = _B()
    ts, bs = B.build_batch(small_tables)
    got = _batch_digests(small_tables)
    assert bs["tables"] == len(small_tables) and bs["graphs_used"] == 1
    for i, t in enumerate(small_tables):
        want, st = _plain_digests(t)
        assert got[i] == want, t.name
        for k in ("raw_boards", "book_entries", "max_layer"):
            assert ts[i][k] == st[k], (t.name, k)


@pytest.mark.parametrize("params", [
    {"expand_chunk": 32, "expand_blocks_per_sm": 2},
    {"expand_chunk": 512, "digit_nibbles": 1},
    {"index_load": 4, "use_graphs": -1},
])
def test_launch_parameters_do_not_change_books(small_tables, params):
    B = _B()
    B.build_batch(small_tables)
    want = _batch_digests(small_tables)
    _, bs = B.build_batch(small_tables, params=params)
    for k, v in params.items():
        assert bs["params"][k] == (0 if k == "use_graphs" and v < 0 else v)
    assert bs["graphs_used"] == (0 if params.get("use_graphs", 1) < 0 else 1)
    assert _batch_digests(small_tables) == want


def test_regrowth_then_remembered_capacities():
    """A fresh set of tables starts from small slices and regrows; the second
    build of the same set fits at once and gives the same books."""
    B = _B()
    tables = [B.make_table("big9", [(3, 3), (3, 2), (3, 1), (3, 0), (2, 3), (2, 2), (2, 1), (2, 0), (1, 3)], 8),
              *B.random_tables(5, seed=99, cells=(6, 7), targets=(6,))]
    ts, bs = B.build_batch(tables)
    assert bs["retries"] > 0
    first = _batch_digests(tables)
    ts2, bs2 = B.build_batch(tables)
    assert bs2["retries"] == 0
    assert _batch_digests(tables) == first
    want, st = _plain_digests(tables[0])
    assert first[0] == want and ts2[0]["raw_boards"] == st["raw_boards"]


def test_small_tables_match_the_oracle():
    import oracle as O
    B = _B()
    tables = [B.make_table("o4", [(3, 3), (3, 2), (2, 3), (2, 2)], 5),
              B.make_table("o5", [(3, 3), (3, 2), (3, 1), (2, 3), (1, 3)], 6),
              B.make_table("o6", [(3, 3), (2, 3), (1, 3), (0, 3), (3, 2), (2, 2)], 6)]
    B.build_batch(tables)
    for i, t in enumerate(tables):
        spec = t.spec()
        ob = O.Build(t.seeds, O.Spec(spec.pattern_masks, spec.success_shifts, 0), t.target, t.steps, t.docheck)
        ob.solve("float32", t.spawn_rate4)
        for L in range(t.steps):
            assert B.batch_book(i, L) == ob.book(L, "float32"), (t.name, L)


def test_batch_writes_the_plain_build_files(small_tables, tmp_root):
    B = _B()
    d_batch = H.fresh(os.path.join(tmp_root, "batch_files") + "/")
    d_plain = H.fresh(os.path.join(tmp_root, "plain_files") + "/")
    tabs = small_tables[:4]
    B.build_batch(tabs, write_dir=d_batch)
    B.build_one_at_a_time(tabs, write_dir=d_plain)
    for t in tabs:
        for L in range(t.steps):
            a = open(os.path.join(d_batch, f"{t.name}_{L}.book"), "rb").read()
            b = open(os.path.join(d_plain, f"{t.name}_{L}.book"), "rb").read()
            assert a == b, (t.name, L)
        sa = open(os.path.join(d_batch, f"{t.name}_stats.txt")).read().splitlines()
        sb = open(os.path.join(d_plain, f"{t.name}_stats.txt")).read().splitlines()
        # same layers, lengths and maxima; the speed and time columns differ
        assert [x.split(",")[:3] for x in sa] == [x.split(",")[:3] for x in sb]


def test_autotune_picks_valid_parameters(small_tables):
    B = _B()
    best, ms = B.autotune(small_tables)
    assert ms > 0
    assert best["expand_chunk"] in (32, 64, 128, 256, 512)
    assert best["expand_blocks_per_sm"] in (2, 3, 6)
    assert best["digit_nibbles"] in (1, 2) and best["index_load"] in (2, 4)
    _, bs = B.build_batch(small_tables)
    assert bs["params"] == best


def test_batch_rejects_bad_input(small_tables):
    B = _B()
    N = H.pkg()._native
    with pytest.raises(N.NativeError):
        B.build_batch([])
    with pytest.raises(N.NativeError):
        B.build_batch(small_tables[:2], params={"expand_chunk": 48})


@pytest.mark.slow
def test_benchmark_batch_of_64_equals_plain_builds():
    """The batched-build benchmark's own workload: the 64 seeded tables of
    random_tables(64) (6-10 free cells, targets 64..512, the largest tables
    10 cells at target 512), built with the autotuner's
    parameters as the benchmark builds them, then every table rebuilt alone
    by the plain path and every book compared byte for byte."""
    B = _B()
    tables = B.random_tables(64)
    B.build_batch(tables)  # capacities settle on the first build
    tuned, _ = B.autotune(tables)
    ts, bs = B.build_batch(tables)
    assert bs["params"] == tuned and bs["tables"] == 64
    assert B.batch_mismatches(tables) == []
    big = [i for i, t in enumerate(tables) if len(t.cells) == 10]
    assert any(tables[i].target == 9 for i in big), "the workload holds 10-cell target-512 tables"
    assert sum(t["raw_boards"] for t in ts) == bs["raw_boards"]


def _shard_rank(rank, world, port, q):
    """One rank of a 2-process batch split (both on GPU 0, gloo for the
    host-side exchange): build this rank's share, report its digests."""
    import datetime
    import sys
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, H.ROOT)
    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    B = importlib.import_module("2048endgametablebase_b200.batch")
    tables = B.random_tables(64)
    mine, ts, bs = B.build_shard(tables, rank, world, device=0)
    dig = B.shard_digests(tables, mine, device=0)
    got = [None] * world
    dist.all_gather_object(got, dig)
    q.put((rank, got))
    dist.destroy_process_group()


@pytest.mark.slow
def test_tables_split_over_two_ranks_equal_the_single_batch():
    """The 64-table benchmark batch split over two ranks by table: the
    union of the ranks' books equals the books of the whole batch built in
    one process, table by table."""
    import socket

    import torch.multiprocessing as mp
    B = _B()
    tables = B.random_tables(64)
    B.build_batch(tables)
    whole = {t.name: d for t, d in zip(tables, _batch_digests(tables))}
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_shard_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = [q.get(timeout=900) for _ in procs]
    finally:
        for p in procs:
            p.join(timeout=120)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    for rank, gathered in got:
        merged = {}
        for part in gathered:
            assert not set(part) & set(merged)  # no table on two ranks
            merged.update(part)
        assert merged == whole, rank
