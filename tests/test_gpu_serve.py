"""Serving loop (egtb_serve_*): books of two tables resident in device
memory, concurrent requests of 1..4096 positions batched into in-flight
slots. Every answer must be the same whether the request ran alone or in the
mix, and the same as the batched book lookup (egtb_book_lookup, which the
reader tests pin to the reference's move_on_dic answers). Integer keys and
float32 answers from the same kernel: bit-exact."""
import os

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu

TABLES = [("L3", 8), ("442", 8)]


@pytest.fixture(scope="module")
def books(tmp_path_factory):
    S = H.serving()
    base = str(tmp_path_factory.mktemp("serve_books", numbered=True))
    out = []
    for pattern, target in TABLES:
        d = os.path.join(base, f"{pattern}_{2 ** target}")
        spec, full, adj = S.build_book(pattern, target, d)
        out.append(S.open_book(d, full, "float32", spec, adj))
    yield out
    for b in out:
        b.close()


def _reference_answers(books, rs):
    """egtb_book_lookup per request (float64, cast to the served float32)."""
    vals = np.zeros((len(rs.pool), 4), dtype=np.float32)
    valid = np.zeros(len(rs.pool), dtype=np.uint8)
    for i in range(len(rs.sizes)):
        a, n = int(rs.offsets[i]), int(rs.sizes[i])
        v, m, _ = books[rs.book_of[i]].lookup(rs.request(i))
        vals[a:a + n] = v.astype(np.float32)
        valid[a:a + n] = m
    return vals, valid


def test_each_answer_same_alone_and_in_the_mix(books):
    S = H.serving()
    rs = S.request_stream(books, n_requests=400, rate_per_s=200_000, seed=7)
    want_v, want_m = _reference_answers(books, rs)
    with S.BookServer(books, slots=4, slot_positions=1 << 16) as srv:
        mix_v, mix_m, lat, wall = srv.replay(rs)
        st = srv.stats()
        # alone: one request at a time, nothing else in flight
        alone_v = np.zeros_like(mix_v)
        alone_m = np.zeros_like(mix_m)
        for i in range(len(rs.sizes)):
            a, n = int(rs.offsets[i]), int(rs.sizes[i])
            v, m, _ = srv.wait(srv.submit(int(rs.book_of[i]), rs.request(i)))
            alone_v[a:a + n], alone_m[a:a + n] = v, m
    assert st["requests"] == len(rs.sizes) and st["positions"] == rs.positions
    assert st["batches"] < st["requests"], st  # requests were batched together
    assert np.array_equal(mix_m, alone_m) and np.array_equal(mix_v.view(np.uint32), alone_v.view(np.uint32))
    assert np.array_equal(mix_m, want_m) and np.array_equal(mix_v.view(np.uint32), want_v.view(np.uint32))
    assert (lat > 0).all() and wall > 0
    # a miss answers 0 in every direction
    assert (mix_v[mix_m == 0] == 0).all()
    # most sampled positions hit, so the stream exercises the search
    assert (mix_m != 0).mean() > 0.5


def test_unbatched_mode_is_one_request_per_launch(books):
    S = H.serving()
    rs = S.request_stream(books, n_requests=60, rate_per_s=0, seed=3)
    want_v, want_m = _reference_answers(books, rs)
    with S.BookServer(books, slots=1, slot_positions=4096, max_requests_per_batch=1) as srv:
        v, m, lat, _ = srv.replay(rs)
        st = srv.stats()
    assert st["batches"] == st["requests"] == st["launches"] == 60
    assert np.array_equal(m, want_m) and np.array_equal(v.view(np.uint32), want_v.view(np.uint32))


def test_admission_by_slot_memory(books):
    """A slot takes requests only while their positions fit its buffers."""
    S = H.serving()
    rs = S.request_stream(books, n_requests=64, rate_per_s=0, seed=5)
    cap = 8192
    with S.BookServer(books, slots=2, slot_positions=cap) as srv:
        srv.replay(rs)
        st = srv.stats()
    assert st["batches"] >= int(np.ceil(rs.positions / cap))


def test_serve_rejects_bad_requests(books):
    S = H.serving()
    N = H.pkg()._native
    with S.BookServer(books, slots=1, slot_positions=4096) as srv:
        with pytest.raises(N.NativeError):
            srv.submit(0, np.zeros(4097, dtype=np.uint64))
        with pytest.raises(N.NativeError):
            srv.submit(5, np.zeros(4, dtype=np.uint64))
        with pytest.raises(N.NativeError):
            srv.submit(0, np.zeros(0, dtype=np.uint64))
        v, m, _ = srv.wait(srv.submit(1, np.zeros(3, dtype=np.uint64)))
        assert v.shape == (3, 4)


def test_registered_buffers_are_answered_in_place(books):
    """Requests whose positions and answer arrays lie in registered memory are
    answered by the kernel in place; the answers equal the staged path's."""
    S = H.serving()
    rs = S.request_stream(books, n_requests=80, rate_per_s=0, seed=9)
    want_v, want_m = _reference_answers(books, rs)
    pool = np.ascontiguousarray(rs.pool)
    vals = np.zeros((len(pool), 4), dtype=np.float32)
    valid = np.zeros(len(pool), dtype=np.uint8)
    with S.BookServer(books, slots=2, slot_positions=1 << 16) as srv:
        for a in (pool, vals, valid):
            srv.register(a)
        tickets = []
        for i in range(len(rs.sizes)):
            a, n = int(rs.offsets[i]), int(rs.sizes[i])
            tickets.append(srv.submit(int(rs.book_of[i]), pool[a:a + n], vals[a:a + n], valid[a:a + n]))
        for t in tickets:
            srv.wait(t)
        N = H.pkg()._native
        with pytest.raises(N.NativeError):
            srv.unregister(np.zeros(4))
        for a in (pool, vals, valid):
            srv.unregister(a)
    assert np.array_equal(valid, want_m) and np.array_equal(vals.view(np.uint32), want_v.view(np.uint32))
