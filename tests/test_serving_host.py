"""Host side of the serving loop (no GPU): the request-stream generator and
its position sampling from book files."""
import ctypes

import numpy as np

import helpers as H


def _fake_books(tmp_path):
    fc = H.fc()
    S = H.serving()
    rec = fc._record_dtype("float32")
    books = []
    for b, (name, layers) in enumerate([("A_64", {3: 100, 4: 50}), ("B_128", {7: 10})]):
        d = tmp_path / name
        d.mkdir()
        for t, n in layers.items():
            r = np.zeros(n, dtype=rec)
            r["board"] = (np.arange(n, dtype=np.uint64) + np.uint64(1000 * t + 10 ** 6 * b)) << np.uint64(4)
            r["success"] = 0.5
            r.tofile(str(d / f"{name}_{t}.book"))
        books.append(S.Book(ctypes.c_void_p(), str(d), name, "float32", 0, len(layers)))
    return books


def test_request_stream_shapes_and_determinism(tmp_path):
    S = H.serving()
    books = _fake_books(tmp_path)
    a = S.request_stream(books, n_requests=200, rate_per_s=1000.0, seed=1, miss_frac=0.0)
    b = S.request_stream(books, n_requests=200, rate_per_s=1000.0, seed=1, miss_frac=0.0)
    assert np.array_equal(a.pool, b.pool) and np.array_equal(a.arrival_us, b.arrival_us)
    assert a.sizes.min() >= 1 and a.sizes.max() <= 4096
    assert a.arrival_us[0] == 0 and (np.diff(a.arrival_us) >= 0).all()
    # mean gap of a Poisson stream at 1000/s is 1000 us
    assert 700 < np.diff(a.arrival_us).mean() < 1300
    assert int(a.offsets[-1]) + int(a.sizes[-1]) == len(a.pool) == a.positions
    # every position comes from the book its request asks
    for i in range(200):
        keys = a.request(i) >> np.uint64(4)
        base = 10 ** 6 * int(a.book_of[i])
        assert ((keys >= base) & (keys < base + 10 ** 5)).all()


def test_perturb_changes_one_nibble():
    S = H.serving()
    rng = np.random.default_rng(0)
    pos = rng.integers(0, 2 ** 63, size=10000, dtype=np.uint64)
    out = S.perturb(pos, 0.05, np.random.default_rng(1))
    diff = pos ^ out
    changed = np.nonzero(diff)[0]
    assert 300 < len(changed) < 700
    for x in diff[changed]:
        nz = [k for k in range(16) if (int(x) >> (4 * k)) & 0xF]
        assert len(nz) == 1


def test_latency_summary():
    S = H.serving()
    s = S.latency_summary(np.arange(1, 101, dtype=np.float64))
    assert abs(s["p50_us"] - 50.5) < 1e-9 and s["max_us"] == 100
