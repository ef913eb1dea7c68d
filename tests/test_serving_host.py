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
    # every position is a record of the book its request asks plus one spawn
    fc = H.fc()
    recs = [set(int(x) for f in sorted(__import__("os").listdir(b.directory))
                for x in np.fromfile(__import__("os").path.join(b.directory, f), dtype=fc._record_dtype("float32"))["board"])
            for b in books]
    for i in range(0, 200, 5):
        for p in a.request(i)[:50]:
            p = int(p)
            spawned = [k for k in range(16) if (p >> (4 * k)) & 0xF in (1, 2) and (p & ~(0xF << (4 * k))) in recs[a.book_of[i]]]
            assert spawned, hex(p)
    assert abs(S.MEAN_REQUEST - 4095 / np.log(4097)) < 10  # log-uniform mean


def test_perturb_changes_one_nibble():
    S = H.serving()
    rng = np.random.default_rng(0)
    pos = rng.integers(0, 2 ** 63, size=10000, dtype=np.uint64) | np.uint64(0xF)  # nibble 0 pinned
    out = S.perturb(pos, 0.05, np.random.default_rng(1))
    diff = pos ^ out
    changed = np.nonzero(diff)[0]
    assert 300 < len(changed) < 700
    for x, y in zip(diff[changed], out[changed]):
        nz = [k for k in range(16) if (int(x) >> (4 * k)) & 0xF]
        assert len(nz) == 1 and nz[0] != 0  # one free cell changed
        assert (int(y) >> (4 * nz[0])) & 0xF != 0xF


def test_request_sizes_log_uniform():
    S = H.serving()
    z = S.request_sizes(200000, np.random.default_rng(3))
    assert z.min() == 1 and z.max() <= 4096
    # log-uniform: about as many requests in 1..63 as in 64..4096
    lo, hi = (z < 64).mean(), (z >= 64).mean()
    assert 0.4 < lo < 0.6 and 0.4 < hi < 0.6


def test_latency_summary():
    S = H.serving()
    s = S.latency_summary(np.arange(1, 101, dtype=np.float64))
    assert abs(s["p50_us"] - 50.5) < 1e-9 and s["max_us"] == 100
