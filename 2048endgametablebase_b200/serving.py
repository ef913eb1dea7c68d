"""Serving loop over device-resident books (libegtb_gpu's egtb_serve_*).

The reference answers one position per Python call from the book files
(BookReader.move_on_dic, engine_core/BookReader.py:96-118, over
ClassicBookReader, native_core/src/ReaderRuntime.cpp:1050-1067). Here the
books of one or more tables are loaded once into device memory and a native
scheduler thread batches concurrent requests of 1..4096 positions into
in-flight slots (continuous batching with admission by slot memory). Each
answer is the move_on_dic answer with last_op 0: float32 success rates for
the four directions up, right, down, left and a mask of the directions with a
numeric value.

    books = [open_book(dir_a, "L3_256", "float32", spec_a, adj_a), ...]
    with BookServer(books, slots=4) as srv:
        t = srv.submit(0, positions)
        values, valid, latency_us = srv.wait(t)
"""
from __future__ import annotations

import ctypes
import importlib
import os
from dataclasses import dataclass

import numpy as np

from . import _native as N

__all__ = ["Book", "BookServer", "RequestStream", "open_book", "build_book", "sample_positions", "sample_book_keys",
           "add_spawn", "perturb", "request_sizes", "request_stream", "latency_summary", "MEAN_REQUEST"]


@dataclass
class Book:
    """One table's books resident in device memory."""
    handle: ctypes.c_void_p
    directory: str
    pattern_full: str
    dtype: str
    nums_adjust: int
    layers: int

    def close(self) -> None:
        if self.handle:
            N.check(N.lib().egtb_book_close(self.handle))
            self.handle = ctypes.c_void_p()

    def lookup(self, positions: np.ndarray, last_op: int = 0):
        """Host-buffer batched move_on_dic (float64 values, op index used)."""
        pos = np.ascontiguousarray(positions, dtype=np.uint64)
        vals = np.zeros((len(pos), 4), dtype=np.float64)
        valid = np.zeros(len(pos), dtype=np.uint8)
        op = np.zeros(len(pos), dtype=np.int8)
        N.check(N.lib().egtb_book_lookup(self.handle, pos.ctypes.data, len(pos), int(last_op), vals.ctypes.data,
                                         valid.ctypes.data, op.ctypes.data))
        return vals, valid, op


def open_book(directory: str, pattern_full: str, dtype: str, spec, nums_adjust: int, device: int = 0) -> Book:
    """Open <directory>/<pattern_full>_<t>.book and load every layer into
    device memory. `spec` is a formation_core.PatternSpec."""
    fc = importlib.import_module(__package__ + ".native_core.formation_core")
    c_spec = spec.to_c()
    ptr = ctypes.c_void_p()
    N.check(N.lib().egtb_book_open(directory.encode(), pattern_full.encode(), fc.dtype_code(dtype),
                                   ctypes.byref(c_spec), int(nums_adjust), int(device), ctypes.byref(ptr)))
    n = ctypes.c_int32(0)
    try:
        N.check(N.lib().egtb_book_load_all(ptr, ctypes.byref(n)))
    except Exception:
        N.lib().egtb_book_close(ptr)
        raise
    return Book(ptr, directory, pattern_full, dtype, int(nums_adjust), int(n.value))


def build_book(pattern: str, target: int, directory: str, device: int = 0, dtype: str = "float32"):
    """Build the classic table `pattern` at 2**target into `directory` with the
    drop-in formation_core.run_pattern_build; returns (spec, pattern_full,
    nums_adjust) for open_book."""
    fc = importlib.import_module(__package__ + ".native_core.formation_core")
    pats = importlib.import_module(__package__ + ".patterns")
    meta = pats.pattern_catalog[pattern]
    s0 = -int(meta["nums_adjust"])
    steps, docheck = pats.steps_and_docheck(s0, target, int(meta["extra_steps"]))
    pattern_full = f"{pattern}_{2 ** target}"
    spec = fc.PatternSpec()
    spec.name = pattern
    spec.pattern_masks = list(meta["pattern_masks"])
    spec.success_shifts = list(meta["success_shifts"])
    spec.symm_mode = pats.SYMM_MODES[meta["canonical_mode"]]
    o = fc.RunOptions()
    o.target, o.steps, o.docheck_step = target, steps, docheck
    o.pathname = os.path.join(directory, pattern_full + "_")
    o.success_rate_dtype = dtype
    o.spawn_rate4 = 0.1
    o.device = int(device)
    os.makedirs(directory, exist_ok=True)
    fc.run_pattern_build(np.asarray(meta["seed_boards"], dtype=np.uint64), spec, o)
    return spec, pattern_full, int(meta["nums_adjust"])


def sample_positions(book: Book, n: int, rng: np.random.Generator) -> np.ndarray:
    """n positions to ask about, drawn like sample_classic_book_state
    (native_core/src/ReaderRuntime.cpp:945-993): a book record chosen
    uniformly over every layer file (weighted by its size), then one spawn (a
    2 with probability 0.9, else a 4) in one of its empty cells, so the
    position is one a player faces before moving."""
    keys = sample_book_keys(book, n, rng)
    return add_spawn(keys, rng)


def sample_book_keys(book: Book, n: int, rng: np.random.Generator) -> np.ndarray:
    """n boards drawn uniformly from the book's own records."""
    fc = importlib.import_module(__package__ + ".native_core.formation_core")
    rec = fc._record_dtype(book.dtype)
    files = []
    for f in os.listdir(book.directory):
        if f.startswith(book.pattern_full + "_") and f.endswith(".book"):
            sz = os.path.getsize(os.path.join(book.directory, f)) // rec.itemsize
            if sz:
                files.append((f, sz))
    files.sort()
    if not files:
        raise RuntimeError(f"no book files of {book.pattern_full} in {book.directory}")
    sizes = np.array([s for _, s in files], dtype=np.int64)
    picks = rng.integers(0, int(sizes.sum()), size=n)
    bounds = np.cumsum(sizes)
    which = np.searchsorted(bounds, picks, side="right")
    order = np.argsort(which, kind="stable")
    cuts = np.searchsorted(which[order], np.arange(len(files) + 1))
    out = np.empty(n, dtype=np.uint64)
    for fi in range(len(files)):
        sel = order[cuts[fi]:cuts[fi + 1]]
        if not len(sel):
            continue
        local = picks[sel] - (bounds[fi] - sizes[fi])
        mm = np.memmap(os.path.join(book.directory, files[fi][0]), dtype=rec, mode="r")
        out[sel] = mm["board"][local]
        del mm
    return out


def _nibbles(b: np.ndarray) -> np.ndarray:
    return ((b[:, None] >> (np.arange(16, dtype=np.uint64) * np.uint64(4))[None, :]) & np.uint64(0xF)).astype(np.int64)


def _pick_where(mask: np.ndarray, rng: np.random.Generator) -> np.ndarray:
    """A uniformly chosen True column per row (-1 for rows with none)."""
    cnt = mask.sum(axis=1)
    r = np.floor(rng.random(len(mask)) * np.maximum(cnt, 1)).astype(np.int64)
    csum = np.cumsum(mask, axis=1)
    col = np.argmax(csum > r[:, None], axis=1)
    return np.where(cnt > 0, col, -1)


def _chunked(fn):
    """Apply a per-board transform in chunks (bounded temporary memory)."""
    def run(boards: np.ndarray, *args):
        out = np.empty_like(boards)
        for a in range(0, len(boards), 1 << 20):
            out[a:a + (1 << 20)] = fn(boards[a:a + (1 << 20)], *args)
        return out
    run.__doc__ = fn.__doc__
    return run


@_chunked
def add_spawn(keys: np.ndarray, rng: np.random.Generator) -> np.ndarray:
    """One spawn per board: a 2 (p 0.9) or a 4 in a uniformly chosen empty cell."""
    pos = keys.copy()
    cell = _pick_where(_nibbles(keys) == 0, rng)
    tile = np.where(rng.random(len(keys)) < 0.9, 1, 2).astype(np.uint64)
    ok = cell >= 0
    pos[ok] |= tile[ok] << (cell[ok].astype(np.uint64) * np.uint64(4))
    return pos


@_chunked
def perturb(positions: np.ndarray, frac: float, rng: np.random.Generator) -> np.ndarray:
    """Change one random free-cell nibble (a cell not pinned at 0xF) of a
    `frac` share of the positions to another value in 0..14 (queries that
    mostly miss; a miss answers 0)."""
    pos = positions.copy()
    sel = np.nonzero(rng.random(len(pos)) < frac)[0]
    if not len(sel):
        return pos
    cell = _pick_where(_nibbles(pos[sel]) != 0xF, rng)
    ok = cell >= 0
    sel, cell = sel[ok], cell[ok].astype(np.uint64)
    shift = cell * np.uint64(4)
    old = ((pos[sel] >> shift) & np.uint64(0xF)).astype(np.int64)
    new = (old + rng.integers(1, 15, size=len(sel))) % 15  # another value in 0..14
    pos[sel] = (pos[sel] & ~(np.uint64(0xF) << shift)) | (new.astype(np.uint64) << shift)
    return pos


def request_sizes(n: int, rng: np.random.Generator, max_size: int = 4096) -> np.ndarray:
    """Log-uniform request sizes in 1..max_size."""
    return np.clip(np.floor(np.exp(rng.random(n) * np.log(max_size + 1))), 1, max_size).astype(np.uint32)


MEAN_REQUEST = float(np.mean(request_sizes(1 << 20, np.random.default_rng(0))))


@dataclass
class RequestStream:
    """A recorded request stream: request i arrives at arrival_us[i], reads
    sizes[i] positions at pool[offsets[i]:] and asks book book_of[i]."""
    pool: np.ndarray
    arrival_us: np.ndarray
    sizes: np.ndarray
    offsets: np.ndarray
    book_of: np.ndarray

    @property
    def positions(self) -> int:
        return int(self.sizes.sum())

    def request(self, i: int) -> np.ndarray:
        return self.pool[int(self.offsets[i]):int(self.offsets[i]) + int(self.sizes[i])]


def request_stream(books: list[Book], n_requests: int, rate_per_s: float, seed: int, miss_frac: float = 0.05,
                   max_size: int = 4096) -> RequestStream:
    """Poisson arrivals at `rate_per_s` requests per second (0: all at once);
    sizes log-uniform in 1..max_size; each request asks one book (uniform),
    its positions sampled from that book's own layers (sample_positions),
    `miss_frac` of them perturbed on one free cell."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1e6 / rate_per_s, size=n_requests) if rate_per_s > 0 else np.zeros(n_requests)
    arrival = np.cumsum(gaps) - (gaps[0] if n_requests else 0.0)
    sizes = request_sizes(n_requests, rng, max_size)
    book_of = rng.integers(0, len(books), size=n_requests).astype(np.int32)
    offsets = np.zeros(n_requests, dtype=np.uint64)
    if n_requests:
        offsets[1:] = np.cumsum(sizes[:-1].astype(np.uint64))
    pool = np.empty(int(sizes.sum()), dtype=np.uint64)
    for b in range(len(books)):
        sel = np.nonzero(book_of == b)[0]
        cnt = int(sizes[sel].sum())
        if not cnt:
            continue
        draws = perturb(sample_positions(books[b], cnt, rng), miss_frac, rng)
        # scatter the draws to the requests of book b, in request order
        starts = offsets[sel].astype(np.int64)
        lens = sizes[sel].astype(np.int64)
        idx = np.repeat(starts - np.concatenate(([0], np.cumsum(lens)[:-1])), lens) + np.arange(cnt)
        pool[idx] = draws
    return RequestStream(pool, arrival.astype(np.float64), sizes, offsets, book_of)


def at_rate(rs: RequestStream, rate_per_s: float, recorded_rate_per_s: float) -> RequestStream:
    """The same requests with their arrival times rescaled from the recorded
    rate to another offered rate (Poisson gaps scale with 1/rate)."""
    return RequestStream(rs.pool, rs.arrival_us * (recorded_rate_per_s / rate_per_s), rs.sizes, rs.offsets,
                         rs.book_of)


def latency_summary(lat_us: np.ndarray) -> dict:
    lat = np.asarray(lat_us, dtype=np.float64)
    return {"p50_us": float(np.percentile(lat, 50)), "p99_us": float(np.percentile(lat, 99)),
            "max_us": float(lat.max()), "mean_us": float(lat.mean())}


class BookServer:
    """Native serving loop over device-resident books (egtb_serve_start)."""

    def __init__(self, books: list[Book], slots: int = 4, slot_positions: int = 1 << 17,
                 max_requests_per_batch: int = 0) -> None:
        self.books = list(books)
        arr = (ctypes.c_void_p * len(self.books))(*[b.handle.value for b in self.books])
        ptr = ctypes.c_void_p()
        N.check(N.lib().egtb_serve_start(arr, len(self.books), int(slots), int(slot_positions),
                                         int(max_requests_per_batch), ctypes.byref(ptr)))
        self._h = ptr
        self._pending: dict[int, tuple] = {}
        self._registered: dict[int, np.ndarray] = {}

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def close(self) -> None:
        if self._h:
            N.check(N.lib().egtb_serve_stop(self._h))
            self._h = ctypes.c_void_p()

    def register(self, array: np.ndarray) -> None:
        """Page-lock and map a C-contiguous array for the server: requests whose
        positions and answer arrays all lie in registered arrays are answered
        in place (no staging copies)."""
        if not array.flags.c_contiguous:
            raise ValueError("register needs a C-contiguous array")
        N.check(N.lib().egtb_serve_register(self._h, array.ctypes.data, array.nbytes))
        self._registered[array.ctypes.data] = array

    def unregister(self, array: np.ndarray) -> None:
        N.check(N.lib().egtb_serve_unregister(self._h, array.ctypes.data))
        self._registered.pop(array.ctypes.data, None)

    def submit(self, book: int, positions: np.ndarray, values: np.ndarray | None = None,
               valid: np.ndarray | None = None) -> int:
        """Queue one request; answers go to `values` ([n, 4] float32) and
        `valid` ([n] uint8) when given (e.g. registered arrays), else to new
        arrays that wait() returns."""
        pos = np.ascontiguousarray(positions, dtype=np.uint64)
        vals = values if values is not None else np.zeros((len(pos), 4), dtype=np.float32)
        valid = valid if valid is not None else np.zeros(len(pos), dtype=np.uint8)
        if vals.shape != (len(pos), 4) or vals.dtype != np.float32 or not vals.flags.c_contiguous:
            raise ValueError("values must be a C-contiguous float32 array of shape (n, 4)")
        if valid.shape != (len(pos),) or valid.dtype != np.uint8:
            raise ValueError("valid must be a uint8 array of shape (n,)")
        t = ctypes.c_uint64(0)
        N.check(N.lib().egtb_serve_submit(self._h, int(book), pos.ctypes.data, len(pos), vals.ctypes.data,
                                          valid.ctypes.data, ctypes.byref(t)))
        self._pending[t.value] = (pos, vals, valid)
        return int(t.value)

    def wait(self, ticket: int, timeout_ms: int = 60000):
        lat = ctypes.c_double(0.0)
        N.check(N.lib().egtb_serve_wait(self._h, int(ticket), int(timeout_ms), ctypes.byref(lat)))
        _, vals, valid = self._pending.pop(ticket)
        return vals, valid, float(lat.value)

    def stats(self) -> dict:
        v = [ctypes.c_uint64(0) for _ in range(4)]
        N.check(N.lib().egtb_serve_stats(self._h, *[ctypes.byref(x) for x in v]))
        return dict(zip(("requests", "positions", "batches", "launches"), (int(x.value) for x in v)))

    def replay(self, rs: RequestStream):
        """Submit the stream at its arrival times from a native driver thread;
        returns (values [P,4] float32, valid [P] uint8, latency_us per request,
        wall_us)."""
        n = len(rs.sizes)
        vals = np.zeros((len(rs.pool), 4), dtype=np.float32)
        valid = np.zeros(len(rs.pool), dtype=np.uint8)
        lat = np.zeros(n, dtype=np.float64)
        wall = ctypes.c_double(0.0)
        pool = np.ascontiguousarray(rs.pool)
        arr = np.ascontiguousarray(rs.arrival_us, dtype=np.float64)
        sizes = np.ascontiguousarray(rs.sizes, dtype=np.uint32)
        offs = np.ascontiguousarray(rs.offsets, dtype=np.uint64)
        bo = np.ascontiguousarray(rs.book_of, dtype=np.int32)
        N.check(N.lib().egtb_serve_replay(self._h, pool.ctypes.data, arr.ctypes.data, sizes.ctypes.data,
                                          offs.ctypes.data, bo.ctypes.data, n, vals.ctypes.data, valid.ctypes.data,
                                          lat.ctypes.data, ctypes.byref(wall)))
        return vals, valid, lat, float(wall.value)
