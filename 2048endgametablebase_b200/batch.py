"""Batched build of many small tables (libegtb_gpu's egtb_build_batch).

The reference builds one table per BookBuilder.start_build call
(engine_core/BookBuilder.py:264 -> run_pattern_build,
native_core/src/BookSolver.cpp:823-832). Here any number of tables of uneven
size are given at once and advance together: one kernel launch per global
layer step for all of them, the per-step loops replayed as CUDA graphs, one
radix sort for every table's layers, one packing pass for every book. Each
table's books are byte for byte the books egtb_build writes for it.

Also here: the synthetic workload of the batched-build benchmark
(random_tables: seeded random connected free regions anchored at the
bottom-right corner, every other cell pinned at 0xF, targets drawn from
64..512) and the one-at-a-time baseline through the plain build
(build_one_at_a_time).
"""
from __future__ import annotations

import ctypes
import importlib
import os
from dataclasses import dataclass, field

import numpy as np

from . import _native as N

__all__ = ["Table", "random_tables", "build_batch", "build_one_at_a_time", "autotune", "batch_book",
           "plain_book", "region_mask", "batch_mismatches"]


def _nibble(r: int, c: int) -> int:
    """Nibble index of row r, column c (row 0 is the high 16 bits)."""
    return (3 - r) * 4 + (3 - c)


def region_mask(cells: list[tuple[int, int]]) -> int:
    """Pattern mask of a free region: every cell outside it pinned at 0xF."""
    free = {_nibble(r, c) for r, c in cells}
    m = 0
    for k in range(16):
        if k not in free:
            m |= 0xF << (4 * k)
    return m


@dataclass
class Table:
    """One table of a batch: its free region, target and seed boards."""
    name: str
    cells: list[tuple[int, int]]
    target: int                    # log2 of the target tile
    seeds: np.ndarray              # uint64 seed boards (layer 0, kept as given)
    steps: int
    docheck: int
    extra_steps: int = 48
    spawn_rate4: float = 0.1
    masks: list[int] = field(default_factory=list)

    @property
    def tile_sum0(self) -> int:
        pats = importlib.import_module(__package__ + ".patterns")
        return pats.tile_sum(int(self.seeds[0]))

    def spec(self):
        fc = importlib.import_module(__package__ + ".native_core.formation_core")
        s = fc.PatternSpec()
        s.name = self.name
        s.pattern_masks = list(self.masks)
        s.success_shifts = [4 * _nibble(r, c) for r, c in sorted(self.cells)]  # a target tile on any free cell
        s.symm_mode = 0
        return s

    def options(self, pathname: str = "", dtype: str = "float32", device: int = 0):
        fc = importlib.import_module(__package__ + ".native_core.formation_core")
        o = fc.RunOptions()
        o.target, o.steps, o.docheck_step = self.target, self.steps, self.docheck
        o.pathname = pathname
        o.success_rate_dtype = dtype
        o.spawn_rate4 = self.spawn_rate4
        o.device = int(device)
        return o


def make_table(name: str, cells: list[tuple[int, int]], target: int, extra_steps: int = 48) -> Table:
    """A table over a free region: seeds are every placement of a 2 and a 4 in
    two distinct free cells (one tile sum), steps and docheck as
    BookBuilder._steps_and_docheck (engine_core/BookBuilder.py:124-128)."""
    pats = importlib.import_module(__package__ + ".patterns")
    mask = region_mask(cells)
    free = sorted(_nibble(r, c) for r, c in cells)
    seeds = [mask | (1 << (4 * a)) | (2 << (4 * b)) for a in free for b in free if a != b]
    s0 = pats.tile_sum(seeds[0])
    steps, docheck = pats.steps_and_docheck(s0, target, extra_steps)
    return Table(name, list(cells), target, np.array(seeds, dtype=np.uint64), steps, docheck, extra_steps,
                 masks=[mask])


def random_region(rng: np.random.Generator, n_cells: int) -> list[tuple[int, int]]:
    """A random connected set of n_cells cells grown from the bottom-right
    corner by adding a uniformly chosen neighbouring cell at a time."""
    cells = [(3, 3)]
    inside = {(3, 3)}
    while len(cells) < n_cells:
        frontier = sorted({(r + dr, c + dc) for r, c in cells for dr, dc in ((0, 1), (0, -1), (1, 0), (-1, 0))
                           if 0 <= r + dr < 4 and 0 <= c + dc < 4} - inside)
        pick = frontier[int(rng.integers(len(frontier)))]
        cells.append(pick)
        inside.add(pick)
    return cells


def random_tables(n: int = 64, seed: int = 0, cells: tuple[int, int] = (6, 10),
                  targets: tuple[int, ...] = (6, 7, 8, 9)) -> list[Table]:
    """The batched-build workload: n tables; table i draws from
    numpy.random.default_rng(seed + i) a free-region size in
    cells[0]..cells[1], a random connected region of that size anchored at
    the bottom-right corner, and a target 2**t with t from `targets`."""
    out = []
    for i in range(n):
        rng = np.random.default_rng(seed + i)
        k = int(rng.integers(cells[0], cells[1] + 1))
        t = int(rng.choice(targets))
        out.append(make_table(f"r{i}_{k}c_{2 ** t}", random_region(rng, k), t))
    return out


class _Args:
    """The C arrays of a batch (kept alive while the call runs)."""

    def __init__(self, tables: list[Table], dtype: str, device: int, write_dir: str | None):
        n = len(tables)
        self.n = n
        self.seeds = [np.ascontiguousarray(t.seeds, dtype=np.uint64) for t in tables]
        self.seed_ptrs = (ctypes.c_void_p * n)(*[s.ctypes.data for s in self.seeds])
        self.n_seeds = (ctypes.c_uint64 * n)(*[len(s) for s in self.seeds])
        self.specs = (N.PatternSpecC * n)(*[t.spec().to_c() for t in tables])
        opts = []
        for t in tables:
            path = os.path.join(write_dir, t.name + "_") if write_dir else ""
            opts.append(t.options(path, dtype, device).to_c(write_files=write_dir is not None))
        self.opts = (N.RunOptionsC * n)(*opts)


def _params(params: dict | None):
    if not params:
        return None
    p = N.BatchParamsC()
    for k, v in params.items():
        setattr(p, k, int(v))
    return p


def build_batch(tables: list[Table], dtype: str = "float32", device: int = 0, params: dict | None = None,
                write_dir: str | None = None):
    """Build every table in one batch. With write_dir, table t's books go to
    <write_dir>/<t.name>_<layer>.book (+ stats.txt); otherwise they stay on the
    device (batch_book). Returns (per-table stats, batch stats) as dicts."""
    a = _Args(tables, dtype, device, write_dir)
    ts = (N.BuildStatsC * a.n)()
    bs = N.BatchStatsC()
    p = _params(params)
    N.check(N.lib().egtb_build_batch(a.n, a.seed_ptrs, a.n_seeds, a.specs, a.opts,
                                     ctypes.byref(p) if p is not None else None, ts, ctypes.byref(bs)))
    return [ts[i].as_dict() for i in range(a.n)], bs.as_dict()


def autotune(tables: list[Table], dtype: str = "float32", device: int = 0):
    """Pick the batch's launch parameters by timing candidate builds; later
    builds of the same tables use them. Returns (params, device ms)."""
    a = _Args(tables, dtype, device, None)
    best = N.BatchParamsC()
    ms = ctypes.c_double(0.0)
    N.check(N.lib().egtb_batch_autotune(a.n, a.seed_ptrs, a.n_seeds, a.specs, a.opts, ctypes.byref(best),
                                        ctypes.byref(ms)))
    return best.as_dict(), float(ms.value)


def build_one_at_a_time(tables: list[Table], dtype: str = "float32", device: int = 0,
                        write_dir: str | None = None) -> list[dict]:
    """The plain path: one egtb_build per table (books kept on the device
    unless write_dir is given). Returns the per-table stats."""
    out = []
    for t in tables:
        seeds = np.ascontiguousarray(t.seeds, dtype=np.uint64)
        path = os.path.join(write_dir, t.name + "_") if write_dir else ""
        spec = t.spec().to_c()
        opts = t.options(path, dtype, device).to_c(write_files=write_dir is not None)
        st = N.BuildStatsC()
        N.check(N.lib().egtb_build(seeds.ctypes.data, len(seeds), ctypes.byref(spec), ctypes.byref(opts),
                                   ctypes.byref(st)))
        out.append(st.as_dict())
    return out


def batch_book(table: int, layer: int, device: int = 0) -> bytes:
    """Book layer `layer` of table `table` of the device's last batch."""
    n = ctypes.c_size_t(0)
    N.check(N.lib().egtb_batch_book_copy(int(device), int(table), int(layer), None, 0, ctypes.byref(n)))
    buf = ctypes.create_string_buffer(max(1, n.value))
    N.check(N.lib().egtb_batch_book_copy(int(device), int(table), int(layer), buf, n.value, ctypes.byref(n)))
    return buf.raw[:n.value]


def plain_book(layer: int, device: int = 0) -> bytes:
    """Book layer `layer` of the device's last plain (egtb_build) build."""
    n = ctypes.c_uint64(0)
    N.check(N.lib().egtb_book_layer_copy(int(device), int(layer), None, 0, ctypes.byref(n)))
    buf = ctypes.create_string_buffer(max(1, n.value))
    N.check(N.lib().egtb_book_layer_copy(int(device), int(layer), buf, n.value, ctypes.byref(n)))
    return buf.raw[:n.value]


def batch_mismatches(tables: list[Table], dtype: str = "float32", device: int = 0) -> list[str]:
    """Check the device's last batch (built from `tables`) against the plain
    path: every table is rebuilt alone by egtb_build and each of its books is
    compared byte for byte with the batch's. Returns the names of the tables
    whose books differ (empty: the batch is exact). The batch's books stay on
    the device through the plain builds (they live in the batch's own buffers)."""
    bad = []
    for i, t in enumerate(tables):
        build_one_at_a_time([t], dtype, device)
        for L in range(t.steps):
            if batch_book(i, L, device) != plain_book(L, device):
                bad.append(t.name)
                break
    return bad


# ------------------------------------------------ batches across GPUs ----
#
# The tables of a batch are independent: across N GPUs each rank builds its
# own share of them as one batch, with no collective on the data path (the
# reference builds every table in its own run, engine_core/BookBuilder.py:264).


def table_weight(t: Table) -> float:
    """Work estimate used to balance tables over GPUs: a table's boards grow
    about sixfold per free cell and with its number of steps."""
    return (6.0 ** len(t.cells)) * t.steps


def shard_tables(tables: list[Table], world: int) -> list[list[int]]:
    """Indexes of the tables each of `world` ranks builds: heaviest first,
    each to the rank with the least work so far (ties to the lowest rank);
    every table goes to exactly one rank, in ascending order within a rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0.0] * world
    share: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(tables)), key=lambda i: (-table_weight(tables[i]), i)):
        r = min(range(world), key=lambda r: (load[r], r))
        share[r].append(i)
        load[r] += table_weight(tables[i])
    return [sorted(s) for s in share]


def build_shard(tables: list[Table], rank: int, world: int, dtype: str = "float32", device: int = 0,
                params: dict | None = None):
    """Build this rank's share of `tables` as one batch on `device`. Returns
    (the share's table indexes, per-table stats, batch stats); the share's
    books are the device's last batch, table k of the share as batch table k."""
    mine = shard_tables(tables, world)[rank]
    if not mine:
        return mine, [], {"raw_boards": 0, "kernel_launches": 0}
    ts, bs = build_batch([tables[i] for i in mine], dtype, device, params)
    return mine, ts, bs


def shard_digests(tables: list[Table], mine: list[int], device: int = 0) -> dict:
    """{table name: SHA-256 of every book layer} of the device's last batch,
    built from the tables listed in `mine` (as build_shard did)."""
    import hashlib
    return {tables[i].name: [hashlib.sha256(batch_book(k, L, device)).hexdigest() for L in range(tables[i].steps)]
            for k, i in enumerate(mine)}
