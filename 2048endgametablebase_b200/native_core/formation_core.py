"""Drop-in replacement of the reference's `formation_core` module for the
classic table-build and book-lookup path, running on the GPU through
libegtb_gpu.so (include/egtb_gpu.h).

Same names, fields, defaults and call signatures as the reference's nanobind
module (native_core/src/bindings_formation.cpp:46-241): SymmMode, PatternSpec,
RunOptions, PatternLayer, run_pattern_generate, run_pattern_solve,
run_pattern_build, ClassicBookReader, find_classic_value,
get_build_progress, reset_build_progress, apply_sym_like. Errors raise
RuntimeError (the reference surfaces C++ exceptions as RuntimeError).
"""
from __future__ import annotations

import ctypes
import enum
import os
from typing import Any

import numpy as np

from .. import _native as N

__all__ = [
    "SymmMode", "PatternSpec", "RunOptions", "PatternLayer", "ClassicBookReader",
    "run_pattern_generate", "run_pattern_solve", "run_pattern_build", "find_classic_value",
    "get_build_progress", "reset_build_progress", "apply_sym_like", "last_build_stats",
]


class SymmMode(enum.IntEnum):
    """native_core/include/FormationRuntime.h:13"""
    Identity = 0
    Full = 1
    Diagonal = 2
    Horizontal = 3
    Min33 = 4
    Min24 = 5
    Min34 = 6


class PatternSpec:
    """PatternSpec, native_core/include/FormationRuntime.h:17-22"""

    def __init__(self) -> None:
        self.name: str = ""
        self.pattern_masks: list[int] = []
        self.success_shifts: list[int] = []
        self.symm_mode: int = int(SymmMode.Identity)

    def to_c(self) -> N.PatternSpecC:
        c = N.PatternSpecC()
        name = str(self.name).encode()[:63]
        c.name = name
        masks = [int(m) & 0xFFFFFFFFFFFFFFFF for m in self.pattern_masks]
        if len(masks) > N.MAX_MASKS:
            raise RuntimeError(f"at most {N.MAX_MASKS} pattern masks are supported")
        for i, m in enumerate(masks):
            c.pattern_masks[i] = m
        c.n_masks = len(masks)
        shifts = [int(s) for s in self.success_shifts]
        if len(shifts) > 16:
            raise RuntimeError("at most 16 success shifts")
        for i, s in enumerate(shifts):
            c.success_shifts[i] = s & 0xFF
        c.n_shifts = len(shifts)
        c.symm_mode = int(self.symm_mode)
        return c


class RunOptions:
    """RunOptions, native_core/include/FormationRuntime.h:24-42 (same defaults),
    plus `device` (CUDA ordinal)."""

    def __init__(self) -> None:
        self.target = 0
        self.steps = 0
        self.docheck_step = 0
        self.pathname = ""
        self.is_free = False
        self.is_variant = False
        self.spawn_rate4 = 0.1
        self.success_rate_dtype = "uint32"
        self.deletion_threshold = 0.0
        self.compress = False
        self.compress_temp_files = False
        self.optimal_branch_only = False
        self.chunked_solve = False
        self.num_threads = 0
        self.direct_io = False
        self.direct_io_queue_depth = 16
        self.direct_io_chunk_mib = 8
        self.device = int(os.environ.get("EGTB_DEVICE", "0"))

    def to_c(self, write_files: bool = True) -> N.RunOptionsC:
        o = N.RunOptionsC()
        o.target = int(self.target)
        o.steps = int(self.steps)
        o.docheck_step = int(self.docheck_step)
        p = str(self.pathname).encode()
        if len(p) >= N.MAX_PATH:
            raise RuntimeError("pathname too long")
        o.pathname = p
        o.is_free = int(bool(self.is_free))
        o.is_variant = int(bool(self.is_variant))
        o.spawn_rate4 = float(self.spawn_rate4)
        o.success_rate_dtype = dtype_code(self.success_rate_dtype)
        o.deletion_threshold = float(self.deletion_threshold)
        o.compress = int(bool(self.compress))
        o.compress_temp_files = int(bool(self.compress_temp_files))
        o.optimal_branch_only = int(bool(self.optimal_branch_only))
        o.chunked_solve = int(bool(self.chunked_solve))
        o.num_threads = int(self.num_threads)
        o.direct_io = int(bool(self.direct_io))
        o.direct_io_queue_depth = int(self.direct_io_queue_depth)
        o.direct_io_chunk_mib = int(self.direct_io_chunk_mib)
        o.device = int(self.device)
        o.write_files = int(bool(write_files))
        return o


def dtype_code(name: str) -> int:
    """success_rate_kind_from_name (native_core/include/FormationRuntime.h:243-255):
    unknown names fall back to uint32."""
    return N.DTYPE_CODES.get(str(name), 0)


def _record_dtype(name: str) -> np.dtype:
    code = dtype_code(name)
    rate = {0: "<u4", 1: "<u8", 2: "<f4", 3: "<f8", 4: "<f4", 5: "<f8"}[code]
    return np.dtype([("board", "<u8"), ("success", rate)])


class PatternLayer:
    """PatternLayer (native_core/include/FormationRuntime.h:207-240): one layer of
    packed {board, success} records."""

    def __init__(self, records: np.ndarray | None = None, dtype_name: str = "uint32") -> None:
        self._dtype_name = dtype_name if dtype_name in N.DTYPE_CODES else "uint32"
        if self._dtype_name.startswith("1-"):
            self._dtype_name = self._dtype_name[2:]
        self.records = records if records is not None else np.zeros(0, dtype=_record_dtype(dtype_name))

    @property
    def size(self) -> int:
        return int(len(self.records))

    @property
    def empty(self) -> bool:
        return self.size == 0

    @property
    def dtype_name(self) -> str:
        return self._dtype_name


_last_stats: dict[str, Any] = {}


def last_build_stats() -> dict[str, Any]:
    """Counters of the last build on this process (no reference counterpart)."""
    return dict(_last_stats)


def _seeds(arr_init) -> np.ndarray:
    a = np.asarray(arr_init)
    if a.ndim != 1:
        raise TypeError("arr_init must be a 1-D uint64 array")
    return np.ascontiguousarray(a, dtype=np.uint64)


# The reference's message when a build runs out of room
# (native_core/src/BookGenerator.cpp:371), which
# BookBuilder._should_retry_build_resume (engine_core/BookBuilder.py:237-243)
# answers with one resumed retry.
CAPACITY_MESSAGE = "The length multiplier is not big enough. Please restart."


def _check_build(rc: int) -> None:
    """N.check for the build calls: a table that does not fit even after the
    library's own regrowth and streamed fallback (EGTB_ERR_CAPACITY) raises
    with the reference's capacity message; the library's detail is chained."""
    if rc == -5:
        detail = N.NativeError(rc, f"EGTB_ERR_CAPACITY: {N.last_error()}")
        raise N.NativeError(rc, CAPACITY_MESSAGE) from detail
    N.check(rc)


def run_pattern_generate(arr_init, pattern_spec: PatternSpec, run_options: RunOptions):
    """run_pattern_generate (native_core/src/BookSolver.cpp:766-782): raw layer files
    plus the success-only books of the last two layers; returns
    (started, layer steps-2, layer steps-1)."""
    seeds = _seeds(arr_init)
    spec = pattern_spec.to_c()
    opts = run_options.to_c()
    started = ctypes.c_int32(0)
    st = N.BuildStatsC()
    _check_build(N.lib().egtb_generate(seeds.ctypes.data, len(seeds), ctypes.byref(spec), ctypes.byref(opts),
                                  ctypes.byref(started), ctypes.byref(st)))
    _last_stats.clear()
    _last_stats.update(st.as_dict())
    rdt = _record_dtype(run_options.success_rate_dtype)
    layers = []
    for t in (int(run_options.steps) - 2, int(run_options.steps) - 1):
        path = f"{run_options.pathname}{t}.book"
        if started.value and os.path.exists(path):
            recs = np.fromfile(path, dtype=rdt)
        else:
            recs = np.zeros(0, dtype=rdt)
        layers.append(PatternLayer(recs, run_options.success_rate_dtype))
    return bool(started.value), layers[0], layers[1]


def run_pattern_solve(d1: PatternLayer, d2: PatternLayer, pattern_spec: PatternSpec, run_options: RunOptions) -> None:
    """run_pattern_solve (native_core/src/BookSolver.cpp:784-821)."""
    spec = pattern_spec.to_c()
    opts = run_options.to_c()
    rdt = _record_dtype(run_options.success_rate_dtype)
    r1 = np.ascontiguousarray(d1.records.astype(rdt, copy=False)) if d1 is not None else np.zeros(0, rdt)
    r2 = np.ascontiguousarray(d2.records.astype(rdt, copy=False)) if d2 is not None else np.zeros(0, rdt)
    st = N.BuildStatsC()
    _check_build(N.lib().egtb_solve(r1.ctypes.data if len(r1) else None, len(r1), r2.ctypes.data if len(r2) else None,
                               len(r2), ctypes.byref(spec), ctypes.byref(opts), ctypes.byref(st)))
    _last_stats.clear()
    _last_stats.update(st.as_dict())


def run_pattern_build(arr_init, pattern_spec: PatternSpec, run_options: RunOptions) -> None:
    """run_pattern_build (native_core/src/BookSolver.cpp:823-832)."""
    seeds = _seeds(arr_init)
    spec = pattern_spec.to_c()
    opts = run_options.to_c()
    st = N.BuildStatsC()
    _check_build(N.lib().egtb_build(seeds.ctypes.data, len(seeds), ctypes.byref(spec), ctypes.byref(opts),
                               ctypes.byref(st)))
    _last_stats.clear()
    _last_stats.update(st.as_dict())


def get_build_progress() -> tuple[int, int]:
    cur, tot = ctypes.c_uint32(0), ctypes.c_uint32(0)
    N.check(N.lib().egtb_get_build_progress(ctypes.byref(cur), ctypes.byref(tot)))
    return int(cur.value), int(tot.value)


def reset_build_progress(total: int = 0) -> None:
    N.check(N.lib().egtb_reset_build_progress(int(total)))


def apply_sym_like(board: int, symm_index: int) -> int:
    """apply_sym_like (native_core/include/SymmetryUtils.h:9-29), on the device."""
    b = np.array([int(board) & 0xFFFFFFFFFFFFFFFF], dtype=np.uint64)
    out = np.zeros(1, dtype=np.uint64)
    N.check(N.lib().egtb_apply_sym(_device(), b.ctypes.data, 1, int(symm_index), out.ctypes.data))
    return int(out[0])


def _device() -> int:
    return int(os.environ.get("EGTB_DEVICE", "0"))


def find_classic_value(pathname: str, filename: str, search_key: int, success_rate_dtype: str = "uint32"):
    """find_classic_value (native_core/src/ReaderRuntime.cpp:1107-1133): the
    normalised value of one key in one book file, None when the file is absent."""
    val = ctypes.c_double(0.0)
    found = ctypes.c_int32(0)
    N.check(N.lib().egtb_find_classic_value(str(pathname).encode(), str(filename).encode(),
                                            int(search_key) & 0xFFFFFFFFFFFFFFFF, dtype_code(success_rate_dtype),
                                            _device(), ctypes.byref(val), ctypes.byref(found)))
    return float(val.value) if found.value else None


# ------------------------------------------------------------------ reader --

_DIRECTIONS = ("up", "right", "down", "left")         # kDirectionNames, ReaderRuntime.cpp:32
_ORDERED_KEYS = ("down", "right", "left", "up")        # kOrderedResultKeys, ReaderRuntime.cpp:33


def _adjust_direction(op: int, direction: str) -> str:
    """adjust_direction, native_core/src/ReaderRuntime.cpp:149-169"""
    d = direction
    if op >= 4:
        d = {"left": "right", "right": "left"}.get(d, d)
    idx = {"up": 0, "right": 1, "down": 2, "left": 3}[d]
    return _DIRECTIONS[(idx + op % 4) % 4]


def _encode_matrix(board) -> tuple[int, int]:
    """encode_board_matrix + board_value_sum (native_core/include/BoardCodec.h:20-74)."""
    enc = 0
    total = 0
    rows = list(board)[:4]
    for r in range(4):
        row = list(rows[r])[:4] if r < len(rows) else []
        for c in range(4):
            v = int(row[c]) & 0xFFFFFFFF if c < len(row) else 0
            total += v
            lv = v.bit_length() - 1 if v else 0
            enc |= (lv & 0xF) << (4 * ((3 - r) * 4 + (3 - c)))
    return enc, total


class ClassicBookReader:
    """ClassicBookReader (native_core/include/ReaderRuntime.h:28-50,
    native_core/src/ReaderRuntime.cpp:1050-1067): move_on_dic answered by the
    batched device lookup over books held in GPU memory."""

    _books: dict[tuple, Any] = {}

    def __init__(self, pattern_spec: PatternSpec, is_variant: bool = False) -> None:
        self.spec_ = pattern_spec
        self.is_variant_ = bool(is_variant)
        self.prefer_max_result_ = pattern_spec.name in ("4442ff", "4442f", "4tiler")
        self.last_operation_index_ = 0

    def _book(self, directory: str, pattern_full: str, dtype: str, nums_adjust: int):
        key = (os.path.abspath(directory), pattern_full, dtype_code(dtype), int(nums_adjust),
               tuple(int(m) for m in self.spec_.pattern_masks), int(self.spec_.symm_mode), _device(),
               self.is_variant_)
        h = ClassicBookReader._books.get(key)
        if h is None:
            spec = self.spec_.to_c()
            ptr = ctypes.c_void_p()
            N.check(N.lib().egtb_book_open(directory.encode(), pattern_full.encode(), dtype_code(dtype),
                                           ctypes.byref(spec), int(nums_adjust), _device(), ctypes.byref(ptr)))
            h = ptr
            if self.is_variant_:
                N.check(N.lib().egtb_book_set_variant(h, 1))
            ClassicBookReader._books[key] = h
        return h

    def _evaluate(self, book, encoded: int, op_mode: int):
        pos = np.array([encoded], dtype=np.uint64)
        vals = np.zeros(4, dtype=np.float64)
        valid = np.zeros(1, dtype=np.uint8)
        op = np.zeros(1, dtype=np.int8)
        N.check(N.lib().egtb_book_lookup(book, pos.ctypes.data, 1, int(op_mode), vals.ctypes.data,
                                         valid.ctypes.data, op.ctypes.data))
        return vals, int(valid[0]), int(op[0])

    @staticmethod
    def _sorted_entries(op: int, vals, mask: int):
        """Entries in kOrderedResultKeys order under the adjusted names, then
        numeric ones by value descending (stable) followed by the others
        (sort_adjusted_entries, ReaderRuntime.cpp:244-269)."""
        entries = []
        for key in _ORDERED_KEYS:
            name = _adjust_direction(op, key)
            slot = _DIRECTIONS.index(name)
            entries.append((name, float(vals[slot]) if mask >> slot & 1 else None))
        numeric = sorted([e for e in entries if e[1] is not None], key=lambda e: -e[1])
        return numeric + [e for e in entries if e[1] is None]

    def move_on_dic(self, board, path_list, pattern_full: str, nums_adjust: int):
        """evaluate_classic_result_candidates, native_core/src/ReaderRuntime.cpp:739-840"""
        if not path_list:
            return {"?": "?"}, ""
        encoded, total = _encode_matrix(board)
        s = total + int(nums_adjust)
        nums = int(s / 2) if s >= 0 else -((-s) // 2)  # C++ integer division
        blank = {"down": "", "right": "", "left": "", "up": ""}
        if nums < 0:
            return blank, ""
        final, best, dtype_out = blank, 0.0, ""
        for directory, dtype in path_list:
            if not os.path.exists(directory) or best > 0.0:
                continue
            # the layer's .book, or its compressed directory (make_classic_lookup_context,
            # ReaderRuntime.cpp:478-497: book_exists || compressed_exists)
            if not (os.path.exists(os.path.join(directory, f"{pattern_full}_{nums}.book")) or
                    os.path.isdir(os.path.join(directory, f"{pattern_full}_{nums}.z"))):
                continue
            book = self._book(directory, pattern_full, dtype, nums_adjust)
            if not self.prefer_max_result_:
                vals, mask, op = self._evaluate(book, encoded, self.last_operation_index_)
                if op >= 0:
                    self.last_operation_index_ = op
                    return dict(self._sorted_entries(op, vals, mask)), dtype
                continue
            ops = [0] if self.is_variant_ else [self.last_operation_index_] + list(range(8))
            for op_index in ops:
                vals, mask, op = self._evaluate(book, encoded, 8 + op_index)
                if op < 0:
                    continue
                self.last_operation_index_ = op
                entries = self._sorted_entries(op, vals, mask)
                first = entries[0][1]
                if first > best:
                    best, final, dtype_out = first, dict(entries), dtype
        return final, dtype_out

    def get_random_state(self, path_list, pattern_full: str, spawn_rate4: float) -> int:
        """sample_classic_book_state, native_core/src/ReaderRuntime.cpp:945-993:
        a random record of a random book among layers 0..9, plus one spawn."""
        rng = np.random.default_rng()
        for directory, dtype in path_list:
            rec = _record_dtype(dtype)
            ids = list(range(10))
            while ids:
                book_id = ids.pop(int(rng.integers(len(ids))))
                path = os.path.join(directory, f"{pattern_full}_{book_id}.book")
                if not os.path.exists(path):
                    continue
                n = os.path.getsize(path) // rec.itemsize
                if n == 0:
                    continue
                k = int(rng.integers(n))
                state = int(np.fromfile(path, dtype=rec, count=1, offset=k * rec.itemsize)["board"][0])
                if state:
                    empties = [i for i in range(16) if (state >> (4 * i)) & 0xF == 0]
                    if not empties:
                        return state
                    pos = empties[int(rng.integers(len(empties)))]
                    val = 2 if rng.random() < spawn_rate4 else 1
                    return state | (val << (4 * pos))
        return 0
