"""ctypes wrapper around the CPU oracle (egtb_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker. The product package never imports
this module.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libegtb_oracle.so")

DTYPES = {"uint32": 0, "uint64": 1, "float32": 2, "float64": 3, "1-float32": 4, "1-float64": 5}
NP_DTYPES = {0: np.uint32, 1: np.uint64, 2: np.float32, 3: np.float64, 4: np.float32, 5: np.float64}


class _Spec(ctypes.Structure):
    _fields_ = [
        ("masks", ctypes.POINTER(ctypes.c_uint64)),
        ("n_masks", ctypes.c_int),
        ("shifts", ctypes.POINTER(ctypes.c_uint8)),
        ("n_shifts", ctypes.c_int),
        ("symm_mode", ctypes.c_int),
        ("is_variant", ctypes.c_int),
    ]


_lib = None


def build() -> str:
    """Compile the oracle with make (gcc is part of the image)."""
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
            os.path.join(HERE, "egtb_oracle.c")
        ):
            build()
        L = ctypes.CDLL(LIB_PATH)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        L.or_generate.restype = ctypes.c_void_p
        L.or_generate.argtypes = [u64p, ctypes.c_size_t, ctypes.POINTER(_Spec), ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.or_num_layers.argtypes = [ctypes.c_void_p]
        L.or_layer_len.restype = ctypes.c_size_t
        L.or_layer_len.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.or_layer_keys.restype = ctypes.c_void_p
        L.or_layer_keys.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.or_layer_rates.restype = ctypes.c_void_p
        L.or_layer_rates.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.or_solve.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.or_free.argtypes = [ctypes.c_void_p]
        L.or_apply_sym.restype = ctypes.c_uint64
        L.or_apply_sym.argtypes = [ctypes.c_uint64, ctypes.c_int]
        L.or_canonical.restype = ctypes.c_uint64
        L.or_canonical.argtypes = [ctypes.c_uint64, ctypes.c_int]
        L.or_move_all_dir_batch.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
        L.or_canonical_batch.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_void_p]
        L.or_row_tables.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.or_row_tables_variant.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.or_move_all_dir_variant_batch.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
        L.or_expand.restype = ctypes.c_size_t
        L.or_expand.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(_Spec), ctypes.c_int, ctypes.c_int,
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        L.or_solve_layer.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                     ctypes.POINTER(_Spec), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        _lib = L
    return _lib


class Spec:
    """Holds the C spec struct and keeps its arrays alive."""

    def __init__(self, masks, shifts, symm_mode, is_variant=False):
        self.masks = np.ascontiguousarray(np.asarray(list(masks), dtype=np.uint64))
        self.shifts = np.ascontiguousarray(np.asarray(list(shifts), dtype=np.uint8))
        self.c = _Spec(
            self.masks.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
            len(self.masks),
            self.shifts.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
            len(self.shifts),
            int(symm_mode),
            int(bool(is_variant)),
        )


def move_all_dir(boards: np.ndarray, variant: bool = False) -> np.ndarray:
    b = np.ascontiguousarray(boards, dtype=np.uint64)
    out = np.zeros((len(b), 4), dtype=np.uint64)
    fn = lib().or_move_all_dir_variant_batch if variant else lib().or_move_all_dir_batch
    fn(b.ctypes.data, len(b), out.ctypes.data)
    return out


def canonical(boards: np.ndarray, mode: int) -> np.ndarray:
    b = np.ascontiguousarray(boards, dtype=np.uint64)
    out = np.zeros(len(b), dtype=np.uint64)
    lib().or_canonical_batch(b.ctypes.data, len(b), int(mode), out.ctypes.data)
    return out


def apply_sym(board: int, idx: int) -> int:
    return int(lib().or_apply_sym(int(board), int(idx)))


def row_tables(variant: bool = False):
    left = np.zeros(65536, dtype=np.uint16)
    right = np.zeros(65536, dtype=np.uint16)
    (lib().or_row_tables_variant if variant else lib().or_row_tables)(left.ctypes.data, right.ctypes.data)
    return left, right


# ---- the advanced algorithm's masked-board primitives (checker only)

class _AdParam(ctypes.Structure):
    _fields_ = [("pos_fixed_32k_mask", ctypes.c_uint64), ("small_tile_sum_limit", ctypes.c_uint32),
                ("target", ctypes.c_uint32), ("num_free_32k", ctypes.c_uint32), ("num_fixed_32k", ctypes.c_uint32)]


def ad_param(small_tile_sum_limit: int, target: int, fixed_shifts, num_free_32k: int) -> _AdParam:
    fixed = 0
    for sh in fixed_shifts:
        fixed |= 0xF << int(sh)
    return _AdParam(fixed, int(small_tile_sum_limit), int(target), int(num_free_32k), len(fixed_shifts))


def _ad_lib():
    L = lib()
    if not getattr(L, "_ad_ready", False):
        P = ctypes.c_void_p
        L.or_ad_move_all_dir_batch.argtypes = [P, ctypes.c_size_t, P, P]
        L.or_ad_mask_board.argtypes = [ctypes.c_uint64, ctypes.c_int]
        L.or_ad_mask_board.restype = ctypes.c_uint64
        L.or_ad_tile_stats.argtypes = [ctypes.c_uint64, ctypes.POINTER(_AdParam), ctypes.c_int, P]
        L.or_ad_validate.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(_AdParam)]
        L.or_ad_unmask.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(_AdParam), P, ctypes.c_size_t]
        L.or_ad_unmask.restype = ctypes.c_size_t
        L._ad_ready = True
    return L


def ad_move_all_dir(boards: np.ndarray):
    b = np.ascontiguousarray(boards, dtype=np.uint64)
    out = np.zeros((len(b), 4), dtype=np.uint64)
    fl = np.zeros((len(b), 4), dtype=np.uint8)
    _ad_lib().or_ad_move_all_dir_batch(b.ctypes.data, len(b), out.ctypes.data, fl.ctypes.data)
    return out, fl


def ad_mask_board(boards: np.ndarray, threshold: int) -> np.ndarray:
    L = _ad_lib()
    return np.array([L.or_ad_mask_board(int(x), int(threshold)) for x in boards], dtype=np.uint64)


def ad_tile_stats(boards: np.ndarray, param: _AdParam, kind: int) -> np.ndarray:
    L = _ad_lib()
    out = np.zeros((len(boards), 8), dtype=np.int64)
    row = np.zeros(8, dtype=np.int64)
    for i, x in enumerate(boards):
        L.or_ad_tile_stats(int(x), ctypes.byref(param), int(kind), row.ctypes.data)
        out[i] = row
    return out


def ad_validate(boards: np.ndarray, sums: np.ndarray, param: _AdParam) -> np.ndarray:
    L = _ad_lib()
    return np.array([L.or_ad_validate(int(x), int(s), ctypes.byref(param)) for x, s in zip(boards, sums)],
                    dtype=np.uint8)


def ad_unmask(boards: np.ndarray, sums: np.ndarray, param: _AdParam):
    L = _ad_lib()
    counts, out = [], []
    buf = np.zeros(1 << 16, dtype=np.uint64)
    for x, s in zip(boards, sums):
        n = L.or_ad_unmask(int(x), int(s), ctypes.byref(param), buf.ctypes.data, len(buf))
        counts.append(n)
        out.append(buf[:min(n, len(buf))].copy())
    return np.array(counts, dtype=np.uint32), (np.concatenate(out) if out else np.zeros(0, dtype=np.uint64))


def expand(parents: np.ndarray, spec: Spec, target: int, do_check: bool):
    p = np.ascontiguousarray(parents, dtype=np.uint64)
    cap = len(p) * 64 + 16
    o1 = np.zeros(cap, dtype=np.uint64)
    o2 = np.zeros(cap, dtype=np.uint64)
    n2 = ctypes.c_size_t(0)
    n1 = lib().or_expand(p.ctypes.data, len(p), ctypes.byref(spec.c), int(target), int(bool(do_check)),
                         o1.ctypes.data, o2.ctypes.data, cap, ctypes.byref(n2))
    return o1[:n1], o2[: n2.value]


def solve_layer(keys0, k1, r1, k2, r2, spec: Spec, target: int, do_check: bool, dtype: str, p4: float):
    d = DTYPES[dtype]
    keys0 = np.ascontiguousarray(keys0, dtype=np.uint64)
    k1 = np.ascontiguousarray(k1, dtype=np.uint64)
    k2 = np.ascontiguousarray(k2, dtype=np.uint64)
    r1 = np.ascontiguousarray(r1, dtype=NP_DTYPES[d])
    r2 = np.ascontiguousarray(r2, dtype=NP_DTYPES[d])
    out = np.zeros(len(keys0), dtype=NP_DTYPES[d])
    lib().or_solve_layer(keys0.ctypes.data, len(keys0), out.ctypes.data, k1.ctypes.data, r1.ctypes.data, len(k1),
                         k2.ctypes.data, r2.ctypes.data, len(k2), ctypes.byref(spec.c), int(target),
                         int(bool(do_check)), d, float(p4))
    return out


class Build:
    """A full forward + backward build held in host memory."""

    def __init__(self, seeds, spec: Spec, target: int, steps: int, docheck: int):
        s = np.ascontiguousarray(seeds, dtype=np.uint64)
        self.spec = spec
        self.h = lib().or_generate(s.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), len(s), ctypes.byref(spec.c),
                                   int(target), int(steps), int(docheck))
        self.steps = steps
        self.dtype = None

    def layer(self, t: int) -> np.ndarray:
        n = lib().or_layer_len(self.h, t)
        p = lib().or_layer_keys(self.h, t)
        if n == 0:
            return np.zeros(0, dtype=np.uint64)
        return np.ctypeslib.as_array((ctypes.c_uint64 * n).from_address(p)).copy()

    def solve(self, dtype: str = "float32", p4: float = 0.1) -> None:
        self.dtype = DTYPES[dtype]
        lib().or_solve(self.h, self.dtype, float(p4))

    def rates(self, t: int) -> np.ndarray:
        n = lib().or_layer_len(self.h, t)
        dt = NP_DTYPES[self.dtype]
        if n == 0:
            return np.zeros(0, dtype=dt)
        p = lib().or_layer_rates(self.h, t)
        return np.frombuffer((ctypes.c_char * (n * np.dtype(dt).itemsize)).from_address(p), dtype=dt).copy()

    def book(self, t: int, dtype: str) -> bytes:
        """The .book bytes of layer t: packed {u64 board; T rate}, rate > zero only
        (compact_live_entries + write_layer_file, native_core/src/BookSolver.cpp:380-394,206-231)."""
        keys, rates = self.layer(t), self.rates(t)
        zero = -1.0 if dtype.startswith("1-") else 0.0
        live = rates > zero
        rec = np.zeros(int(live.sum()), dtype=[("board", "<u8"), ("rate", rates.dtype)])
        rec["board"] = keys[live]
        rec["rate"] = rates[live]
        return rec.tobytes()

    def live(self, t: int, dtype: str):
        """(keys, rates) of book t: the entries with rate > zero."""
        keys, rates = self.layer(t), self.rates(t)
        live = rates > rates.dtype.type(_ZERO[dtype])
        return keys[live], rates[live]

    def books(self, dtype: str, deletion: float = 0.0, optimal: bool = False, variant: bool = False) -> list:
        """Every .book's bytes with the reference's post-passes applied.

        deletion > 0 (BookSolver.cpp:589-593): after solving layer i the book of
        layer i+2 keeps only rates above T(deletion * (max - zero) + zero), so
        books 2..steps-1 are thinned (books 0 and 1 never are; a thinned book is
        never read by a later solve).
        optimal (keep_only_optimal_branches_impl, BookSolver.cpp:611-735): for
        i = 21..steps-1, book i keeps the entries that are the best move of a
        position of the (already thinned) book i-2 plus a 4 or of book i-1 plus
        a 2: first strictly largest rate over the moves left, right, up, down
        that moved and stay in the pattern; no move above zero marks entry 0."""
        steps = self.steps
        books = [self.live(t, dtype) for t in range(steps)]
        if deletion > 0.0:
            T = books[0][1].dtype.type
            thr = _threshold(T, deletion, dtype)
            for t in range(2, steps):
                k, r = books[t]
                keep = r > thr
                books[t] = (k[keep], r[keep])
        if optimal:
            zero = books[0][1].dtype.type(_ZERO[dtype])
            for i in range(21, steps):
                k2, r2 = books[i]
                mark = np.zeros(len(k2), dtype=bool)
                if len(k2):
                    for parents, v in ((books[i - 2][0], 2), (books[i - 1][0], 1)):
                        _mark_best_moves(parents, v, k2, r2, zero, self.spec, variant, mark)
                books[i] = (k2[mark], r2[mark])
        out = []
        for k, r in books:
            rec = np.zeros(len(k), dtype=[("board", "<u8"), ("rate", r.dtype)])
            rec["board"] = k
            rec["rate"] = r
            out.append(rec.tobytes())
        return out

    def __del__(self):
        try:
            lib().or_free(self.h)
        except Exception:
            pass


_ZERO = {"uint32": 0, "uint64": 0, "float32": 0.0, "float64": 0.0, "1-float32": -1.0, "1-float64": -1.0}
_MAX = {"uint32": 4e9, "uint64": 1.6e18, "float32": 1.0, "float64": 1.0, "1-float32": 0.0, "1-float64": 0.0}


def _threshold(T, deletion: float, dtype: str):
    """static_cast<T>(deletion * double(max - zero) + double(zero)): truncation for
    the integer kinds, rounding to nearest for float."""
    x = deletion * (_MAX[dtype] - _ZERO[dtype]) + _ZERO[dtype]
    return T(int(x)) if np.issubdtype(T, np.integer) else T(x)


def _is_pattern(boards: np.ndarray, masks: np.ndarray) -> np.ndarray:
    if len(masks) == 0:
        return np.ones(boards.shape, dtype=bool)
    ok = np.zeros(boards.shape, dtype=bool)
    for m in masks:
        ok |= (boards & np.uint64(m)) == np.uint64(m)
    return ok


def _mark_best_moves(parents, v, k2, r2, zero, spec, variant, mark):
    """find_optimal_branches (BookSolver.cpp:611-645) over one parent book."""
    parents = np.asarray(parents, dtype=np.uint64)
    n2 = len(k2)
    for cell in range(16):
        sel = parents[((parents >> np.uint64(4 * cell)) & np.uint64(0xF)) == 0]
        if len(sel) == 0:
            continue
        spawned = sel | np.uint64(v << (4 * cell))
        mv = move_all_dir(spawned, variant)                                  # (n, 4)
        valid = (mv != spawned[:, None]) & _is_pattern(mv, spec.masks)
        key = canonical(mv.reshape(-1), int(spec.c.symm_mode)).reshape(mv.shape)
        pos = np.searchsorted(k2, key)
        posc = np.minimum(pos, n2 - 1)
        found = valid & (pos < n2) & (k2[posc] == key)
        rate = np.where(found, r2[posc], zero)
        best = np.full(len(sel), zero, dtype=r2.dtype)
        best_index = np.zeros(len(sel), dtype=np.int64)
        for d in range(4):
            up = found[:, d] & (rate[:, d] > best)
            best = np.where(up, rate[:, d], best)
            best_index = np.where(up, posc[:, d], best_index)
        mark[best_index] = True


def free_inits(t32ks: int, t2s: int) -> np.ndarray:
    """generate_free_inits (engine_core/BookBuilder.py:149-182) restated on the
    oracle's primitives: boards with t32ks 32768 tiles and t2s 2-tiles (at most
    10^6, combinations in lexicographic order), sorted and unique; then board
    by board the moves {left, right, up, down} that equal their full-symmetry
    canonical form, stopping once (boards - 3) are collected; sorted, unique."""
    from itertools import combinations
    boards = []
    for walls in combinations(range(16), t32ks):
        base = sum(0xF << (4 * p) for p in walls)
        for twos in combinations([p for p in range(16) if p not in walls], t2s):
            if len(boards) >= 1_000_000:
                break
            boards.append(base | sum(1 << (4 * p) for p in twos))
    gen = np.unique(np.array(boards, dtype=np.uint64))
    moves = move_all_dir(gen)
    canon = canonical(moves.reshape(-1), 1).reshape(moves.shape)
    out = []
    for i in range(len(gen)):
        for d in range(4):
            if moves[i, d] == canon[i, d]:
                out.append(moves[i, d])
        if len(out) >= len(gen) - 3:
            break
    return np.unique(np.array(out, dtype=np.uint64))


# ------------------------------------------------------------------ reader --
# ClassicBookReader.move_on_dic restated (native_core/src/ReaderRuntime.cpp).

_DIRECTION_NAMES = ("up", "right", "down", "left")      # kDirectionNames, :32
_ORDERED_KEYS = ("down", "right", "left", "up")         # kOrderedResultKeys, :33
_DTYPE_INFO = {"uint32": (4e9, 0.0), "uint64": (1.6e18, 0.0), "float32": (1.0, 0.0), "float64": (1.0, 0.0),
               "1-float32": (0.0, -1.0), "1-float64": (0.0, -1.0)}  # dtype_info_for_name, :190-206
_REC = {"uint32": "<u4", "uint64": "<u8", "float32": "<f4", "float64": "<f8", "1-float32": "<f4", "1-float64": "<f8"}


def _apply_operation(m, op: int):
    """apply_operation (:127-147) on a 4x4 list matrix."""
    a = np.array(m, dtype=np.int64)
    left = lambda x: np.array([[x[r][3 - c] for r in range(4)] for c in range(4)])   # rotated[3-c][r] = x[r][c]
    right = lambda x: np.array([[x[3 - r][c] for r in range(4)] for c in range(4)])  # rotated[c][3-r] = x[r][c]
    half = lambda x: x[::-1, ::-1]
    flip = lambda x: x[:, ::-1]
    out = {0: a, 1: left(a), 2: half(a), 3: right(a), 4: flip(a), 5: flip(left(a)), 6: flip(half(a)),
           7: flip(right(a))}[op]
    return out.tolist()


def _encode(m) -> int:
    """encode_board_matrix (BoardCodec.h:20-29): log2 of each tile, row 0 high."""
    b = 0
    for r in range(4):
        for c in range(4):
            v = int(m[r][c])
            b |= (v.bit_length() - 1 if v >= 2 else 0) << (4 * ((3 - r) * 4 + (3 - c)))
    return b


def _adjust_direction(op: int, name: str) -> str:
    """adjust_direction (:149-169)."""
    if op >= 4 and name in ("left", "right"):
        name = "right" if name == "left" else "left"
    idx = {"up": 0, "right": 1, "down": 2, "left": 3}[name]
    return _DIRECTION_NAMES[(idx + op % 4) % 4]


def _round_half_away(x: float) -> float:
    f = math.floor(abs(x))
    r = f + (1.0 if abs(x) - f >= 0.5 else 0.0)
    return math.copysign(r, x)


def _present(raw, dtype: str) -> float:
    """normalize_raw_value + maybe_round_value (:208-214, :271-277); the -Ofast
    build divides by 10^9 as a multiplication by its reciprocal."""
    max_scale = _DTYPE_INFO[dtype][0]
    v = float(raw)
    if np.issubdtype(np.dtype(_REC[dtype]), np.integer) and max_scale > 1.0:
        v = v / max_scale
    if "32" in dtype and abs(v) > 1e-7:
        v = _round_half_away(v * 1e9) * (1.0 / 1e9)
    return v


def _file_lookup(path: str, key: int, dtype: str):
    """find_success_entry_in_file (:279-316): binary search over the records as
    they lie in the file; a miss reads as the dtype's zero."""
    rec = np.fromfile(path, dtype=[("board", "<u8"), ("rate", _REC[dtype])])
    n = len(rec)
    left, right = 0, n - 1
    while n and left <= right:
        mid = (left + right) // 2
        b = int(rec["board"][mid])
        if b == key:
            return _present(rec["rate"][mid], dtype)
        if b < key:
            left = mid + 1
        else:
            if mid == 0:
                break
            right = mid - 1
    return _present(_DTYPE_INFO[dtype][1], dtype)


class Reader:
    """ClassicBookReader (:1050-1067) with move_on_dic (evaluate_classic_result_candidates, :739-840)."""

    def __init__(self, masks, symm_mode: int, is_variant: bool = False, prefer_max: bool = False):
        self.masks = np.asarray(list(masks), dtype=np.uint64)
        self.symm = int(symm_mode)
        self.variant = bool(is_variant)
        self.prefer_max = bool(prefer_max)
        self.last_op = 0

    def _trie_lookup(self, zdir: str, stem: str, dtype: str):
        import ztrie
        layer = ztrie.TrieLayer.from_dir(zdir, stem, dtype)

        def lookup(key):
            raw = layer.search(key)
            return _present(_DTYPE_INFO[dtype][1] if raw is None else raw, dtype)
        return lookup

    def move_on_dic(self, board, path_list, pattern_full: str, nums_adjust: int):
        if not path_list:
            return [("?", "?")], ""
        s = sum(int(v) for row in board for v in row) + int(nums_adjust)
        nums = int(s / 2) if s >= 0 else -((-s) // 2)  # C++ division
        blank = [("down", ""), ("right", ""), ("left", ""), ("up", "")]
        if nums < 0:
            return blank, ""
        final, best, dt_out = blank, 0.0, ""
        ops = [0] if self.variant else [self.last_op] + list(range(8))  # operation_sequence, :171-182
        for directory, dtype in path_list:
            path = os.path.join(directory, f"{pattern_full}_{nums}.book")
            zdir = os.path.join(directory, f"{pattern_full}_{nums}.z")
            # a .book first, else its compressed .z directory (make_classic_lookup_context,
            # ReaderRuntime.cpp:478-497; find_classic_value_with_context, :520-545)
            if not os.path.exists(directory) or best > 0.0 or not (os.path.exists(path) or os.path.isdir(zdir)):
                continue
            lookup = (lambda key, p=path, dt=dtype: _file_lookup(p, key, dt)) if os.path.exists(path) else \
                self._trie_lookup(zdir, f"{pattern_full}_{nums}.", dtype)
            for op in ops:
                enc = _encode(_apply_operation(board, op))
                if not _is_pattern(np.array([enc], dtype=np.uint64), self.masks)[0]:
                    continue
                mv = move_all_dir(np.array([enc], dtype=np.uint64), self.variant)[0]
                values = [None] * 4  # in _ORDERED_KEYS order
                slot_of_move = (2, 1, 3, 0)  # left, right, up, down -> down/right/left/up slots
                for d in range(4):
                    m = int(mv[d])
                    if m == enc or not _is_pattern(np.array([m], dtype=np.uint64), self.masks)[0]:
                        continue
                    key = int(canonical(np.array([m], dtype=np.uint64), self.symm)[0])
                    values[slot_of_move[d]] = lookup(key)
                entries = [(_adjust_direction(op, k), values[i]) for i, k in enumerate(_ORDERED_KEYS)]
                numeric = [e for e in entries if e[1] is not None]
                others = [e for e in entries if e[1] is None]
                numeric.sort(key=lambda e: -e[1])  # stable, descending (sort_adjusted_entries, :244-269)
                if not numeric:
                    continue
                self.last_op = op
                result = numeric + others
                if self.prefer_max:
                    if numeric[0][1] > best:
                        best, final, dt_out = numeric[0][1], result, dtype
                else:
                    return result, dtype
        return final, dt_out
