"""Generate the golden fixtures in tests/golden/ by running the REFERENCE's own
classic-path code (compiled from its sources by `make -C oracle ref`).

The reference ships no golden vectors, known-answer tests or fixtures, so the
fixtures are outputs of the reference itself, run in this container:

  cases.json   per build case: the PatternSpec/RunOptions inputs, every raw
               layer's length and SHA-256 (run_pattern_generate writes them) and
               every .book file's SHA-256 (run_pattern_build writes them)
  prims.npz    board primitives on seeded random boards: move_all_dir (classic
               and variant movers), canonical_by_mode for modes 0-6,
               apply_sym_like 0-7, row tables of both movers
  ad_prims.npz the advanced algorithm's masked-board primitives on seeded
               random boards: m_move_all_dir with its mask_new_tile flags,
               mask_board, tile_sum_and_32k_count / 2 / 4, validate and
               unmask_board under four parameter sets, the masked row rule, the tiles-combination
               table of init_masker
  reader.json  ClassicBookReader.move_on_dic answers on positions sampled from
               the books of the small cases
  free5_32.npz one complete small build (raw layers and books) as data

Usage:  python tests/golden/make_golden.py            # small cases
        python tests/golden/make_golden.py --full     # + full-size L3-256, 442-512
Reads the reference's pattern catalog from the reference's source tree
($EGTB_REFERENCE_ROOT, default /root/reference; this container only); the
fixtures carry every input, so nothing reads the reference tree later.
"""
from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import reference as R  # noqa: E402

GOLDEN = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("EGTB_REFERENCE_ROOT", "/root/reference")
REF_CATALOG = os.path.join(REF_ROOT, "docs_and_configs", "patterns_config.json")
WORK = os.environ.get("GOLDEN_WORK", "/dev/shm/egtb_golden")


def _cellmask(free):
    m = 0
    for r in range(4):
        for c in range(4):
            if (r, c) not in free:
                m |= 0xF << (4 * ((3 - r) * 4 + (3 - c)))
    return m


def _board(tiles, base):
    b = base
    for (r, c), v in tiles.items():
        b |= v << (4 * ((3 - r) * 4 + (3 - c)))
    return b


def custom_patterns() -> dict:
    """Small patterns, in the reference's catalog format, that cover the
    symmetry modes the reference's small catalog entries do not reach quickly."""
    pats = {}
    d9 = [(r, c) for r in range(3) for c in range(3)]
    m = _cellmask(d9)
    pats["diag9"] = {"valid pattern": [hex(m)], "target pos": hex(0xFFFFFFFFFFFFFFFF & ~m),
                     "canonical mode": "diagonal",
                     "seed boards": [hex(_board({(0, 0): 1, (0, 1): 2}, m)), hex(_board({(0, 0): 2, (1, 1): 1}, m))],
                     "extra steps": 24}
    h8 = [(r, c) for r in range(2) for c in range(4)]
    m = _cellmask(h8)
    pats["horiz8"] = {"valid pattern": [hex(m)], "target pos": hex(0xFFFFFFFFFFFFFFFF & ~m),
                      "canonical mode": "horizontal",
                      "seed boards": [hex(_board({(1, 0): 1, (1, 1): 2}, m)), hex(_board({(1, 3): 2, (0, 3): 1}, m))],
                      "extra steps": 48}
    cells = [(r, c) for r in range(4) for c in range(4)]
    for n_free in (5, 6):
        fb = 0
        for (r, c) in cells[n_free:]:
            fb |= 0xF << (4 * ((3 - r) * 4 + (3 - c)))
        pats[f"free{n_free}"] = {"valid pattern": [], "target pos": "0xffffffffffffffff", "canonical mode": "full",
                                 "seed boards": [hex(fb | (1 << 60) | (2 << 56))], "extra steps": 16}
    return pats


# builds whose books are rewritten with a deletion threshold (BookSolver.cpp:589-593)
DELETION_CASES = [("L3", 5, "float32", 0.3), ("442", 6, "uint32", 0.5), ("diag9", 6, "float64", 0.7)]
# builds followed by the optimal-branch pass (keep_only_optimal_branches_impl, BookSolver.cpp:688-735)
OPTIMAL_CASES = [("L3", 6, "float32"), ("442", 6, "uint32"), ("diag9", 6, "float64"), ("44", 6, "1-float32")]
# variant boards (wall-merge mover, VBoardMover) of the catalog's "variant"
# category, each with its own symmetry mode (min24, min33, min34)
VARIANT_CASES = [("2x4", 7, "float32"), ("2x4", 8, "uint32"), ("3x3", 7, "float64"), ("3x4", 7, "float32")]

SMALL_CASES = [
    ("44", 6, "float32"), ("44", 7, "uint32"),
    ("L3", 5, "float32"), ("L3", 5, "uint32"), ("L3", 5, "uint64"), ("L3", 5, "float64"),
    ("L3", 5, "1-float32"), ("L3", 5, "1-float64"),
    ("442", 6, "float32"), ("diag9", 6, "float32"), ("horiz8", 6, "float32"),
    ("free5", 5, "float32"), ("free6", 5, "float32"), ("LL", 5, "float32"), ("t", 6, "uint32"),
]
FULL_CASES = [("L3", 8, "float32"), ("442", 9, "float32")]
# the 13-cell diagonal table (config-2 family) at the largest target the
# reference can build here (2.25e9 boards, ~45 GB of files, ~10 min)
HUGE_CASES = [("4432", 7, "float32")]
# forward prefixes of tables too large to build here: the first `steps` steps of
# run_pattern_generate at the table's own docheck_step (the 13-cell diagonal
# table at 1024: 560 steps, ~1 TB of raw layers). No success check happens
# before docheck_step (504), so these raw layers are the whole table's.
PREFIX_CASES = [("4432", 10, 130)]
# builds with compress=True: books over 2 MiB (layers 3 and up) become trie +
# xz-block directories <name>_<t>.z (TrieCompression.cpp:326-354, called from
# BookSolver.cpp:596-597 and CompressionBridge.cpp:41-59)
COMPRESS_CASES = [("442", 9, "float32"), ("442", 9, "uint32")]
# float32 tables against the float64 build of the same pattern (the reference's
# own builds): the largest and mean |r32 - r64| over every book entry
FP64_CASES = [("L3", 8), ("442", 9)]


def sha(path: str) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 24), b""):
            h.update(chunk)
    return h.hexdigest()


def run_case(catalog, pat, target, dtype, deletion=0.0, optimal=False, variant=False):
    masks, shifts, symm, seeds, steps, docheck, s0 = R.pattern_params(catalog[pat], target)
    T = 2 ** target
    name = f"{pat}_{T}"
    tag = f"{name}_{dtype}" + (f"_del{deletion}" if deletion else "") + ("_opt" if optimal else "")
    gdir = R.fresh_dir(os.path.join(WORK, tag, "gen") + "/")
    bdir = R.fresh_dir(os.path.join(WORK, tag, "build") + "/")
    spec, o = R.make_spec_options(masks, shifts, symm, target, steps, docheck, gdir + name + "_", dtype,
                                  is_variant=variant)
    started, last0, last1 = R.run_generate(seeds, spec, o)
    raw_len, raw_sha = [], []
    for t in range(steps - 2):
        p = gdir + f"{name}_{t}"
        raw_len.append(os.path.getsize(p) // 8)
        raw_sha.append(sha(p))
    spec, o = R.make_spec_options(masks, shifts, symm, target, steps, docheck, bdir + name + "_", dtype,
                                  deletion_threshold=deletion, optimal_branch_only=optimal, is_variant=variant)
    R.run_build(seeds, spec, o)
    book_len, book_sha = [], []
    rec = 12 if dtype in ("uint32", "float32", "1-float32") else 16
    for t in range(steps):
        p = bdir + f"{name}_{t}.book"
        book_len.append(os.path.getsize(p) // rec)
        book_sha.append(sha(p))
    case = {
        "pattern": pat, "target": target, "dtype": dtype, "spawn_rate4": 0.1,
        "masks": [hex(m) for m in masks], "shifts": shifts, "symm_mode": symm,
        "seeds": [hex(int(s)) for s in seeds], "steps": steps, "docheck_step": docheck,
        "tile_sum0": s0, "pattern_full": name,
        "raw_len": raw_len, "raw_sha256": raw_sha,
        "partial_len": [int(last0.size), int(last1.size)],
        "book_len": book_len, "book_sha256": book_sha,
    }
    if optimal:
        case["optimal_branch_only"] = True
    if variant:
        case["is_variant"] = True
    if deletion:
        case["deletion_threshold"] = deletion
        lines = open(bdir + name + "_stats.txt").read().splitlines()
        case["stats_columns"] = [",".join(x.split(",")[:3]) for x in lines]
    if (pat, target, dtype) in HUGE_CASES:
        import shutil
        shutil.rmtree(gdir, ignore_errors=True)
    return case, bdir


def run_prefix(catalog, pat, target, steps):
    masks, shifts, symm, seeds, full_steps, docheck, s0 = R.pattern_params(catalog[pat], target)
    T = 2 ** target
    name = f"{pat}_{T}"
    gdir = R.fresh_dir(os.path.join(WORK, f"{name}_prefix{steps}", "gen") + "/")
    spec, o = R.make_spec_options(masks, shifts, symm, target, steps, docheck, gdir + name + "_", "float32")
    started, last0, last1 = R.run_generate(seeds, spec, o)
    raw_len, raw_sha = [], []
    for t in range(steps - 2):
        p = gdir + f"{name}_{t}"
        raw_len.append(os.path.getsize(p) // 8)
        raw_sha.append(sha(p))
        os.remove(p)
    import shutil
    shutil.rmtree(os.path.dirname(gdir.rstrip("/")), ignore_errors=True)
    return {
        "pattern": pat, "target": target, "dtype": "float32", "spawn_rate4": 0.1,
        "masks": [hex(m) for m in masks], "shifts": shifts, "symm_mode": symm,
        "seeds": [hex(int(s)) for s in seeds], "steps": steps, "full_steps": full_steps,
        "docheck_step": docheck, "tile_sum0": s0, "pattern_full": name,
        "raw_len": raw_len, "raw_sha256": raw_sha,
        "partial_len": [int(last0.size), int(last1.size)],
        "size_class": "prefix",
    }


def run_fp64_error(catalog, pat, target):
    import importlib
    sys.path.insert(0, ROOT)
    P = importlib.import_module("2048endgametablebase_b200.precision")
    masks, shifts, symm, seeds, steps, docheck, s0 = R.pattern_params(catalog[pat], target)
    name = f"{pat}_{2 ** target}"
    books = {}
    for dtype in ("float32", "float64"):
        bdir = R.fresh_dir(os.path.join(WORK, f"{name}_{dtype}_fp64err") + "/")
        spec, o = R.make_spec_options(masks, shifts, symm, target, steps, docheck, bdir + name + "_", dtype)
        R.run_build(seeds, spec, o)
        books[dtype] = [open(bdir + f"{name}_{t}.book", "rb").read() for t in range(steps)]
        import shutil
        shutil.rmtree(bdir, ignore_errors=True)
    r = P.compare_books(books["float32"], "float32", books["float64"], "float64")
    r["board"] = hex(r["board"])
    return r


def run_compress_case(catalog, pat, target, dtype, rng):
    """A compressed build by the reference: per layer, the .book digest or the
    digests of the four files of its .z directory; plus move_on_dic answers on
    the compressed table for positions sampled from the uncompressed books
    (their answers on the uncompressed table are recorded beside them)."""
    import shutil
    case, plain_dir = run_case(catalog, pat, target, dtype)
    masks, shifts, symm, seeds, steps, docheck, s0 = R.pattern_params(catalog[pat], target)
    name = f"{pat}_{2 ** target}"
    zdir = R.fresh_dir(os.path.join(WORK, f"{name}_{dtype}_compressed", "build") + "/")
    spec, o = R.make_spec_options(masks, shifts, symm, target, steps, docheck, zdir + name + "_", dtype)
    o.compress = True
    R.run_build(seeds, spec, o)
    layers = []
    for t in range(steps):
        b = zdir + f"{name}_{t}.book"
        z = zdir + f"{name}_{t}.z"
        if os.path.isdir(z):
            stem = f"{name}_{t}."
            layers.append({"kind": "z", "sha256": {sfx: sha(os.path.join(z, stem + sfx)) for sfx in ("i", "ii", "s", "z")}})
        else:
            layers.append({"kind": "book", "sha256": sha(b) if os.path.exists(b) else None})
    case = dict(case, compress=True, size_class="compressed", layers=layers)
    answers = reader_fixture(case, plain_dir, rng, n_pos=400)
    fc = R.module()
    sp = fc.PatternSpec()
    sp.name = pat
    sp.pattern_masks = [int(m, 16) for m in case["masks"]]
    sp.success_shifts = case["shifts"]
    sp.symm_mode = case["symm_mode"]
    reader = fc.ClassicBookReader(sp, False)
    differ = 0
    for a in answers:
        res, dt = reader.move_on_dic(a["board"], [(zdir, dtype)], name, -case["tile_sum0"])
        got = [[k, v] for k, v in res.items()]
        differ += got != a["result"]
        a["result"], a["dtype"] = got, dt
    case["reader_answers_differing_from_uncompressed"] = differ
    shutil.rmtree(os.path.dirname(zdir.rstrip("/")), ignore_errors=True)
    return case, answers


def prims_fixture():
    L = ctypes.CDLL(os.path.join(R.REF_DIR, "libref_prims.so"))
    rng = np.random.default_rng(2048)
    n = 20000
    # random boards with small tiles, a share of 0xF cells and empty cells
    cells = rng.integers(0, 16, size=(n, 16))
    cells = np.where(rng.random((n, 16)) < 0.35, 0, cells)
    boards = np.zeros(n, dtype=np.uint64)
    for k in range(16):
        boards |= cells[:, k].astype(np.uint64) << np.uint64(4 * k)
    out = {"boards": boards}
    mv = np.zeros(n * 4, dtype=np.uint64)
    L.ref_move_all_dir_batch(boards.ctypes.data, ctypes.c_size_t(n), mv.ctypes.data)
    out["moves"] = mv.reshape(n, 4)
    mv = np.zeros(n * 4, dtype=np.uint64)
    L.ref_move_all_dir_variant_batch(boards.ctypes.data, ctypes.c_size_t(n), mv.ctypes.data)
    out["moves_variant"] = mv.reshape(n, 4)
    for mode in range(7):
        c = np.zeros(n, dtype=np.uint64)
        L.ref_canonical_batch(boards.ctypes.data, ctypes.c_size_t(n), mode, c.ctypes.data)
        out[f"canonical_{mode}"] = c
    for idx in range(8):
        c = np.zeros(n, dtype=np.uint64)
        L.ref_apply_sym_batch(boards.ctypes.data, ctypes.c_size_t(n), idx, c.ctypes.data)
        out[f"sym_{idx}"] = c
    left = np.zeros(65536, dtype=np.uint16)
    right = np.zeros(65536, dtype=np.uint16)
    L.ref_row_tables(left.ctypes.data, right.ctypes.data)
    out["row_left"] = left
    out["row_right"] = right
    left = np.zeros(65536, dtype=np.uint16)
    right = np.zeros(65536, dtype=np.uint16)
    L.ref_row_tables_variant(left.ctypes.data, right.ctypes.data)
    out["row_left_variant"] = left
    out["row_right_variant"] = right
    np.savez_compressed(os.path.join(GOLDEN, "prims.npz"), **out)


# masked-board parameter sets of the advanced algorithm: (small_tile_sum_limit,
# target, fixed 32k shifts, num_free_32k)
AD_PARAMS = [(96, 10, [], 0), (96, 11, [60, 56], 2), (160, 9, [0, 4, 8], 1), (32, 12, [12], 3)]


def _pack(cells: np.ndarray) -> np.ndarray:
    boards = np.zeros(len(cells), dtype=np.uint64)
    for k in range(16):
        boards |= cells[:, k].astype(np.uint64) << np.uint64(4 * k)
    return boards


def ad_prims_fixture():
    """The advanced algorithm's masked-board primitives, from the reference's
    own BoardMoverAD / BoardMaskerAD (oracle/_ref/libref_ad_prims.so)."""
    L = ctypes.CDLL(os.path.join(R.REF_DIR, "libref_ad_prims.so"))
    P, Z, U = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32
    L.ref_ad_move_all_dir_batch.argtypes = [P, Z, P, P]
    L.ref_ad_mask_board_batch.argtypes = [P, Z, ctypes.c_int, P]
    L.ref_ad_tile_stats_batch.argtypes = [P, Z, U, U, P, Z, U, ctypes.c_int, P]
    L.ref_ad_validate_batch.argtypes = [P, Z, P, U, U, P, Z, U, P]
    L.ref_ad_tiles_combinations.argtypes = [P, P]
    L.ref_ad_unmask_batch.argtypes = [P, Z, P, U, U, P, Z, U, P, P, Z]
    L.ref_ad_unmask_batch.restype = ctypes.c_size_t
    rng = np.random.default_rng(4096)
    n = 4000
    # mover: small tiles, equal neighbours common (merges into 32 and 64+), some 0xF
    vals = np.array([0, 1, 2, 3, 4, 5, 6, 7, 15])
    prob = np.array([0.30, 0.08, 0.08, 0.08, 0.10, 0.14, 0.10, 0.04, 0.08])
    mover_boards = _pack(rng.choice(vals, size=(n, 16), p=prob))
    out = {"mover_boards": mover_boards}
    mv = np.zeros(n * 4, dtype=np.uint64)
    fl = np.zeros(n * 4, dtype=np.uint8)
    L.ref_ad_move_all_dir_batch(mover_boards.ctypes.data, ctypes.c_size_t(n), mv.ctypes.data, fl.ctypes.data)
    out["mover_moves"], out["mover_flags"] = mv.reshape(n, 4), fl.reshape(n, 4)
    # masker and tile statistics: any nibble
    boards = _pack(rng.integers(0, 16, size=(n, 16)))
    out["boards"] = boards
    for th in (6, 5, 9):
        m = np.zeros(n, dtype=np.uint64)
        L.ref_ad_mask_board_batch(boards.ctypes.data, ctypes.c_size_t(n), ctypes.c_int(th), m.ctypes.data)
        out[f"mask_{th}"] = m
    for i, (limit, target, fixed, nfree) in enumerate(AD_PARAMS):
        fx = np.array(fixed, dtype=np.uint8)
        for kind in (1, 2, 4):
            st = np.zeros(n * 8, dtype=np.int64)
            L.ref_ad_tile_stats_batch(boards.ctypes.data, ctypes.c_size_t(n), ctypes.c_uint32(limit),
                                      ctypes.c_uint32(target), fx.ctypes.data, ctypes.c_size_t(len(fx)),
                                      ctypes.c_uint32(nfree), ctypes.c_int(kind), st.ctypes.data)
            out[f"stats_{i}_{kind}"] = st.reshape(n, 8)
        # validate: boards whose 32k count (tiles of 64 and up outside the fixed
        # cells) is num_free_32k .. num_free_32k + 9, where the reference's
        # table lookup stays inside its table; small tiles mostly
        cells = rng.choice(np.arange(16), size=(4 * n, 16),
                           p=np.r_[[0.3], np.full(5, 0.5 / 5), np.full(10, 0.2 / 10)])
        cand = _pack(cells)
        st = np.zeros(len(cand) * 8, dtype=np.int64)
        L.ref_ad_tile_stats_batch(cand.ctypes.data, ctypes.c_size_t(len(cand)), ctypes.c_uint32(limit),
                                  ctypes.c_uint32(target), fx.ctypes.data, ctypes.c_size_t(len(fx)),
                                  ctypes.c_uint32(nfree), ctypes.c_int(2), st.ctypes.data)
        st = st.reshape(len(cand), 8)
        keep = (st[:, 1] >= nfree) & (st[:, 1] <= nfree + 9)
        vb = cand[keep][:n]
        small = st[keep][:n, 0].astype(np.int64)
        large = 64 * rng.integers(0, 300, size=len(vb))
        orig = (small + ((nfree + len(fixed)) << 15) + large).astype(np.uint32)
        ok = np.zeros(len(vb), dtype=np.uint8)
        L.ref_ad_validate_batch(vb.ctypes.data, ctypes.c_size_t(len(vb)), orig.ctypes.data, ctypes.c_uint32(limit),
                                ctypes.c_uint32(target), fx.ctypes.data, ctypes.c_size_t(len(fx)),
                                ctypes.c_uint32(nfree), ok.ctypes.data)
        out[f"validate_{i}_boards"], out[f"validate_{i}_sums"], out[f"validate_{i}"] = vb, orig, ok
    lens = np.zeros(2560, dtype=np.uint8)
    vals16 = np.zeros(2560 * 16, dtype=np.uint8)
    L.ref_ad_tiles_combinations(lens.ctypes.data, vals16.ctypes.data)
    # unmask_board: masked boards (small tiles and 0xF cells) whose 32k count is
    # num_free_32k .. num_free_32k + 4, tile sums mostly of large tiles that a
    # combination exists for (a few arbitrary ones)
    for i, (limit, target, fixed, nfree) in enumerate(AD_PARAMS):
        fx = np.array(fixed, dtype=np.uint8)
        fmask = 0
        for sh in fixed:
            fmask |= 0xF << sh
        cells = rng.choice(np.r_[np.arange(6), [15]], size=(8 * 400, 16), p=[0.35, 0.1, 0.1, 0.1, 0.1, 0.05, 0.2])
        cand = _pack(cells)
        free_f = np.zeros(len(cand), dtype=np.int64)
        small = np.zeros(len(cand), dtype=np.int64)
        for k in range(16):
            nib = (cand >> np.uint64(4 * k)) & np.uint64(0xF)
            if (fmask >> (4 * k)) & 0xF:
                continue
            free_f += (nib == 15)
            small += np.where((nib > 0) & (nib < 15), 1 << nib.astype(np.int64), 0)
        c = free_f - nfree
        keep = (c >= 0) & (c <= 4)
        ub, small, c = cand[keep][:400], small[keep][:400], c[keep][:400]
        large = np.zeros(len(ub), dtype=np.int64)
        for j in range(len(ub)):
            ok = np.flatnonzero(lens[256 * c[j]: 256 * c[j] + 256]) if c[j] > 0 else np.array([], dtype=np.int64)
            if len(ok) and rng.random() < 0.85:
                large[j] = 64 * int(rng.choice(ok)) + int(rng.integers(0, 64))
            else:
                large[j] = 64 * int(rng.integers(0, 256))
        orig = (small + ((nfree + len(fixed)) << 15) + large).astype(np.uint32)
        counts = np.zeros(len(ub), dtype=np.uint32)
        total = L.ref_ad_unmask_batch(ub.ctypes.data, len(ub), orig.ctypes.data, limit, target, fx.ctypes.data,
                                      len(fx), nfree, counts.ctypes.data, None, 0)
        got = np.zeros(max(1, total), dtype=np.uint64)
        L.ref_ad_unmask_batch(ub.ctypes.data, len(ub), orig.ctypes.data, limit, target, fx.ctypes.data, len(fx),
                              nfree, counts.ctypes.data, got.ctypes.data, total)
        out[f"unmask_{i}_boards"], out[f"unmask_{i}_sums"] = ub, orig
        out[f"unmask_{i}_counts"], out[f"unmask_{i}"] = counts, got[:total]
    out["combo_lens"], out["combo_vals"] = lens, vals16.reshape(2560, 16)
    # the masked row rule: each row alone on an otherwise empty board
    rows = np.arange(65536, dtype=np.uint64)
    mv = np.zeros(65536 * 4, dtype=np.uint64)
    fl = np.zeros(65536 * 4, dtype=np.uint8)
    L.ref_ad_move_all_dir_batch(rows.ctypes.data, ctypes.c_size_t(65536), mv.ctypes.data, fl.ctypes.data)
    mv = mv.reshape(65536, 4)
    out["row_left"] = (mv[:, 0] & np.uint64(0xFFFF)).astype(np.uint16)
    out["row_right"] = (mv[:, 1] & np.uint64(0xFFFF)).astype(np.uint16)
    out["row_flag"] = fl.reshape(65536, 4)[:, 0]
    np.savez_compressed(os.path.join(GOLDEN, "ad_prims.npz"), **out)


def decode(board: int):
    return [[(1 << v) if (v := (board >> (4 * ((3 - r) * 4 + (3 - c)))) & 0xF) else 0 for c in range(4)]
            for r in range(4)]


def reader_fixture(case, bdir, rng, n_pos=60):
    """move_on_dic answers for positions sampled like sample_classic_book_state
    (native_core/src/ReaderRuntime.cpp:945-993): a book key plus one spawn, then
    a random orientation; one in eight gets a random free-cell nibble changed."""
    fc = R.module()
    spec = fc.PatternSpec()
    spec.name = case["pattern"]
    spec.pattern_masks = [int(m, 16) for m in case["masks"]]
    spec.success_shifts = case["shifts"]
    spec.symm_mode = case["symm_mode"]
    variant = bool(case.get("is_variant"))
    reader = fc.ClassicBookReader(spec, variant)
    rec = 12 if case["dtype"] in ("uint32", "float32", "1-float32") else 16
    path_list = [(bdir, case["dtype"])]
    out = []
    nonempty = [t for t, n in enumerate(case["book_len"]) if n > 0]
    if not nonempty:
        return out
    for _ in range(n_pos):
        t = int(rng.choice(nonempty))
        data = np.fromfile(bdir + f"{case['pattern_full']}_{t}.book", dtype=np.uint8)
        recs = data.reshape(-1, rec)
        key = int(recs[int(rng.integers(len(recs)))][:8].view(np.uint64)[0])
        empties = [i for i in range(16) if (key >> (4 * i)) & 0xF == 0]
        if not empties:
            continue
        i = int(rng.choice(empties))
        v = 2 if rng.random() < 0.1 else 1
        pos = key | (v << (4 * i))
        if rng.random() < 0.125:
            j = int(rng.integers(16))
            if (pos >> (4 * j)) & 0xF != 0xF:
                pos = (pos & ~(0xF << (4 * j))) | (int(rng.integers(0, 6)) << (4 * j))
        # a variant reader tries the board as given only (operation_sequence,
        # ReaderRuntime.cpp:171-182): most variant positions stay unrotated
        op = int(rng.integers(8)) if not variant or rng.random() < 0.25 else 0
        board = decode(pos)
        b = np.array(board)
        if op in (1, 5):
            b = np.rot90(b, 1)
        elif op in (2, 6):
            b = np.rot90(b, 2)
        elif op in (3, 7):
            b = np.rot90(b, 3)
        if op >= 4:
            b = b[:, ::-1]
        board = b.tolist()
        res, dt = reader.move_on_dic(board, path_list, case["pattern_full"], -case["tile_sum0"])
        out.append({"board": board, "result": [[k, v] for k, v in res.items()], "dtype": dt})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--full", action="store_true", help="also the full-size L3-256 and 442-512 builds")
    ap.add_argument("--huge", action="store_true", help="also the 4432-128 build (needs ~45 GB of disk in GOLDEN_WORK)")
    ap.add_argument("--prefix", action="store_true",
                    help="also the forward prefix of the 13-cell diagonal table at 1024 (~30 GB in GOLDEN_WORK)")
    ap.add_argument("--compress", action="store_true",
                    help="also the compressed (trie + xz) builds of 442-512")
    ap.add_argument("--fp64", action="store_true",
                    help="also the float32-vs-float64 rate error of the full-size L3-256 and 442-512 tables")
    ap.add_argument("--only", default="", help="comma-separated case keys to (re)generate")
    args = ap.parse_args()
    R.build(REF_ROOT)
    catalog = json.load(open(REF_CATALOG))
    catalog.update(custom_patterns())
    only = set(filter(None, args.only.split(",")))
    if not only or "prims" in only:
        prims_fixture()
    if not only or "ad_prims" in only:
        ad_prims_fixture()
    cases_path = os.path.join(GOLDEN, "cases.json")
    cases = json.load(open(cases_path)) if os.path.exists(cases_path) else {}
    reader = {}
    rng = np.random.default_rng(7)
    todo = SMALL_CASES + (FULL_CASES if args.full else []) + (HUGE_CASES if args.huge else [])
    for pat, target, dtype in todo:
        key = f"{pat}_{2 ** target}_{dtype}"
        if only and key not in only:
            continue
        print("case", key, flush=True)
        case, bdir = run_case(catalog, pat, target, dtype)
        case["size_class"] = ("full" if (pat, target, dtype) in FULL_CASES else
                              "huge" if (pat, target, dtype) in HUGE_CASES else "small")
        cases[key] = case
        if case["size_class"] == "small" and pat in ("44", "L3", "diag9", "horiz8", "free6", "442"):
            reader[key] = reader_fixture(case, bdir, rng)
        if case["size_class"] == "huge":
            import shutil
            shutil.rmtree(os.path.dirname(bdir.rstrip("/")), ignore_errors=True)
        if key == "free5_32_float32":
            data = {}
            for t in range(case["steps"]):
                raw = bdir + f"free5_32_{t}.book"
                data[f"book_{t}"] = np.fromfile(raw, dtype=np.uint8)
            np.savez_compressed(os.path.join(GOLDEN, "free5_32.npz"), **data)
    for pat, target, steps in (PREFIX_CASES if args.prefix else []):
        key = f"{pat}_{2 ** target}_prefix{steps}"
        if only and key not in only:
            continue
        print("case", key, flush=True)
        cases[key] = run_prefix(catalog, pat, target, steps)
    for pat, target, dtype in (COMPRESS_CASES if args.compress else []):
        key = f"{pat}_{2 ** target}_{dtype}_compressed"
        if only and key not in only:
            continue
        print("case", key, flush=True)
        cases[key], reader[key] = run_compress_case(catalog, pat, target, dtype, np.random.default_rng(17))
    for pat, target in (FP64_CASES if args.fp64 else []):
        key = f"{pat}_{2 ** target}_fp64_error"
        if only and key not in only:
            continue
        print("case", key, flush=True)
        cases[key] = dict(run_fp64_error(catalog, pat, target), pattern=pat, target=target, size_class="fp64_error")
    for pat, target, dtype, thr in DELETION_CASES:
        key = f"{pat}_{2 ** target}_{dtype}_del{thr}"
        if only and key not in only:
            continue
        print("case", key, flush=True)
        case, _ = run_case(catalog, pat, target, dtype, thr)
        case["size_class"] = "deletion"
        cases[key] = case
    for pat, target, dtype in OPTIMAL_CASES:
        key = f"{pat}_{2 ** target}_{dtype}_opt"
        if only and key not in only:
            continue
        print("case", key, flush=True)
        case, _ = run_case(catalog, pat, target, dtype, optimal=True)
        case["size_class"] = "optimal"
        cases[key] = case
    for pat, target, dtype in VARIANT_CASES:
        key = f"{pat}_{2 ** target}_{dtype}"
        if only and key not in only:
            continue
        print("case", key, flush=True)
        case, bdir = run_case(catalog, pat, target, dtype, variant=True)
        case["size_class"] = "variant"
        cases[key] = case
        reader[key] = reader_fixture(case, bdir, rng)
    json.dump(cases, open(cases_path, "w"), indent=0)
    if reader:
        rpath = os.path.join(GOLDEN, "reader.json")
        old = json.load(open(rpath)) if os.path.exists(rpath) else {}
        old.update(reader)
        json.dump(old, open(rpath, "w"))
    print("wrote", cases_path)


if __name__ == "__main__":
    main()
