"""GPU builds through the drop-in formation_core (C ABI) against the
reference's own layer files and books (SHA-256 per file, tests/golden)."""
import os

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def _generate(case, d):
    F = H.fc()
    spec, o = H.spec_options(case, d + case["pattern_full"] + "_")
    started, l0, l1 = F.run_pattern_generate(H.seeds(case), spec, o)
    return started, l0, l1


@pytest.mark.parametrize("key", H.SMALL_CASES + H.VARIANT_CPU_CASES)
def test_generate_raw_layers_bit_exact(key, tmp_root):
    case = H.cases()[key]
    d = H.fresh(os.path.join(tmp_root, "gen_" + key) + "/")
    started, l0, l1 = _generate(case, d)
    assert started
    steps = case["steps"]
    name = case["pattern_full"]
    for t in range(steps - 2):
        p = d + f"{name}_{t}"
        if t == steps - 2:
            continue
        assert os.path.exists(p), p
        assert os.path.getsize(p) // 8 == case["raw_len"][t], (key, t)
        assert H.sha(p) == case["raw_sha256"][t], (key, t)
    # the last two layers are written as success-only books
    for t in (steps - 2, steps - 1):
        assert H.sha(d + f"{name}_{t}.book") == case["book_sha256"][t], (key, t)
    assert l0.size == case["book_len"][steps - 2] and l1.size == case["book_len"][steps - 1]


@pytest.mark.parametrize("key", H.SMALL_CASES + H.VARIANT_CASES)
def test_build_books_bit_exact(key, tmp_root):
    case = H.cases()[key]
    F = H.fc()
    d = H.fresh(os.path.join(tmp_root, "build_" + key) + "/")
    spec, o = H.spec_options(case, d + case["pattern_full"] + "_")
    F.run_pattern_build(H.seeds(case), spec, o)
    name = case["pattern_full"]
    for t in range(case["steps"]):
        p = d + f"{name}_{t}.book"
        assert H.sha(p) == case["book_sha256"][t], (key, t)
    # no raw layer is left behind, as after the reference's solve
    assert not any(os.path.exists(d + f"{name}_{t}") for t in range(case["steps"]))
    st = F.last_build_stats()
    assert st["raw_boards"] >= sum(case["raw_len"])
    assert st["book_entries"] == sum(case["book_len"])
    lines = open(d + f"{name}_stats.txt").read().splitlines()
    assert lines[0] == "layer,length,max success rate,speed,deletion_threshold,time"


@pytest.mark.slow
@pytest.mark.parametrize("key", H.FULL_CASES)
def test_full_size_build_bit_exact(key, tmp_root):
    """The benchmark tables at full size (L3-256, 442-512)."""
    case = H.cases()[key]
    F = H.fc()
    d = H.fresh(os.path.join(tmp_root, "full_" + key) + "/")
    spec, o = H.spec_options(case, d + case["pattern_full"] + "_")
    F.run_pattern_build(H.seeds(case), spec, o)
    name = case["pattern_full"]
    bad = [t for t in range(case["steps"]) if H.sha(d + f"{name}_{t}.book") != case["book_sha256"][t]]
    assert not bad, bad[:10]
    st = F.last_build_stats()
    assert st["raw_boards"] >= sum(case["raw_len"])
    assert st["book_entries"] == sum(case["book_len"])
    H.fresh(d)


@pytest.mark.parametrize("key", ["L3_32_float32", "diag9_64_float32", "L3_32_uint32"])
def test_generate_then_solve_matches_build(key, tmp_root):
    """run_pattern_generate + run_pattern_solve (the file-based path) give the reference's books."""
    case = H.cases()[key]
    F = H.fc()
    d = H.fresh(os.path.join(tmp_root, "gs_" + key) + "/")
    spec, o = H.spec_options(case, d + case["pattern_full"] + "_")
    started, l0, l1 = F.run_pattern_generate(H.seeds(case), spec, o)
    F.run_pattern_solve(l0, l1, spec, o)
    name = case["pattern_full"]
    for t in range(case["steps"]):
        assert H.sha(d + f"{name}_{t}.book") == case["book_sha256"][t], (key, t)


def test_resume_after_interrupted_forward(tmp_root):
    """Raw layers from an interrupted run: the forward restarts at the first missing step."""
    case = H.cases()["L3_32_float32"]
    F = H.fc()
    d = H.fresh(os.path.join(tmp_root, "resume") + "/")
    name = case["pattern_full"]
    spec, o = H.spec_options(case, d + name + "_")
    F.run_pattern_generate(H.seeds(case), spec, o)
    # keep raw layers 0..20 only, as if the run stopped after step 20
    for f in os.listdir(d):
        stem = f.split("_")[-1]
        if stem.endswith(".book") or (stem.isdigit() and int(stem) > 20):
            os.remove(d + f)
    F.run_pattern_build(H.seeds(case), spec, o)
    for t in range(case["steps"]):
        assert H.sha(d + f"{name}_{t}.book") == case["book_sha256"][t], t


def test_resume_after_interrupted_solve(tmp_root):
    """Books of the top layers present: the solve restarts below them."""
    case = H.cases()["44_64_float32"]
    F = H.fc()
    d = H.fresh(os.path.join(tmp_root, "resume2") + "/")
    name = case["pattern_full"]
    spec, o = H.spec_options(case, d + name + "_")
    started, l0, l1 = F.run_pattern_generate(H.seeds(case), spec, o)
    F.run_pattern_solve(l0, l1, spec, o)
    # drop the books of layers 0..30 and put their raw layers back
    F2 = H.fresh(os.path.join(tmp_root, "resume2_raw") + "/")
    spec2, o2 = H.spec_options(case, F2 + name + "_")
    F.run_pattern_generate(H.seeds(case), spec2, o2)
    for t in range(31):
        os.remove(d + f"{name}_{t}.book")
        os.replace(F2 + f"{name}_{t}", d + f"{name}_{t}")
    F.run_pattern_solve(F.PatternLayer(), F.PatternLayer(), spec, o)
    for t in range(case["steps"]):
        assert H.sha(d + f"{name}_{t}.book") == case["book_sha256"][t], t


def test_progress_reaches_total(tmp_root):
    case = H.cases()["44_64_float32"]
    F = H.fc()
    d = H.fresh(os.path.join(tmp_root, "progress") + "/")
    spec, o = H.spec_options(case, d + case["pattern_full"] + "_")
    F.reset_build_progress(0)
    F.run_pattern_build(H.seeds(case), spec, o)
    cur, tot = F.get_build_progress()
    assert tot == 2 * case["steps"] and cur == tot


def test_invalid_options_raise(tmp_root):
    F = H.fc()
    case = H.cases()["44_64_float32"]
    spec, o = H.spec_options(case, os.path.join(tmp_root, "bad_"))
    # compressed books are files: a device-only build asking for them is refused
    import ctypes
    N = H.pkg()._native
    o.compress = True
    seeds = H.seeds(case)
    c_spec, c_opt = spec.to_c(), o.to_c(write_files=False)
    rc = N.lib().egtb_build(seeds.ctypes.data, len(seeds), ctypes.byref(c_spec), ctypes.byref(c_opt), None)
    assert rc == -7 and "compress" in N.last_error()
    o.compress = False
    spec.symm_mode = 7
    with pytest.raises(RuntimeError, match="symmetry"):
        F.run_pattern_build(H.seeds(case), spec, o)


def test_variant_tables_are_refused_by_the_batched_build():
    """The batched build moves every table with the classic rule: a variant
    table in a batch is an error (build it with egtb_build)."""
    import ctypes
    import importlib
    B = importlib.import_module("2048endgametablebase_b200.batch")
    N = H.pkg()._native
    a = B._Args(B.random_tables(2, seed=3), "float32", 0, None)
    a.opts[1].is_variant = 1
    ts = (N.BuildStatsC * a.n)()
    bs = N.BatchStatsC()
    rc = N.lib().egtb_build_batch(a.n, a.seed_ptrs, a.n_seeds, a.specs, a.opts, None, ts, ctypes.byref(bs))
    assert rc == -7 and "variant" in N.last_error()


@pytest.mark.slow
@pytest.mark.parametrize("key", [k for k, v in H.cases().items() if v.get("size_class") == "huge"])
def test_huge_build_in_memory_bit_exact(key):
    """The 13-cell diagonal table at target 128 (2.25e9 boards, 17.9 GB of books),
    built in device memory and read back layer by layer."""
    import ctypes
    import hashlib
    case = H.cases()[key]
    N = H.pkg()._native
    spec, o = H.spec_options(case, "/nonexistent/unused_")
    c_spec, c_opt = spec.to_c(), o.to_c(write_files=False)
    st = N.BuildStatsC()
    s = H.seeds(case)
    N.check(N.lib().egtb_build(s.ctypes.data, len(s), ctypes.byref(c_spec), ctypes.byref(c_opt), ctypes.byref(st)))
    assert st.raw_boards == sum(case["raw_len"])
    assert st.book_entries == sum(case["book_len"])
    buf = np.empty(max(case["book_len"]) * 12 + 16, dtype=np.uint8)
    size = ctypes.c_uint64(0)
    for t in range(case["steps"]):
        N.check(N.lib().egtb_book_layer_copy(0, t, buf.ctypes.data, buf.nbytes, ctypes.byref(size)))
        assert hashlib.sha256(buf[: size.value].tobytes()).hexdigest() == case["book_sha256"][t], t


@pytest.mark.parametrize("key", [k for k, v in H.cases().items() if v.get("size_class") == "deletion"])
def test_deletion_threshold_books_bit_exact(key, tmp_root):
    """deletion_threshold > 0: after layer i is solved, the book of layer i+2
    keeps only rates above the threshold (BookSolver.cpp:589-593); the books
    and the stats.txt columns must equal the reference's."""
    case = H.cases()[key]
    F = H.fc()
    d = H.fresh(os.path.join(tmp_root, "del_" + key) + "/")
    spec, o = H.spec_options(case, d + case["pattern_full"] + "_")
    o.deletion_threshold = case["deletion_threshold"]
    F.run_pattern_build(H.seeds(case), spec, o)
    name = case["pattern_full"]
    for t in range(case["steps"]):
        assert H.sha(d + f"{name}_{t}.book") == case["book_sha256"][t], (key, t)
    lines = open(d + f"{name}_stats.txt").read().splitlines()
    assert [",".join(x.split(",")[:3]) for x in lines] == case["stats_columns"]


def test_deletion_threshold_needs_files():
    import ctypes
    case = H.cases()["L3_32_float32"]
    N = H.pkg()._native
    spec, o = H.spec_options(case, "/nonexistent/unused_")
    o.deletion_threshold = 0.3
    c_spec, c_opt = spec.to_c(), o.to_c(write_files=False)
    s = H.seeds(case)
    assert N.lib().egtb_build(s.ctypes.data, len(s), ctypes.byref(c_spec), ctypes.byref(c_opt), None) == -7


OPTIMAL_CASES = [k for k, v in H.cases().items() if v.get("size_class") == "optimal"]


@pytest.mark.parametrize("key", OPTIMAL_CASES)
def test_optimal_branch_books_bit_exact(key, tmp_root):
    """optimal_branch_only: after the solve, book i (i >= 21) keeps only the
    entries that are the best move of a position of thinned book i-2 plus a
    4 or of thinned book i-1 plus a 2 (BookSolver.cpp:611-735); every book
    must equal the reference's, and the progress counts 3 * steps."""
    case = H.cases()[key]
    F = H.fc()
    d = H.fresh(os.path.join(tmp_root, "opt_" + key) + "/")
    spec, o = H.spec_options(case, d + case["pattern_full"] + "_")
    o.optimal_branch_only = True
    F.reset_build_progress(0)
    F.run_pattern_build(H.seeds(case), spec, o)
    cur, tot = F.get_build_progress()
    assert tot == 3 * case["steps"] and cur == tot
    name = case["pattern_full"]
    for t in range(case["steps"]):
        assert H.sha(d + f"{name}_{t}.book") == case["book_sha256"][t], (key, t)
    assert not os.path.exists(d + name + "_optlayer")


def test_optimal_branch_resumes_after_marker(tmp_root):
    """An interrupted pass leaves "<path>optlayer" with the last thinned
    layer: a rerun solves nothing and thins only the layers above it."""
    case = H.cases()["L3_64_float32_opt"]
    F = H.fc()
    name = case["pattern_full"]
    done = H.fresh(os.path.join(tmp_root, "opt_done") + "/")
    spec, o = H.spec_options(case, done + name + "_")
    o.optimal_branch_only = True
    F.run_pattern_build(H.seeds(case), spec, o)
    d = H.fresh(os.path.join(tmp_root, "opt_resume") + "/")
    spec, o = H.spec_options(case, d + name + "_")
    F.run_pattern_build(H.seeds(case), spec, o)  # books not thinned
    for t in range(21, 41):
        os.replace(done + f"{name}_{t}.book", d + f"{name}_{t}.book")
    with open(d + name + "_optlayer", "w") as f:
        f.write("40")
    o.optimal_branch_only = True
    F.run_pattern_solve(F.PatternLayer(), F.PatternLayer(), spec, o)
    for t in range(case["steps"]):
        assert H.sha(d + f"{name}_{t}.book") == case["book_sha256"][t], t
    assert not os.path.exists(d + name + "_optlayer")


def test_optimal_branch_needs_files():
    import ctypes
    case = H.cases()["L3_32_float32"]
    N = H.pkg()._native
    spec, o = H.spec_options(case, "/nonexistent/unused_")
    o.optimal_branch_only = True
    c_spec, c_opt = spec.to_c(), o.to_c(write_files=False)
    s = H.seeds(case)
    assert N.lib().egtb_build(s.ctypes.data, len(s), ctypes.byref(c_spec), ctypes.byref(c_opt), None) == -7
