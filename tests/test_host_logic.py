"""Host-side logic that mirrors the reference's Python layer: pattern catalog
parsing, steps/docheck, option defaults, reader result ordering."""
import numpy as np
import pytest

import helpers as H


def patterns():
    import importlib
    return importlib.import_module("2048endgametablebase_b200.patterns")


def test_builtin_catalog_matches_golden_cases():
    P = patterns()
    for key in ("L3_32_float32", "442_64_float32", "L3_256_float32", "442_512_float32"):
        case = H.cases()[key]
        meta = P.pattern_catalog[case["pattern"]]
        assert [hex(int(m)) for m in meta["pattern_masks"]] == case["masks"]
        assert list(meta["success_shifts"]) == case["shifts"]
        assert [hex(int(s)) for s in meta["seed_boards"]] == case["seeds"]
        assert -meta["nums_adjust"] == case["tile_sum0"]
        steps, docheck = P.steps_and_docheck(case["tile_sum0"], case["target"], meta["extra_steps"])
        assert (steps, docheck) == (case["steps"], case["docheck_step"])


def test_4432_is_diagonal_with_13_free_cells():
    P = patterns()
    meta = P.pattern_catalog["4432"]
    assert meta["canonical_mode"] == "diagonal"
    assert bin(int(meta["pattern_masks"][0])).count("1") == 12  # three pinned cells


def test_seed_filter_keeps_the_first_tile_sum():
    P = patterns()
    e = P.parse_entry("x", {"valid pattern": ["0xf"], "seed boards": ["0x12f", "0x11f", "0x21f"]})
    assert [hex(int(b)) for b in e["seed_boards"]] == ["0x12f", "0x21f"]


def test_success_shifts_from_target_pos():
    P = patterns()
    assert P.find_f_nibble_positions(0xF000000) == [24]
    assert P.find_f_nibble_positions(0xFFFFFFFFFFFFFFFF) == list(range(0, 64, 4))


def test_run_options_defaults_match_reference():
    F = H.fc()
    o = F.RunOptions()
    assert (o.spawn_rate4, o.success_rate_dtype, o.direct_io_queue_depth, o.direct_io_chunk_mib) == (
        0.1, "uint32", 16, 8)
    assert F.dtype_code("nonsense") == 0 and F.dtype_code("1-float64") == 5


def test_adjust_direction_is_a_bijection_per_op():
    F = H.fc()
    for op in range(8):
        names = {F._adjust_direction(op, d) for d in ("up", "right", "down", "left")}
        assert names == {"up", "right", "down", "left"}


def test_sorted_entries_are_stable_and_descending():
    F = H.fc()
    vals = np.array([0.5, 0.9, 0.5, 0.1])  # up, right, down, left
    entries = F.ClassicBookReader._sorted_entries(0, vals, 0b0111)
    # kOrderedResultKeys order is down, right, left, up; left has no value
    assert entries == [("right", 0.9), ("down", 0.5), ("up", 0.5), ("left", None)]


def test_encode_matrix_and_c_division():
    F = H.fc()
    enc, total = F._encode_matrix([[2, 0, 0, 0], [0, 4, 0, 0], [0, 0, 0, 0], [0, 0, 0, 32768]])
    assert enc == (1 << 60) | (2 << 40) | (15 << 0)
    assert total == 2 + 4 + 32768


@pytest.mark.parametrize("key", ["L3_32_float32", "diag9_64_float32"])
def test_reader_fixture_ordering_rules(key):
    """Every golden answer is in the reference's order: numeric values
    descending, then the unmoved directions."""
    for entry in H.reader_cases()[key]:
        vals = [v for _, v in entry["result"] if isinstance(v, float)]
        assert vals == sorted(vals, reverse=True)
        kinds = [isinstance(v, float) for _, v in entry["result"]]
        assert kinds == sorted(kinds, reverse=True)


def test_capacity_failure_raises_the_reference_message(monkeypatch):
    """A build that cannot fit even after regrowth and the streamed fallback
    (EGTB_ERR_CAPACITY) raises the reference's "length multiplier" message, so
    BookBuilder's one resumed retry still applies; other errors keep theirs."""
    F = H.fc()
    N = H.pkg()._native
    bb = __import__("importlib").import_module("2048endgametablebase_b200.engine_core.BookBuilder")

    class FakeLib:
        def __init__(self, rc):
            self.rc = rc

        def egtb_build(self, *args):
            return self.rc

        def egtb_last_error(self, buf, n):
            return 0

    case = H.cases()["L3_32_float32"]
    spec, o = H.spec_options(case, "/nonexistent/unused_")
    for rc, retry in ((-5, True), (-7, False)):
        monkeypatch.setattr(N, "lib", lambda rc=rc: FakeLib(rc))
        with pytest.raises(N.NativeError) as ei:
            F.run_pattern_build(H.seeds(case), spec, o)
        assert ei.value.code == rc
        assert bb._should_retry_build_resume(ei.value) is retry
        if retry:
            assert str(ei.value) == F.CAPACITY_MESSAGE


# The catalog entries of the reference's variant patterns (its
# patterns_config.json format), parsed as the build reads them.
_VARIANT_ENTRIES = {
    "2x4": {"category": "variant", "valid pattern": [], "target pos": "0xffffffff0000", "canonical mode": "min24",
            "seed boards": ["0xffff00000000ffff"], "extra steps": 48},
    "3x3": {"category": "variant", "valid pattern": [], "target pos": "0xfff0fff0fff00000", "canonical mode": "min33",
            "seed boards": ["0x000f000f000fffff"], "extra steps": 60},
    "3x4": {"category": "variant", "valid pattern": [], "target pos": "0xffffffffffff0000", "canonical mode": "min34",
            "seed boards": ["0x000000000000ffff"], "extra steps": 60},
}


@pytest.mark.parametrize("key", H.VARIANT_CASES)
def test_variant_catalog_entries_match_golden_cases(key):
    """Masks, success shifts, symmetry mode, seeds, steps and docheck of the
    variant patterns as the golden cases (made by the reference) hold them."""
    P = patterns()
    case = H.cases()[key]
    meta = P.parse_entry(case["pattern"], _VARIANT_ENTRIES[case["pattern"]])
    assert [hex(int(m)) for m in meta["pattern_masks"]] == case["masks"]
    assert list(meta["success_shifts"]) == case["shifts"]
    assert P.SYMM_MODES[meta["canonical_mode"]] == case["symm_mode"]
    assert [hex(int(s)) for s in meta["seed_boards"]] == case["seeds"]
    assert -meta["nums_adjust"] == case["tile_sum0"]
    steps, docheck = P.steps_and_docheck(case["tile_sum0"], case["target"], meta["extra_steps"])
    assert (steps, docheck) == (case["steps"], case["docheck_step"])
    assert case.get("is_variant") is True


def test_compare_books_counts_missing_keys_as_zero():
    import importlib
    P = importlib.import_module("2048endgametablebase_b200.precision")

    def book(pairs, dt):
        rec = np.dtype([("key", "<u8"), ("rate", dt)])
        return np.array(pairs, dtype=rec).tobytes()

    a = [book([(1, 0.5), (3, 0.25)], "<f4"), book([], "<f4")]
    b = [book([(1, 0.5), (2, 0.125), (3, 0.2500001)], "<f8"), book([(7, 1e-9)], "<f8")]
    r = P.compare_books(a, "float32", b, "float64")
    assert r["entries"] == 4 and r["only_in_b"] == 2 and r["only_in_a"] == 0
    assert r["max_abs_err"] == 0.125 and r["layer"] == 0 and r["board"] == 2
    assert r["rate_a"] == 0.0 and r["rate_b"] == 0.125
