"""The CPU oracle (oracle/egtb_oracle.c) against the reference's own outputs
(tests/golden, produced by tests/golden/make_golden.py from the reference
compiled out of its sources). This pins the oracle the GPU tests check against."""
import numpy as np
import pytest

import helpers as H
import oracle as O


def test_row_tables_match_reference():
    p = H.prims()
    left, right = O.row_tables()
    assert np.array_equal(left, p["row_left"])
    assert np.array_equal(right, p["row_right"])


def test_moves_match_reference():
    p = H.prims()
    assert np.array_equal(O.move_all_dir(p["boards"]), p["moves"])


def test_variant_row_tables_and_moves_match_reference():
    """The variant boards' wall-merge mover (VBoardMover)."""
    p = H.prims()
    left, right = O.row_tables(variant=True)
    assert np.array_equal(left, p["row_left_variant"])
    assert np.array_equal(right, p["row_right_variant"])
    assert np.array_equal(O.move_all_dir(p["boards"], variant=True), p["moves_variant"])


@pytest.mark.parametrize("mode", range(7))
def test_canonical_match_reference(mode):
    p = H.prims()
    assert np.array_equal(O.canonical(p["boards"], mode), p[f"canonical_{mode}"])


@pytest.mark.parametrize("idx", range(8))
def test_symmetries_match_reference(idx):
    p = H.prims()
    b = p["boards"][:2000]
    got = np.array([O.apply_sym(int(x), idx) for x in b], dtype=np.uint64)
    assert np.array_equal(got, p[f"sym_{idx}"][:2000])


def _build(case):
    spec = O.Spec([int(m, 16) for m in case["masks"]], case["shifts"], case["symm_mode"],
                  case.get("is_variant", False))
    return O.Build(H.seeds(case), spec, case["target"], case["steps"], case["docheck_step"])


@pytest.mark.parametrize("key", H.SMALL_CPU_CASES + H.VARIANT_CPU_CASES)
def test_oracle_raw_layers_and_books(key):
    case = H.cases()[key]
    b = _build(case)
    steps = case["steps"]
    for t in range(steps - 2):
        layer = b.layer(t)
        assert len(layer) == case["raw_len"][t], (key, t)
        assert H.sha_bytes(layer.astype("<u8").tobytes()) == case["raw_sha256"][t], (key, t)
    assert [len(b.layer(steps - 2)), len(b.layer(steps - 1))] >= [0, 0]
    b.solve(case["dtype"], case["spawn_rate4"])
    for t in range(steps):
        book = b.book(t, case["dtype"])
        assert H.sha_bytes(book) == case["book_sha256"][t], (key, t)


def test_free5_book_data_fixture():
    """One complete build kept as data: the oracle's books byte for byte."""
    case = H.cases()["free5_32_float32"]
    data = np.load(H.os.path.join(H.GOLDEN, "free5_32.npz"))
    b = _build(case)
    b.solve("float32", 0.1)
    for t in range(case["steps"]):
        assert b.book(t, "float32") == data[f"book_{t}"].tobytes(), t


POST_PASS_CASES = [k for k, v in H.cases().items() if v.get("size_class") in ("deletion", "optimal")]


@pytest.mark.parametrize("key", POST_PASS_CASES)
def test_oracle_post_pass_books(key):
    """The oracle's restated post-passes (deletion threshold, optimal branch)
    give the reference's books byte for byte."""
    case = H.cases()[key]
    b = _build(case)
    b.solve(case["dtype"], case["spawn_rate4"])
    books = b.books(case["dtype"], case.get("deletion_threshold", 0.0), case.get("optimal_branch_only", False),
                    case.get("is_variant", False))
    for t in range(case["steps"]):
        assert H.sha_bytes(books[t]) == case["book_sha256"][t], (key, t)


READER_CPU_CASES = sorted(k for k in H.reader_cases() if k in set(H.SMALL_CPU_CASES + H.VARIANT_CPU_CASES))


@pytest.mark.parametrize("key", READER_CPU_CASES)
def test_oracle_reader_answers(key, tmp_path):
    """The oracle's move_on_dic over the oracle's own books gives the reference
    reader's answers, position after position (the reader's last operation
    carries over, as in the reference)."""
    case = H.cases()[key]
    b = _build(case)
    b.solve(case["dtype"], case["spawn_rate4"])
    books = b.books(case["dtype"])
    name = case["pattern_full"]
    for t, data in enumerate(books):
        (tmp_path / f"{name}_{t}.book").write_bytes(data)
    reader = O.Reader([int(m, 16) for m in case["masks"]], case["symm_mode"], case.get("is_variant", False))
    for i, entry in enumerate(H.reader_cases()[key]):
        res, dt = reader.move_on_dic(entry["board"], [(str(tmp_path), case["dtype"])], name, -case["tile_sum0"])
        assert [[k, v] for k, v in res] == entry["result"], (key, i, entry["board"])
        assert dt == entry["dtype"], (key, i)


# ------------------------------------------------- compressed books (.z) ----

COMPRESSED_CASES = sorted(k for k, v in H.cases().items() if v.get("size_class") == "compressed")


def test_compression_rule_selects_the_reference_layers():
    """Layers 3 and up whose book passes 2 MiB are the ones the reference
    compressed (CompressionBridge.cpp:41-59)."""
    import ztrie
    for key in COMPRESSED_CASES:
        case = H.cases()[key]
        rec = 12 if case["dtype"] in ("uint32", "float32") else 16
        for t, layer in enumerate(case["layers"]):
            name = f"{case['pattern_full']}_{t}.book"
            assert ztrie.wants_compression(name, case["book_len"][t] * rec) == (layer["kind"] == "z"), (key, t)


@pytest.fixture(scope="module")
def oracle_442():
    case = H.cases()["442_512_float32"]
    b = _build(case)
    return b


@pytest.mark.parametrize("dtype", ["float32", "uint32"])
def test_oracle_compressed_layers_equal_the_reference(oracle_442, dtype):
    """The oracle's restatement of the trie + xz format, on the oracle's own
    442-512 books, writes the reference's .z files byte for byte (smallest,
    middle and last compressed layers)."""
    import ztrie
    case = H.cases()[f"442_512_{dtype}_compressed"]
    oracle_442.solve(dtype, 0.1)
    zl = [t for t, layer in enumerate(case["layers"]) if layer["kind"] == "z"]
    for t in (zl[0], zl[len(zl) // 2], zl[-1]):
        book = oracle_442.book(t, dtype)
        assert H.sha_bytes(book) == case["book_sha256"][t]
        stem = f"{case['pattern_full']}_{t}."
        files = ztrie.compress_book(book, dtype, stem)
        for sfx, want in case["layers"][t]["sha256"].items():
            assert H.sha_bytes(files[stem + sfx]) == want, (dtype, t, sfx)


def test_oracle_trie_search_finds_every_entry(oracle_442):
    """The restated reader search over a compressed layer returns each book
    entry's rate, and a miss for boards that are not in the layer."""
    import ztrie
    oracle_442.solve("float32", 0.1)
    case = H.cases()["442_512_float32_compressed"]
    t = [t for t, layer in enumerate(case["layers"]) if layer["kind"] == "z"][0]
    book = oracle_442.book(t, "float32")
    stem = f"{case['pattern_full']}_{t}."
    layer = ztrie.TrieLayer(ztrie.compress_book(book, "float32", stem), stem, "float32")
    rec = np.frombuffer(book, dtype=[("key", "<u8"), ("rate", "<f4")])
    for i in range(0, len(rec), 97):
        assert layer.search(int(rec["key"][i])) == rec["rate"][i].item(), i
    assert layer.search(int(rec["key"][0]) - 1) is None


def test_oracle_reader_on_the_compressed_table(oracle_442, tmp_path):
    """The oracle's reader over the oracle's own 442-512 table laid out as the
    reference's compressed build left it (171 layers as .z directories, the
    rest as .book files) gives the reference reader's answers on that build."""
    import ztrie
    key = "442_512_float32_compressed"
    case = H.cases()[key]
    oracle_442.solve("float32", 0.1)
    name = case["pattern_full"]
    answers = H.reader_cases()[key]
    # the layers the positions read (a position's layer is its tile sum's)
    wanted = {(sum(v for row in e["board"] for v in row) - case["tile_sum0"]) // 2 for e in answers}
    for t, layer in enumerate(case["layers"]):
        if t not in wanted:
            continue
        book = oracle_442.book(t, "float32")
        if layer["kind"] == "z":
            zdir = tmp_path / f"{name}_{t}.z"
            zdir.mkdir()
            for fname, data in ztrie.compress_book(book, "float32", f"{name}_{t}.").items():
                (zdir / fname).write_bytes(data)
        else:
            (tmp_path / f"{name}_{t}.book").write_bytes(book)
    reader = O.Reader([int(m, 16) for m in case["masks"]], case["symm_mode"])
    for i, entry in enumerate(answers):
        res, dt = reader.move_on_dic(entry["board"], [(str(tmp_path), case["dtype"])], name, -case["tile_sum0"])
        assert [[k, v] for k, v in res] == entry["result"], (i, entry["board"])
        assert dt == entry["dtype"]
