"""ClassicBookReader.move_on_dic on the GPU (books resident in device memory)
against the reference reader's answers on the same books (tests/golden/reader.json).
The books are built by the GPU path, which the build tests pin to the
reference's files."""
import os

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def built(tmp_root):
    F = H.fc()
    out = {}
    for key in H.reader_cases():
        case = H.cases()[key]
        d = H.fresh(os.path.join(tmp_root, "reader_" + key) + "/")
        spec, o = H.spec_options(case, d + case["pattern_full"] + "_")
        F.run_pattern_build(H.seeds(case), spec, o)
        out[key] = d
    return out


@pytest.mark.parametrize("key", sorted(H.reader_cases()))
def test_move_on_dic_matches_reference(key, built):
    F = H.fc()
    case = H.cases()[key]
    spec, _ = H.spec_options(case, "")
    reader = F.ClassicBookReader(spec, bool(case.get("is_variant", False)))
    path_list = [(built[key].rstrip("/"), case["dtype"])]
    for i, entry in enumerate(H.reader_cases()[key]):
        res, dt = reader.move_on_dic(entry["board"], path_list, case["pattern_full"], -case["tile_sum0"])
        got = [[k, v] for k, v in res.items()]
        assert got == entry["result"], (key, i, entry["board"], got, entry["result"])
        assert dt == entry["dtype"]


def test_missing_layer_and_negative_layer(built):
    F = H.fc()
    key = "L3_32_float32"
    case = H.cases()[key]
    spec, _ = H.spec_options(case, "")
    reader = F.ClassicBookReader(spec, False)
    path_list = [(built[key].rstrip("/"), case["dtype"])]
    # a board whose layer index is beyond the table: no file, blank answers
    big = [[2048, 1024, 0, 0], [0, 0, 0, 0], [0, 32768, 32768, 32768], [0, 32768, 32768, 32768]]
    res, dt = reader.move_on_dic(big, path_list, case["pattern_full"], -case["tile_sum0"])
    assert res == {"down": "", "right": "", "left": "", "up": ""} and dt == ""
    res, dt = reader.move_on_dic([[0] * 4] * 4, path_list, case["pattern_full"], -case["tile_sum0"])
    assert res == {"down": "", "right": "", "left": "", "up": ""}
    res, dt = reader.move_on_dic(big, [], case["pattern_full"], -case["tile_sum0"])
    assert res == {"?": "?"}


def test_find_classic_value(built):
    F = H.fc()
    key = "L3_32_float32"
    case = H.cases()[key]
    d = built[key]
    name = case["pattern_full"]
    rec = np.dtype([("board", "<u8"), ("rate", "<f4")])
    data = np.fromfile(d + f"{name}_10.book", dtype=rec)
    for r in data[:: max(1, len(data) // 50)]:
        v = F.find_classic_value(d, f"{name}_10.book", int(r["board"]), "float32")
        assert v == float(r["rate"])
    assert F.find_classic_value(d, f"{name}_10.book", 12345, "float32") == 0.0
    assert F.find_classic_value(d, "nope.book", 12345, "float32") is None
