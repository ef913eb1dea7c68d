"""Compressed books (compress=True): the reference turns every book of layer 3
and up that passes 2 MiB into a trie + xz-block directory <name>_<t>.z
(TrieCompression.cpp:326-354). A GPU build with compress=True must leave
exactly the reference's files: the same layers as .book, the same four files
in every .z directory, byte for byte. The reader's answers on such a table
are checked in test_gpu_reader.py (golden answers of the reference's reader
on its own compressed table)."""
import os
import shutil

import pytest

import helpers as H

pytestmark = pytest.mark.gpu

COMPRESSED = sorted(k for k, v in H.cases().items() if v.get("size_class") == "compressed")


@pytest.mark.parametrize("key", COMPRESSED)
def test_compressed_build_files_equal_the_reference(key, tmp_root):
    case = H.cases()[key]
    F = H.fc()
    d = H.fresh(os.path.join(tmp_root, "zbuild_" + key) + "/")
    name = case["pattern_full"]
    spec, o = H.spec_options(case, d + name + "_")
    assert o.compress
    F.run_pattern_build(H.seeds(case), spec, o)
    for t, layer in enumerate(case["layers"]):
        book, zdir = d + f"{name}_{t}.book", d + f"{name}_{t}.z"
        if layer["kind"] == "z":
            assert not os.path.exists(book) and os.path.isdir(zdir), t
            assert sorted(os.listdir(zdir)) == sorted(f"{name}_{t}." + s for s in ("i", "ii", "s", "z")), t
            for sfx, want in layer["sha256"].items():
                assert H.sha(os.path.join(zdir, f"{name}_{t}.{sfx}")) == want, (t, sfx)
        else:
            assert not os.path.exists(zdir), t
            assert H.sha(book) == layer["sha256"], t
    shutil.rmtree(d, ignore_errors=True)


def test_compressed_streamed_solve_equals_the_reference(tmp_root, monkeypatch):
    """The same through the layer-by-layer solve (generate + solve, the
    streamed path): compression runs once the books are final."""
    monkeypatch.setenv("EGTB_STREAM_LAYERS", "1")
    key = COMPRESSED[0]
    case = H.cases()[key]
    F = H.fc()
    d = H.fresh(os.path.join(tmp_root, "zsolve_" + key) + "/")
    name = case["pattern_full"]
    spec, o = H.spec_options(case, d + name + "_")
    started, l0, l1 = F.run_pattern_generate(H.seeds(case), spec, o)
    F.run_pattern_solve(l0, l1, spec, o)
    for t, layer in enumerate(case["layers"]):
        if layer["kind"] == "z":
            for sfx, want in layer["sha256"].items():
                assert H.sha(d + f"{name}_{t}.z/{name}_{t}.{sfx}") == want, (t, sfx)
        else:
            assert H.sha(d + f"{name}_{t}.book") == layer["sha256"], t
    shutil.rmtree(d, ignore_errors=True)
