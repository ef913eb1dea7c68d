"""Streamed build: layers leave the device as each one closes (sorted there,
copied through pinned host buffers into their raw layer files) and the
solve streams them back, so a table needs device memory for a window of
layers instead of all of them. EGTB_STREAM_LAYERS=1 forces this path (it is
taken by itself when a table outgrows device memory); every file must equal
the reference's."""
import os
import shutil

import pytest

import helpers as H

pytestmark = pytest.mark.gpu


@pytest.fixture
def streamed(monkeypatch):
    monkeypatch.setenv("EGTB_STREAM_LAYERS", "1")


@pytest.mark.parametrize("key", H.SMALL_CASES)
def test_streamed_generate_raw_layers_bit_exact(key, tmp_root, streamed):
    case = H.cases()[key]
    F = H.fc()
    d = H.fresh(os.path.join(tmp_root, "sgen_" + key) + "/")
    spec, o = H.spec_options(case, d + case["pattern_full"] + "_")
    started, l0, l1 = F.run_pattern_generate(H.seeds(case), spec, o)
    assert started
    steps = case["steps"]
    name = case["pattern_full"]
    for t in range(steps - 2):
        p = d + f"{name}_{t}"
        assert os.path.getsize(p) // 8 == case["raw_len"][t], (key, t)
        assert H.sha(p) == case["raw_sha256"][t], (key, t)
    for t in (steps - 2, steps - 1):
        assert H.sha(d + f"{name}_{t}.book") == case["book_sha256"][t], (key, t)


@pytest.mark.parametrize("key", ["L3_32_float32", "diag9_64_float32", "horiz8_64_float32", "free6_32_float32",
                                 "t_64_uint32"] + list(H.FULL_CASES))
def test_streamed_build_books_bit_exact(key, tmp_root, streamed):
    case = H.cases()[key]
    F = H.fc()
    d = H.fresh(os.path.join(tmp_root, "sbuild_" + key) + "/")
    spec, o = H.spec_options(case, d + case["pattern_full"] + "_")
    F.run_pattern_build(H.seeds(case), spec, o)
    name = case["pattern_full"]
    for t in range(case["steps"]):
        assert H.sha(d + f"{name}_{t}.book") == case["book_sha256"][t], (key, t)
    assert not any(os.path.exists(d + f"{name}_{t}") for t in range(case["steps"]))
    shutil.rmtree(d, ignore_errors=True)


def test_streamed_diagonal_1024_prefix_matches_128(tmp_root, streamed):
    """The 13-cell diagonal table at target 1024, first 62 steps, streamed:
    layers 0..56 come before any success check of either target, so they
    equal the 4432-128 table's raw layers."""
    case = dict(H.cases()["4432_128_float32"])
    F = H.fc()
    pats = __import__("importlib").import_module("2048endgametablebase_b200.patterns")
    steps_full, docheck = pats.steps_and_docheck(case["tile_sum0"], 10, 48)
    assert docheck == 504
    case.update(target=10, steps=62, docheck_step=docheck)
    d = H.fresh(os.path.join(tmp_root, "s4432_1024") + "/")
    spec, o = H.spec_options(case, d + "4432_1024_")
    started, _, _ = F.run_pattern_generate(H.seeds(case), spec, o)
    assert started
    ref = H.cases()["4432_128_float32"]
    for t in range(57):
        p = d + f"4432_1024_{t}"
        assert os.path.getsize(p) // 8 == ref["raw_len"][t], t
        assert H.sha(p) == ref["raw_sha256"][t], t
    # past the 128 table's first success check its parents with a 128 tile are
    # skipped, so each later 1024 layer holds the 128 layer (and more)
    for t in range(57, 60):
        assert os.path.getsize(d + f"4432_1024_{t}") // 8 >= ref["raw_len"][t], t
    shutil.rmtree(d, ignore_errors=True)


def test_build_falls_back_to_streamed_layers_when_the_table_does_not_fit(tmp_root):
    """A build whose layer arena cannot be allocated is built with streamed
    layers by itself (generate + solve through files), books unchanged. The
    allocation limit stands in for a smaller device; it is read once per
    process, so the build runs in a child process."""
    import json
    import subprocess
    import sys
    key = "L3_256_float32"
    case = H.cases()[key]
    d = H.fresh(os.path.join(tmp_root, "fallback_" + key) + "/")
    code = f"""
import json, sys
sys.path.insert(0, {H.ROOT!r}); sys.path.insert(0, {os.path.join(H.ROOT, "tests")!r})
import helpers as H
import ctypes
case = H.cases()[{key!r}]
F = H.fc()
N = H.pkg()._native
spec, o = H.spec_options(case, {d!r} + case["pattern_full"] + "_")
# without files there is no streamed path: under the limit the table must not fit
seeds = H.seeds(case)
c_spec, c_opt = spec.to_c(), o.to_c(write_files=False)
rc = N.lib().egtb_build(seeds.ctypes.data, len(seeds), ctypes.byref(c_spec), ctypes.byref(c_opt), None)
assert rc == -5, rc
F.run_pattern_build(seeds, spec, o)
print(json.dumps(F.last_build_stats()))
"""
    env = dict(os.environ, EGTB_MAX_ALLOC_BYTES=str(512 << 20))
    env.pop("EGTB_STREAM_LAYERS", None)
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stderr[-2000:]
    name = case["pattern_full"]
    for t in range(case["steps"]):
        assert H.sha(d + f"{name}_{t}.book") == case["book_sha256"][t], t
    assert not any(os.path.exists(d + f"{name}_{t}") for t in range(case["steps"]))
    shutil.rmtree(d, ignore_errors=True)
