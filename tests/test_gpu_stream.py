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


def _hash_and_remove(path):
    h = H.sha(path)
    n = os.path.getsize(path) // 8
    os.remove(path)
    return n, h


@pytest.mark.slow
def test_streamed_diagonal_1024_prefix_bit_exact(tmp_root, streamed):
    """The 13-cell diagonal table at target 1024 (560 steps, ~1 TB of raw
    layers in all): its first 130 steps, streamed, every raw layer 0..127
    (3.8e9 boards) byte-identical to the reference's own generate of the same
    prefix (SHA-256 per layer). No success check happens before step 504, so
    these are the whole table's layers."""
    from concurrent.futures import ThreadPoolExecutor
    case = H.cases()["4432_1024_prefix130"]
    assert case["docheck_step"] == 504 and case["full_steps"] == 560
    F = H.fc()
    d = H.fresh(os.path.join(tmp_root, "s4432_1024") + "/")
    spec, o = H.spec_options(case, d + "4432_1024_")
    started, l0, l1 = F.run_pattern_generate(H.seeds(case), spec, o)
    assert started
    steps = case["steps"]
    with ThreadPoolExecutor(16) as ex:
        got = list(ex.map(_hash_and_remove, [d + f"4432_1024_{t}" for t in range(steps - 2)]))
    for t, (n, h) in enumerate(got):
        assert n == case["raw_len"][t], t
        assert h == case["raw_sha256"][t], t
    assert [l0.size, l1.size] == case["partial_len"]
    shutil.rmtree(d, ignore_errors=True)


@pytest.mark.slow
def test_streamed_diagonal_256_solve_is_self_consistent(tmp_root, streamed):
    """The 13-cell diagonal table at target 256 (176 steps, ~6e9 boards; the
    reference's build of it does not fit the machine that made the golden
    files): streamed generate, then streamed solve. Boards sampled from raw
    layers on both sides of the success check (docheck_step 120) must carry
    in their book (0 when absent) exactly the rate the CPU oracle recomputes
    from the GPU's own books of the next two layers, bit for bit."""
    import numpy as np
    import oracle as O
    base = H.cases()["4432_128_float32"]
    pats = __import__("importlib").import_module("2048endgametablebase_b200.patterns")
    steps, docheck = pats.steps_and_docheck(base["tile_sum0"], 8, 48)
    assert (steps, docheck) == (176, 120)
    case = dict(base, target=8, steps=steps, docheck_step=docheck)
    F = H.fc()
    d = H.fresh(os.path.join(tmp_root, "s4432_256") + "/")
    name = "4432_256"
    spec, o = H.spec_options(case, d + name + "_")
    started, l0, l1 = F.run_pattern_generate(H.seeds(case), spec, o)
    assert started
    rng = np.random.default_rng(256)
    layers = [30, 90, 119, 120, 121, 122, 150, 172, steps - 3]
    sample = {}
    for t in layers:
        raw = np.fromfile(d + f"{name}_{t}", dtype="<u8")
        assert raw.size and np.all(raw[1:] > raw[:-1]), t
        sample[t] = np.sort(rng.choice(raw, size=min(2048, raw.size), replace=False))
    F.run_pattern_solve(l0, l1, spec, o)
    assert not any(os.path.exists(d + f"{name}_{t}") for t in range(steps))
    rec = np.dtype([("key", "<u8"), ("rate", "<f4")])

    def book(t):
        b = np.fromfile(d + f"{name}_{t}.book", dtype=rec)
        return b["key"].copy(), b["rate"].copy()

    ospec = O.Spec([int(m, 16) for m in case["masks"]], case["shifts"], case["symm_mode"])
    checked = 0
    for t in layers:
        k0, r0 = book(t)
        k1, r1 = book(t + 1)
        k2, r2 = book(t + 2)
        want = O.solve_layer(sample[t], k1, r1, k2, r2, ospec, 8, t > docheck, "float32", 0.1)
        pos = np.minimum(np.searchsorted(k0, sample[t]), max(k0.size - 1, 0))
        hit = (k0.size > 0) & (k0[pos] == sample[t])
        got = np.where(hit, r0[pos] if k0.size else 0, np.float32(0))
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), t
        assert np.all(hit == (want > 0)), t
        checked += sample[t].size
    assert checked > 10_000
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
