"""Seed boards of free patterns (BookBuilder.generate_free_inits, reference
engine_core/BookBuilder.py:149-182) from the device primitives, against the
oracle's restatement on its own primitives (pinned to the reference's by
test_oracle_golden), and start_build of a free pattern."""
import importlib
import json
import os

import numpy as np
import pytest

import helpers as H
import oracle as O

pytestmark = pytest.mark.gpu


def _bb():
    return importlib.import_module("2048endgametablebase_b200.engine_core.BookBuilder")


@pytest.mark.parametrize("t32ks,t2s", [(0, 2), (1, 3), (2, 4), (4, 5), (6, 2)])
def test_free_inits_match_oracle(t32ks, t2s):
    got = _bb().generate_free_inits(t32ks, t2s)
    want = O.free_inits(t32ks, t2s)
    assert got.dtype == np.uint64 and np.array_equal(got, want), (t32ks, t2s, len(got), len(want))


def test_start_build_of_a_free_pattern(tmp_root):
    """A free pattern whose seed is 11 walls and two 2s: start_build generates
    the seeds and builds; the books equal a build from the oracle's seeds."""
    walls = sum(0xF << (4 * k) for k in range(5, 16))
    cfg = {"free5w": {"category": "free", "valid pattern": [], "target pos": "0xffffffffffffffff",
                      "canonical mode": "full", "seed boards": [hex(walls | 1 | (1 << 4))], "extra steps": 16}}
    path = os.path.join(tmp_root, "free_patterns.json")
    json.dump(cfg, open(path, "w"))
    pats = importlib.import_module("2048endgametablebase_b200.patterns")
    pats.use_catalog(path)
    bb = _bb()
    try:
        d = H.fresh(os.path.join(tmp_root, "free5w_start") + "/")
        assert bb.start_build("free5w", 6, d + "free5w_64_")
        seeds = O.free_inits(11, 2)
        meta = pats.pattern_catalog["free5w"]
        steps, docheck = pats.steps_and_docheck(-int(meta["nums_adjust"]), 6, 16)
        F = H.fc()
        spec = F.PatternSpec()
        spec.name = "free5w"
        spec.pattern_masks = []
        spec.success_shifts = [4 * k for k in range(16)]
        spec.symm_mode = 1
        o = F.RunOptions()
        o.target, o.steps, o.docheck_step = 6, steps, docheck
        d2 = H.fresh(os.path.join(tmp_root, "free5w_ref") + "/")
        o.pathname = d2 + "free5w_64_"
        o.success_rate_dtype = bb.SingletonConfig().config.get("success_rate_dtype", "uint32")
        o.spawn_rate4 = float(bb.SingletonConfig().config["4_spawn_rate"])
        F.run_pattern_build(seeds, spec, o)
        n = 0
        for t in range(steps):
            a, b = d + f"free5w_64_{t}.book", d2 + f"free5w_64_{t}.book"
            assert os.path.exists(a) == os.path.exists(b), t
            if os.path.exists(a):
                assert H.sha(a) == H.sha(b), t
                n += 1
        assert n > 0
    finally:
        pats.use_catalog(os.environ.get("EGTB_PATTERNS_CONFIG") or None)
