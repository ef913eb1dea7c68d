"""Shared helpers of the test suite."""
from __future__ import annotations

import hashlib
import importlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pkg():
    return importlib.import_module("2048endgametablebase_b200")


def serving():
    return importlib.import_module("2048endgametablebase_b200.serving")


def fc():
    return importlib.import_module("2048endgametablebase_b200.native_core.formation_core")


def cases() -> dict:
    return json.load(open(os.path.join(GOLDEN, "cases.json")))


def reader_cases() -> dict:
    return json.load(open(os.path.join(GOLDEN, "reader.json")))


def prims():
    return np.load(os.path.join(GOLDEN, "prims.npz"))


def ad_prims():
    return np.load(os.path.join(GOLDEN, "ad_prims.npz"))


def ad():
    return importlib.import_module("2048endgametablebase_b200.formation_ad")


# the masked-board parameter sets of tests/golden/make_golden.py (AD_PARAMS):
# (small_tile_sum_limit, target, fixed 32k shifts, num_free_32k)
AD_PARAMS = [(96, 10, [], 0), (96, 11, [60, 56], 2), (160, 9, [0, 4, 8], 1), (32, 12, [12], 3)]


def ad_param(i: int):
    limit, target, fixed, nfree = AD_PARAMS[i]
    A = ad()
    return A.build_mask_param(A.AdvancedPatternSpec(num_free_32k=nfree, fixed_32k_shifts=fixed,
                                                    small_tile_sum_limit=limit, target=target))


def sha(path: str) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 24), b""):
            h.update(chunk)
    return h.hexdigest()


def sha_bytes(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def spec_options(case: dict, pathname: str):
    F = fc()
    spec = F.PatternSpec()
    spec.name = case["pattern"]
    spec.pattern_masks = [int(m, 16) for m in case["masks"]]
    spec.success_shifts = list(case["shifts"])
    spec.symm_mode = int(case["symm_mode"])
    o = F.RunOptions()
    o.target = case["target"]
    o.steps = case["steps"]
    o.docheck_step = case["docheck_step"]
    o.pathname = pathname
    o.success_rate_dtype = case["dtype"]
    o.spawn_rate4 = case["spawn_rate4"]
    o.is_variant = bool(case.get("is_variant", False))
    o.compress = bool(case.get("compress", False))
    return spec, o


def seeds(case: dict) -> np.ndarray:
    return np.array([int(s, 16) for s in case["seeds"]], dtype=np.uint64)


def fresh(path: str) -> str:
    import shutil
    shutil.rmtree(path, ignore_errors=True)
    os.makedirs(path, exist_ok=True)
    return path


SMALL_CPU_CASES = [k for k, v in cases().items() if v.get("size_class") == "small" and sum(v["raw_len"]) < 3_000_000]
SMALL_CASES = [k for k, v in cases().items() if v.get("size_class") == "small"]
FULL_CASES = [k for k, v in cases().items() if v.get("size_class") == "full"]
# variant boards (wall-merge mover, min24/min33/min34 symmetry); the CPU oracle
# takes the ones it finishes in seconds
VARIANT_CASES = [k for k, v in cases().items() if v.get("size_class") == "variant"]
VARIANT_CPU_CASES = [k for k in VARIANT_CASES if sum(cases()[k]["raw_len"]) < 3_000_000]
