"""Driver for the reference's own classic-path code compiled into oracle/_ref/.

TEST INFRASTRUCTURE ONLY (checker and CPU baseline). Loads the reference's
formation_core module built by `make -C oracle ref` from the reference's
sources, with its AVX-512 sort plug-in bookgen_native.so preloaded so the
reference's dlopen("bookgen_native.so") (native_core/src/BookGeneratorUtils.cpp:86-90)
finds it.
"""
from __future__ import annotations

import ctypes
import glob
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
SYMM = {"identity": 0, "full": 1, "diagonal": 2, "horizontal": 3, "min33": 4, "min24": 5, "min34": 6}

_fc = None


def available() -> bool:
    return bool(glob.glob(os.path.join(REF_DIR, "formation_core*.so")))


# the reference's source tree (only in the container that compiles it)
REF_ROOT = os.environ.get("EGTB_REFERENCE_ROOT", "/root/reference")


def build(ref_root: str = REF_ROOT) -> bool:
    """Compile the reference's classic path from its sources (only where they exist)."""
    if not os.path.isdir(ref_root):
        return available()
    subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref", f"REF={ref_root}", f"PYTHON={sys.executable}"],
                   check=True)
    return available()


def module():
    global _fc
    if _fc is None:
        if not available():
            raise RuntimeError("reference formation_core is not built (make -C oracle ref)")
        bg = os.path.join(REF_DIR, "bookgen_native.so")
        if os.path.exists(bg):
            ctypes.CDLL(bg, mode=ctypes.RTLD_GLOBAL)
        if REF_DIR not in sys.path:
            sys.path.insert(0, REF_DIR)
        import formation_core  # noqa: E402  (the reference's module)

        _fc = formation_core
    return _fc


def tile_sum(board: int) -> int:
    """Sum of tile values of an encoded board (each 0xF cell counts 32768)."""
    s = 0
    for i in range(16):
        v = (int(board) >> (4 * i)) & 0xF
        if v:
            s += 1 << v
    return s


def pattern_params(entry: dict, target: int):
    """Masks, success shifts, symmetry, seeds, steps and docheck_step of a pattern,
    as the reference derives them (Config.py:179-282, engine_core/BookBuilder.py:111-128)."""
    masks = [int(m, 16) for m in entry.get("valid pattern", [])]
    tp = int(entry.get("target pos", "0xffffffffffffffff"), 16)
    shifts = [4 * i for i in range(16) if (tp >> (4 * i)) & 0xF == 0xF]
    seeds = [int(s, 16) for s in entry.get("seed boards", ["0xffffffff"])]
    s0 = tile_sum(seeds[0])
    seeds = np.array([s for s in seeds if tile_sum(s) == s0], dtype=np.uint64)
    extra = int(entry.get("extra steps", 36))
    t = 2 ** int(target)
    steps = int(t / 2 + extra)
    docheck = int(t / 2) - s0 % t // 2
    symm = SYMM.get(entry.get("canonical mode", "identity"), 0)
    return masks, shifts, symm, seeds, steps, docheck, s0


def make_spec_options(masks, shifts, symm, target, steps, docheck, pathname, dtype="float32", p4=0.1, threads=0,
                      deletion_threshold=0.0, optimal_branch_only=False, is_variant=False):
    fc = module()
    spec = fc.PatternSpec()
    spec.name = "oracle"
    spec.pattern_masks = [int(m) for m in masks]
    spec.success_shifts = [int(s) for s in shifts]
    spec.symm_mode = int(symm)
    o = fc.RunOptions()
    o.target = int(target)
    o.steps = int(steps)
    o.docheck_step = int(docheck)
    o.pathname = pathname
    o.success_rate_dtype = dtype
    o.spawn_rate4 = float(p4)
    o.direct_io = False
    o.num_threads = int(threads or os.cpu_count() or 4)
    o.deletion_threshold = float(deletion_threshold)
    o.optimal_branch_only = bool(optimal_branch_only)
    o.is_variant = bool(is_variant)
    return spec, o


def fresh_dir(path: str) -> str:
    shutil.rmtree(path, ignore_errors=True)
    os.makedirs(path, exist_ok=True)
    # the reference keeps a length-factor history next to the build directory
    lf = os.path.join(os.path.dirname(path.rstrip("/")), "length_factors_list.txt")
    if os.path.exists(lf):
        os.remove(lf)
    return path


def run_generate(seeds, spec, options):
    return module().run_pattern_generate(np.ascontiguousarray(seeds, dtype=np.uint64), spec, options)


def run_build(seeds, spec, options):
    module().run_pattern_build(np.ascontiguousarray(seeds, dtype=np.uint64), spec, options)
