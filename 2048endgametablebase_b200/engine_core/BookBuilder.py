"""BookBuilder mirror (reference engine_core/BookBuilder.py) for the classic
path: resolves a pattern name into PatternSpec / RunOptions and runs the
build on the GPU through the drop-in formation_core.

Same entry points and semantics as the reference: start_build(pattern,
target, pathname) (:264-317), _steps_and_docheck (:124-128),
save_config_to_txt (:131-146), the one resume-retry on the
"length multiplier" message (:237-261).
"""
from __future__ import annotations

import logging
import os

import numpy as np

from .. import patterns
from ..native_core import formation_core
from .config import SingletonConfig

logger = logging.getLogger("debug_logger")

_SYMM_MODE_BY_NAME = {name: formation_core.SymmMode(v) for name, v in patterns.SYMM_MODES.items()}


def _symm_mode_value(name: str) -> int:
    return int(_SYMM_MODE_BY_NAME.get(name, formation_core.SymmMode.Identity).value)


def _build_native_run_options(target, steps, pathname, docheck_step, is_free, is_variant, spawn_rate4):
    """_build_native_run_options, engine_core/BookBuilder.py:44-73"""
    config = SingletonConfig().config
    options = formation_core.RunOptions()
    options.target = int(target)
    options.steps = int(steps)
    options.docheck_step = int(docheck_step)
    options.pathname = str(pathname)
    options.is_free = bool(is_free)
    options.is_variant = bool(is_variant)
    options.spawn_rate4 = float(spawn_rate4)
    options.success_rate_dtype = str(config.get("success_rate_dtype", "uint32"))
    options.deletion_threshold = float(config.get("deletion_threshold", 0.0))
    options.compress = bool(config.get("compress", False))
    options.compress_temp_files = bool(config.get("compress_temp_files", False))
    options.optimal_branch_only = bool(config.get("optimal_branch_only", False))
    options.chunked_solve = bool(config.get("chunked_solve", False))
    options.direct_io = bool(config.get("direct_io", True))
    options.direct_io_queue_depth = int(config.get("direct_io_queue_depth", 16))
    options.direct_io_chunk_mib = int(config.get("direct_io_chunk_mib", 8))
    options.num_threads = int(max(4, min(32, os.cpu_count() or 2)))
    return options


def _build_native_pattern_spec(pattern: str):
    """_build_native_pattern_spec, engine_core/BookBuilder.py:76-88"""
    meta = patterns.pattern_catalog.get(pattern)
    if meta is None:
        raise KeyError(f"Unknown pattern: {pattern}")
    spec = formation_core.PatternSpec()
    spec.name = pattern
    spec.pattern_masks = list(meta.get("pattern_masks", ()))
    spec.success_shifts = list(meta.get("success_shifts", ()))
    spec.symm_mode = _symm_mode_value(meta.get("canonical_mode", "identity"))
    return spec


def _resolve_build_meta(pattern: str):
    """_resolve_build_meta, engine_core/BookBuilder.py:111-121"""
    meta = patterns.pattern_catalog.get(pattern)
    if meta is None:
        raise KeyError(f"Unknown pattern: {pattern}")
    tile_sum = -int(meta.get("nums_adjust", 0))
    seed_boards = np.asarray(meta.get("seed_boards", ()), dtype=np.uint64)
    if seed_boards.size == 0:
        raise ValueError(f"Pattern {pattern} has no seed boards")
    extra_steps = int(meta.get("extra_steps", 36))
    return meta, tile_sum, seed_boards, extra_steps


_steps_and_docheck = patterns.steps_and_docheck


def save_config_to_txt(output_path: str) -> None:
    """save_config_to_txt, engine_core/BookBuilder.py:131-146"""
    keys = ["compress", "optimal_branch_only", "compress_temp_files", "advanced_algo", "direct_io",
            "direct_io_queue_depth", "direct_io_chunk_mib", "deletion_threshold", "4_spawn_rate",
            "success_rate_dtype"]
    with open(output_path, "w", encoding="utf-8") as f:
        for key in keys:
            f.write(f"{key}: {str(SingletonConfig().config.get(key, '?'))}\n")


def _run_classic_build(pattern, arr_init, target, steps, pathname, docheck_step, is_free, is_variant, spawn_rate4):
    spec = _build_native_pattern_spec(pattern)
    options = _build_native_run_options(target, steps, pathname, docheck_step, is_free, is_variant, spawn_rate4)
    formation_core.run_pattern_build(np.asarray(arr_init, dtype=np.uint64), spec, options)


def _should_retry_build_resume(exc: Exception) -> bool:
    message = str(exc).strip()
    if not message:
        return False
    if message == "The length multiplier is not big enough. Please restart.":
        return True
    return message.startswith("length multiplier ")


def _run_with_single_resume_retry(build_label: str, build_fn) -> None:
    retried = False
    while True:
        try:
            build_fn()
            return
        except Exception as exc:  # noqa: BLE001
            if retried or not _should_retry_build_resume(exc):
                raise
            retried = True
            logger.warning("%s interrupted (%s); re-entering build once.", build_label, exc)


def generate_free_inits(t32ks: int, t2s: int) -> np.ndarray:
    """Seed boards of a free pattern (generate_free_inits,
    engine_core/BookBuilder.py:149-182): every board with t32ks 32768 tiles
    and t2s 2-tiles (combinations in lexicographic order, at most 10^6),
    sorted and unique; then, board by board in that order, its four moves
    (left, right, up, down) that are their own full-symmetry canonical form,
    stopping after the board at which at least (boards - 3) have been
    collected; the result sorted and unique. The moves and canonical forms
    are the device primitives (egtb_move_all_dir, egtb_canonical)."""
    from itertools import combinations

    from . import Calculator as C

    cap = 1_000_000
    boards = []
    for walls in combinations(range(16), t32ks):
        base = 0
        for p in walls:
            base |= 0xF << (4 * p)
        rest = [p for p in range(16) if p not in walls]
        for twos in combinations(rest, t2s):
            if len(boards) >= cap:
                break
            b = base
            for p in twos:
                b |= 1 << (4 * p)
            boards.append(b)
    gen = np.unique(np.array(boards, dtype=np.uint64))
    if len(gen) == 0:
        return gen
    moved = C.move_all_dir(gen)                                    # (n, 4)
    keep = moved == C.canonical_full(moved.reshape(-1)).reshape(moved.shape)
    # collected after each board, in order; stop at the first board that reaches n - 3
    cum = np.cumsum(keep.sum(axis=1))
    hit = np.nonzero(cum >= len(gen) - 3)[0]
    last = int(hit[0]) if len(hit) else len(gen) - 1
    return np.unique(moved[: last + 1][keep[: last + 1]])


def start_build(pattern: str, target: int, pathname: str) -> bool:
    """start_build, engine_core/BookBuilder.py:264-317 (classic algorithm)."""
    config = SingletonConfig().config
    if config.get("advanced_algo", False):
        raise RuntimeError("the advanced (masked-board) algorithm is not built")
    spawn_rate4 = float(config["4_spawn_rate"])
    _, tile_sum, seed_boards, extra_steps = _resolve_build_meta(pattern)
    steps, docheck_step = _steps_and_docheck(tile_sum, target, extra_steps)
    is_variant = pattern in patterns.category_info.get("variant", [])
    save_config_to_txt(pathname + "config.txt")
    if pattern.startswith("free"):
        # BookBuilder.py:275-283: the seeds of a free pattern are generated
        # when its extra tiles are all 2s that fit the free cells
        seed = int(seed_boards[0])
        num_32k = sum(1 for k in range(16) if (seed >> (4 * k)) & 0xF == 0xF)
        extra = tile_sum - 32768 * num_32k
        arr_init = generate_free_inits(num_32k, extra // 2) if extra <= (15 - num_32k) * 2 else seed_boards
        is_free = True
    else:
        arr_init = seed_boards
        masks = patterns.pattern_catalog[pattern]["pattern_masks"]
        inter = 0
        if masks:
            inter = ~0 & 0xFFFFFFFFFFFFFFFF
            for m in masks:
                inter &= int(m)
        fixed = patterns.find_f_nibble_positions(inter) if masks else []
        is_free = (len(fixed) < 4) and (tile_sum < 180000)
    _run_with_single_resume_retry(
        f"Classic build {pattern}_{2 ** target}",
        lambda: _run_classic_build(pattern, arr_init, target, steps, pathname, docheck_step, is_free, is_variant,
                                   spawn_rate4),
    )
    return True
