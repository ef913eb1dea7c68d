"""BookBuilder mirror (reference engine_core/BookBuilder.py) for the classic
path: resolves a pattern name into PatternSpec / RunOptions and runs the
build on the GPU through the drop-in formation_core.

Same entry points and behaviour as the reference's module: start_build(pattern,
target, pathname) (:264-317), save_config_to_txt (:131-146), the seeds of
free patterns (generate_free_inits, :149-182) and one resumed retry after the
"length multiplier" capacity failure (:237-261). The build itself is planned
here as a BuildPlan (catalog entry -> PatternSpec, RunOptions, seeds).
"""
from __future__ import annotations

import logging
import os
from dataclasses import dataclass

import numpy as np

from .. import patterns
from ..native_core import formation_core
from .config import SingletonConfig

logger = logging.getLogger("debug_logger")

# RunOptions fields taken from the configuration: field -> (config key,
# default, conversion). The reference's BookBuilder fills the same fields
# from SingletonConfig with these defaults (engine_core/BookBuilder.py:44-73).
_CONFIG_OPTIONS = {
    "success_rate_dtype": ("success_rate_dtype", "uint32", str),
    "deletion_threshold": ("deletion_threshold", 0.0, float),
    "compress": ("compress", False, bool),
    "compress_temp_files": ("compress_temp_files", False, bool),
    "optimal_branch_only": ("optimal_branch_only", False, bool),
    "chunked_solve": ("chunked_solve", False, bool),
    "direct_io": ("direct_io", True, bool),
    "direct_io_queue_depth": ("direct_io_queue_depth", 16, int),
    "direct_io_chunk_mib": ("direct_io_chunk_mib", 8, int),
}

# config.txt keys, in the order the reference writes them (BookBuilder.py:131-146)
_CONFIG_TXT_KEYS = ("compress", "optimal_branch_only", "compress_temp_files", "advanced_algo", "direct_io",
                    "direct_io_queue_depth", "direct_io_chunk_mib", "deletion_threshold", "4_spawn_rate",
                    "success_rate_dtype")

# what run_pattern_build raises when the table outgrows its buffers; the
# reference retries such a build once, resuming from its files
_CAPACITY_MESSAGE = formation_core.CAPACITY_MESSAGE
_CAPACITY_PREFIX = "length multiplier "


def _symm_mode_value(name: str) -> int:
    """Integer symmetry mode of a catalog "canonical mode" name (identity if unknown)."""
    return int(patterns.SYMM_MODES.get(name, int(formation_core.SymmMode.Identity)))


@dataclass
class BuildPlan:
    """Everything one classic build needs, resolved from the catalog."""
    pattern: str
    target: int
    pathname: str
    seeds: np.ndarray
    steps: int
    docheck_step: int
    is_free: bool
    is_variant: bool
    spawn_rate4: float

    def spec(self):
        meta = patterns.pattern_catalog[self.pattern]
        s = formation_core.PatternSpec()
        s.name = self.pattern
        s.pattern_masks = [int(m) for m in meta.get("pattern_masks", ())]
        s.success_shifts = [int(x) for x in meta.get("success_shifts", ())]
        s.symm_mode = _symm_mode_value(meta.get("canonical_mode", "identity"))
        return s

    def options(self):
        config = SingletonConfig().config
        o = formation_core.RunOptions()
        o.target, o.steps, o.docheck_step = int(self.target), int(self.steps), int(self.docheck_step)
        o.pathname = str(self.pathname)
        o.is_free, o.is_variant = bool(self.is_free), bool(self.is_variant)
        o.spawn_rate4 = float(self.spawn_rate4)
        for field_name, (key, default, conv) in _CONFIG_OPTIONS.items():
            setattr(o, field_name, conv(config.get(key, default)))
        o.num_threads = max(4, min(32, os.cpu_count() or 2))
        return o

    def run(self) -> None:
        formation_core.run_pattern_build(np.asarray(self.seeds, dtype=np.uint64), self.spec(), self.options())


def _steps_and_docheck(tile_sum: int, target: int, extra_steps: int):
    return patterns.steps_and_docheck(tile_sum, target, extra_steps)


def save_config_to_txt(output_path: str) -> None:
    """config.txt beside the books: one "key: value" line per build setting."""
    config = SingletonConfig().config
    with open(output_path, "w", encoding="utf-8") as f:
        f.writelines(f"{k}: {config.get(k, '?')}\n" for k in _CONFIG_TXT_KEYS)


def _should_retry_build_resume(exc: Exception) -> bool:
    """True for the capacity failure that a resumed second attempt can fix."""
    text = str(exc).strip()
    return bool(text) and (text == _CAPACITY_MESSAGE or text.startswith(_CAPACITY_PREFIX))


def _build_with_one_resume(label: str, build) -> None:
    """Run build(); after a capacity failure run it once more (it resumes from
    the layer files already written). Any other failure, or a second one,
    propagates."""
    for attempt in (1, 2):
        try:
            build()
            return
        except Exception as exc:  # noqa: BLE001
            if attempt == 2 or not _should_retry_build_resume(exc):
                raise
            logger.warning("%s interrupted (%s); re-entering build once.", label, exc)


def _free_pattern_seeds(seeds: np.ndarray, tile_sum: int) -> np.ndarray:
    """A free pattern's start layer: generated (generate_free_inits) when its
    extra tiles are 2s that fit the free cells, else its catalog seeds."""
    first = int(seeds[0])
    walls = sum((first >> (4 * k)) & 0xF == 0xF for k in range(16))
    extra = tile_sum - 32768 * walls
    return generate_free_inits(walls, extra // 2) if extra <= (15 - walls) * 2 else seeds


def _counts_as_free(pattern: str, tile_sum: int) -> bool:
    """A catalog pattern whose masks pin fewer than four cells in common
    (and whose start sum is small) is built with is_free set."""
    masks = patterns.pattern_catalog[pattern]["pattern_masks"]
    if not masks:
        return tile_sum < 180000
    common = 0xFFFFFFFFFFFFFFFF
    for m in masks:
        common &= int(m)
    return len(patterns.find_f_nibble_positions(common)) < 4 and tile_sum < 180000


def plan_build(pattern: str, target: int, pathname: str) -> BuildPlan:
    """Resolve a catalog pattern and target into a BuildPlan."""
    meta = patterns.pattern_catalog.get(pattern)
    if meta is None:
        raise KeyError(f"Unknown pattern: {pattern}")
    seeds = np.asarray(meta.get("seed_boards", ()), dtype=np.uint64)
    if seeds.size == 0:
        raise ValueError(f"Pattern {pattern} has no seed boards")
    tile_sum = -int(meta.get("nums_adjust", 0))
    steps, docheck = _steps_and_docheck(tile_sum, target, int(meta.get("extra_steps", 36)))
    free = pattern.startswith("free")
    return BuildPlan(pattern, int(target), pathname,
                     _free_pattern_seeds(seeds, tile_sum) if free else seeds, steps, docheck,
                     True if free else _counts_as_free(pattern, tile_sum),
                     pattern in patterns.category_info.get("variant", []),
                     float(SingletonConfig().config["4_spawn_rate"]))


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
    """start_build (reference engine_core/BookBuilder.py:264-317), classic
    algorithm: write config.txt, then build the table through the drop-in
    formation_core, resuming once after a capacity failure."""
    if SingletonConfig().config.get("advanced_algo", False):
        raise RuntimeError("the advanced (masked-board) algorithm is not built")
    plan = plan_build(pattern, target, pathname)
    save_config_to_txt(pathname + "config.txt")
    _build_with_one_resume(f"Classic build {pattern}_{2 ** int(target)}", plan.run)
    return True
