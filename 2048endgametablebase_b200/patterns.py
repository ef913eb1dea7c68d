"""Pattern catalog in the reference's patterns_config.json format.

load_patterns_from_file restates Config.load_patterns_from_file
(Config.py:179-282) for the fields the classic build/lookup path reads:
  valid pattern  -> pattern_masks (hex strings, with or without 0x)
  target pos     -> success_shifts (every 0xF nibble, find_f_nibble_positions, Config.py:153-159)
  canonical mode -> canonical_mode
  seed boards    -> seed_boards, keeping only those with the first seed's tile sum (Config.py:241-248)
  extra steps    -> extra_steps (default 36)
and nums_adjust = -(seed tile sum), each 0xF cell counting 32768.

BUILTIN holds the catalog entries of the three tables this package
benchmarks (L3, 442, 4432), so the package runs without the reference's
configuration files; any reference patterns_config.json can be loaded instead.
"""
from __future__ import annotations

import json
import os
from typing import Any

import numpy as np

BUILTIN: dict[str, dict[str, Any]] = {
    # L-shaped 10-cell region, identity symmetry, success anywhere
    "L3": {"category": "10 space", "valid pattern": ["0xfff0fff"], "target pos": "0xffffffffffffffff",
           "canonical mode": "identity", "seed boards": ["0x100000001fff2fff", "0x000000012fff1fff"],
           "extra steps": 48},
    # bottom row + two cells of row 2 pinned, success at row 2 column 1
    "442": {"category": "10 space", "valid pattern": ["0xffffff"], "target pos": "0xf000000",
            "canonical mode": "identity", "seed boards": ["0x1000000021ffffff", "0x0000000112ffffff"],
            "extra steps": 48},
    # three corner cells pinned, diagonal symmetry, success at row 2 column 2
    "4432": {"category": "others", "valid pattern": ["0xf00ff"], "target pos": "0xf00000",
             "canonical mode": "diagonal", "seed boards": ["0x00001000121f21ff", "0x00010000121f21ff"],
             "extra steps": 48},
}

SYMM_MODES = {"identity": 0, "full": 1, "diagonal": 2, "horizontal": 3, "min33": 4, "min24": 5, "min34": 6}


def tile_sum(board: int) -> int:
    """Sum of the tile values of an encoded board; 0xF counts 32768."""
    s = 0
    for i in range(16):
        v = (int(board) >> (4 * i)) & 0xF
        if v:
            s += 1 << v
    return s


def find_f_nibble_positions(board: int) -> list[int]:
    return [4 * i for i in range(16) if (int(board) >> (4 * i)) & 0xF == 0xF]


def parse_entry(name: str, data: dict[str, Any]) -> dict[str, Any]:
    masks = tuple(int(m, 16) for m in data.get("valid pattern", []))
    shifts = tuple(find_f_nibble_positions(int(data.get("target pos", "0xffffffffffffffff"), 16)))
    seeds_raw = [int(s, 16) for s in data.get("seed boards", ["0xffffffff"])]
    s0 = tile_sum(seeds_raw[0])
    seeds = np.array([s for s in seeds_raw if tile_sum(s) == s0], dtype=np.uint64)
    return {
        "name": name,
        "category": data.get("category", "others"),
        "pattern_masks": masks,
        "success_shifts": shifts,
        "canonical_mode": data.get("canonical mode", "identity"),
        "seed_boards": seeds,
        "nums_adjust": -s0,
        "extra_steps": data.get("extra steps", 36),
    }


def load_patterns_from_file(file_path: str | None = None) -> tuple[dict, dict]:
    """(category_info, pattern_catalog) from a patterns_config.json, or the
    built-in entries when file_path is None."""
    raw = BUILTIN if file_path is None else json.load(open(file_path, encoding="utf-8"))
    category_info: dict[str, list[str]] = {}
    catalog: dict[str, dict[str, Any]] = {}
    for name, data in raw.items():
        category_info.setdefault(data.get("category", "others"), []).append(name)
        catalog[name] = parse_entry(name, data)
    if "others" in category_info:
        category_info["others"] = category_info.pop("others")
    return category_info, catalog


def steps_and_docheck(tile_sum0: int, target: int, extra_steps: int) -> tuple[int, int]:
    """_steps_and_docheck, engine_core/BookBuilder.py:124-128"""
    target_tile = int(2 ** target)
    steps = int(target_tile / 2 + extra_steps)
    docheck_step = int(target_tile / 2) - tile_sum0 % target_tile // 2
    return steps, docheck_step


_env_path = os.environ.get("EGTB_PATTERNS_CONFIG")
category_info, pattern_catalog = load_patterns_from_file(_env_path if _env_path else None)


def use_catalog(file_path: str | None) -> None:
    """Replace the active catalog (e.g. with the reference's patterns_config.json)."""
    global category_info, pattern_catalog
    ci, pc = load_patterns_from_file(file_path)
    category_info.clear()
    category_info.update(ci)
    pattern_catalog.clear()
    pattern_catalog.update(pc)
