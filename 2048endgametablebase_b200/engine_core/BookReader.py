"""BookReader mirror (reference engine_core/BookReader.py:39-161) for the
classic books, answered by the GPU reader of the drop-in formation_core."""
from __future__ import annotations

from typing import Any

import numpy as np

from .. import patterns
from ..native_core import formation_core
from .BookBuilder import _symm_mode_value
from .config import SingletonConfig


class BookReader:
    _native_readers: dict[str, Any] = {}

    @classmethod
    def _get_native_reader(cls, pattern: str):
        reader = cls._native_readers.get(pattern)
        if reader is not None:
            return reader
        meta = patterns.pattern_catalog.get(pattern)
        if meta is None:
            return None
        spec = formation_core.PatternSpec()
        spec.name = pattern
        spec.pattern_masks = list(meta.get("pattern_masks", ()))
        spec.success_shifts = list(meta.get("success_shifts", ()))
        spec.symm_mode = _symm_mode_value(meta.get("canonical_mode", "identity"))
        reader = formation_core.ClassicBookReader(spec, pattern in patterns.category_info.get("variant", []))
        cls._native_readers[pattern] = reader
        return reader

    @classmethod
    def move_on_dic(cls, board, pattern: str, target: str, pattern_full: str):
        del target
        meta = patterns.pattern_catalog.get(pattern)
        reader = cls._get_native_reader(pattern)
        spawn_rate4 = SingletonConfig().config["4_spawn_rate"]
        path_list = SingletonConfig().config["filepath_map"].get((pattern_full, spawn_rate4), [])
        if meta is None or reader is None:
            return {"?": "?"}, ""
        return reader.move_on_dic(np.asarray(board).tolist(), path_list, pattern_full, int(meta.get("nums_adjust", 0)))

    @classmethod
    def get_random_state(cls, path_list: list, pattern_full: str) -> np.uint64:
        pattern = pattern_full.split("_", 1)[0]
        reader = cls._get_native_reader(pattern)
        if reader is None:
            return np.uint64(0)
        return np.uint64(reader.get_random_state(path_list, pattern_full,
                                                 float(SingletonConfig().config["4_spawn_rate"])))


class BookReaderDispatcher:
    """Classic-only dispatcher (the advanced-algorithm reader is not built)."""

    _book_reader = BookReader

    def __init__(self):
        self.use_ad = False

    def move_on_dic(self, board, pattern: str, target: str, pattern_full: str):
        return self._book_reader.move_on_dic(board, pattern, target, pattern_full)

    def get_random_state(self, path_list: list, pattern_full: str):
        return self._book_reader.get_random_state(path_list, pattern_full)

    def dispatch(self, path_list: list, pattern: str, target) -> None:
        self.use_ad = False
