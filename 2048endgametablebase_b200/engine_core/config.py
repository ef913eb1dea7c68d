"""Configuration consulted by the build and reader mirrors.

The reference keeps these keys in SingletonConfig().config (Config.py:383-493,
defaults :469-493); only the keys the classic build/lookup path reads are
kept, with the reference's defaults.
"""
from __future__ import annotations

import threading

DEFAULTS = {
    "4_spawn_rate": 0.1,
    "success_rate_dtype": "uint32",
    "deletion_threshold": 0.0,
    "compress": False,
    "optimal_branch_only": False,
    "compress_temp_files": False,
    "advanced_algo": False,
    "chunked_solve": False,
    "direct_io": True,
    "direct_io_queue_depth": 16,
    "direct_io_chunk_mib": 8,
    "filepath_map": {},
}


class SingletonConfig:
    """Process-wide configuration dict (SingletonConfig, Config.py:383)."""

    _instance = None
    _lock = threading.Lock()

    def __new__(cls):
        with cls._lock:
            if cls._instance is None:
                inst = super().__new__(cls)
                inst.config = {k: (dict(v) if isinstance(v, dict) else v) for k, v in DEFAULTS.items()}
                cls._instance = inst
        return cls._instance
