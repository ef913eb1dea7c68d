"""B200-native classic endgame-tablebase build and book lookup.

Layout:
  csrc/          CUDA kernels (sm_100a) and the C ABI of libegtb_gpu.so
  _native.py     ctypes binding of include/egtb_gpu.h
  native_core/   drop-in `formation_core` module (the reference's nanobind surface)
  engine_core/   BookBuilder / BookReader / Calculator mirrors of the reference's Python API
  patterns.py    pattern catalog loader (the reference's patterns_config.json format)
  serving.py     continuous-batching lookup server over device-resident books

The package directory name starts with a digit, so import it with
importlib.import_module("2048endgametablebase_b200").
"""
from ._native import LIB_PATH, NativeError, device_count, lib  # noqa: F401

__version__ = "0.1.0"
