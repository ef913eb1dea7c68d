"""Error of a table's success rates against a float64 recomputation.

The reference keeps success rates in the run's dtype (`success_rate_dtype`,
native_core/src/BookSolver.cpp:784-821; records `SuccessEntry`,
native_core/include/FormationRuntime.h:191-199): every board's rate is summed
in double (recalculate_layer, BookSolver.cpp:413-470) and then cast to the
dtype, and the layers below read the cast values. A float32 table therefore
differs from the float64 table of the same pattern by the rounding of every
cast, carried down through the layers. This module builds a table in both
dtypes on the device and compares the books entry by entry; a key missing
from one book (its rate was exactly zero there) counts as rate 0.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N

__all__ = ["parse_book", "compare_books", "device_books", "rate_error_vs_fp64"]

_RATE = {"float32": np.float32, "float64": np.float64, "uint32": np.uint32, "uint64": np.uint64,
         "1-float32": np.float32, "1-float64": np.float64}


def parse_book(data: bytes, dtype: str) -> tuple[np.ndarray, np.ndarray]:
    """Keys (uint64, ascending) and rates (float64) of one .book layer: packed
    little-endian {u64 board; T rate} records."""
    rt = np.dtype(_RATE[dtype])
    rec = np.dtype([("key", "<u8"), ("rate", rt.newbyteorder("<"))], align=False)
    arr = np.frombuffer(data, dtype=rec)
    return arr["key"].copy(), arr["rate"].astype(np.float64)


def compare_books(books_a: list[bytes], dtype_a: str, books_b: list[bytes], dtype_b: str) -> dict:
    """Entry-by-entry |rate_a - rate_b| over the union of both tables' keys,
    layer by layer: max and mean, the layer and board of the max, and both
    rates there."""
    if len(books_a) != len(books_b):
        raise ValueError(f"tables have {len(books_a)} and {len(books_b)} layers")
    worst = {"max_abs_err": 0.0, "layer": -1, "board": 0, "rate_a": 0.0, "rate_b": 0.0}
    total, n, only_a, only_b = 0.0, 0, 0, 0
    for L, (a, b) in enumerate(zip(books_a, books_b)):
        ka, ra = parse_book(a, dtype_a)
        kb, rb = parse_book(b, dtype_b)
        keys = np.union1d(ka, kb)
        if keys.size == 0:
            continue
        va = np.zeros(keys.size)
        vb = np.zeros(keys.size)
        va[np.searchsorted(keys, ka)] = ra
        vb[np.searchsorted(keys, kb)] = rb
        d = np.abs(va - vb)
        i = int(np.argmax(d))
        if d[i] > worst["max_abs_err"]:
            worst = {"max_abs_err": float(d[i]), "layer": L, "board": int(keys[i]), "rate_a": float(va[i]),
                     "rate_b": float(vb[i])}
        total += float(d.sum())
        n += int(keys.size)
        only_a += int(keys.size - kb.size)
        only_b += int(keys.size - ka.size)
    worst.update(mean_abs_err=total / max(n, 1), entries=n, only_in_a=only_a, only_in_b=only_b)
    return worst


def device_books(seeds: np.ndarray, spec, options) -> list[bytes]:
    """Build one table on the device (no files; formation_core spec/options)
    and return every layer's .book bytes."""
    seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
    c_spec, c_opt = spec.to_c(), options.to_c(write_files=False)
    st = N.BuildStatsC()
    N.check(N.lib().egtb_build(seeds.ctypes.data, len(seeds), ctypes.byref(c_spec), ctypes.byref(c_opt),
                               ctypes.byref(st)))
    dev = int(options.device)
    out = []
    for L in range(int(options.steps)):
        n = ctypes.c_uint64(0)
        N.check(N.lib().egtb_book_layer_copy(dev, L, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(max(1, n.value))
        N.check(N.lib().egtb_book_layer_copy(dev, L, buf, n.value, ctypes.byref(n)))
        out.append(buf.raw[:n.value])
    return out


def rate_error_vs_fp64(seeds: np.ndarray, spec, options) -> dict:
    """Build the table with options.success_rate_dtype (float32 unless set)
    and again with float64, on the device, and compare every book entry."""
    import copy

    dt = options.success_rate_dtype or "float32"
    o32 = copy.copy(options)
    o32.success_rate_dtype = dt
    o64 = copy.copy(options)
    o64.success_rate_dtype = "float64"
    a = device_books(seeds, spec, o32)
    b = device_books(seeds, spec, o64)
    r = compare_books(a, dt, b, "float64")
    r["dtype"] = dt
    return r
