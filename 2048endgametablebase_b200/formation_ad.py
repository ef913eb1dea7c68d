"""Masked-board primitives of the advanced algorithm on the GPU.

The reference's advanced (masked-board) build holds every tile of 64 and up
as a 0xF ("32k") nibble. These are its board-level primitives, batched over
numpy arrays of uint64 boards and run by the library's CUDA kernels, with the
reference's names (namespace FormationAD):

  m_move_all_dir                 native_core/src/BoardMoverAD.cpp:171-178
  mask_board                     native_core/src/BoardMaskerAD.cpp:112-121
  tile_sum_and_32k_count(2, 4)   native_core/src/BoardMaskerAD.cpp:123-144,
                                 :169-190, :219-257
  validate                       native_core/src/BoardMaskerAD.cpp:409-443
  unmask_board                   native_core/src/BoardMaskerAD.cpp:445-512
  build_mask_param               native_core/src/BoardMaskerAD.cpp:102-110

There is no CPU fallback: without the library or a device every call raises.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _native as N

_ERR_CAPACITY = -5  # EGTB_ERR_CAPACITY: the output did not fit; counts and total are filled


@dataclass
class AdvancedMaskParam:
    """AdvancedMaskParam (native_core/include/FormationRuntime.h:98-104)."""
    small_tile_sum_limit: int = 96
    target: int = 0
    pos_fixed_32k_mask: int = 0
    num_free_32k: int = 0
    num_fixed_32k: int = 0

    def to_c(self) -> N.AdParamC:
        return N.AdParamC(int(self.pos_fixed_32k_mask), int(self.small_tile_sum_limit), int(self.target),
                          int(self.num_free_32k), int(self.num_fixed_32k))


@dataclass
class AdvancedPatternSpec:
    """The fields of AdvancedPatternSpec (FormationRuntime.h:88-96) the masker reads."""
    num_free_32k: int = 0
    fixed_32k_shifts: list = field(default_factory=list)
    small_tile_sum_limit: int = 96
    target: int = 0


def fixed_32k_mask(fixed_shifts) -> int:
    """0xF at every fixed 32k cell (BoardMaskerAD.cpp:94-100)."""
    return sum(0xF << int(s) for s in fixed_shifts) & 0xFFFFFFFFFFFFFFFF


def build_mask_param(spec: AdvancedPatternSpec) -> AdvancedMaskParam:
    return AdvancedMaskParam(small_tile_sum_limit=int(spec.small_tile_sum_limit), target=int(spec.target),
                             pos_fixed_32k_mask=fixed_32k_mask(spec.fixed_32k_shifts),
                             num_free_32k=int(spec.num_free_32k), num_fixed_32k=len(spec.fixed_32k_shifts))


def _boards(boards) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(boards, dtype=np.uint64).reshape(-1))


def m_move_all_dir(boards, device: int = 0):
    """(moves, flags): moves[i] = left, right, up, down of boards[i] under the
    masked rule; flags[i] = mask_new_tile of each (a merge made a 32k tile)."""
    b = _boards(boards)
    moves = np.zeros((len(b), 4), dtype=np.uint64)
    flags = np.zeros((len(b), 4), dtype=np.uint8)
    N.check(N.lib().egtb_ad_move_all_dir(device, b.ctypes.data, len(b), moves.ctypes.data, flags.ctypes.data))
    return moves, flags.astype(bool)


def mask_board(boards, threshold: int = 6, device: int = 0) -> np.ndarray:
    b = _boards(boards)
    out = np.zeros(len(b), dtype=np.uint64)
    N.check(N.lib().egtb_ad_mask_board(device, b.ctypes.data, len(b), int(threshold), out.ctypes.data))
    return out


def _tile_stats(boards, param: AdvancedMaskParam, kind: int, device: int) -> dict:
    b = _boards(boards)
    out = (N.AdTileCountC * max(1, len(b)))()
    c = param.to_c()
    N.check(N.lib().egtb_ad_tile_stats(device, b.ctypes.data, len(b), ctypes.byref(c), kind, ctypes.addressof(out)))
    a = np.frombuffer(out, dtype=np.dtype([(f, np.uint64 if f == "pos_bitmap" else
                                            (np.int32 if f == "count_32k" else np.uint32))
                                           for f, _ in N.AdTileCountC._fields_]), count=len(b))
    return {f: a[f].copy() for f in a.dtype.names}


def tile_sum_and_32k_count(boards, param: AdvancedMaskParam, device: int = 0) -> dict:
    """total_sum, count_32k, pos_bitmap with only 0xF counted as 32k."""
    d = _tile_stats(boards, param, 1, device)
    return {k: d[k] for k in ("total_sum", "count_32k", "pos_bitmap")}


def tile_sum_and_32k_count2(boards, param: AdvancedMaskParam, device: int = 0) -> dict:
    """total_sum, count_32k, pos_bitmap with every tile of 64 and up counted as 32k."""
    d = _tile_stats(boards, param, 2, device)
    return {k: d[k] for k in ("total_sum", "count_32k", "pos_bitmap")}


def tile_sum_and_32k_count4(boards, param: AdvancedMaskParam, device: int = 0) -> dict:
    """count2's fields plus pos_rank, merged_tile_found, merged_tile, is_success."""
    d = _tile_stats(boards, param, 4, device)
    d["is_success"] = d["is_success"].astype(bool)
    return d


def validate(boards, original_sums, param: AdvancedMaskParam, device: int = 0) -> np.ndarray:
    """Per board: can this masked board stand for a real board of the pattern
    whose tile sum is original_sums[i]?"""
    b = _boards(boards)
    s = np.ascontiguousarray(np.asarray(original_sums, dtype=np.uint32).reshape(-1))
    if len(s) != len(b):
        raise ValueError("one original sum per board")
    out = np.zeros(len(b), dtype=np.uint8)
    c = param.to_c()
    N.check(N.lib().egtb_ad_validate(device, b.ctypes.data, len(b), s.ctypes.data, ctypes.byref(c), out.ctypes.data))
    return out.astype(bool)


def unmask_board(boards, original_sums, param: AdvancedMaskParam, device: int = 0):
    """(counts, unmasked): every board each masked board stands for, in the
    reference's order; unmasked holds all boards' results one after another
    (counts[i] of them for boards[i])."""
    b = _boards(boards)
    s = np.ascontiguousarray(np.asarray(original_sums, dtype=np.uint32).reshape(-1))
    if len(s) != len(b):
        raise ValueError("one original sum per board")
    counts = np.zeros(len(b), dtype=np.uint32)
    c = param.to_c()
    total = ctypes.c_uint64(0)
    cap = 16 * max(1, len(b))
    out = np.zeros(cap, dtype=np.uint64)
    rc = N.lib().egtb_ad_unmask(device, b.ctypes.data, len(b), s.ctypes.data, ctypes.byref(c), counts.ctypes.data,
                                out.ctypes.data, cap, ctypes.byref(total))
    if rc == _ERR_CAPACITY and total.value > cap:
        out = np.zeros(int(total.value), dtype=np.uint64)
        rc = N.lib().egtb_ad_unmask(device, b.ctypes.data, len(b), s.ctypes.data, ctypes.byref(c),
                                    counts.ctypes.data, out.ctypes.data, len(out), ctypes.byref(total))
    N.check(rc)
    return counts, out[:int(total.value)]


def row_tables():
    """(moves, flags) of the masked row rule, computed on the host: moves[r] =
    left xor | right xor << 16, flags[r] = the left merge made a 32k tile."""
    moves = np.zeros(65536, dtype=np.uint32)
    flags = np.zeros(65536, dtype=np.uint8)
    N.check(N.lib().egtb_ad_row_tables(moves.ctypes.data, flags.ctypes.data))
    return moves, flags


def tiles_combinations():
    """(lens, vals): init_masker's tiles-combination table, entry a + 256 b."""
    lens = np.zeros(2560, dtype=np.uint8)
    vals = np.zeros((2560, 16), dtype=np.uint8)
    N.check(N.lib().egtb_ad_tiles_combinations(lens.ctypes.data, vals.ctypes.data))
    return lens, vals
