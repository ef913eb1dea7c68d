"""Calculator mirror (reference engine_core/Calculator.py:80-324): board
symmetries and canonical forms, evaluated by libegtb_gpu's batched device
primitives. Every function takes one board or an array of boards."""
from __future__ import annotations

import os

import numpy as np

from .. import _native as N


def _dev() -> int:
    return int(os.environ.get("EGTB_DEVICE", "0"))


def _batch(boards):
    a = np.atleast_1d(np.asarray(boards, dtype=np.uint64))
    return np.ascontiguousarray(a), np.ndim(boards) == 0


def _sym(boards, idx: int):
    a, scalar = _batch(boards)
    out = np.zeros_like(a)
    N.check(N.lib().egtb_apply_sym(_dev(), a.ctypes.data, len(a), int(idx), out.ctypes.data))
    return np.uint64(out[0]) if scalar else out


def _canon(boards, mode: int):
    a, scalar = _batch(boards)
    out = np.zeros_like(a)
    N.check(N.lib().egtb_canonical(_dev(), a.ctypes.data, len(a), int(mode), out.ctypes.data))
    return np.uint64(out[0]) if scalar else out


def ReverseLR(board):
    return _sym(board, 1)


def ReverseUD(board):
    return _sym(board, 2)


def ReverseUL(board):
    return _sym(board, 3)


def ReverseUR(board):
    return _sym(board, 4)


def Rotate180(board):
    return _sym(board, 5)


def RotateL(board):
    return _sym(board, 6)


def RotateR(board):
    return _sym(board, 7)


def canonical_identity(board):
    return _canon(board, 0)


def canonical_full(board):
    return _canon(board, 1)


def canonical_diagonal(board):
    return _canon(board, 2)


def canonical_horizontal(board):
    return _canon(board, 3)


def canonical_min33(board):
    """Minimum over the eight symmetries of the 3x3 board (Calculator.py:315-317)."""
    return _canon(board, 4)


def canonical_min24(board):
    """Minimum over the mirrors and half turn of the 2x4 board (Calculator.py:319-321)."""
    return _canon(board, 5)


def canonical_min34(board):
    """Minimum over the symmetries of the 3x4 board (Calculator.py:323-325)."""
    return _canon(board, 6)


def move_all_dir(boards):
    """{left, right, up, down} of every board (CommonMover.h:136-139)."""
    a, scalar = _batch(boards)
    out = np.zeros((len(a), 4), dtype=np.uint64)
    N.check(N.lib().egtb_move_all_dir(_dev(), a.ctypes.data, len(a), out.ctypes.data))
    return tuple(np.uint64(x) for x in out[0]) if scalar else out


def move_all_dir_variant(boards):
    """move_all_dir of the variant boards' mover: 0xF cells are walls
    (VBoardMover, native_core/include/VBoardMover.h)."""
    a, scalar = _batch(boards)
    out = np.zeros((len(a), 4), dtype=np.uint64)
    N.check(N.lib().egtb_move_all_dir_variant(_dev(), a.ctypes.data, len(a), out.ctypes.data))
    return tuple(np.uint64(x) for x in out[0]) if scalar else out


def is_success(board_encoded, target_stacked, mask=np.uint64(0xFFFFFFFFFFFFFFFF)):
    """SWAR zero-nibble test (Calculator.is_success, engine_core/Calculator.py:75-81)."""
    board_encoded = np.uint64(board_encoded) & np.uint64(mask)
    diff = board_encoded ^ np.uint64(target_stacked)
    mask_7 = np.uint64(0x7777777777777777)
    result = ~(((diff & mask_7) + mask_7) | diff | mask_7)
    return bool(result != 0)
