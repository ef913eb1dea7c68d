"""Board primitives on the device (libegtb_gpu egtb_move_all_dir /
egtb_canonical / egtb_apply_sym) against the reference's own primitives."""
import ctypes

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def _call(name, boards, *args, width=1):
    N = H.pkg()._native
    b = np.ascontiguousarray(boards, dtype=np.uint64)
    out = np.zeros(len(b) * width, dtype=np.uint64)
    fn = getattr(N.lib(), name)
    if args:
        N.check(fn(0, b.ctypes.data, len(b), *args, out.ctypes.data))
    else:
        N.check(fn(0, b.ctypes.data, len(b), out.ctypes.data))
    return out.reshape(len(b), width) if width > 1 else out


def test_device_present():
    assert H.pkg().device_count() >= 1


def test_moves():
    p = H.prims()
    assert np.array_equal(_call("egtb_move_all_dir", p["boards"], width=4), p["moves"])


def test_variant_moves():
    """The variant boards' wall-merge mover (VBoardMover)."""
    p = H.prims()
    assert np.array_equal(_call("egtb_move_all_dir_variant", p["boards"], width=4), p["moves_variant"])


@pytest.mark.parametrize("mode", range(7))
def test_canonical(mode):
    p = H.prims()
    assert np.array_equal(_call("egtb_canonical", p["boards"], mode), p[f"canonical_{mode}"])


@pytest.mark.parametrize("idx", range(8))
def test_symmetries(idx):
    p = H.prims()
    assert np.array_equal(_call("egtb_apply_sym", p["boards"], idx), p[f"sym_{idx}"])


def test_unknown_mode_is_an_error():
    N = H.pkg()._native
    b = np.zeros(4, dtype=np.uint64)
    out = np.zeros(4, dtype=np.uint64)
    rc = N.lib().egtb_canonical(0, b.ctypes.data, 4, 7, out.ctypes.data)
    assert rc == -1 and "symmetry" in N.last_error()
