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


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_canonical(mode):
    p = H.prims()
    assert np.array_equal(_call("egtb_canonical", p["boards"], mode), p[f"canonical_{mode}"])


@pytest.mark.parametrize("idx", range(8))
def test_symmetries(idx):
    p = H.prims()
    assert np.array_equal(_call("egtb_apply_sym", p["boards"], idx), p[f"sym_{idx}"])


def test_unsupported_mode_is_an_error():
    N = H.pkg()._native
    b = np.zeros(4, dtype=np.uint64)
    out = np.zeros(4, dtype=np.uint64)
    rc = N.lib().egtb_canonical(0, b.ctypes.data, 4, 5, out.ctypes.data)
    assert rc == -7 and "symmetry" in N.last_error()
