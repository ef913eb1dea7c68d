"""Bounded device waits. The layer sort's look-back waits on other blocks'
counts; with egtb_set_spin_limit(1) those waits give up after two polls, the
kernel records the timeout and returns (nothing spins on), the build reports
EGTB_ERR_TIMEOUT, and the next build on the same device is exact again."""
import ctypes

import pytest

import helpers as H

pytestmark = pytest.mark.gpu

EGTB_ERR_TIMEOUT = -6


def _device_build(case):
    N = H.pkg()._native
    spec, o = H.spec_options(case, "")
    seeds = H.seeds(case)
    c_spec, c_opt = spec.to_c(), o.to_c(write_files=False)
    st = N.BuildStatsC()
    rc = N.lib().egtb_build(seeds.ctypes.data, len(seeds), ctypes.byref(c_spec), ctypes.byref(c_opt),
                            ctypes.byref(st))
    return rc, st


def _book_digests(case):
    B = __import__("importlib").import_module("2048endgametablebase_b200.batch")
    return [H.sha_bytes(B.plain_book(L)) for L in range(case["steps"])]


def test_look_back_wait_gives_up_with_timeout_and_library_stays_usable():
    N = H.pkg()._native
    # 442-512 layers span up to 83 sort tiles, sorted by 296 concurrent blocks:
    # tiles look back on predecessors that have not published yet
    big = H.cases()["442_512_float32"]
    N.check(N.lib().egtb_set_spin_limit(1))
    try:
        rc, _ = _device_build(big)
        msg = N.last_error()
    finally:
        N.check(N.lib().egtb_set_spin_limit(0))
    assert rc == EGTB_ERR_TIMEOUT, (rc, msg)
    assert "bounded device wait" in msg
    # the same device builds exactly again, with the default limit
    small = H.cases()["L3_32_float32"]
    rc, _ = _device_build(small)
    assert rc == 0, N.last_error()
    assert _book_digests(small) == small["book_sha256"]
    rc, st = _device_build(big)
    assert rc == 0, N.last_error()
    assert st.raw_boards == sum(big["raw_len"])
    assert _book_digests(big) == big["book_sha256"]
