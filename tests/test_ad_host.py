"""Host side of the advanced algorithm's masked-board primitives (no GPU):
the masked row rule and init_masker's tiles-combination table as the library
builds them, against the reference's own (tests/golden/ad_prims.npz, written
by the reference's BoardMoverAD / BoardMaskerAD). Where the reference's code
is built here (oracle/_ref), it must reproduce the fixture."""
import ctypes
import os

import numpy as np
import pytest

import helpers as H


def test_masked_row_rule_matches_reference():
    g = H.ad_prims()
    moves, flags = H.ad().row_tables()
    rows = np.arange(65536, dtype=np.uint32)
    assert np.array_equal((rows ^ (moves & 0xFFFF)).astype(np.uint16), g["row_left"])
    assert np.array_equal((rows ^ (moves >> 16)).astype(np.uint16), g["row_right"])
    assert np.array_equal(flags, g["row_flag"])
    # the rule's own corners: 32 + 32 -> 0xF with the flag, 0xF + 0xF stays
    assert (0x5500 ^ (moves[0x5500] & 0xFFFF)) == 0xF000 and flags[0x5500] == 1
    assert (0xFF00 ^ (moves[0xFF00] & 0xFFFF)) == 0xFF00 and flags[0xFF00] == 0
    assert (0x4400 ^ (moves[0x4400] & 0xFFFF)) == 0x5000 and flags[0x4400] == 0


def test_tiles_combinations_match_reference():
    g = H.ad_prims()
    lens, vals = H.ad().tiles_combinations()
    assert np.array_equal(lens, g["combo_lens"])
    for e in np.flatnonzero(lens):
        assert np.array_equal(vals[e, :lens[e]], g["combo_vals"][e, :lens[e]]), e
    # 64 x 3 = 192 as three 64s; one 1024 for 1024 / 1 tile
    assert list(vals[3 + 256 * 3, :lens[3 + 256 * 3]]) == [6, 6, 6]
    assert list(vals[16 + 256 * 1, :lens[16 + 256 * 1]]) == [10]


def test_mask_param_from_spec():
    p = H.ad_param(1)
    assert p.pos_fixed_32k_mask == (0xF << 60) | (0xF << 56)
    assert (p.num_fixed_32k, p.num_free_32k, p.target, p.small_tile_sum_limit) == (2, 2, 11, 96)


@pytest.mark.skipif(not os.path.exists(os.path.join(H.ROOT, "oracle", "_ref", "libref_ad_prims.so")),
                    reason="the reference's code is not built here (make -C oracle ref)")
def test_reference_reproduces_fixture():
    L = ctypes.CDLL(os.path.join(H.ROOT, "oracle", "_ref", "libref_ad_prims.so"))
    L.ref_ad_move_all_dir_batch.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]
    g = H.ad_prims()
    b = np.ascontiguousarray(g["mover_boards"])
    mv = np.zeros(len(b) * 4, dtype=np.uint64)
    fl = np.zeros(len(b) * 4, dtype=np.uint8)
    L.ref_ad_move_all_dir_batch(b.ctypes.data, len(b), mv.ctypes.data, fl.ctypes.data)
    assert np.array_equal(mv.reshape(-1, 4), g["mover_moves"])
    assert np.array_equal(fl.reshape(-1, 4), g["mover_flags"])
