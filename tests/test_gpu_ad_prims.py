"""The advanced algorithm's masked-board primitives on the device
(egtb_ad_*) against the reference's own BoardMoverAD / BoardMaskerAD outputs
(tests/golden/ad_prims.npz): bit-exact."""
import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def test_masked_moves_and_flags():
    g = H.ad_prims()
    moves, flags = H.ad().m_move_all_dir(g["mover_boards"])
    assert np.array_equal(moves, g["mover_moves"])
    assert np.array_equal(flags.astype(np.uint8), g["mover_flags"])
    assert 0.05 < flags.mean() < 0.95  # the workload does make 32k tiles


@pytest.mark.parametrize("threshold", [6, 5, 9])
def test_mask_board(threshold):
    g = H.ad_prims()
    assert np.array_equal(H.ad().mask_board(g["boards"], threshold), g[f"mask_{threshold}"])


@pytest.mark.parametrize("i", range(len(H.AD_PARAMS)))
@pytest.mark.parametrize("kind", [1, 2, 4])
def test_tile_stats(i, kind):
    g = H.ad_prims()
    A = H.ad()
    fn = {1: A.tile_sum_and_32k_count, 2: A.tile_sum_and_32k_count2, 4: A.tile_sum_and_32k_count4}[kind]
    got = fn(g["boards"], H.ad_param(i))
    want = g[f"stats_{i}_{kind}"]
    assert np.array_equal(got["total_sum"].astype(np.int64), want[:, 0])
    assert np.array_equal(got["count_32k"].astype(np.int64), want[:, 1])
    pos = (want[:, 2].astype(np.uint64) & np.uint64(0xFFFFFFFF)) | (want[:, 3].astype(np.uint64) << np.uint64(32))
    assert np.array_equal(got["pos_bitmap"], pos)
    if kind == 4:
        assert np.array_equal(got["pos_rank"].astype(np.int64), want[:, 4])
        assert np.array_equal(got["merged_tile_found"].astype(np.int64), want[:, 5])
        assert np.array_equal(got["merged_tile"].astype(np.int64), want[:, 6])
        assert np.array_equal(got["is_success"].astype(np.int64), want[:, 7])


@pytest.mark.parametrize("i", range(len(H.AD_PARAMS)))
def test_validate(i):
    g = H.ad_prims()
    got = H.ad().validate(g[f"validate_{i}_boards"], g[f"validate_{i}_sums"], H.ad_param(i))
    want = g[f"validate_{i}"].astype(bool)
    assert np.array_equal(got, want)
    assert 0 < want.mean() < 1  # both answers occur


def test_empty_and_bad_arguments():
    A = H.ad()
    m, f = A.m_move_all_dir(np.zeros(0, dtype=np.uint64))
    assert m.shape == (0, 4)
    with pytest.raises(Exception):
        A._tile_stats(np.zeros(4, dtype=np.uint64), H.ad_param(0), 3, 0)
    with pytest.raises(ValueError):
        A.validate(np.zeros(4, dtype=np.uint64), np.zeros(3, dtype=np.uint32), H.ad_param(0))


@pytest.mark.parametrize("i", range(len(H.AD_PARAMS)))
def test_unmask_board(i):
    """Every board a masked board stands for, in the reference's permutation order."""
    g = H.ad_prims()
    counts, boards = H.ad().unmask_board(g[f"unmask_{i}_boards"], g[f"unmask_{i}_sums"], H.ad_param(i))
    assert np.array_equal(counts, g[f"unmask_{i}_counts"])
    assert np.array_equal(boards, g[f"unmask_{i}"])
    assert counts.max() > 1 and (counts == 0).any()  # expansions and rejections both occur


def test_unmask_reports_capacity():
    """Too small an output: EGTB_ERR_CAPACITY with the counts and total filled."""
    import ctypes
    g = H.ad_prims()
    N = H.pkg()._native
    b = np.ascontiguousarray(g["unmask_1_boards"])
    s = np.ascontiguousarray(g["unmask_1_sums"])
    counts = np.zeros(len(b), dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint64)
    total = ctypes.c_uint64(0)
    c = H.ad_param(1).to_c()
    rc = N.lib().egtb_ad_unmask(0, b.ctypes.data, len(b), s.ctypes.data, ctypes.byref(c), counts.ctypes.data,
                                out.ctypes.data, 4, ctypes.byref(total))
    assert rc == -5 and total.value == g["unmask_1_counts"].sum()
    assert np.array_equal(counts, g["unmask_1_counts"])
