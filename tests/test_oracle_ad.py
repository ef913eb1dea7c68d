"""The oracle's plain-C restatement of the advanced algorithm's masked-board
primitives (oracle/egtb_oracle.c) against the reference's own outputs
(tests/golden/ad_prims.npz): the checker pinned, on CPU."""
import numpy as np
import pytest

import helpers as H
import oracle as O


def _param(i):
    limit, target, fixed, nfree = H.AD_PARAMS[i]
    return O.ad_param(limit, target, fixed, nfree)


def test_masked_moves_and_flags():
    g = H.ad_prims()
    moves, flags = O.ad_move_all_dir(g["mover_boards"])
    assert np.array_equal(moves, g["mover_moves"])
    assert np.array_equal(flags, g["mover_flags"])


@pytest.mark.parametrize("threshold", [6, 5, 9])
def test_mask_board(threshold):
    g = H.ad_prims()
    assert np.array_equal(O.ad_mask_board(g["boards"][:1000], threshold), g[f"mask_{threshold}"][:1000])


@pytest.mark.parametrize("i", range(len(H.AD_PARAMS)))
@pytest.mark.parametrize("kind", [1, 2, 4])
def test_tile_stats(i, kind):
    g = H.ad_prims()
    assert np.array_equal(O.ad_tile_stats(g["boards"][:1000], _param(i), kind), g[f"stats_{i}_{kind}"][:1000])


@pytest.mark.parametrize("i", range(len(H.AD_PARAMS)))
def test_validate(i):
    g = H.ad_prims()
    got = O.ad_validate(g[f"validate_{i}_boards"][:2000], g[f"validate_{i}_sums"][:2000], _param(i))
    assert np.array_equal(got, g[f"validate_{i}"][:2000])


@pytest.mark.parametrize("i", range(len(H.AD_PARAMS)))
def test_unmask(i):
    g = H.ad_prims()
    counts, boards = O.ad_unmask(g[f"unmask_{i}_boards"], g[f"unmask_{i}_sums"], _param(i))
    assert np.array_equal(counts, g[f"unmask_{i}_counts"])
    assert np.array_equal(boards, g[f"unmask_{i}"])
