"""egtb_sort_unique_u64 (device sort + unique of caller-owned keys) against numpy."""
import ctypes

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def _sort_unique(keys: np.ndarray) -> np.ndarray:
    import torch
    N = H.pkg()._native
    n = len(keys)
    d_in = torch.from_numpy(keys.view(np.int64).copy()).cuda() if n else torch.zeros(1, dtype=torch.int64, device="cuda")
    d_out = torch.zeros(max(n, 1), dtype=torch.int64, device="cuda")
    d_cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    st = torch.cuda.current_stream()
    N.check(N.lib().egtb_sort_unique_u64(0, d_in.data_ptr(), n, d_out.data_ptr(), d_cnt.data_ptr(), st.cuda_stream))
    st.synchronize()
    m = int(d_cnt.item())
    return d_out[:m].cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("n", [0, 1, 2, 4095, 4096, 4097, 100_000, 1_000_003])
def test_random_keys_with_repeats(n):
    rng = np.random.default_rng(n)
    pool = rng.integers(0, 2 ** 63, size=max(1, n // 3), dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=max(1, n // 3), dtype=np.uint64)
    keys = rng.choice(pool, size=n) if n else np.zeros(0, dtype=np.uint64)
    assert np.array_equal(_sort_unique(keys), np.unique(keys))


def test_skewed_board_like_keys():
    """Few distinct high nibbles, the shape of real layers."""
    rng = np.random.default_rng(5)
    n = 3_000_000
    cells = rng.integers(0, 6, size=(n, 16)).astype(np.uint64)
    cells[:, :6] = 15
    cells[:, 12:] = np.where(rng.random((n, 4)) < 0.8, 0, cells[:, 12:])
    keys = np.zeros(n, dtype=np.uint64)
    for k in range(16):
        keys |= cells[:, k] << np.uint64(4 * k)
    assert np.array_equal(_sort_unique(keys), np.unique(keys))


def test_all_equal_and_extremes():
    keys = np.array([2 ** 64 - 1] * 5000 + [0] * 3 + [7] * 9000, dtype=np.uint64)
    assert np.array_equal(_sort_unique(keys), np.array([0, 7, 2 ** 64 - 1], dtype=np.uint64))


def test_aliasing_is_rejected():
    import torch
    N = H.pkg()._native
    d = torch.zeros(8, dtype=torch.int64, device="cuda")
    rc = N.lib().egtb_sort_unique_u64(0, d.data_ptr(), 8, d.data_ptr(), d.data_ptr(), None)
    assert rc == -1 and "alias" in N.last_error()
