"""egtb_sort_unique_u64_noalloc: the sort + unique of caller-owned device keys
for callers that cannot let the library allocate device memory (their pool
holds it all, or cudaMalloc/cudaFree would stall a latency-critical path).
Its scratch is a static device array, so it is checked here against the
allocating entry point, egtb_sort_unique_u64, on two calls in a row (the
second call finds the first call's contents in the shared array)."""
import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu

LIMIT = 1 << 20


def _keys(seed: int, n: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    pool = rng.integers(0, 2 ** 62, size=max(1, n // 4), dtype=np.uint64) * np.uint64(4)
    return rng.choice(pool, size=n)


def _run(fn_name: str, keys: np.ndarray):
    import torch
    N = H.pkg()._native
    n = len(keys)
    d_in = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    d_out = torch.full((max(n, 1),), -1, dtype=torch.int64, device="cuda")
    d_cnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    st = torch.cuda.current_stream()
    N.check(getattr(N.lib(), fn_name)(0, d_in.data_ptr(), n, d_out.data_ptr(), d_cnt.data_ptr(), st.cuda_stream))
    st.synchronize()
    m = int(d_cnt.item())
    return d_out[:m].cpu().numpy().view(np.uint64)


def test_noalloc_matches_allocating_entry_point_twice():
    for call, (seed, n) in enumerate([(11, LIMIT), (12, 300_001)]):
        keys = _keys(seed, n)
        want = _run("egtb_sort_unique_u64", keys)
        got = _run("egtb_sort_unique_u64_noalloc", keys)
        assert got.dtype == want.dtype and len(got) == len(want), call
        assert np.array_equal(got, want), call  # integer keys: bit-exact
        assert np.array_equal(got, np.unique(keys)), call


def test_noalloc_rejects_sizes_beyond_its_limit():
    import torch
    N = H.pkg()._native
    d = torch.zeros(2, dtype=torch.int64, device="cuda")
    rc = N.lib().egtb_sort_unique_u64_noalloc(0, d.data_ptr(), LIMIT + 1, d.data_ptr() + 8, d.data_ptr(), None)
    assert rc == -1 and "limit" in N.last_error()
