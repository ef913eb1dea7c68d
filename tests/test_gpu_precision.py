"""Error of float32 success rates against a float64 recomputation of the same
table. Both dtypes are built on the device and compared entry by entry; the
result must be the reference's own float32-vs-float64 difference (recorded
from the reference's builds in tests/golden/cases.json), and it stays under
the stated bound."""
import importlib

import pytest

import helpers as H

# largest |r32 - r64| over every entry of the L3-256 and 442-512 books
# (3.06e-7 and 2.78e-7; means 1.7e-8 and 1.6e-8)
# (the reference's builds give the same figures; see the golden cases)
MAX_ABS_ERR_BOUND = 4e-7


def _P():
    return importlib.import_module("2048endgametablebase_b200.precision")


@pytest.mark.gpu
@pytest.mark.slow
@pytest.mark.parametrize("key", ["L3_256", "442_512"])
def test_float32_rates_against_float64_recomputation(key):
    want = H.cases()[key + "_fp64_error"]
    case = H.cases()[key + "_float32"]
    spec, o = H.spec_options(case, "")
    got = _P().rate_error_vs_fp64(H.seeds(case), spec, o)
    assert got["entries"] == want["entries"]
    assert got["max_abs_err"] == want["max_abs_err"]
    assert got["layer"] == want["layer"] and hex(got["board"]) == want["board"]
    assert got["mean_abs_err"] == pytest.approx(want["mean_abs_err"], rel=1e-9)
    assert got["max_abs_err"] <= MAX_ABS_ERR_BOUND
