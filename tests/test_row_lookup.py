"""The device path finds the row of a cell or y-face index as
floor((idx + 0.5) * rcp(nx)) in FP32 (rowOf in csrc/rq_solver.cu) instead of an
integer division. This restates that arithmetic with IEEE FP32 (numpy float32:
correctly rounded reciprocal and product, as __frcp_rn and the FP32 multiply) and
checks it against idx // nx for every index below the 2^21 bound that rq_problem_create
enforces, for the mesh widths the generators produce."""
import numpy as np
import pytest

NX = list(range(1, 65)) + [96, 100, 127, 128, 200, 255, 256, 400, 512, 1000, 1024, 2047]


@pytest.mark.parametrize("nx", NX)
def test_fp32_row_lookup_is_exact_below_bound(nx):
    idx = np.arange(1 << 21, dtype=np.int64)
    rcp = np.float32(1.0) / np.float32(nx)
    q = (idx.astype(np.float32) + np.float32(0.5)) * rcp
    assert q.dtype == np.float32
    rows = np.floor(q).astype(np.int64)
    np.testing.assert_array_equal(rows, idx // nx)
