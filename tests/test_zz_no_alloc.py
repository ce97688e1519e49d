"""The allocation-free dot product (mfixgpu_dot_product_par_noalloc).

Hosts that own all device memory or run under a fixed device-memory budget
cannot let a library allocate; this entry point keeps its scratch in a fixed
array inside the library.  The test calls it through the C ABI twice in a row,
on different data, and compares each result with mfixgpu_dot_product_par
within the dot-product tolerance of the other tests (1e-13 relative); it also
checks that a length beyond the fixed scratch is refused.  This file is
collected last so that it runs after every other test as well as alone.
"""
import numpy as np
import pytest

from mfix_b200 import leq

pytestmark = pytest.mark.gpu


def test_noalloc_dot_matches_allocating_entry_point_twice(cuda):
    rng = np.random.default_rng(2024)
    for n in (1_000_003, 257):  # two calls in a row: the shared scratch is reused
        x, y = rng.standard_normal(n), rng.standard_normal(n)
        dx = cuda.from_numpy(x).cuda()
        dy = cuda.from_numpy(y).cuda()
        out = cuda.zeros(1, dtype=cuda.float64, device="cuda")
        rc = leq.dot_product_par_noalloc(dx.data_ptr(), dy.data_ptr(), n, out.data_ptr())
        assert rc == 0, leq.last_error()
        cuda.cuda.synchronize()
        got = float(out.item())
        ref = leq.dot_product_par(dx.data_ptr(), dy.data_ptr(), n)
        assert abs(got - ref) <= 1e-13 * max(1.0, float(np.abs(x * y).sum()))


def test_noalloc_rejects_length_beyond_scratch(cuda):
    d = cuda.zeros(4, dtype=cuda.float64, device="cuda")
    rc = leq.dot_product_par_noalloc(d.data_ptr(), d.data_ptr(), leq.NOALLOC_MAX_N + 1, d.data_ptr())
    assert rc == leq.IER_ARGS
    assert "MFIXGPU_NOALLOC_MAX_N" in leq.last_error()
