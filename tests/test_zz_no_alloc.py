"""The allocation-free dot product (mfixgpu_dot_product_par_noalloc).

Hosts that own all device memory or run under a fixed device-memory budget
cannot let a library allocate; this entry point keeps its scratch in a fixed
array inside the library.  The tests call it through the C ABI and compare
each result with an exactly rounded sum of the products (math.fsum), with
numpy's dot and with mfixgpu_dot_product_par, within the dot-product tolerance
of the other tests (1e-13 of sum |r1*r2|): two calls in a row on different
data (the shared scratch is reused), a length that fills whole chunks of the
scratch exactly, the empty vector (the result is written as zero), a
non-default stream, and a length beyond the fixed scratch, which is refused.
This file is collected last so that it runs after every other test as well as
alone.
"""
import math

import numpy as np
import pytest

from mfix_b200 import leq

pytestmark = pytest.mark.gpu

CHUNK = 1 << 17  # elements each block of the kernel reduces (the scratch holds one partial sum per chunk)


def _check(cuda, x, y, stream=None):
    n = len(x)
    pad = np.zeros(1)  # an empty tensor may have no address: the buffers keep one element
    dx = cuda.from_numpy(np.concatenate([x, pad])).cuda()
    dy = cuda.from_numpy(np.concatenate([y, pad])).cuda()
    out = cuda.full((1,), 12345.0, dtype=cuda.float64, device="cuda")  # stale value: the call must overwrite it
    cuda.cuda.synchronize()
    if stream is None:
        rc = leq.dot_product_par_noalloc(dx.data_ptr(), dy.data_ptr(), n, out.data_ptr())
    else:
        rc = leq.dot_product_par_noalloc(dx.data_ptr(), dy.data_ptr(), n, out.data_ptr(), stream.cuda_stream)
        stream.synchronize()
    assert rc == 0, leq.last_error()
    cuda.cuda.synchronize()
    got = float(out.item())
    exact = math.fsum((x * y).tolist())
    scale = max(1.0, float(np.abs(x * y).sum()))
    assert abs(got - exact) <= 1e-13 * scale
    assert abs(got - float(np.dot(x, y))) <= 1e-13 * scale
    if n > 0:
        ref = leq.dot_product_par(dx.data_ptr(), dy.data_ptr(), n)
        assert abs(got - ref) <= 1e-13 * scale
    return got


def test_noalloc_dot_two_calls_in_a_row(cuda):
    rng = np.random.default_rng(2024)
    for n in (1_000_003, 257):  # two calls in a row: the shared scratch is reused
        _check(cuda, rng.standard_normal(n), rng.standard_normal(n))


def test_noalloc_dot_whole_chunks_and_empty(cuda):
    rng = np.random.default_rng(7)
    n = 2 * CHUNK  # every block reduces a full chunk, none a partial one
    _check(cuda, rng.standard_normal(n), rng.standard_normal(n))
    _check(cuda, rng.standard_normal(CHUNK), rng.uniform(-1, 1, CHUNK))
    assert _check(cuda, np.zeros(0), np.zeros(0)) == 0.0


def test_noalloc_dot_on_a_stream(cuda):
    rng = np.random.default_rng(11)
    s = cuda.cuda.Stream()
    for n in (300_001, 5):
        _check(cuda, rng.standard_normal(n), rng.standard_normal(n), stream=s)


def test_noalloc_rejects_length_beyond_scratch(cuda):
    d = cuda.zeros(4, dtype=cuda.float64, device="cuda")
    rc = leq.dot_product_par_noalloc(d.data_ptr(), d.data_ptr(), leq.NOALLOC_MAX_N + 1, d.data_ptr())
    assert rc == leq.IER_ARGS
    assert "MFIXGPU_NOALLOC_MAX_N" in leq.last_error()
