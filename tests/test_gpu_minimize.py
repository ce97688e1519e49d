"""MINIMIZE_DOTPRODUCTS / ICHECK_BICGS for the FP64 drop-in (METHOD 2).

With the reference's MINIMIZE_DOTPRODUCTS set, LEQ_BICGS0 skips the Snorm exit
and forms and tests Rnorm only every ICHECK_BICGS-th iteration
(model/leq_bicgs.f:372,411,439); LEQ_BICGSt tests every fifth
(model/leq_bicgst.f:514).  The GPU drop-in against the oracle in the same mode:
the same IER, an iteration count that is a multiple of ICHECK_BICGS inside the
oracle's envelope, A/B scaled bit for bit, the true residual of the scaled system
<= 1.01 TOL.
"""
import numpy as np
import pytest

import oracle as O
from mfix_b200 import leq
from mfix_b200 import systems as S

pytestmark = pytest.mark.gpu


def _with(opts, fn):
    old = {k: leq.get_option(k) for k in opts}
    try:
        for k, v in opts.items():
            assert leq.set_option(k, v) == 0
        return fn()
    finally:
        for k, v in old.items():
            leq.set_option(k, v)


@pytest.mark.parametrize("icheck", [1, 3, 7])
@pytest.mark.parametrize("make", [lambda: S.conv_diff(20, 26, 18, seed=30),
                                  lambda: S.conv_diff(40, 33, 1, seed=31, do_k=False)], ids=["3d", "2d"])
def test_minimize_matches_oracle(make, icheck):
    s = make()
    ref = s.copy()
    st_ref = O.leq_bicgs(ref, icheck=icheck)
    counts = []
    for eps in (0.0, 1e-15, -1e-15):
        t = s.copy()
        t.b *= 1.0 + eps
        counts.append(O.leq_bicgs(t, icheck=icheck)["iterations"])
    gpu = s.copy()
    ier = _with({"minimize_dotproducts": 1, "icheck_bicgs": icheck}, lambda: leq.solve_system(gpu))
    st = leq.last_stats()
    assert ier == st_ref["ier"] == 0, leq.last_error()
    assert st["iterations"] % icheck == 0
    assert min(counts) - icheck <= st["iterations"] <= max(counts) + icheck
    assert np.array_equal(gpu.a, ref.a) and np.array_equal(gpu.b, ref.b)
    r0 = O.true_resid(ref, np.zeros(s.n))
    assert O.true_resid(ref, gpu.x) <= 1.01 * s.tol * r0


def test_minimize_transposed_every_fifth():
    s = S.conv_diff(18, 22, 14, seed=32)
    ref = s.copy()
    st_ref = O.leq_bicgst(ref, minimize=True)
    gpu = s.copy()
    ier = _with({"minimize_dotproducts": 1, "do_transpose": 1}, lambda: leq.solve_system(gpu))
    st = leq.last_stats()
    assert ier == st_ref["ier"] == 0, leq.last_error()
    assert st["iterations"] % 5 == 0 and abs(st["iterations"] - st_ref["iterations"]) <= 5
    assert np.array_equal(gpu.b, ref.b)
