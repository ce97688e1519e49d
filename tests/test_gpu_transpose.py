"""DO_TRANSPOSE (model/solve_lin_eq.f:139-150): METHOD 2 through LEQ_BICGSt
(model/leq_bicgst.f), served by the drop-in with option "do_transpose".

Against the oracle's restatement of LEQ_BICGSt: the same IER, an iteration
count inside the oracle's rounding envelope, A_M left as the caller passed it
(SOLVE_LIN_EQ scales a transposed copy and discards it), B_M scaled in place
bit for bit, and the true residual of the scaled system <= 1.01 TOL.  Cases:
red/black sweeps in 3-D (an even IMAX2), I sweeps in 3-D and 2-D, and red/black
letters in 2-D, which LEQ_MSOLVEt does not serve (the preconditioner is the
copy alone).  Red/black sweeps in 3-D with an odd IMAX2 (LEQ_MSOLVEt's loop
wraps within a row) return MFIXGPU_ERR_UNSUPPORTED.
"""
import numpy as np
import pytest

import oracle as O
from mfix_b200 import leq
from mfix_b200 import systems as S

pytestmark = pytest.mark.gpu


def _envelope(s, sweep):
    counts = []
    for eps in (0.0, 1e-15, -1e-15, 2e-15):
        t = s.copy()
        t.b *= 1.0 + eps
        counts.append(O.leq_bicgst(t, sweep)["iterations"])
    return min(counts) - 1, max(counts) + 1


CASES = [
    ("rb_3d", lambda: S.conv_diff(14, 17, 11, seed=30), "RSRS"),
    ("isis_3d", lambda: S.conv_diff(11, 13, 9, seed=31), "ISIS"),
    ("isis_2d", lambda: S.conv_diff(26, 21, 1, seed=32, do_k=False), "ISIS"),
    ("rb_2d_copy_only", lambda: S.conv_diff(20, 17, 1, seed=33, do_k=False), "RSRS"),
]


@pytest.mark.parametrize("name,make,sweep", CASES, ids=[c[0] for c in CASES])
def test_transposed_matches_oracle(name, make, sweep):
    s = make()
    ref = s.copy()
    st_ref = O.leq_bicgst(ref, sweep)
    lo, hi = _envelope(s, sweep)
    gpu = s.copy()
    assert leq.set_option("do_transpose", 1) == 0
    try:
        ier = leq.solve_system(gpu, sweep=sweep)
        st = leq.last_stats()
    finally:
        leq.set_option("do_transpose", 0)
    assert ier == st_ref["ier"] == 0, leq.last_error()
    assert lo <= st["iterations"] <= hi, (st["iterations"], lo, hi)
    assert np.array_equal(gpu.a, s.a)  # A_M as passed: the scaled copy is discarded
    assert np.array_equal(gpu.b, ref.b)  # B_M scaled in place
    scaled = s.copy()
    O.scale(scaled)
    r0 = O.true_resid(scaled, np.zeros(s.n))
    assert O.true_resid(scaled, gpu.x) <= 1.01 * s.tol * r0
    assert np.linalg.norm(gpu.x - ref.x) <= 1e-6 * np.linalg.norm(ref.x)


def test_transposed_odd_imax2_red_black_not_served():
    s = S.conv_diff(13, 10, 8, seed=34)  # IMAX2 = 15
    assert leq.set_option("do_transpose", 1) == 0
    try:
        ier = leq.solve_system(s.copy(), sweep="RSRS")
        ier_i = leq.solve_system(s.copy(), sweep="ISIS")  # I sweeps are served at any size
    finally:
        leq.set_option("do_transpose", 0)
    assert ier == leq.IER_UNSUPPORTED
    assert ier_i == 0
