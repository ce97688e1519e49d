"""J-line kernel with the rows past a line's register passes staged by cp.async.

With option "line_stage" 1 the warp J-line kernel copies the operand rows beyond
its first register passes (right-hand side, four off-line coefficients, four
neighbour lines, three factors) into shared memory before those passes start
and forms their right-hand sides from the copies; with 0 every row goes through
register passes.  Both evaluate the same operations in the same order, so the
solves agree bit for bit and in their iteration counts: FP64 and mixed forms,
lines with a short last pass (MFIX's 2^m + 2), several lines per warp, 2-D, a
flagged (pivoting) line, cyclic boxes and an uneven batch.
"""
import numpy as np
import pytest

import oracle as O
from mfix_b200 import leq
from mfix_b200 import systems as S

pytestmark = pytest.mark.gpu

CASES = [
    # JMAX2 = 132: one 128-row pass of four-row groups plus a 4-row tail
    ("tail_132", lambda: S.conv_diff(10, 130, 8, seed=80)),
    # JMAX2 = 258 as in the 256^3 benchmark, on a thin box
    ("tail_258", lambda: S.conv_diff(5, 256, 4, seed=81)),
    # two register passes before the staged rows (JMAX2 = 386)
    ("tail_386", lambda: S.conv_diff(4, 384, 3, seed=82)),
    ("odd_line", lambda: S.conv_diff(9, 141, 7, seed=83)),
    ("conv2d", lambda: S.conv_diff(40, 150, 1, seed=84, do_k=False)),
    ("cyclic", lambda: S.conv_diff_cyclic(9, 134, 7, seed=85, cyc=7)),
    ("pressure", lambda: S.pressure_like(12, 140, 10, seed=86, nspheres=3, rmin=3, rmax=5, itmax=3000)),
]


def _solve(s, stage, precision, lanes=0):
    m = s.copy()
    assert leq.set_option("line_stage", stage) == 0
    assert leq.set_option("precision", precision) == 0
    assert leq.set_option("line_lanes", lanes) == 0
    try:
        ier = leq.solve_system(m)
        st = leq.last_stats()
    finally:
        leq.set_option("precision", 0)
        leq.set_option("line_stage", 1)
        leq.set_option("line_lanes", 0)
    return ier, st, m


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_staged_rows_match_register_passes(name, make, precision):
    s = make()
    ier1, st1, m1 = _solve(s, 1, precision)
    ier0, st0, m0 = _solve(s, 0, precision)
    assert ier1 == ier0, leq.last_error()
    assert st1["iterations"] == st0["iterations"]
    assert st1["fp64_fallback"] == st0["fp64_fallback"]
    assert np.array_equal(m1.x, m0.x)
    assert np.array_equal(m1.a, m0.a) and np.array_equal(m1.b, m0.b)
    if ier1 == 0:
        ref = s.copy()
        O.scale(ref)
        r0 = O.true_resid(ref, np.zeros(s.n))
        assert O.true_resid(ref, m1.x) <= 1.01 * s.tol * r0


@pytest.mark.parametrize("lanes", [4, 8, 16])
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_several_lines_per_warp(lanes, precision):
    s = S.conv_diff(11, 66, 9, seed=87)
    ier1, st1, m1 = _solve(s, 1, precision, lanes)
    ier0, st0, m0 = _solve(s, 0, precision, lanes)
    assert ier1 == ier0 == 0, leq.last_error()
    assert st1["iterations"] == st0["iterations"]
    assert np.array_equal(m1.x, m0.x)


def test_pivoting_line():
    # a line whose elimination interchanges rows runs DGTSV's pivoting path; the
    # staged copies of its rows are ignored like the register loads
    s = S.conv_diff(7, 140, 6, seed=88)
    # line (i=3, k=3), row j = 20: a tiny diagonal against a large coupling from
    # the next row (A(-2) of row j = 21, DGTSV's DL)
    c = (3 - 1) * s.jmax2 + (3 - 1) * s.jmax2 * s.imax2 + 19
    s.a[3, c] = 1e-3 * s.a[3, c]
    s.a[1, c + 1] = -4.0 * abs(s.a[3, c + 1])
    for precision in (0, 1):
        ier1, st1, m1 = _solve(s, 1, precision)
        ier0, st0, m0 = _solve(s, 0, precision)
        assert ier1 == ier0
        assert st1["iterations"] == st0["iterations"]
        assert np.array_equal(m1.x, m0.x)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_batch(precision):
    sizes = [(17, 130, 13), (12, 258, 9), (9, 66, 9), (33, 98, 1), (8, 386, 5), (21, 33, 17)]
    systems = [S.conv_diff(i, j, k, seed=90 + q, do_k=k > 1) for q, (i, j, k) in enumerate(sizes)]
    out = {}
    for stage in (1, 0):
        batch = [t.copy() for t in systems]
        assert leq.set_option("line_stage", stage) == 0
        try:
            rc, res = leq.batch_solve(batch, precision=precision)
        finally:
            leq.set_option("line_stage", 1)
        assert rc == 0, leq.last_error()
        assert all(r.ier == 0 for r in res)
        out[stage] = (batch, [r.iterations for r in res])
    assert out[1][1] == out[0][1]
    for a, b in zip(out[1][0], out[0][0]):
        assert np.array_equal(a.x, b.x)
