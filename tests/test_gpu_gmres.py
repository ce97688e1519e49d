"""METHOD 3 (LEQ_GMRES, model/leq_gmres.f) and METHOD 4 (BiCGSTAB, then GMRES on
a breakdown, model/solve_lin_eq.f:161-171) through the drop-in entry point,
against the oracle's restatements on the same inputs.

Checked: IER (0 or 1) and the Arnoldi step count equal to the oracle's within
one (the GPU sums the dot products in another order); the solution within 1e-6
of the oracle's; A_M and B_M untouched by GMRES; B = 0 gives Var = 0; an ITMAX
too small for convergence gives IER 1 after exactly ITMAX steps; METHOD 4 hands
a BiCGSTAB breakdown (IER -2) to GMRES on the scaled system from BiCGSTAB's
result, IER reset to 0, ITER_TOT from BiCGSTAB only.
"""
import numpy as np
import pytest

import oracle as O
from mfix_b200 import leq
from mfix_b200 import systems as S

pytestmark = pytest.mark.gpu

CASES = [
    ("conv3d", lambda: S.conv_diff(14, 20, 12, seed=3)),
    ("conv2d", lambda: S.conv_diff(21, 19, 1, seed=5, do_k=False)),
    ("odd", lambda: S.conv_diff(9, 31, 7, seed=7)),
    ("pressure", lambda: S.pressure_like(14, 20, 12, seed=3, nspheres=4, rmin=2, rmax=5)),
    ("kat", lambda: S.known_answer(8, 40, 6, seed=4)[0]),
]


def _close(x, y, rel):
    return np.linalg.norm(x - y) <= rel * max(np.linalg.norm(y), 1e-300)


@pytest.mark.parametrize("sweep", ["RSRS", "ISIS"])
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_gmres_matches_oracle(cuda, name, make, sweep):
    s = make()
    s.itmax = 200
    ref = s.copy()
    st_ref = O.leq_gmres(ref, sweep=sweep)
    got = s.copy()
    before = leq.iter_tot(2)
    ier = leq.solve_system(got, method=3, sweep=sweep, vno=2)
    st = leq.last_stats()
    assert ier == st_ref["ier"] == 0, leq.last_error()
    assert abs(st["iterations"] - st_ref["iterations"]) <= 1
    assert leq.iter_tot(2) == before  # GMRES keeps no ITER_TOT
    assert np.array_equal(got.a, s.a) and np.array_equal(got.b, s.b)
    assert _close(got.x, ref.x, 1e-6)


def test_gmres_itmax_reached(cuda):
    s = S.conv_diff(16, 22, 14, seed=11)
    s.itmax = 5
    ref = s.copy()
    st_ref = O.leq_gmres(ref)
    got = s.copy()
    assert leq.solve_system(got, method=3) == st_ref["ier"] == 1
    assert leq.last_stats()["iterations"] == st_ref["iterations"] == 5
    assert _close(got.x, ref.x, 1e-9)


def test_gmres_zero_rhs(cuda):
    s = S.conv_diff(8, 9, 7, seed=1)
    s.b[:] = 0.0
    s.x[:] = 3.0
    assert leq.solve_system(s, method=3) == 0
    assert not np.any(s.x)


@pytest.mark.parametrize("case", ["ratio", "singular_row"])
def test_method4_hands_breakdown_to_gmres(cuda, case):
    if case == "ratio":  # one unpreconditioned iteration leaves ||R|| above 0.2 ||R0||: IER -2
        s = S.pressure_like(14, 20, 12, seed=3, nspheres=4, rmin=2, rmax=5)
        s.itmax = 1
        pc = "NONE"
    else:  # a zero row: IER -2 before any iteration
        s = S.conv_diff(10, 12, 9, seed=2)
        s.itmax = 30
        s.a[:, 5 * s.jmax2 + 3 + 4 * s.jmax2 * s.imax2] = 0.0
        pc = "LINE"
    ref = s.copy()
    st_b = O.leq_bicgs(ref, pc=pc)
    assert st_b["ier"] == -2
    st_g = O.leq_gmres(ref)  # on the scaled system, from BiCGSTAB's result
    got = s.copy()
    before = leq.iter_tot(4)
    ier = leq.solve_system(got, method=4, pc=pc, vno=4)
    assert ier == st_g["ier"], leq.last_error()
    assert leq.iter_tot(4) - before == st_b["iter_tot_add"]
    assert np.array_equal(got.a, ref.a) and np.array_equal(got.b, ref.b)  # BiCGSTAB's scaling came back
    assert _close(got.x, ref.x, 1e-6)


@pytest.mark.parametrize("lanes", [1, 2, 32])
def test_method4_singular_row_each_line_shape(cuda, lanes):
    """The zero row's J-line meets a zero pivot in DGTSV (INFO != 0, the line is left
    unchanged) inside the GMRES preconditioner, whose right-hand side is a work
    vector of its own: every line-kernel shape (one lane per line included) gives
    the oracle's VAR."""
    s = S.conv_diff(10, 12, 9, seed=2)
    s.itmax = 30
    s.a[:, 5 * s.jmax2 + 3 + 4 * s.jmax2 * s.imax2] = 0.0
    ref = s.copy()
    assert O.leq_bicgs(ref, pc="LINE")["ier"] == -2
    st_g = O.leq_gmres(ref)
    assert leq.set_option("line_lanes", lanes) == 0
    try:
        got = s.copy()
        ier = leq.solve_system(got, method=4, pc="LINE", vno=4)
    finally:
        leq.set_option("line_lanes", 0)
    assert ier == st_g["ier"], leq.last_error()
    assert _close(got.x, ref.x, 1e-9)
