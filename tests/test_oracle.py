"""CPU checks of the oracle (the C restatement of the reference path).

Pins: DGTSV bit-for-bit against LAPACK's dgtsv (scipy), MATVEC against an
independent numpy restatement, the LINE preconditioner's exactness on a single
J-line, the identity of the reference's ISIS and KSKS orders, the
known-answer recipe of model/test_lin_eq.f, and the IER rules of
model/leq_bicgs.f.
"""
import numpy as np
import pytest
import scipy.linalg.lapack as lapack

import oracle as O
from mfix_b200 import systems as S


def test_dgtsv_matches_lapack_bitwise():
    rng = np.random.default_rng(0)
    interchanges = 0
    for t in range(3000):
        n = int(rng.integers(2, 50))
        dl, d, du, b = (rng.standard_normal(n - 1), rng.standard_normal(n), rng.standard_normal(n - 1),
                        rng.standard_normal(n))
        if t % 3 == 0:
            d = d * 10.0
        else:
            interchanges += 1
        info, x = O.dgtsv(dl, d, du, b)
        _, _, _, xr, info_r = lapack.dgtsv(dl, d, du, b.reshape(-1, 1))
        assert info == info_r
        if info == 0:
            assert np.array_equal(x, xr.ravel())
    assert interchanges > 1000


def test_dgtsv_zero_pivot_info():
    # exact zero pivot at row 2 (1-based)
    dl = np.array([0.0, 0.0])
    d = np.array([1.0, 0.0, 1.0])
    du = np.array([0.0, 0.0])
    info, _ = O.dgtsv(dl, d, du, np.ones(3))
    _, _, _, _, info_r = lapack.dgtsv(dl, d, du, np.ones((3, 1)))
    assert info == info_r == 2
    info, _ = O.dgtsv(np.zeros(0), np.zeros(1), np.zeros(0), np.ones(1))
    assert info == 1


@pytest.mark.parametrize("dims,do_k", [((7, 9, 5), True), ((12, 10, 1), False), ((3, 40, 3), True)])
def test_matvec_matches_numpy(dims, do_k):
    s = S.conv_diff(*dims, seed=1, do_k=do_k)
    x = np.random.default_rng(1).standard_normal(s.n)
    ref = S.matvec_np(s.imax2, s.jmax2, s.kmax2, s.do_k, s.a, x)
    np.testing.assert_allclose(O.matvec(s, x), ref, rtol=1e-14, atol=1e-14)


def _single_line(L=23, seed=2):
    rng = np.random.default_rng(seed)
    a = np.zeros((7, L))
    a[1, 1:] = rng.random(L - 1)
    a[5, :-1] = rng.random(L - 1)
    a[3] = -(a[1] + a[5] + 0.5)
    return S.System(1, L, 1, 1, a, rng.standard_normal(L), np.zeros(L), 1e-10, 50, "line")


def test_line_preconditioner_is_exact_on_one_line():
    s = _single_line()
    rc, v, _ = O.msolve(s, s.b, "RSRS", "LINE")
    assert rc == 0
    np.testing.assert_allclose(O.matvec(s, v), s.b, rtol=0, atol=1e-13)
    st = O.leq_bicgs(s)
    assert st["ier"] == 0 and st["iterations"] == 1


def test_isis_equals_ksks():
    """Both lexicographic orders see the same neighbour values (model/leqsol_mod.f:567-582)."""
    s = S.conv_diff(8, 9, 7, seed=3)
    O.scale(s)
    b = np.random.default_rng(3).standard_normal(s.n)
    _, v1, _ = O.msolve(s, b, "ISIS")
    _, v2, _ = O.msolve(s, b, "KSKS")
    assert np.array_equal(v1, v2)


def test_noop_letters_copy_b():
    s = S.conv_diff(5, 6, 4, seed=4)
    O.scale(s)
    b = np.random.default_rng(4).standard_normal(s.n)
    _, v, _ = O.msolve(s, b, "JSJS")
    assert np.array_equal(v, b)


def test_known_answer_recipe():
    s, x_act = S.known_answer(10, 12, 9, seed=5)
    st = O.leq_bicgs(s)
    assert st["ier"] == 0
    assert np.linalg.norm(s.x - x_act) / np.linalg.norm(x_act) < 1e-9


def test_ier_rules():
    s = S.conv_diff(6, 7, 5, seed=6)
    z = s.copy()
    z.b[:] = 0.0
    st = O.leq_bicgs(z)
    assert st["ier"] == 0 and st["exit_kind"] == 2 and st["iter_tot_add"] == 0
    sg = s.copy()
    sg.a[:, 50] = 0.0
    st = O.leq_bicgs(sg)
    assert st["ier"] == -2 and st["exit_kind"] == 4
    t = S.pressure_like(12, 12, 12, seed=7, nspheres=2, rmin=2, rmax=3)
    t.itmax = 2
    st = O.leq_bicgs(t)
    assert st["ier"] in (-1, -2) and st["iterations"] == 3 and st["iter_tot_add"] == 3
    t0 = S.conv_diff(6, 6, 6, seed=8)
    t0.itmax = 0
    st = O.leq_bicgs(t0)
    assert st["ier"] == 0  # REAL(0) <= TOL*Rnorm0 after an empty loop
    st = O.leq_bicgs(s.copy(), pc="ILU ")
    assert st["ier"] == -10


def test_unit_scaling_rows():
    s = S.conv_diff(6, 5, 4, seed=9)
    assert O.scale(s) == 0
    m = np.abs(s.a).max(axis=0)
    np.testing.assert_allclose(m, 1.0, rtol=2e-16, atol=0)


def test_truth_solver_reaches_1e14():
    s = S.conv_diff(12, 12, 12, seed=10)
    O.scale(s)
    x, rel = O.truth(s)
    assert rel <= 1e-14


def test_convergence_residual_below_tol():
    s = S.conv_diff(16, 18, 14, seed=11)
    ref = s.copy()
    O.leq_bicgs(ref)
    r0 = O.true_resid(ref, np.zeros(s.n))
    assert O.true_resid(ref, ref.x) / r0 <= 1.01e-8
