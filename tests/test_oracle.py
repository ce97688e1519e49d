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


# ---------------------------------------------------------------- LEQ_CG0 (METHOD 5)
def _cg_numpy(s, k):
    """k iterations of textbook unpreconditioned CG from x = 0 on the
    diagonal-scaled system, numpy vector operations (an independent restatement
    of model/leq_cg.f:271-410 with MSOLVE0)."""
    t = s.copy()
    O.scale_diag(t)
    mv = lambda v: S.matvec_np(t.imax2, t.jmax2, t.kmax2, t.do_k, t.a, v)
    x = np.zeros(t.n)
    r = t.b - mv(x)
    p = np.zeros(t.n)
    rho_old = 0.0
    for i in range(1, k + 1):
        z = r.copy()
        rho = float(r @ z)
        p = z.copy() if i == 1 else z + (rho / rho_old) * p
        q = mv(p)
        alpha = rho / float(p @ q)
        r = r - alpha * q
        x = x + alpha * p
        rho_old = rho
    return x


def test_cg_iterates_match_numpy():
    s = S.diffusion_sym(12, 17, 9, seed=3)
    for k in (1, 4, 12):
        t = s.copy()
        t.tol = 0.0  # never converged: the oracle runs exactly k iterations
        t.itmax = k
        st = O.leq_cg(t, pc="NONE")
        assert st["iterations"] == k + 1 and st["ier"] in (-1, -2)
        xr = _cg_numpy(s, k)
        assert np.max(np.abs(t.x - xr)) <= 1e-10 * np.max(np.abs(xr))


def test_cg_converges_on_symmetric_systems():
    for dims, do_k in (((14, 20, 12), True), ((21, 19, 1), False), ((40, 3, 30), True)):
        s = S.diffusion_sym(*dims, seed=5, do_k=do_k)
        for pc in ("LINE", "DIAG", "NONE"):
            t = s.copy()
            st = O.leq_cg(t, pc=pc)
            ref = s.copy()
            O.scale_diag(ref)
            assert st["ier"] == 0 and st["exit_kind"] == 0
            assert st["iter_tot_add"] == st["iterations"] + 1
            assert O.true_resid(ref, t.x) <= s.tol * O.true_resid(ref, np.zeros(s.n)) * 1.01
            assert np.array_equal(t.a, ref.a) and np.array_equal(t.b, ref.b)  # rows scaled by 1/A(0)


def test_cg_ier_rules():
    s = S.diffusion_sym(8, 9, 7, seed=1)
    # R = 0: rho(0) = 0 at i = 1 -> IER 0, no iteration (model/leq_cg.f:294-303)
    t = s.copy()
    t.b[:] = 0.0
    st = O.leq_cg(t)
    assert st["ier"] == 0 and st["exit_kind"] == 2 and st["iter_tot_add"] == 0
    assert not np.any(t.x)
    # ITMAX = 0: the loop does not run; Rnorm = 0 < 0.2 Rnorm0 -> IER -1, ITER_TOT += 1
    t = s.copy()
    t.itmax = 0
    st = O.leq_cg(t)
    assert st["ier"] == -1 and st["iter_tot_add"] == 1
    # the reference's CG on a non-symmetric scaled operator diverges: IER -2 after ITMAX
    p = S.pressure_like(14, 20, 12, seed=3, nspheres=4, rmin=2, rmax=5, itmax=60)
    st = O.leq_cg(p)
    assert st["ier"] == -2 and st["iterations"] == 61 and st["iter_tot_add"] == 61


# ---------------------------------------------------------------- LEQ_GMRES0 (METHOD 3)
def _gmres_numpy(s, m, sweep="RSRS"):
    """m steps of left-preconditioned GMRES from x0 = s.x, the least-squares
    problem solved by numpy (an independent restatement of
    model/leq_gmres.f:220-507 without its Givens rotations)."""
    prec = lambda v: O.msolve(s, np.ascontiguousarray(v), sweep=sweep)[1]
    mv = lambda v: S.matvec_np(s.imax2, s.jmax2, s.kmax2, s.do_k, s.a, v)
    r = prec(s.b - mv(s.x))
    beta = np.linalg.norm(r)
    V = [r / beta]
    H = np.zeros((m + 1, m))
    for i in range(m):
        w = prec(mv(V[i]))
        for k in range(i + 1):
            H[k, i] = w @ V[k]
            w = w - H[k, i] * V[k]
        H[i + 1, i] = np.linalg.norm(w)
        V.append(w / H[i + 1, i])
    e1 = np.zeros(m + 1)
    e1[0] = beta
    y = np.linalg.lstsq(H, e1, rcond=None)[0]
    return s.x + np.array(V[:m]).T @ y


@pytest.mark.parametrize("m", [1, 5, 15])
def test_gmres_iterate_matches_numpy(m):
    s = S.conv_diff(11, 16, 9, seed=4)
    t = s.copy()
    t.tol = 0.0  # never converged: ITMAX steps, then the update with all m vectors
    t.itmax = m
    st = O.leq_gmres(t)
    assert st["ier"] == 1 and st["iterations"] == m
    xr = _gmres_numpy(s, m)
    assert np.max(np.abs(t.x - xr)) <= 1e-9 * np.max(np.abs(xr))


def test_gmres_converges_and_leaves_a_b():
    for s in (S.conv_diff(14, 20, 12, seed=3), S.conv_diff(21, 19, 1, seed=5, do_k=False),
              S.pressure_like(14, 20, 12, seed=3, nspheres=4, rmin=2, rmax=5, itmax=200)):
        s.itmax = 200
        t = s.copy()
        st = O.leq_gmres(t)
        assert st["ier"] == 0 and st["exit_kind"] == 0 and st["iter_tot_add"] == 0
        assert np.array_equal(t.a, s.a) and np.array_equal(t.b, s.b)  # no unit scaling in GMRES
        # ERROR is the preconditioned residual; the true one follows it within a few orders
        assert O.true_resid(s, t.x) <= 1e-5 * O.true_resid(s, np.zeros(s.n))


def test_gmres_zero_rhs_and_itmax():
    s = S.conv_diff(8, 9, 7, seed=1)
    t = s.copy()
    t.b[:] = 0.0
    t.x[:] = 3.0
    st = O.leq_gmres(t)  # model/leq_gmres.f:64-70: Var = 0, no iteration
    assert st["ier"] == 0 and st["exit_kind"] == 2 and not np.any(t.x)
    t = s.copy()
    t.itmax = 3
    st = O.leq_gmres(t)
    assert st["ier"] == 1 and st["iterations"] == 3


def test_sor_is_one_jacobi_step():
    """LEQ_SOR as the reference has it: every pass starts from the same VAR, so
    the result is one point-Jacobi step on the diagonal-scaled rows."""
    s = S.conv_diff(6, 7, 5, seed=1)
    s.x = np.random.default_rng(0).standard_normal(s.n)
    s.itmax = 4
    t = s.copy()
    st = O.leq_sor(t)
    a = s.a / s.a[3]
    a[3] = 1.0
    b = s.b / s.a[3]
    xj = s.x + (b - S.matvec_np(s.imax2, s.jmax2, s.kmax2, s.do_k, a, s.x))
    assert np.max(np.abs(xj - t.x)) <= 1e-14 * np.max(np.abs(xj))
    assert np.array_equal(t.a[3], np.ones(s.n)) and st["iter_tot_add"] == 5


@pytest.mark.parametrize("cyc,do_k", [(1, True), (2, True), (4, True), (7, True), (3, False)])
def test_cyclic_matvec_and_known_answer(cyc, do_k):
    """Cyclic axes: the oracle's LEQ_MATVEC equals an independent numpy restatement
    of the wrapped increments, and a system built from a known x (b = A x) is solved
    back to it."""
    s = S.conv_diff_cyclic(9, 11, 7 if do_k else 1, seed=12, cyc=cyc, do_k=do_k)
    rng = np.random.default_rng(cyc)
    x = rng.standard_normal(s.n)
    y_np = S.matvec_np(s.imax2, s.jmax2, s.kmax2, s.do_k, s.a, x, cyc=s.cyc)
    assert np.allclose(O.matvec(s, x), y_np, rtol=1e-13, atol=1e-13)
    assert not np.allclose(y_np, S.matvec_np(s.imax2, s.jmax2, s.kmax2, s.do_k, s.a, x))  # the wrap matters
    t = s.copy()
    wall = t.a[3] == -1.0
    x_act = rng.uniform(0.5, 1.5, s.n)
    x_act[wall] = 0.0
    t.b = S.matvec_np(t.imax2, t.jmax2, t.kmax2, t.do_k, t.a, x_act, cyc=t.cyc)
    t.x[:] = 0.0
    t.tol = 1e-12
    st = O.leq_bicgs(t)
    assert st["ier"] == 0
    assert np.linalg.norm(t.x - x_act) <= 1e-8 * np.linalg.norm(x_act)


def _rb_serial(s, b):
    """LEQ_MSOLVE's 'R' letter (model/leqsol_mod.f:382-391 in 2-D, :497-522 in 3-D)
    in a serial build's loop order, in plain Python: Var = B, then the J-lines
    (i + k) odd first in k-outer / i-inner order, each a tridiagonal solve whose
    right-hand side takes the wrapped I and K neighbours."""
    n = s.n
    A = s.a.reshape(7, s.kmax2, s.imax2, s.jmax2)
    B = b.reshape(s.kmax2, s.imax2, s.jmax2)
    V = B.copy()
    ni = S.neighbour_index
    im, ip = ni(s.imax2, -1, bool(s.cyc & 1)), ni(s.imax2, 1, bool(s.cyc & 1))
    km, kp = ni(s.kmax2, -1, bool(s.cyc & 4)), ni(s.kmax2, 1, bool(s.cyc & 4))
    first = 1 if s.do_k else 0   # 2-D: i odd (1-based) first, i.e. i + k even with k = 1
    for colour in (first, 1 - first):
        for k in range(s.kmax2):
            for i in range(s.imax2):
                if ((i + 1) + (k + 1)) % 2 != colour:
                    continue
                r = B[k, i] - A[2, k, i] * V[k, im[i]] - A[4, k, i] * V[k, ip[i]]
                if s.do_k:
                    r = r - A[0, k, i] * V[km[k], i] - A[6, k, i] * V[kp[k], i]
                dl, d, du = A[1, k, i][1:], A[3, k, i], A[5, k, i][:-1]
                _, _, _, x, info = lapack.dgtsv(dl.copy(), d.copy(), du.copy(), r.copy())
                assert info == 0
                V[k, i] = x
    assert V.size == n
    return V.reshape(-1)


@pytest.mark.parametrize("dims,cyc,do_k", [((11, 7, 9), 5, True), ((11, 6, 8), 7, True), ((13, 8, 1), 1, False)])
def test_cyclic_red_black_serial_order(dims, cyc, do_k):
    """With an odd number of interior cells along a cyclic axis the first and last
    interior lines share a colour; the oracle sweeps them in the serial loop order."""
    s = S.conv_diff_cyclic(*dims, seed=13, cyc=cyc, do_k=do_k)
    O.scale(s)
    x = np.random.default_rng(2).standard_normal(s.n)
    rc, v, _ = O.msolve(s, x, "RRRR"[:1] + "   ")
    assert rc == 0
    ref = _rb_serial(s, x)
    assert np.max(np.abs(v - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_minimize_dotproducts_mode():
    """MINIMIZE_DOTPRODUCTS (model/leq_bicgs.f:372,411,439): no Snorm exit and the
    Rnorm test every ICHECK_BICGS-th iteration, so a converged solve stops on a
    multiple of ICHECK_BICGS; with ICHECK_BICGS = 1 it is the plain iteration."""
    s = S.conv_diff(14, 17, 12, seed=21)
    base = s.copy()
    st0 = O.leq_bicgs(base)
    one = s.copy()
    st1 = O.leq_bicgs(one, icheck=1)
    assert st1["ier"] == st0["ier"] == 0 and st1["iterations"] == st0["iterations"]
    assert np.array_equal(one.x, base.x)
    for k in (3, 7):
        t = s.copy()
        stk = O.leq_bicgs(t, icheck=k)
        assert stk["ier"] == 0 and stk["iterations"] % k == 0
        assert st0["iterations"] <= stk["iterations"] < st0["iterations"] + k
        sc = s.copy()
        O.scale(sc)
        assert O.true_resid(sc, t.x) <= s.tol * O.true_resid(sc, np.zeros(s.n)) * 1.01
    tr = s.copy()
    stt = O.leq_bicgst(tr, minimize=True)
    assert stt["ier"] == 0 and stt["iterations"] % 5 == 0
