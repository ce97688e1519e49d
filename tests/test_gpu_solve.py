"""Whole-solve parity of the drop-in (mfixgpu_solve_lin_eq_) against the oracle.

For each seeded system the GPU and the oracle run LEQ_BICGS from the same
inputs.  Checked: the same IER and exit reason, an iteration count inside the
oracle's own rounding envelope (its counts when B_M is perturbed by 1e-15
relative; BiCGSTAB's count is that sensitive on some systems),
the unit-scaled A_M/B_M written back bit for bit, the true relative residual
||b - A x|| / ||b - A x0|| <= TOL * 1.01 (the reference's own test is on the
recursive residual, model/leq_bicgs.f:455), an error against a 1e-14 FP64
solution no larger than ten times the oracle's own error (or 1e-10), plus
ITER_TOT accounting.
"""
import numpy as np
import pytest

import oracle as O
from mfix_b200 import leq
from mfix_b200 import systems as S

pytestmark = pytest.mark.gpu


def _run_both(s, sweep="RSRS", pc="LINE", method=2, vno=3):
    ref = s.copy()
    st_ref = O.leq_bicgs(ref, sweep, pc)
    gpu = s.copy()
    leq.reset_iter_tot()
    ier = leq.solve_system(gpu, method=method, sweep=sweep, pc=pc, vno=vno)
    st = leq.last_stats()
    return ref, st_ref, gpu, ier, st


def _envelope(s, sweep, pc):
    counts = []
    for eps in (0.0, 1e-15, -1e-15, 2e-15):
        t = s.copy()
        t.b *= (1.0 + eps)
        counts.append(O.leq_bicgs(t, sweep, pc)["iterations"])
    return min(counts) - 1, max(counts) + 1


def _true_rel(s_scaled, x):
    r0 = O.true_resid(s_scaled, np.zeros(s_scaled.n))
    return O.true_resid(s_scaled, x) / r0 if r0 > 0 else 0.0


SOLVES = [
    ("conv3d_20", lambda: S.conv_diff(20, 20, 20, seed=0), "RSRS", "LINE"),
    ("conv3d_uneven", lambda: S.conv_diff(17, 31, 9, seed=1), "RSRS", "LINE"),
    ("conv2d", lambda: S.conv_diff(40, 33, 1, seed=2, do_k=False), "RSRS", "LINE"),
    ("pressure", lambda: S.pressure_like(18, 24, 14, seed=3, nspheres=5, rmin=2, rmax=5, itmax=2000), "RSRS", "LINE"),
    ("kat", lambda: S.known_answer(12, 14, 10, seed=4)[0], "RSRS", "LINE"),
    ("diag", lambda: S.conv_diff(12, 12, 12, seed=5), "RSRS", "DIAG"),
    ("none", lambda: S.conv_diff(10, 12, 8, seed=6), "RSRS", "NONE"),
    ("isis", lambda: S.conv_diff(11, 13, 7, seed=7), "ISIS", "LINE"),
    ("asas", lambda: S.conv_diff(9, 10, 8, seed=8), "ASAS", "LINE"),
    # JMAX2 = 602: lines longer than the autotuner's 17 rows per lane at 32 lanes
    ("long_lines", lambda: S.conv_diff(4, 600, 3, seed=14), "RSRS", "LINE"),
]


@pytest.mark.parametrize("name,make,sweep,pc", SOLVES, ids=[c[0] for c in SOLVES])
def test_drop_in_matches_oracle(name, make, sweep, pc):
    s = make()
    ref, st_ref, gpu, ier, st = _run_both(s, sweep, pc)
    assert ier == st_ref["ier"] == 0, (ier, st_ref, leq.last_error())
    assert st["exit_kind"] == st_ref["exit_kind"]
    lo, hi = _envelope(s, sweep, pc)
    assert lo <= st["iterations"] <= hi, (st["iterations"], lo, hi)
    # unit scaling written back exactly as LEQ_BICGS0 leaves A_M / B_M
    assert np.array_equal(gpu.a, ref.a) and np.array_equal(gpu.b, ref.b)
    assert _true_rel(ref, gpu.x) <= s.tol * 1.01 + 1e-15
    truth = ref.copy()
    truth.x[:] = 0.0
    x_truth, rel = O.truth(truth)
    assert rel <= 1e-13
    nt = np.linalg.norm(x_truth)
    err_ref = np.linalg.norm(ref.x - x_truth) / nt
    err_gpu = np.linalg.norm(gpu.x - x_truth) / nt
    assert err_gpu <= max(10 * err_ref, 1e-10), (err_gpu, err_ref)
    assert leq.iter_tot(3) == st["iter_tot_add"]
    if st["exit_kind"] == 0:  # converged on Rnorm: ITER_TOT += ITER + 1 (model/leq_bicgs.f:458)
        assert st["iter_tot_add"] == st["iterations"] + 1


def test_known_answer_recovers_x():
    s, x_act = S.known_answer(16, 18, 14, seed=11)
    ier = leq.solve_system(s)
    assert ier == 0
    assert np.linalg.norm(s.x - x_act) / np.linalg.norm(x_act) < 1e-8


def test_ier_singular_row():
    s = S.conv_diff(8, 8, 8, seed=12)
    p = 3 + 3 * s.jmax2 + 3 * s.jmax2 * s.imax2
    s.a[:, p] = 0.0
    ref = s.copy()
    st_ref = O.leq_bicgs(ref)
    ier = leq.solve_system(s)
    assert ier == st_ref["ier"] == -2
    assert leq.last_stats()["exit_kind"] == 4
    assert np.array_equal(s.a, ref.a) and np.array_equal(s.b, ref.b)  # all other rows scaled


def test_ier_zero_rhs_converged_immediately():
    s = S.conv_diff(8, 9, 7, seed=13)
    s.b[:] = 0.0
    ier = leq.solve_system(s)
    assert ier == 0 and leq.last_stats()["exit_kind"] == 2
    assert not s.x.any()


@pytest.mark.parametrize("itmax", [0, 1, 3])
def test_ier_itmax_exhausted(itmax):
    s = S.pressure_like(16, 16, 16, seed=14, nspheres=3, rmin=2, rmax=4)
    s.itmax = itmax
    ref, st_ref, gpu, ier, st = _run_both(s)
    assert ier == st_ref["ier"]
    assert st["iterations"] == st_ref["iterations"]
    assert st["iter_tot_add"] == st_ref["iter_tot_add"]


def test_unsupported_method_and_pc():
    s = S.conv_diff(6, 6, 6, seed=15)
    assert leq.solve_system(s.copy(), method=6) == leq.IER_UNSUPPORTED
    assert leq.solve_system(s.copy(), pc="line") == leq.IER_UNSUPPORTED
    assert leq.solve_system(s.copy(), pc="ILU ") == leq.IER_UNSUPPORTED


def test_phase_slice_m():
    """A_M(:,:,M) / B_M(:,M) are found from the whole arrays and M."""
    s0 = S.conv_diff(9, 10, 8, seed=16)
    s1 = S.conv_diff(9, 10, 8, seed=17)
    a_m = np.stack([s0.a, s1.a])
    b_m = np.stack([s0.b, s1.b])
    assert leq.init_geometry(s0.imax2, s0.jmax2, s0.kmax2, 1, s0.n, 1) == 0
    var = np.zeros(s0.n)
    ier = leq.solve_lin_eq("U_s", 3, var, a_m, b_m, 1, 500, 2, "RSRS", 1e-8, "LINE")
    assert ier == 0
    ref = s1.copy()
    O.leq_bicgs(ref)
    assert np.array_equal(a_m[1], ref.a) and np.array_equal(a_m[0], s0.a)  # only phase 1 scaled
    assert np.linalg.norm(var - ref.x) <= 1e-6 * np.linalg.norm(ref.x)


def test_solution_vs_truth():
    s = S.conv_diff(24, 24, 24, seed=18)
    ref = s.copy()
    O.scale(ref)
    x_truth, rel = O.truth(ref)
    assert rel <= 1e-13
    ier = leq.solve_system(s)
    assert ier == 0
    err = np.linalg.norm(s.x - x_truth) / np.linalg.norm(x_truth)
    assert err < 1e-6


def test_deferred_phase_calls_equal_single_calls():
    """The phases M = 0..2 of one A_M(:,:,0:DIMENSION_M), as the SIMPLE loop
    solves them back to back (model/solve_vel_star.f:308-331), deferred and
    flushed as one batch: each phase's result, IER and ITER_TOT contribution
    equal its single call's, bit for bit."""
    phases = [S.conv_diff(12, 15, 10, seed=70 + m) for m in range(3)]
    s0 = phases[0]
    n = s0.n
    a = np.ascontiguousarray(np.stack([p.a for p in phases]))  # A_M(DIMENSION_3, -3:3, 0:2)
    b = np.ascontiguousarray(np.stack([p.b for p in phases]))  # B_M(DIMENSION_3, 0:2)
    assert leq.init_geometry(s0.imax2, s0.jmax2, s0.kmax2, s0.do_k, n, 2) == 0
    a1, b1 = a.copy(), b.copy()
    x1 = [np.zeros(n) for _ in range(3)]
    t0 = leq.iter_tot(3)
    iers1 = [leq.solve_lin_eq("U_s", 3, x1[m], a1, b1, m, 500, 2, "RSRS", 1e-8, "LINE") for m in range(3)]
    single_tot = leq.iter_tot(3) - t0
    a2, b2 = a.copy(), b.copy()
    x2 = [np.zeros(n) for _ in range(3)]
    t0 = leq.iter_tot(3)
    cells = [leq.defer_lin_eq("U_s", 3, x2[m], a2, b2, m, 500, 2, "RSRS", 1e-8, "LINE") for m in range(3)]
    assert leq.pending_lin_eq() == 3
    assert leq.flush_lin_eq() == 0, leq.last_error()
    assert leq.pending_lin_eq() == 0
    assert [c.value for c in cells] == iers1 == [0, 0, 0]
    assert leq.iter_tot(3) - t0 == single_tot
    for m in range(3):
        assert np.array_equal(x1[m], x2[m])
    assert np.array_equal(a1, a2) and np.array_equal(b1, b2)  # every slice came back unit-scaled
