"""The mixed-precision form and the batched solver on the GPU.

Mixed form (FP32 BiCGSTAB, FP64 solution accumulation and reliable updates):
IER 0, the FP64 true relative residual of the scaled system <= TOL, and a
solution within 1e-6 of the FP64 drop-in's, never handing over to FP64.  On the
well-conditioned convection-diffusion systems it takes no more than 1.3x the
FP64 iterations; the near-singular pressure-like systems (zero wall coupling,
diagonal excess 1e-6, so a diagonal-dominance margin of 1e-6) are deflated
(the constant mode over the coupled rows solved exactly in every
preconditioner application) and take no more iterations than the FP64 drop-in.
With deflation off they go to the FP64 drop-in before any FP32 iteration.
Batch: uneven systems solved together give results bit-identical to each
system solved alone, in both precisions.
"""
import numpy as np
import pytest

import oracle as O
from mfix_b200 import leq
from mfix_b200 import systems as S

pytestmark = pytest.mark.gpu


def _true_rel(s_scaled, x):
    return O.true_resid(s_scaled, x) / O.true_resid(s_scaled, np.zeros(s_scaled.n))


@pytest.mark.parametrize("make,near_singular", [
    (lambda: S.conv_diff(24, 30, 20, seed=0), False),
    (lambda: S.pressure_like(30, 40, 26, seed=1, nspheres=6, rmin=3, rmax=7, itmax=3000), True),
    (lambda: S.conv_diff(50, 41, 1, seed=2, do_k=False), False),
    (lambda: S.known_answer(14, 16, 12, seed=3)[0], False),
], ids=["conv3d", "pressure", "conv2d", "kat"])
def test_mixed_converges_to_tol(make, near_singular):
    s = make()
    ref = s.copy()
    st_ref = O.leq_bicgs(ref)
    m = s.copy()
    assert leq.set_option("precision", 1) == 0
    try:
        ier = leq.solve_system(m)
        st = leq.last_stats()
    finally:
        leq.set_option("precision", 0)
    assert ier == 0, leq.last_error()
    assert np.array_equal(m.a, ref.a) and np.array_equal(m.b, ref.b)
    assert _true_rel(ref, m.x) <= s.tol * 1.01
    assert np.linalg.norm(m.x - ref.x) <= 1e-6 * np.linalg.norm(ref.x)
    assert st["fp64_fallback"] == 0
    assert st["outer_steps"] >= 1
    assert st["deflated"] == (1 if near_singular else 0)
    if not near_singular:
        assert st["iterations"] <= 1.3 * st_ref["iterations"] + 2
    else:  # margin 1e-6 < 1e-4: deflated, and no slower than FP64 in iterations
        assert st["iterations"] <= st_ref["iterations"] + 2


def test_margin_routing_threshold():
    """The routing follows the options: below mixed_min_margin a system is
    deflated (default) or, with deflate = 0, solved by the FP64 drop-in before any
    FP32 iteration; with mixed_min_margin = 0 the pressure-like system is
    attempted in FP32 without deflation (and may still hand over later)."""
    s = S.pressure_like(20, 22, 18, seed=5, nspheres=3, rmin=2, rmax=4, itmax=3000)
    assert leq.get_option("deflate") == 1
    assert leq.set_option("precision", 1) == 0 and leq.set_option("deflate", 0) == 0
    try:
        m = s.copy()
        assert leq.solve_system(m) == 0
        st = leq.last_stats()
        assert st["fp64_fallback"] == 1 and st["mixed_iterations"] == 0 and st["deflated"] == 0
    finally:
        leq.set_option("deflate", 1)
        leq.set_option("precision", 0)
    assert leq.set_option("precision", 1) == 0 and leq.set_option("mixed_min_margin", 0.0) == 0
    try:
        m = s.copy()
        assert leq.solve_system(m) == 0
        st = leq.last_stats()
        assert st["deflated"] == 0
        assert st["fp64_fallback"] == 0 or st["mixed_iterations"] > 0
    finally:
        leq.set_option("mixed_min_margin", 1e-4)
        leq.set_option("precision", 0)
    c = S.conv_diff(20, 22, 18, seed=6)  # margin 1e-3: stays in the mixed form
    assert leq.set_option("precision", 1) == 0
    try:
        assert leq.solve_system(c) == 0
        assert leq.last_stats()["fp64_fallback"] == 0
    finally:
        leq.set_option("precision", 0)


def test_mixed_itmax_hands_over_to_fp64():
    """ITMAX spent in FP32 without reaching TOL: the FP64 drop-in re-solves from
    the initial guess and its verdict is the result, bit for bit."""
    s = S.conv_diff(20, 22, 18, seed=6, itmax=8)
    f = s.copy()
    ier_f = leq.solve_system(f)
    st_f = leq.last_stats()
    assert ier_f in (-1, -2)
    m = s.copy()
    assert leq.set_option("precision", 1) == 0
    try:
        ier_m = leq.solve_system(m)
        st_m = leq.last_stats()
    finally:
        leq.set_option("precision", 0)
    assert ier_m == ier_f, leq.last_error()
    assert st_m["fp64_fallback"] == 1 and st_m["iterations"] == st_f["iterations"]
    assert np.array_equal(m.x, f.x) and np.array_equal(m.a, f.a) and np.array_equal(m.b, f.b)


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_equals_alone(precision):
    sizes = [(9, 12, 7), (20, 15, 11), (5, 40, 6), (16, 16, 16), (31, 9, 4), (7, 7, 33)]
    systems = [S.conv_diff(*d, seed=q) for q, d in enumerate(sizes)]
    systems.append(S.pressure_like(14, 18, 12, seed=9, nspheres=3, rmin=2, rmax=4, itmax=2000))
    together = [s.copy() for s in systems]
    rc, res = leq.batch_solve(together, precision=precision)
    assert rc == 0, leq.last_error()
    for q, s in enumerate(systems):
        alone = s.copy()
        rc1, r1 = leq.batch_solve([alone], precision=precision)
        assert rc1 == 0
        assert res[q].ier == r1[0].ier == 0
        assert res[q].iterations == r1[0].iterations
        assert np.array_equal(together[q].x, alone.x)  # bit-identical alone and in the mix
        ref = s.copy()
        O.leq_bicgs(ref)
        assert _true_rel(ref, together[q].x) <= s.tol * 1.01


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_with_a_long_line(precision):
    # JMAX2 = 602: more than 17 rows per lane at every width, so the autotuner
    # gives that length 32 lanes (or one lane per line for all) while it times
    # the batch's other lengths; results as alone and within TOL
    systems = [S.conv_diff(4, 600, 3, seed=50), S.conv_diff(9, 20, 8, seed=51), S.conv_diff(6, 41, 5, seed=52)]
    together = [s.copy() for s in systems]
    rc, res = leq.batch_solve(together, precision=precision)
    assert rc == 0, leq.last_error()
    for q, s in enumerate(systems):
        alone = s.copy()
        rc1, r1 = leq.batch_solve([alone], precision=precision)
        assert rc1 == 0
        assert res[q].ier == r1[0].ier == 0
        assert res[q].iterations == r1[0].iterations
        assert np.array_equal(together[q].x, alone.x)
        ref = s.copy()
        O.leq_bicgs(ref)
        assert _true_rel(ref, together[q].x) <= s.tol * 1.01


def test_batch_rejects_sequential_letters():
    systems = [S.conv_diff(6, 6, 6, seed=q) for q in range(2)]
    rc, _ = leq.batch_solve(systems, sweep="ISIS")
    assert rc == leq.IER_UNSUPPORTED


@pytest.mark.parametrize("lanes", [1, 4])
@pytest.mark.parametrize("precision", [0, 1])
def test_forced_lanes_per_line(lanes, precision):
    """Every line kernel shape gives a correct solve: one lane per line (each lane
    runs a whole line) and the warp-cooperative shapes."""
    s = S.conv_diff(12, 31, 10, seed=40)
    ref = s.copy()
    st_ref = O.leq_bicgs(ref)
    assert leq.set_option("line_lanes", lanes) == 0 and leq.set_option("precision", precision) == 0
    try:
        m = s.copy()
        assert leq.solve_system(m) == 0, leq.last_error()
    finally:
        leq.set_option("line_lanes", 0)
        leq.set_option("precision", 0)
    assert np.array_equal(m.a, ref.a)
    assert _true_rel(ref, m.x) <= s.tol * 1.01
    assert np.linalg.norm(m.x - ref.x) <= 1e-6 * np.linalg.norm(ref.x)


def _pivoting(s, seed=0):
    """One row per J-line on a few lines with its diagonal shrunk a hundredfold:
    DGTSV takes a row interchange there, so those lines run the exact
    elimination (the system still converges)."""
    t = s.copy()
    rng = np.random.default_rng(seed)
    lines = rng.choice(t.imax2 * t.kmax2, size=6, replace=False)
    for li in lines:
        i, k = li % t.imax2, li // t.imax2
        if 0 < i < t.imax2 - 1 and 0 < k < t.kmax2 - 1:
            base = i * t.jmax2 + k * t.jmax2 * t.imax2
            t.a[3, base + int(rng.integers(2, t.jmax2 - 2))] *= 0.01
    return t


@pytest.mark.parametrize("lanes", [1, 32])
def test_pivoting_lines_each_shape(lanes):
    """J-lines on which DGTSV interchanges rows take the exact elimination in both
    line kernel shapes (one lane per line, 32 lanes per line), alone and batched."""
    s = _pivoting(S.conv_diff(14, 47, 12, seed=94), seed=3)
    ref = s.copy()
    st_ref = O.leq_bicgs(ref)
    assert leq.set_option("line_lanes", lanes) == 0
    try:
        m = s.copy()
        ier = leq.solve_system(m)
        st = leq.last_stats()
        pair = [s.copy(), S.conv_diff(9, 20, 8, seed=95)]
        rc, res = leq.batch_solve(pair, precision=0)
    finally:
        leq.set_option("line_lanes", 0)
    assert ier == st_ref["ier"] == 0, leq.last_error()
    assert st["line_fallbacks"] > 0
    assert np.array_equal(m.a, ref.a)
    assert _true_rel(ref, m.x) <= s.tol * 1.01
    assert np.linalg.norm(m.x - ref.x) <= 1e-6 * np.linalg.norm(ref.x)
    assert rc == 0 and res[0].ier == 0
    assert np.array_equal(pair[0].x, m.x)  # the same bits in a batch


def _scaled_ref(s):
    ref = s.copy()
    O.scale(ref)
    return ref
