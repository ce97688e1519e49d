"""Parity at the benchmark configurations, through the drop-in entry point.

The 64x64x64 convection-diffusion system (66^3 = 287,496 cells with the wall
layer, seed 0, LINE preconditioner, RSRS sweeps, ITMAX 500, TOL 1e-8) is the
configuration the reference's own CPU path runs.  It is solved through
mfixgpu_solve_lin_eq_ (gfortran's convention, the call a Fortran host makes)
in the FP64 drop-in and in the mixed form, and compared with the oracle (the
reference's LEQ_BICGS restated in C) on the same inputs:

* the same IER and exit reason;
* an iteration count inside the oracle's own rounding envelope (its counts
  when B_M is perturbed by 1e-15 relative) for the FP64 drop-in; the mixed
  form's inner count within 1.3x of the oracle's;
* the unit-scaled A_M / B_M written back bit for bit (model/leq_bicgs.f:194-233);
* the true relative residual ||b - A x|| / ||b - A x0|| of the scaled system
  <= 1.01 TOL (the reference tests its recursive residual, :455);
* the error against an FP64 solution solved to a true residual of 1e-14,
  ||x - x_truth|| / ||x_truth||, no larger than ten times the oracle's own error.

The 2-D 64x64 counterpart (NO_K, the LEQ_ISWEEP branch) is checked the same way.
"""
import numpy as np
import pytest

import oracle as O
from mfix_b200 import leq
from mfix_b200 import systems as S

pytestmark = pytest.mark.gpu


def _envelope(s):
    counts = []
    for eps in (0.0, 1e-15, -1e-15, 2e-15):
        t = s.copy()
        t.b *= 1.0 + eps
        counts.append(O.leq_bicgs(t)["iterations"])
    return min(counts) - 1, max(counts) + 1


def _true_rel(s_scaled, x):
    return O.true_resid(s_scaled, x) / O.true_resid(s_scaled, np.zeros(s_scaled.n))


@pytest.fixture(scope="module", params=["3d", "2d"])
def config(request):
    """The system, the oracle's solve of it, its iteration envelope and the 1e-14 truth."""
    if request.param == "3d":
        s = S.conv_diff(64, 64, 64, seed=0, itmax=500, tol=1e-8)
    else:
        s = S.conv_diff(64, 64, 1, seed=0, itmax=500, tol=1e-8, do_k=False)
    ref = s.copy()
    st_ref = O.leq_bicgs(ref)
    lo, hi = _envelope(s)
    t = ref.copy()
    t.x[:] = 0.0
    x_truth, rel = O.truth(t)
    assert rel <= 1e-13
    err_ref = np.linalg.norm(ref.x - x_truth) / np.linalg.norm(x_truth)
    return s, ref, st_ref, (lo, hi), x_truth, err_ref


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_config_matches_oracle(config, precision):
    s, ref, st_ref, (lo, hi), x_truth, err_ref = config
    assert st_ref["ier"] == 0
    gpu = s.copy()
    assert leq.set_option("precision", precision) == 0
    try:
        ier = leq.solve_system(gpu)
        st = leq.last_stats()
    finally:
        leq.set_option("precision", 0)
    assert ier == st_ref["ier"] == 0, leq.last_error()
    assert st["exit_kind"] == st_ref["exit_kind"] == 0
    if precision == 0:
        assert lo <= st["iterations"] <= hi, (st["iterations"], lo, hi)
    else:
        assert st["fp64_fallback"] == 0 and st["outer_steps"] >= 1
        assert st["iterations"] <= 1.3 * st_ref["iterations"] + 2
    assert np.array_equal(gpu.a, ref.a) and np.array_equal(gpu.b, ref.b)
    assert _true_rel(ref, gpu.x) <= s.tol * 1.01
    err = np.linalg.norm(gpu.x - x_truth) / np.linalg.norm(x_truth)
    assert err <= max(10 * err_ref, 1e-10), (err, err_ref)
    # and the two solutions agree with each other to the accuracy the tolerance allows
    assert np.linalg.norm(gpu.x - ref.x) / np.linalg.norm(ref.x) <= 20 * max(err_ref, 1e-10)
