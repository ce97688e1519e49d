"""METHOD 5 (LEQ_CG, model/leq_cg.f) through the drop-in entry point, against
the oracle's restatement on the same inputs.

Checked: the diagonal scaling of A_M/B_M bit for bit; IER, the exit and the
ITER_TOT contribution equal to the oracle's; iteration counts within one of
the oracle's (the GPU sums the dot products in another order); the solution
within 1e-6 of the oracle's and the true residual of the scaled system within
TOL; the rho = 0 exit, ITMAX = 0 and the divergence of CG on a non-symmetric
scaled operator (IER -2), as the reference has them.
"""
import numpy as np
import pytest

import oracle as O
from mfix_b200 import leq
from mfix_b200 import systems as S

pytestmark = pytest.mark.gpu

CASES = [
    ("sym3d", lambda: S.diffusion_sym(14, 20, 12, seed=5)),
    ("sym2d", lambda: S.diffusion_sym(21, 19, 1, seed=6, do_k=False)),
    ("sym_odd", lambda: S.diffusion_sym(9, 31, 7, seed=7)),
    ("sym_long_lines", lambda: S.diffusion_sym(6, 300, 5, seed=8)),
]


def _scaled(s):
    t = s.copy()
    O.scale_diag(t)
    return t


@pytest.mark.parametrize("pc", ["LINE", "DIAG", "NONE"])
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_cg_matches_oracle(cuda, name, make, pc):
    s = make()
    ref = s.copy()
    st_ref = O.leq_cg(ref, pc=pc)
    got = s.copy()
    before = leq.iter_tot(1)
    ier = leq.solve_system(got, method=5, pc=pc, vno=1)
    st = leq.last_stats()
    assert ier == st_ref["ier"] == 0, leq.last_error()
    assert st["exit_kind"] == st_ref["exit_kind"]
    assert abs(st["iterations"] - st_ref["iterations"]) <= 1
    assert leq.iter_tot(1) - before == st["iter_tot_add"] == st["iterations"] + 1
    assert np.array_equal(got.a, ref.a) and np.array_equal(got.b, ref.b)
    sc = _scaled(s)
    assert O.true_resid(sc, got.x) <= s.tol * O.true_resid(sc, np.zeros(s.n)) * 1.01
    assert np.linalg.norm(got.x - ref.x) <= 1e-6 * np.linalg.norm(ref.x)


def test_cg_rho_zero_and_itmax_zero(cuda):
    s = S.diffusion_sym(8, 9, 7, seed=1)
    z = s.copy()
    z.b[:] = 0.0
    assert leq.solve_system(z, method=5) == 0
    st = leq.last_stats()
    assert st["exit_kind"] == 2 and st["iter_tot_add"] == 0 and not np.any(z.x)
    t = s.copy()
    t.itmax = 0
    ref = s.copy()
    ref.itmax = 0
    st_ref = O.leq_cg(ref)
    assert leq.solve_system(t, method=5) == st_ref["ier"] == -1
    assert leq.last_stats()["iter_tot_add"] == st_ref["iter_tot_add"] == 1


def test_cg_diverges_like_the_reference(cuda):
    """Rows with different diagonals make the scaled operator non-symmetric and
    the reference's CG diverges; the drop-in reports the same IER -2 after the
    same ITMAX + 1 counter."""
    p = S.pressure_like(14, 20, 12, seed=3, nspheres=4, rmin=2, rmax=5, itmax=60)
    ref = p.copy()
    st_ref = O.leq_cg(ref)
    got = p.copy()
    assert leq.solve_system(got, method=5) == st_ref["ier"] == -2
    st = leq.last_stats()
    assert st["iterations"] == st_ref["iterations"] == 61 and st["iter_tot_add"] == 61


def test_cg_ignores_mixed_precision_option(cuda):
    s = S.diffusion_sym(12, 15, 10, seed=9)
    a, b = s.copy(), s.copy()
    assert leq.solve_system(a, method=5) == 0
    assert leq.set_option("precision", 1) == 0
    try:
        assert leq.solve_system(b, method=5) == 0
    finally:
        leq.set_option("precision", 0)
    assert np.array_equal(a.x, b.x)  # CG runs its FP64 form whatever the option


def test_unsupported_methods_still_refused(cuda):
    s = S.diffusion_sym(6, 6, 6, seed=2)
    for m in (6, 0, -1):
        assert leq.solve_system(s.copy(), method=m) == leq.IER_UNSUPPORTED
