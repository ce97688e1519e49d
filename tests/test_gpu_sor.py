"""METHOD 1 (LEQ_SOR, model/leq_sor.f) through the drop-in entry point against
the oracle: rows scaled by 1/A(0) with A(0) set to one, bit for bit; VAR one
point-Jacobi step from the caller's VAR (every one of the ITMAX passes starts
from the same VAR and VAR takes the last pass once); ITER_TOT(VNO) set, not
increased, to ITMAX + 1; ITMAX = 0 leaves VAR alone."""
import numpy as np
import pytest

import oracle as O
from mfix_b200 import leq
from mfix_b200 import systems as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make", [lambda: S.conv_diff(13, 17, 11, seed=1),
                                  lambda: S.conv_diff(21, 19, 1, seed=5, do_k=False),
                                  lambda: S.known_answer(8, 40, 6, seed=4)[0]], ids=["3d", "2d", "kat"])
def test_sor_matches_oracle(cuda, make):
    s = make()
    s.x = np.random.default_rng(3).standard_normal(s.n)
    s.itmax = 7
    ref = s.copy()
    st_ref = O.leq_sor(ref)
    prime = s.copy()
    prime.itmax = 500
    assert leq.solve_system(prime, vno=5) == 0  # a BiCGSTAB solve adds to ITER_TOT(5) first
    assert leq.iter_tot(5) > 8
    got = s.copy()
    assert leq.solve_system(got, method=1, vno=5) == 0
    assert leq.iter_tot(5) == st_ref["iter_tot_add"] == 8  # set to ITMAX + 1
    assert np.array_equal(got.a, ref.a) and np.array_equal(got.b, ref.b)
    assert np.max(np.abs(got.x - ref.x)) <= 1e-14 * np.max(np.abs(ref.x))


def test_sor_itmax_zero_leaves_var(cuda):
    s = S.conv_diff(9, 10, 8, seed=2)
    s.x = np.full(s.n, 0.5)
    s.itmax = 0
    got = s.copy()
    assert leq.solve_system(got, method=1, vno=6) == 0
    assert np.all(got.x == 0.5) and leq.iter_tot(6) == 1
