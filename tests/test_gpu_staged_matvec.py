"""The mixed form's matvecs with operands staged by bulk copies.

k_matvec_staged streams the off-diagonals, the row sums, x and its line / plane
neighbours and the reduction's second vector into shared memory through
cp.async.bulk copies counted on mbarriers; each thread owns the same cells, in
the same order, as in the register-load kernels it replaces.  So a mixed-form
solve with "staged_matvec" 1 (x's i/k neighbour lines staged too) or 2 (read
from global memory) and with 0 gives the same solution bit for bit and
the same iteration counts: single systems (odd and even JMAX2, 2-D, cyclic axes
whose wrapped neighbours lie outside the staged windows, a deflated near-singular
system) and an uneven batch, several systems per block.
"""
import numpy as np
import pytest

import oracle as O
from mfix_b200 import leq
from mfix_b200 import systems as S

pytestmark = pytest.mark.gpu

CASES = [
    ("conv3d_even", lambda: S.conv_diff(30, 38, 22, seed=60)),
    ("conv3d_odd", lambda: S.conv_diff(27, 33, 19, seed=61)),
    ("conv2d", lambda: S.conv_diff(90, 71, 1, seed=62, do_k=False)),
    ("cyclic_xyz", lambda: S.conv_diff_cyclic(21, 26, 17, seed=63, cyc=7)),
    ("pressure", lambda: S.pressure_like(30, 40, 26, seed=64, nspheres=6, rmin=3, rmax=7, itmax=3000)),
]


def _mixed(s, staged):
    m = s.copy()
    assert leq.set_option("staged_matvec", staged) == 0
    assert leq.set_option("precision", 1) == 0
    try:
        ier = leq.solve_system(m)
        st = leq.last_stats()
    finally:
        leq.set_option("precision", 0)
        leq.set_option("staged_matvec", 2)
    return ier, st, m


@pytest.mark.parametrize("variant", [1, 2], ids=["windows", "no_windows"])
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_staged_matches_register_loads(name, make, variant):
    s = make()
    ier1, st1, m1 = _mixed(s, variant)
    ier0, st0, m0 = _mixed(s, 0)
    assert ier1 == ier0 == 0, leq.last_error()
    assert st1["iterations"] == st0["iterations"] and st1["outer_steps"] == st0["outer_steps"]
    assert st1["fp64_fallback"] == st0["fp64_fallback"] == 0
    assert np.array_equal(m1.x, m0.x)
    if name == "pressure":
        assert st1["deflated"] == 1
    ref = s.copy()
    O.scale(ref)
    r0 = O.true_resid(ref, np.zeros(s.n))
    assert O.true_resid(ref, m1.x) <= 1.01 * s.tol * r0


@pytest.mark.parametrize("variant", [1, 2], ids=["windows", "no_windows"])
def test_staged_batch_matches_register_loads(variant):
    sizes = [(17, 23, 13), (40, 12, 31), (9, 64, 9), (33, 33, 1), (26, 18, 21)]
    systems = [S.conv_diff(i, j, k, seed=70 + q, do_k=k > 1) for q, (i, j, k) in enumerate(sizes)]
    out = {}
    for staged in (variant, 0):
        batch = [t.copy() for t in systems]
        assert leq.set_option("staged_matvec", staged) == 0
        try:
            rc, res = leq.batch_solve(batch, precision=1)
        finally:
            leq.set_option("staged_matvec", 2)
        assert rc == 0, leq.last_error()
        assert all(r.ier == 0 for r in res)
        out[staged] = (batch, [r.iterations for r in res])
    assert out[variant][1] == out[0][1]
    for a, b in zip(out[variant][0], out[0][0]):
        assert np.array_equal(a.x, b.x)
