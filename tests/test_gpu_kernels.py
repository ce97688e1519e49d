"""Per-routine parity of the CUDA kernels against the CPU oracle.

Each routine is called through its C entry point on device arrays and
compared with the oracle's restatement of the same reference routine:
LEQ_MATVEC, LEQ_MSOLVE for every sweep letter, LEQ_MSOLVE1 and
DOT_PRODUCT_PAR.  Tolerance: 1e-13 relative (max norm) for MATVEC and the
dot product, 1e-12 for the preconditioner (the GPU eliminates each line in a
different order than DGTSV; both are backward stable on these lines).
"""
import numpy as np
import pytest

import oracle as O
from mfix_b200 import leq
from mfix_b200 import systems as S

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _rel(x, y):
    return float(np.max(np.abs(x - y)) / max(np.max(np.abs(y)), 1e-300))


CASES = [
    ("conv3d", lambda: S.conv_diff(13, 17, 11, seed=1)),
    ("conv3d_odd", lambda: S.conv_diff(9, 30, 7, seed=2)),
    ("pressure3d", lambda: S.pressure_like(14, 20, 12, seed=3, nspheres=4, rmin=2, rmax=5)),
    ("kat", lambda: S.known_answer(8, 40, 6, seed=4)[0]),
    ("conv2d", lambda: S.conv_diff(21, 19, 1, seed=5, do_k=False)),
    ("long_lines", lambda: S.conv_diff(6, 384, 5, seed=6)),
    ("short_lines", lambda: S.conv_diff(10, 2, 10, seed=7)),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_matvec(cuda, name, make):
    s = make()
    rng = np.random.default_rng(0)
    x = rng.standard_normal(s.n)
    ref = O.matvec(s, x)
    da, dx = _dev(cuda, s.a), _dev(cuda, x)
    dy = cuda.empty(s.n, dtype=cuda.float64, device="cuda")
    rc = leq.leq_matvec(leq.geom(s.imax2, s.jmax2, s.kmax2, s.do_k), da.data_ptr(), dx.data_ptr(), dy.data_ptr())
    assert rc == 0, leq.last_error()
    assert _rel(dy.cpu().numpy(), ref) <= 1e-13


@pytest.mark.parametrize("n", [1, 7, 4096, 300_001])
def test_dot_product_par(cuda, n):
    rng = np.random.default_rng(n)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    ref = O.dot(x, y)
    dx, dy = _dev(cuda, x), _dev(cuda, y)  # keep both tensors alive across the call
    got = leq.dot_product_par(dx.data_ptr(), dy.data_ptr(), n)
    assert abs(got - ref) <= 1e-13 * max(1.0, float(np.abs(x * y).sum()))
    # fixed-order reduction: the same value every time
    got2 = leq.dot_product_par(dx.data_ptr(), dy.data_ptr(), n)
    assert got == got2


SWEEPS = ["RSRS", "RRRR", "R   ", "ISIS", "KSKS", "ASAS", "SRSR", "JSJS", "IRIS"]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("sweep", SWEEPS)
def test_msolve_line(cuda, name, make, sweep):
    s = make()
    if sweep.startswith("A") and s.imax2 * s.kmax2 > 20000:
        pytest.skip("ASAS schedule check kept to small grids")
    O.scale(s)  # the solver applies the preconditioner to the unit-scaled system
    rng = np.random.default_rng(1)
    b = rng.standard_normal(s.n)
    rc_ref, ref, _ = O.msolve(s, b, sweep, "LINE")
    assert rc_ref == 0
    da, db = _dev(cuda, s.a), _dev(cuda, b)
    dv = cuda.zeros(s.n, dtype=cuda.float64, device="cuda")
    rc = leq.leq_msolve(leq.geom(s.imax2, s.jmax2, s.kmax2, s.do_k), db.data_ptr(), da.data_ptr(), dv.data_ptr(),
                        sweep, "LINE")
    assert rc == 0, leq.last_error()
    assert _rel(dv.cpu().numpy(), ref) <= 1e-12


@pytest.mark.parametrize("pc", ["DIAG", "NONE"])
def test_msolve_diag_none(cuda, pc):
    s = S.conv_diff(11, 13, 9, seed=8)
    O.scale(s)
    b = np.random.default_rng(2).standard_normal(s.n)
    _, ref, _ = O.msolve(s, b, "RSRS", pc)
    da, db = _dev(cuda, s.a), _dev(cuda, b)
    dv = cuda.zeros(s.n, dtype=cuda.float64, device="cuda")
    rc = leq.leq_msolve(leq.geom(s.imax2, s.jmax2, s.kmax2, s.do_k), db.data_ptr(), da.data_ptr(), dv.data_ptr(),
                        "RSRS", pc)
    assert rc == 0, leq.last_error()
    assert np.array_equal(dv.cpu().numpy(), ref)  # b / A(0) and a copy are exact


def test_msolve_pivoting_lines(cuda):
    """Lines that are not diagonally dominant take the exact pivoting DGTSV path."""
    s = S.conv_diff(7, 25, 6, seed=9)
    O.scale(s)
    rng = np.random.default_rng(3)
    # make some J-couplings dominate their rows so DGTSV interchanges rows
    sel = rng.random(s.n) < 0.15
    s.a[1][sel] *= 6.0
    s.a[5][sel] *= 6.0
    b = rng.standard_normal(s.n)
    rc_ref, ref, skips = O.msolve(s, b, "RSRS", "LINE")
    da, db = _dev(cuda, s.a), _dev(cuda, b)
    dv = cuda.zeros(s.n, dtype=cuda.float64, device="cuda")
    rc = leq.leq_msolve(leq.geom(s.imax2, s.jmax2, s.kmax2, s.do_k), db.data_ptr(), da.data_ptr(), dv.data_ptr(),
                        "RSRS", "LINE")
    assert rc == 0
    assert _rel(dv.cpu().numpy(), ref) <= 1e-11


def test_msolve_singular_line_left_unchanged(cuda):
    """DGTSV INFO != 0 leaves the J-line as it was (model/leqsol_mod.f:910-914)."""
    s = S.conv_diff(6, 10, 5, seed=10)
    O.scale(s)
    n = s.n
    # zero the tridiagonal of one interior line -> exact zero pivot
    i, k = 3, 3
    base = (i - 1) * s.jmax2 + (k - 1) * s.jmax2 * s.imax2
    s.a[1][base:base + s.jmax2] = 0.0
    s.a[3][base:base + s.jmax2] = 0.0
    s.a[5][base:base + s.jmax2] = 0.0
    b = np.random.default_rng(4).standard_normal(n)
    rc_ref, ref, skips = O.msolve(s, b, "RSRS", "LINE")
    assert skips > 0
    da, db = _dev(cuda, s.a), _dev(cuda, b)
    dv = cuda.zeros(n, dtype=cuda.float64, device="cuda")
    rc = leq.leq_msolve(leq.geom(s.imax2, s.jmax2, s.kmax2, s.do_k), db.data_ptr(), da.data_ptr(), dv.data_ptr(),
                        "RSRS", "LINE")
    assert rc == 0
    got = dv.cpu().numpy()
    assert np.array_equal(got[base:base + s.jmax2], ref[base:base + s.jmax2])
    assert _rel(got, ref) <= 1e-12
