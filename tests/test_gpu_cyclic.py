"""Cyclic boxes (CYCLIC_X / CYCLIC_Y / CYCLIC_Z of a serial run).

The interior cells' neighbour increments wrap along the cyclic axes
(model/set_increments.f:73-113); the J-lines of the LINE preconditioner stay
open tridiagonals (model/leqsol_mod.f:907-909) whose right-hand sides take the
wrapped I and K neighbours.  Against the oracle (the same increments, checked
against an independent numpy restatement in the CPU tests): LEQ_MATVEC to
1e-13 and LEQ_MSOLVE (red/black and lexicographic letters) to 1e-12 on device
arrays (with an odd number of interior cells along a cyclic axis the first and
last interior lines share a red/black colour and run in the reference's serial
loop order); whole drop-in solves with the same IER, an iteration count inside the
oracle's rounding envelope, A_M / B_M scaled bit for bit, the true residual of
the scaled system <= 1.01 TOL and an error against a 1e-14 FP64 solution no
larger than ten times the oracle's own; the mixed form to TOL.
"""
import numpy as np
import pytest

import oracle as O
from mfix_b200 import leq
from mfix_b200 import systems as S

pytestmark = pytest.mark.gpu

CYCLIC = [
    ("x", lambda: S.conv_diff_cyclic(12, 15, 9, seed=40, cyc=1)),
    ("y", lambda: S.conv_diff_cyclic(10, 16, 8, seed=41, cyc=2)),
    ("z", lambda: S.conv_diff_cyclic(9, 13, 12, seed=42, cyc=4)),
    ("xyz", lambda: S.conv_diff_cyclic(11, 14, 10, seed=43, cyc=7)),
    ("xy_2d", lambda: S.conv_diff_cyclic(24, 21, 1, seed=44, cyc=3, do_k=False)),
    # odd numbers of interior cells: the wrapped lines share a red/black colour
    ("xz_odd", lambda: S.conv_diff_cyclic(11, 12, 9, seed=47, cyc=5)),
    ("x_2d_odd", lambda: S.conv_diff_cyclic(23, 14, 1, seed=48, cyc=1, do_k=False)),
]


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _rel(x, y):
    return float(np.max(np.abs(x - y)) / max(np.max(np.abs(y)), 1e-300))


@pytest.mark.parametrize("name,make", CYCLIC, ids=[c[0] for c in CYCLIC])
def test_cyclic_routines(cuda, name, make):
    s = make()
    g = leq.geom(s.imax2, s.jmax2, s.kmax2, s.do_k, cyclic=s.cyc)
    rng = np.random.default_rng(1)
    x = rng.standard_normal(s.n)
    da, dx = _dev(cuda, s.a), _dev(cuda, x)
    dy = cuda.empty(s.n, dtype=cuda.float64, device="cuda")
    assert leq.leq_matvec(g, da.data_ptr(), dx.data_ptr(), dy.data_ptr()) == 0, leq.last_error()
    assert _rel(dy.cpu().numpy(), O.matvec(s, x)) <= 1e-13
    sc = s.copy()
    O.scale(sc)
    dsa = _dev(cuda, sc.a)
    for sweep in ("RSRS", "ISIS"):
        rc, ref, _ = O.msolve(sc, x, sweep)
        assert rc == 0
        dv = cuda.empty(s.n, dtype=cuda.float64, device="cuda")
        assert leq.leq_msolve(g, dx.data_ptr(), dsa.data_ptr(), dv.data_ptr(), sweep) == 0, leq.last_error()
        assert _rel(dv.cpu().numpy(), ref) <= 1e-12, sweep


def _envelope(s):
    counts = []
    for eps in (0.0, 1e-15, -1e-15, 2e-15):
        t = s.copy()
        t.b *= 1.0 + eps
        counts.append(O.leq_bicgs(t)["iterations"])
    return min(counts) - 1, max(counts) + 1


@pytest.mark.parametrize("name,make", CYCLIC, ids=[c[0] for c in CYCLIC])
def test_cyclic_drop_in_matches_oracle(name, make):
    s = make()
    ref = s.copy()
    st_ref = O.leq_bicgs(ref)
    lo, hi = _envelope(s)
    gpu = s.copy()
    ier = leq.solve_system(gpu)
    st = leq.last_stats()
    assert ier == st_ref["ier"] == 0, leq.last_error()
    assert lo <= st["iterations"] <= hi, (st["iterations"], lo, hi)
    assert np.array_equal(gpu.a, ref.a) and np.array_equal(gpu.b, ref.b)
    r0 = O.true_resid(ref, np.zeros(s.n))
    assert O.true_resid(ref, gpu.x) <= 1.01 * s.tol * r0
    t = ref.copy()
    t.x[:] = 0.0
    x_truth, rel = O.truth(t)
    assert rel <= 1e-13
    nt = np.linalg.norm(x_truth)
    err_ref = np.linalg.norm(ref.x - x_truth) / nt
    assert np.linalg.norm(gpu.x - x_truth) / nt <= max(10 * err_ref, 1e-10)


def test_cyclic_mixed_form():
    s = S.conv_diff_cyclic(16, 18, 14, seed=45, cyc=7)
    ref = s.copy()
    O.leq_bicgs(ref)
    m = s.copy()
    assert leq.set_option("precision", 1) == 0
    try:
        ier = leq.solve_system(m)
        st = leq.last_stats()
    finally:
        leq.set_option("precision", 0)
    assert ier == 0 and st["fp64_fallback"] == 0, leq.last_error()
    r0 = O.true_resid(ref, np.zeros(s.n))
    assert O.true_resid(ref, m.x) <= 1.01 * s.tol * r0


def test_cyclic_sequential_letters():
    """ASAS (the I-, K- and J-line sweeps in the reference's loop orders) on a cyclic box."""
    s = S.conv_diff_cyclic(9, 10, 8, seed=46, cyc=5)
    ref = s.copy()
    st_ref = O.leq_bicgs(ref, "ASAS")
    gpu = s.copy()
    ier = leq.solve_system(gpu, sweep="ASAS")
    assert ier == st_ref["ier"] == 0, leq.last_error()
    assert np.linalg.norm(gpu.x - ref.x) <= 1e-6 * np.linalg.norm(ref.x)
