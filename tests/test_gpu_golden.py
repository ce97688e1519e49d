"""The CUDA path against the committed golden fixtures (tests/golden).

Every LEQ_BICGS case runs through the drop-in entry point mfixgpu_solve_lin_eq_:
the same IER and exit reason, an iteration count inside the golden envelope
(widened by one), the unit-scaled A_M / B_M equal to the golden digests bit
for bit, and VAR within 1e-6 (relative) of the golden oracle solution (both
stop at a relative residual of 1e-8).  The DGTSV fixtures run as single
J-lines through LEQ_MSOLVE's LINE preconditioner: each line within 1e-12 of
LAPACK, and lines with an exact zero pivot left as SETGUESS leaves them
(model/leqsol_mod.f:910-914).
"""
import hashlib
import os

import numpy as np
import pytest

from mfix_b200 import leq

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def test_drop_in_matches_golden(cuda):
    from tests.golden.make_golden import CASES

    z = np.load(os.path.join(G, "leq_bicgs_small.npz"))
    cases = {c[0]: c for c in CASES}
    for nm in list(z["names"]):
        g = lambda f: z[f"{nm}__{f}"]
        _, make, sweep, pc = cases[nm]
        s = make()
        ier = leq.solve_system(s, sweep=sweep, pc=pc)
        st = leq.last_stats()
        assert ier == int(g("ier")) and st["exit_kind"] == int(g("exit_kind")), (nm, ier, leq.last_error())
        lo, hi = g("env")
        assert lo - 1 <= st["iterations"] <= hi + 1, (nm, st["iterations"], lo, hi)
        assert _sha(s.a) == str(g("a_sha")) and _sha(s.b) == str(g("b_sha")), nm
        gx = g("x")
        assert np.linalg.norm(s.x - gx) <= 1e-6 * np.linalg.norm(gx), nm


def test_jline_matches_lapack_golden(cuda):
    torch = cuda
    z = np.load(os.path.join(G, "dgtsv_lapack.npz"))
    offs = z["offs"]
    for q in range(len(offs) - 1):
        a0, a1 = int(offs[q]), int(offs[q + 1])
        n = a1 - a0
        # one J-line (IMAX2 = KMAX2 = 1, 2-D): A(-2) = DL shifted down, A(0) = D, A(2) = DU
        A = np.zeros((7, n))
        A[1, 1:] = z["dl"][a0:a1 - 1]
        A[3] = z["d"][a0:a1]
        A[5, :-1] = z["du"][a0:a1 - 1]
        b = z["b"][a0:a1].copy()
        da = torch.from_numpy(A).cuda()
        db = torch.from_numpy(b).cuda()
        dv = torch.zeros(n, dtype=torch.float64, device="cuda")
        rc = leq.leq_msolve(leq.geom(1, n, 1, 0), db.data_ptr(), da.data_ptr(), dv.data_ptr(), "R   ", "LINE")
        assert rc == 0, leq.last_error()
        got = dv.cpu().numpy()
        if int(z["info"][q]) == 0:
            ref = z["x"][a0:a1]
            assert np.max(np.abs(got - ref)) <= 1e-12 * max(np.max(np.abs(ref)), 1.0), q
        else:
            assert np.array_equal(got, b), q  # DGTSV INFO != 0: the line keeps VAR = B
