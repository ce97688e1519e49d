"""The oracle against the committed golden fixtures (tests/golden, made by
tests/golden/make_golden.py): DGTSV bit for bit against LAPACK's dgtsv, the
known-answer systems of model/test_lin_eq.f, and LEQ_BICGS verdicts,
iteration envelopes and unit-scaled A_M / B_M digests on small systems."""
import hashlib
import os

import numpy as np
import pytest

import oracle as O
from mfix_b200 import systems as S

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def _load(name):
    return np.load(os.path.join(G, name), allow_pickle=False)


def test_dgtsv_matches_lapack_golden():
    z = _load("dgtsv_lapack.npz")
    offs = z["offs"]
    pivots = 0
    for q in range(len(offs) - 1):
        a, b = offs[q], offs[q + 1]
        n = b - a
        info, x = O.dgtsv(z["dl"][a:b - 1], z["d"][a:b], z["du"][a:b - 1], z["b"][a:b])
        assert info == z["info"][q]
        if info == 0:
            assert np.array_equal(x, z["x"][a:b]), q
        else:
            pivots += 1
    assert pivots >= 3  # the zero-pivot cases are in the set


def _cases():
    from tests.golden.make_golden import CASES  # the generator calls that made the fixtures
    return CASES


def test_leq_bicgs_matches_golden():
    z = _load("leq_bicgs_small.npz")
    names = list(z["names"])
    cases = {c[0]: c for c in _cases()}
    assert sorted(names) == sorted(cases)
    for nm in names:
        g = lambda f: z[f"{nm}__{f}"]
        _, make, sweep, pc = cases[nm]
        s = make()
        assert _sha(s.a) == str(g("a_in_sha")) and _sha(s.b) == str(g("b_in_sha")), nm  # generator pinned
        ref = s.copy()
        st = O.leq_bicgs(ref, sweep, pc)
        assert st["ier"] == int(g("ier")) and st["exit_kind"] == int(g("exit_kind")), nm
        lo, hi = g("env")
        assert lo <= st["iterations"] <= hi, nm
        assert _sha(ref.a) == str(g("a_sha")) and _sha(ref.b) == str(g("b_sha")), nm
        gx = g("x")
        # OpenMP reductions: the oracle's sums depend on its thread count
        assert np.linalg.norm(ref.x - gx) <= 1e-6 * np.linalg.norm(gx), nm


def test_known_answer_golden():
    z = _load("kat_systems.npz")
    for q in range(int(z["count"])):
        dims = z[f"k{q}__dims"]
        do_k = bool(dims[3])
        imax, jmax, kmax = int(dims[0]) - 2, int(dims[1]) - 2, (int(dims[2]) - 2 if do_k else 1)
        s, x_act = S.known_answer(imax, jmax, kmax, seed=int(z[f"k{q}__seed"]), do_k=do_k)
        assert np.array_equal(x_act, z[f"k{q}__x_act"])
        assert _sha(s.b) == str(z[f"k{q}__b_sha"])
        st = O.leq_bicgs(s)
        assert st["ier"] == int(z[f"k{q}__ier"]) == 0
        assert np.linalg.norm(s.x - x_act) / np.linalg.norm(x_act) < 1e-8
