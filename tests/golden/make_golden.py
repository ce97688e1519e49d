"""Generates the golden fixtures of tests/golden (run from the repository root).

* dgtsv_lapack.npz: tridiagonal systems solved by LAPACK's dgtsv as scipy
  ships it, the routine the reference vendors as model/DGTSV.f (NRHS = 1):
  diagonally dominant lines, lines that force row interchanges, and exact
  zero pivots (INFO > 0).
* kat_systems.npz: the known-answer recipe of model/test_lin_eq.f:63-117
  (x_act and B = A x_act) on small boxes, with the oracle's LEQ_BICGS verdict.
* leq_bicgs_small.npz: small seeded systems of every generator, each with the
  oracle's LEQ_BICGS result (IER, ITER, ITER_TOT increment, exit kind, norms,
  VAR), the range of iteration counts the oracle gives when B_M is perturbed
  by a few ulps (BiCGSTAB's count is that sensitive), and SHA-256 digests of
  the unit-scaled A_M / B_M (model/leq_bicgs.f:194-233), which any
  implementation of the scaling must reproduce bit for bit.

    python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np
import scipy.linalg.lapack as lapack

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from mfix_b200 import systems as S  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def dgtsv_cases():
    rng = np.random.default_rng(20240)
    dl_all, d_all, du_all, b_all, x_all, info, offs = [], [], [], [], [], [], [0]
    for t in range(240):
        n = int(rng.integers(2, 41))
        dl, d, du, b = (rng.standard_normal(n - 1), rng.standard_normal(n), rng.standard_normal(n - 1),
                        rng.standard_normal(n))
        if t % 3 == 0:
            d = d * 8.0  # dominant: no interchanges
        if t % 40 == 7:  # exact zero pivot at a row
            k = int(rng.integers(0, n))
            d[k] = 0.0
            if k > 0:
                dl[k - 1] = 0.0
            if k < n - 1:
                du[k] = 0.0
        _, _, _, x, inf = lapack.dgtsv(dl, d, du, b.reshape(-1, 1))
        dl_all.append(np.append(dl, 0.0))
        du_all.append(np.append(du, 0.0))
        d_all.append(d)
        b_all.append(b)
        x_all.append(x.ravel() if inf == 0 else np.full(n, np.nan))
        info.append(inf)
        offs.append(offs[-1] + n)
    cat = np.concatenate
    np.savez_compressed(os.path.join(HERE, "dgtsv_lapack.npz"), dl=cat(dl_all), d=cat(d_all), du=cat(du_all),
                        b=cat(b_all), x=cat(x_all), info=np.array(info), offs=np.array(offs))


def envelope(s, sweep, pc):
    counts = []
    for eps in (0.0, 1e-15, -1e-15, 2e-15):
        t = s.copy()
        t.b *= (1.0 + eps)
        counts.append(O.leq_bicgs(t, sweep, pc)["iterations"])
    return min(counts), max(counts)


CASES = [
    # name, generator call, sweep, pc
    ("conv3d", lambda: S.conv_diff(8, 9, 7, seed=1), "RSRS", "LINE"),
    ("conv3d_odd_j", lambda: S.conv_diff(7, 11, 6, seed=2), "RSRS", "LINE"),
    ("conv2d", lambda: S.conv_diff(14, 12, 1, seed=3, do_k=False), "RSRS", "LINE"),
    ("pressure", lambda: S.pressure_like(9, 10, 8, seed=4, nspheres=2, rmin=1.5, rmax=3.0, itmax=2000), "RSRS", "LINE"),
    ("diag", lambda: S.conv_diff(7, 8, 6, seed=5), "RSRS", "DIAG"),
    ("none", lambda: S.conv_diff(6, 7, 5, seed=6), "RSRS", "NONE"),
    ("isis", lambda: S.conv_diff(6, 8, 5, seed=7), "ISIS", "LINE"),
    ("asas", lambda: S.conv_diff(6, 7, 6, seed=8), "ASAS", "LINE"),
]


def leq_cases():
    out = {}
    for name, make, sweep, pc in CASES:
        s = make()
        ref = s.copy()
        st = O.leq_bicgs(ref, sweep, pc)
        lo, hi = envelope(s, sweep, pc)
        out[name] = dict(dims=np.array([s.imax2, s.jmax2, s.kmax2, s.do_k]), sweep=sweep, pc=pc, tol=s.tol,
                         itmax=s.itmax, ier=st["ier"], iterations=st["iterations"],
                         iter_tot_add=st["iter_tot_add"], exit_kind=st["exit_kind"], rnorm0=st["rnorm0"],
                         rnorm=st["rnorm"], x=ref.x, env=np.array([lo, hi]), a_sha=sha(ref.a), b_sha=sha(ref.b),
                         a_in_sha=sha(s.a), b_in_sha=sha(s.b))
    flat = {f"{k}__{f}": v for k, d in out.items() for f, v in d.items()}
    np.savez_compressed(os.path.join(HERE, "leq_bicgs_small.npz"), names=np.array(list(out)), **flat)


def kat_cases():
    res = {}
    for q, dims in enumerate([(8, 10, 6), (12, 9, 1), (6, 14, 7)]):
        do_k = dims[2] > 1
        s, x_act = S.known_answer(*dims, seed=30 + q, do_k=do_k)
        ref = s.copy()
        st = O.leq_bicgs(ref)
        res[f"k{q}__dims"] = np.array([s.imax2, s.jmax2, s.kmax2, s.do_k])
        res[f"k{q}__seed"] = 30 + q
        res[f"k{q}__x_act"] = x_act
        res[f"k{q}__ier"] = st["ier"]
        res[f"k{q}__iterations"] = st["iterations"]
        res[f"k{q}__b_sha"] = sha(s.b)
    np.savez_compressed(os.path.join(HERE, "kat_systems.npz"), count=3, **res)


if __name__ == "__main__":
    dgtsv_cases()
    leq_cases()
    kat_cases()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
