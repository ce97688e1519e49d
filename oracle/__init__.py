"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the CPU oracle (leq_oracle.c).

The oracle restates MFIX 2016-1's FP64 LEQ_BICGS path in C (see
leq_oracle.h for the reference lines each routine follows).  Only the tests,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may load
it; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_leq.so")
_lib = None

_dp = C.POINTER(C.c_double)


class Geom(C.Structure):
    _fields_ = [("imax2", C.c_int), ("jmax2", C.c_int), ("kmax2", C.c_int), ("do_k", C.c_int), ("n", C.c_int64),
                ("cyclic", C.c_int), ("pad", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("ier", C.c_int), ("iterations", C.c_int), ("iter_tot_add", C.c_int), ("exit_kind", C.c_int),
                ("line_info_skips", C.c_int), ("rnorm0", C.c_double), ("rnorm", C.c_double)]


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.orc_matvec.argtypes = [C.POINTER(Geom), vp, vp, vp]
        L.orc_dot.argtypes = [vp, vp, C.c_int64]
        L.orc_dot.restype = C.c_double
        L.orc_dgtsv.argtypes = [C.c_int, vp, vp, vp, vp]
        L.orc_dgtsv.restype = C.c_int
        L.orc_iksweep.argtypes = [C.POINTER(Geom), C.c_int, C.c_int, vp, vp, vp]
        L.orc_iksweep.restype = C.c_int
        L.orc_msolve.argtypes = [C.POINTER(Geom), vp, vp, vp, C.c_char_p, C.POINTER(C.c_int)]
        L.orc_msolve.restype = C.c_int
        L.orc_msolve1.argtypes = [C.POINTER(Geom), vp, vp, vp]
        L.orc_scale.argtypes = [C.POINTER(Geom), vp, vp]
        L.orc_scale.restype = C.c_int
        L.orc_uniform.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
        L.orc_uniform.restype = C.c_double
        L.orc_leq_bicgs.argtypes = [C.POINTER(Geom), vp, vp, vp, C.c_char_p, C.c_double, C.c_char_p, C.c_int,
                                    C.c_uint64, C.POINTER(Stats)]
        L.orc_leq_bicgs.restype = C.c_int
        L.orc_leq_bicgs_icheck.argtypes = [C.POINTER(Geom), vp, vp, vp, C.c_char_p, C.c_double, C.c_char_p,
                                           C.c_int, C.c_uint64, C.c_int, C.POINTER(Stats)]
        L.orc_leq_bicgs_icheck.restype = C.c_int
        L.orc_leq_bicgs_sample.argtypes = [C.POINTER(Geom), vp, vp, vp, C.c_char_p, C.c_double, C.c_char_p,
                                           C.c_int, C.c_uint64, C.c_int, C.POINTER(Stats)]
        L.orc_leq_bicgs_sample.restype = C.c_int
        L.orc_leq_cg.argtypes = [C.POINTER(Geom), vp, vp, vp, C.c_char_p, C.c_double, C.c_char_p, C.c_int,
                                 C.POINTER(Stats)]
        L.orc_leq_cg.restype = C.c_int
        L.orc_scale_diag.argtypes = [C.POINTER(Geom), vp, vp]
        L.orc_leq_gmres.argtypes = [C.POINTER(Geom), vp, vp, vp, C.c_char_p, C.c_double, C.c_int, C.POINTER(Stats)]
        L.orc_leq_gmres.restype = C.c_int
        L.orc_leq_sor.argtypes = [C.POINTER(Geom), vp, vp, vp, C.c_int, C.POINTER(Stats)]
        L.orc_leq_sor.restype = C.c_int
        L.orc_true_resid.argtypes = [C.POINTER(Geom), vp, vp, vp]
        L.orc_true_resid.restype = C.c_double
        L.orc_truth_solve.argtypes = [C.POINTER(Geom), vp, vp, vp, C.c_double, C.c_int, C.c_uint64, _dp]
        L.orc_truth_solve.restype = C.c_int
        L.orc_truth_refine.argtypes = [C.POINTER(Geom), vp, vp, vp, C.c_double, C.c_double, C.c_int, C.c_uint64, _dp]
        L.orc_truth_refine.restype = C.c_int
        L.orc_num_threads.restype = C.c_int
        L.orc_leq_bicgst.argtypes = [C.POINTER(Geom), vp, vp, vp, C.c_char_p, C.c_double, C.c_char_p, C.c_int,
                                     C.c_uint64, C.c_int, C.POINTER(Stats)]
        L.orc_leq_bicgst.restype = C.c_int
        L.orc_msolve_t.argtypes = [C.POINTER(Geom), vp, vp, vp, C.c_char_p, C.POINTER(C.c_int)]
        L.orc_msolve_t.restype = C.c_int
        L.orc_conv_source_pp_g.argtypes = [C.POINTER(Geom), C.c_void_p, vp, vp, vp]
        L.orc_calc_resid_pp.argtypes = [C.POINTER(Geom), vp, vp, C.c_double]
        L.orc_calc_resid_pp.restype = C.c_double
        _lib = L
    return _lib


def _p(a: np.ndarray) -> int:
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def geom(s) -> Geom:
    return Geom(s.imax2, s.jmax2, s.kmax2, s.do_k, s.n, getattr(s, "cyc", 0), 0)


def matvec(s, x: np.ndarray, a: np.ndarray | None = None) -> np.ndarray:
    y = np.empty(s.n)
    lib().orc_matvec(C.byref(geom(s)), _p(s.a if a is None else a), _p(x), _p(y))
    return y


def dot(x: np.ndarray, y: np.ndarray) -> float:
    return lib().orc_dot(_p(x), _p(y), x.size)


def dgtsv(dl: np.ndarray, d: np.ndarray, du: np.ndarray, b: np.ndarray):
    """DGTSV (NRHS=1) on copies; returns (info, x)."""
    dl, d, du, b = (np.ascontiguousarray(v, dtype=np.float64).copy() for v in (dl, d, du, b))
    n = d.size
    if n > 1:
        info = lib().orc_dgtsv(n, _p(dl), _p(d), _p(du), _p(b))
    else:
        z = np.zeros(1)
        info = lib().orc_dgtsv(n, _p(z), _p(d), _p(z), _p(b))
    return info, b


def msolve(s, b: np.ndarray, sweep: str = "RSRS", pc: str = "LINE", a: np.ndarray | None = None):
    """LEQ_MSOLVE (LINE) / LEQ_MSOLVE1 (DIAG) / copy (NONE); returns (rc, var, skips)."""
    var = np.zeros(s.n)
    A = s.a if a is None else a
    if pc == "DIAG":
        lib().orc_msolve1(C.byref(geom(s)), _p(b), _p(A), _p(var))
        return 0, var, 0
    if pc == "NONE":
        return 0, b.copy(), 0
    sk = C.c_int(0)
    rc = lib().orc_msolve(C.byref(geom(s)), _p(b), _p(A), _p(var), sweep.ljust(4)[:4].encode(), C.byref(sk))
    return rc, var, sk.value


def scale(s) -> int:
    """Unit scaling of s.a / s.b in place (model/leq_bicgs.f:194-233)."""
    return lib().orc_scale(C.byref(geom(s)), _p(s.a), _p(s.b))


def uniform(seed: int, tag: int, idx: int) -> float:
    return lib().orc_uniform(seed, tag, idx)


def leq_bicgs(s, sweep: str = "RSRS", pc: str = "LINE", seed: int = 0x5EED, max_exec: int | None = None,
              icheck: int = 0) -> dict:
    """LEQ_BICGS on s (in place: s.x solution, s.a / s.b scaled).  Returns the stats.
    icheck > 0: MINIMIZE_DOTPRODUCTS with ICHECK_BICGS = icheck."""
    st = Stats()
    sw = sweep.ljust(4)[:4].encode()
    pcs = pc.ljust(4)[:4].encode()
    if icheck > 0:
        lib().orc_leq_bicgs_icheck(C.byref(geom(s)), _p(s.x), _p(s.a), _p(s.b), sw, s.tol, pcs, s.itmax, seed,
                                   int(icheck), C.byref(st))
    elif max_exec is None:
        lib().orc_leq_bicgs(C.byref(geom(s)), _p(s.x), _p(s.a), _p(s.b), sw, s.tol, pcs, s.itmax, seed,
                            C.byref(st))
    else:
        lib().orc_leq_bicgs_sample(C.byref(geom(s)), _p(s.x), _p(s.a), _p(s.b), sw, s.tol, pcs, s.itmax, seed,
                                   max_exec, C.byref(st))
    return {k: getattr(st, k) for k, _ in Stats._fields_}


def leq_bicgst(s, sweep: str = "RSRS", pc: str = "LINE", seed: int = 0x5EED, minimize: bool = False) -> dict:
    """LEQ_BICGSt (DO_TRANSPOSE) on s: s.x solution, s.b scaled, s.a left as given.
    minimize: MINIMIZE_DOTPRODUCTS (the Rnorm test every fifth iteration)."""
    st = Stats()
    lib().orc_leq_bicgst(C.byref(geom(s)), _p(s.x), _p(s.a), _p(s.b), sweep.ljust(4)[:4].encode(), s.tol,
                         pc.ljust(4)[:4].encode(), s.itmax, seed, int(bool(minimize)), C.byref(st))
    return {k: getattr(st, k) for k, _ in Stats._fields_}


def msolve_t(s, b: np.ndarray, sweep: str = "RSRS", a: np.ndarray | None = None) -> np.ndarray:
    """LEQ_MSOLVEt on s's (scaled) A: var = M^{-1} b."""
    var = np.zeros(s.n)
    lib().orc_msolve_t(C.byref(geom(s)), _p(b), _p(s.a if a is None else a), _p(var), sweep.ljust(4)[:4].encode(),
                       None)
    return var


def leq_cg(s, sweep: str = "RSRS", pc: str = "LINE") -> dict:
    """LEQ_CG (METHOD 5) on s (in place: s.x solution, s.a / s.b scaled by the diagonal)."""
    st = Stats()
    lib().orc_leq_cg(C.byref(geom(s)), _p(s.x), _p(s.a), _p(s.b), sweep.ljust(4)[:4].encode(), s.tol,
                     pc.ljust(4)[:4].encode(), s.itmax, C.byref(st))
    return {k: getattr(st, k) for k, _ in Stats._fields_}


def leq_gmres(s, sweep: str = "RSRS") -> dict:
    """LEQ_GMRES (METHOD 3) on s (s.x updated; A and B untouched).  IER 0 or 1."""
    st = Stats()
    lib().orc_leq_gmres(C.byref(geom(s)), _p(s.x), _p(s.a), _p(s.b), sweep.ljust(4)[:4].encode(), s.tol, s.itmax,
                        C.byref(st))
    return {k: getattr(st, k) for k, _ in Stats._fields_}


def leq_sor(s) -> dict:
    """LEQ_SOR (METHOD 1) on s in place (rows scaled by 1/A(0), A(0) = 1; s.x one
    point-Jacobi step).  iter_tot_add is the value ITER_TOT(VNO) is set to."""
    st = Stats()
    lib().orc_leq_sor(C.byref(geom(s)), _p(s.x), _p(s.a), _p(s.b), s.itmax, C.byref(st))
    return {k: getattr(st, k) for k, _ in Stats._fields_}


def scale_diag(s) -> None:
    """LEQ_CG0's unit scaling of s in place (rows divided by their diagonal)."""
    lib().orc_scale_diag(C.byref(geom(s)), _p(s.a), _p(s.b))


def true_resid(s, x: np.ndarray, a: np.ndarray | None = None, b: np.ndarray | None = None) -> float:
    return lib().orc_true_resid(C.byref(geom(s)), _p(s.a if a is None else a), _p(s.b if b is None else b), _p(x))


def truth(s, rtol: float = 1e-14, max_steps: int = 60, seed: int = 0x7A7E) -> tuple[np.ndarray, float]:
    """FP64 solution of the (already scaled) system to a long-double true residual of rtol."""
    x = s.x.copy()
    rel = C.c_double(0.0)
    lib().orc_truth_solve(C.byref(geom(s)), _p(s.a), _p(s.b), _p(x), rtol, max_steps, seed, C.byref(rel))
    return x, rel.value


def truth_from(s, x0: np.ndarray, r0: float, rtol: float = 1e-14, max_steps: int = 60,
               seed: int = 0x7A7E) -> tuple[np.ndarray, float]:
    """Refines the guess x0 of the (already scaled) system until ||b - A x|| <= rtol * r0
    (long-double residuals); returns x and ||b - A x|| / r0."""
    x = np.array(x0, dtype=np.float64, copy=True)
    rel = C.c_double(0.0)
    lib().orc_truth_refine(C.byref(geom(s)), _p(s.a), _p(s.b), _p(x), float(r0), rtol, max_steps, seed, C.byref(rel))
    return x, rel.value


class PPFieldsC(C.Structure):
    _fields_ = [("flag", C.c_void_p), ("rop_ge", C.c_void_p), ("rop_gn", C.c_void_p), ("rop_gt", C.c_void_p),
                ("ayz", C.c_void_p), ("axz", C.c_void_p), ("axy", C.c_void_p), ("u_g", C.c_void_p),
                ("v_g", C.c_void_p), ("w_g", C.c_void_p), ("rop_g", C.c_void_p), ("rop_go", C.c_void_p),
                ("vol", C.c_void_p), ("sum_r_g", C.c_void_p), ("d_e", C.c_void_p), ("d_n", C.c_void_p),
                ("d_t", C.c_void_p), ("mmax", C.c_int), ("close_packed", C.c_void_p), ("rop_se", C.c_void_p),
                ("rop_sn", C.c_void_p), ("rop_st", C.c_void_p), ("u_s", C.c_void_p), ("v_s", C.c_void_p),
                ("w_s", C.c_void_p), ("rop_s", C.c_void_p), ("rop_so", C.c_void_p), ("sum_r_s", C.c_void_p),
                ("odt", C.c_double), ("ijk_p_g", C.c_longlong)]


def conv_source_pp_g(f):
    """CONV_PP_G + SOURCE_PP_G restated in C: (A_M(:,:,0) as (7, n), B_M(:,0), B_MMAX(:,0))."""
    c = PPFieldsC()
    for name, _ in PPFieldsC._fields_:
        if name in ("mmax", "odt", "ijk_p_g"):
            continue
        arr = getattr(f, name)
        setattr(c, name, arr.ctypes.data if arr is not None else None)
    c.mmax, c.odt, c.ijk_p_g = f.mmax, f.odt, f.ijk_p_g
    g = Geom(f.imax2, f.jmax2, f.kmax2, f.do_k, f.n)
    a = np.zeros((7, f.n))
    b = np.zeros(f.n)
    bm = np.zeros(f.n)
    lib().orc_conv_source_pp_g(C.byref(g), C.byref(c), _p(a), _p(b), _p(bm))
    return a, b, bm


def calc_resid_pp(f, b: np.ndarray, norm: float) -> float:
    """CALC_RESID_PP's RESID of b over the fluid cells."""
    g = Geom(f.imax2, f.jmax2, f.kmax2, f.do_k, f.n)
    return lib().orc_calc_resid_pp(C.byref(g), f.flag.ctypes.data, _p(b), norm)


def num_threads() -> int:
    return lib().orc_num_threads()
