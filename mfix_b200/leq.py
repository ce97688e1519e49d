"""Python mirror of the reference's linear-solver interface over the C ABI.

``solve_lin_eq`` keeps SOLVE_LIN_EQ's dummy list and meaning
(model/solve_lin_eq.f:17-78): VAR is updated in place, A_M(:,:,M) and
B_M(:,M) come back unit-scaled as LEQ_BICGS0 leaves them
(model/leq_bicgs.f:194-233), and the return value is IER.  It calls the
gfortran-convention entry point ``mfixgpu_solve_lin_eq_`` exactly as a Fortran
host would, hidden CHARACTER lengths included.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import lib

IER_UNSUPPORTED = -10
IER_NOMEM = -11
IER_DGTSV = -12
IER_CUDA = -13
IER_ARGS = -14
IER_INCOMPLETE = -15
IER_NOGEOM = -16
IER_CANCELLED = -17

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class Stats(C.Structure):
    _fields_ = [("ier", C.c_int), ("iterations", C.c_int), ("iter_tot_add", C.c_int), ("exit_kind", C.c_int),
                ("line_skips", C.c_int), ("line_fallbacks", C.c_int), ("outer_steps", C.c_int), ("pad", C.c_int),
                ("rnorm0", C.c_double), ("rnorm", C.c_double), ("seconds", C.c_double), ("device_ms", C.c_double),
                ("jline_ms", C.c_double), ("jline_launches", C.c_int), ("fp64_fallback", C.c_int),
                ("kernel_launches", C.c_longlong), ("mixed_iterations", C.c_int), ("deflated", C.c_int)]


class Geom(C.Structure):
    _fields_ = [("imax2", C.c_int), ("jmax2", C.c_int), ("kmax2", C.c_int), ("do_k", C.c_int),
                ("dimension_3", C.c_int64), ("cyclic", C.c_int), ("pad", C.c_int)]


class SystemC(C.Structure):
    _fields_ = [("imax2", C.c_int), ("jmax2", C.c_int), ("kmax2", C.c_int), ("do_k", C.c_int),
                ("dimension_3", C.c_int64), ("a_m", C.c_void_p), ("b_m", C.c_void_p), ("var", C.c_void_p),
                ("tol", C.c_double), ("itmax", C.c_int), ("ier", C.c_int), ("iterations", C.c_int),
                ("outer_steps", C.c_int), ("exit_kind", C.c_int), ("fp64_fallback", C.c_int),
                ("rnorm0", C.c_double), ("rnorm", C.c_double)]


class ServerConfigC(C.Structure):
    _fields_ = [("precision", C.c_int), ("max_systems", C.c_int), ("check_every", C.c_int), ("device", C.c_int),
                ("hbm_budget", C.c_double), ("inner_tol", C.c_double), ("sweep", C.c_char * 4),
                ("pc", C.c_char * 4)]


class RequestC(C.Structure):
    _fields_ = [("status", C.c_int), ("ier", C.c_int), ("iterations", C.c_int), ("iter_tot_add", C.c_int),
                ("exit_kind", C.c_int), ("outer_steps", C.c_int), ("fp64_fallback", C.c_int),
                ("mixed_iterations", C.c_int), ("rnorm0", C.c_double), ("rnorm", C.c_double),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_start", C.c_double), ("t_done", C.c_double)]


class ServerCountersC(C.Structure):
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong), ("queued", C.c_longlong),
                ("copying", C.c_longlong), ("running", C.c_longlong), ("commits", C.c_longlong),
                ("iterations", C.c_longlong), ("kernel_launches", C.c_longlong), ("fp64_fallbacks", C.c_longlong),
                ("max_running", C.c_longlong), ("reserved_bytes", C.c_double), ("peak_reserved_bytes", C.c_double),
                ("budget_bytes", C.c_double), ("seconds", C.c_double), ("busy_ms", C.c_double * 2)]


class PPFieldsC(C.Structure):
    """mfixgpu_pp_fields: the fields SOLVE_PP_G assembles the pressure correction from."""
    _fields_ = [("flag", C.c_void_p), ("rop_ge", C.c_void_p), ("rop_gn", C.c_void_p), ("rop_gt", C.c_void_p),
                ("ayz", C.c_void_p), ("axz", C.c_void_p), ("axy", C.c_void_p), ("u_g", C.c_void_p),
                ("v_g", C.c_void_p), ("w_g", C.c_void_p), ("rop_g", C.c_void_p), ("rop_go", C.c_void_p),
                ("vol", C.c_void_p), ("sum_r_g", C.c_void_p), ("d_e", C.c_void_p), ("d_n", C.c_void_p),
                ("d_t", C.c_void_p), ("mmax", C.c_int), ("ro_g0_defined", C.c_int), ("close_packed", C.c_void_p),
                ("rop_se", C.c_void_p), ("rop_sn", C.c_void_p), ("rop_st", C.c_void_p), ("u_s", C.c_void_p),
                ("v_s", C.c_void_p), ("w_s", C.c_void_p), ("rop_s", C.c_void_p), ("rop_so", C.c_void_p),
                ("sum_r_s", C.c_void_p), ("odt", C.c_double), ("ijk_p_g", C.c_longlong), ("on_device", C.c_int),
                ("pad", C.c_int)]


PP_ARRAYS = ("flag", "rop_ge", "rop_gn", "rop_gt", "ayz", "axz", "axy", "u_g", "v_g", "w_g", "rop_g", "rop_go", "vol",
             "sum_r_g", "d_e", "d_n", "d_t", "rop_se", "rop_sn", "rop_st", "u_s", "v_s", "w_s", "rop_s", "rop_so",
             "sum_r_s")


def pp_struct(f, device_ptrs: dict | None = None) -> PPFieldsC:
    """The C record of a :class:`mfix_b200.systems.PPFields` (host arrays), or of
    device pointers given by name in device_ptrs (on_device set)."""
    c = PPFieldsC()
    for name in PP_ARRAYS:
        if device_ptrs is not None:
            setattr(c, name, device_ptrs.get(name) or None)
        else:
            arr = getattr(f, name)
            setattr(c, name, arr.ctypes.data if arr is not None else None)
    c.mmax = f.mmax
    c.ro_g0_defined = 1
    c.close_packed = f.close_packed.ctypes.data if f.mmax > 0 else None
    c.odt = f.odt
    c.ijk_p_g = f.ijk_p_g
    c.on_device = 1 if device_ptrs is not None else 0
    return c


def conv_source_pp_g(f, a_m, b_m, b_mmax, device_ptrs: dict | None = None) -> int:
    """mfixgpu_conv_source_pp_g: A_M(:,:,0), B_M(:,0), B_MMAX(:,0) assembled on the device
    (numpy arrays, or device addresses with device_ptrs)."""
    c = pp_struct(f, device_ptrs)
    if device_ptrs is not None:
        return lib().mfixgpu_conv_source_pp_g(C.byref(c), a_m, b_m, b_mmax)
    return lib().mfixgpu_conv_source_pp_g(C.byref(c), _ptr(a_m), _ptr(b_m), _ptr(b_mmax))


def solve_pp_g(f, normg: float, pp_g: np.ndarray, itmax: int = 500, method: int = 2, sweep: str = "RSRS",
               tol: float = 1e-8, pc: str = "LINE") -> tuple[int, float]:
    """SOLVE_PP_G(NORMG, RESG, IER) through mfixgpu_solve_pp_g_ with equation 1's LEQ settings:
    returns (IER, RESG); PP_G is written in place."""
    c = pp_struct(f)
    ier = C.c_int(0)
    resg = C.c_double(0.0)
    lib().mfixgpu_solve_pp_g_(C.byref(c), C.byref(C.c_double(normg)), _ptr(pp_g), C.byref(resg),
                              C.byref(C.c_int(itmax)), C.byref(C.c_int(method)), sweep.encode(),
                              C.byref(C.c_double(tol)), pc.encode(), C.byref(ier), len(sweep), len(pc))
    return ier.value, resg.value


REQ_ZERO_GUESS = 1
REQ_WRITE_AB = 2
REQ_ON_DEVICE = 4


def _declare(L: C.CDLL) -> None:
    L.mfixgpu_last_kernel_times.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_longlong), C.c_int]
    L.mfixgpu_last_kernel_times.restype = C.c_int
    L.mfixgpu_server_create.argtypes = [C.POINTER(ServerConfigC), C.POINTER(C.c_void_p)]
    L.mfixgpu_server_create.restype = C.c_int
    L.mfixgpu_server_submit.argtypes = [C.c_void_p, C.POINTER(SystemC), C.c_int]
    L.mfixgpu_server_submit.restype = C.c_longlong
    L.mfixgpu_server_poll.argtypes = [C.c_void_p, C.c_longlong, C.POINTER(RequestC)]
    L.mfixgpu_server_poll.restype = C.c_int
    L.mfixgpu_server_wait.argtypes = [C.c_void_p, C.c_longlong, C.c_double, C.POINTER(RequestC)]
    L.mfixgpu_server_wait.restype = C.c_int
    L.mfixgpu_server_wait_any.argtypes = [C.c_void_p, C.c_double, C.POINTER(C.c_longlong), C.POINTER(RequestC)]
    L.mfixgpu_server_wait_any.restype = C.c_int
    L.mfixgpu_server_counters_get.argtypes = [C.c_void_p, C.POINTER(ServerCountersC)]
    L.mfixgpu_server_counters_get.restype = C.c_int
    L.mfixgpu_server_cancel_queued.argtypes = [C.c_void_p]
    L.mfixgpu_server_cancel_queued.restype = C.c_int
    L.mfixgpu_server_destroy.argtypes = [C.c_void_p]
    L.mfixgpu_server_destroy.restype = C.c_int
    L.mfixgpu_init_geometry.argtypes = [_ip, _ip, _ip, _ip, C.POINTER(C.c_int64), _ip]
    L.mfixgpu_init_geometry.restype = C.c_int
    L.mfixgpu_init_cyclic.argtypes = [_ip, _ip, _ip]
    L.mfixgpu_init_cyclic.restype = C.c_int
    L.mfixgpu_solve_lin_eq_.argtypes = [C.c_char_p, _ip, C.c_void_p, C.c_void_p, C.c_void_p, _ip, _ip, _ip,
                                        C.c_char_p, _dp, C.c_char_p, _ip, C.c_size_t, C.c_size_t, C.c_size_t]
    L.mfixgpu_solve_lin_eq_.restype = None
    L.mfixgpu_solve_lin_eq.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                       C.c_int, C.c_int, C.c_char_p, C.c_int, C.c_double, C.c_char_p, C.c_int, _ip]
    L.mfixgpu_solve_lin_eq.restype = None
    L.mfixgpu_solve_lin_eq_defer_.argtypes = L.mfixgpu_solve_lin_eq_.argtypes
    L.mfixgpu_solve_lin_eq_defer_.restype = None
    L.mfixgpu_solve_lin_eq_flush.argtypes = []
    L.mfixgpu_solve_lin_eq_flush.restype = C.c_int
    L.mfixgpu_solve_lin_eq_pending.argtypes = []
    L.mfixgpu_solve_lin_eq_pending.restype = C.c_int
    L.mfixgpu_iter_tot.argtypes = [C.c_int]
    L.mfixgpu_iter_tot.restype = C.c_int
    L.mfixgpu_reset_iter_tot.argtypes = []
    L.mfixgpu_reset_iter_tot.restype = None
    L.mfixgpu_last_stats.argtypes = [C.POINTER(Stats)]
    L.mfixgpu_last_stats.restype = C.c_int
    L.mfixgpu_last_error.argtypes = []
    L.mfixgpu_last_error.restype = C.c_char_p
    L.mfixgpu_set_option.argtypes = [C.c_char_p, C.c_double]
    L.mfixgpu_set_option.restype = C.c_int
    L.mfixgpu_get_option.argtypes = [C.c_char_p]
    L.mfixgpu_get_option.restype = C.c_double
    L.mfixgpu_finalize.argtypes = []
    L.mfixgpu_finalize.restype = None
    L.mfixgpu_leq_matvec.argtypes = [C.POINTER(Geom), C.c_void_p, C.c_void_p, C.c_void_p]
    L.mfixgpu_leq_matvec.restype = C.c_int
    L.mfixgpu_leq_msolve.argtypes = [C.POINTER(Geom), C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_char_p]
    L.mfixgpu_leq_msolve.restype = C.c_int
    L.mfixgpu_dot_product_par.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, _dp]
    L.mfixgpu_dot_product_par.restype = C.c_int
    L.mfixgpu_batch_solve.argtypes = [C.POINTER(SystemC), C.c_int, C.c_char_p, C.c_char_p, C.c_int, C.c_int]
    L.mfixgpu_batch_solve.restype = C.c_int
    L.mfixgpu_dot_product_par_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    L.mfixgpu_dot_product_par_noalloc.restype = C.c_int
    L.mfixgpu_conv_source_pp_g.argtypes = [C.POINTER(PPFieldsC), C.c_void_p, C.c_void_p, C.c_void_p]
    L.mfixgpu_conv_source_pp_g.restype = C.c_int
    L.mfixgpu_solve_pp_g_.argtypes = [C.POINTER(PPFieldsC), _dp, C.c_void_p, _dp, _ip, _ip, C.c_char_p, _dp,
                                      C.c_char_p, _ip, C.c_size_t, C.c_size_t]
    L.mfixgpu_solve_pp_g_.restype = None
    L.mfixgpu_autotune_cache.argtypes = [C.c_char_p]
    L.mfixgpu_autotune_cache.restype = C.c_int
    L.mfixgpu_autotune_table.argtypes = [C.POINTER(C.c_int), C.c_int]
    L.mfixgpu_autotune_table.restype = C.c_int


def _ptr(a: np.ndarray) -> int:
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise TypeError("arrays must be C-contiguous float64 (Fortran A_M/B_M order)")
    return a.ctypes.data


def init_geometry(imax2: int, jmax2: int, kmax2: int, do_k: int, dimension_3: int, dimension_m: int = 0) -> int:
    """mfixgpu_init_geometry: the module data SOLVE_LIN_EQ relies on."""
    L = lib()
    return L.mfixgpu_init_geometry(C.byref(C.c_int(imax2)), C.byref(C.c_int(jmax2)), C.byref(C.c_int(kmax2)),
                                   C.byref(C.c_int(do_k)), C.byref(C.c_int64(dimension_3)),
                                   C.byref(C.c_int(dimension_m)))


def solve_lin_eq(vname: str, vno: int, var: np.ndarray, a_m: np.ndarray, b_m: np.ndarray, m: int, itmax: int,
                 method: int, sweep: str, tol1: float, pc: str) -> int:
    """SOLVE_LIN_EQ(VNAME, VNO, VAR, A_M, B_M, M, ITMAX, METHOD, SWEEP, TOL1, PC, IER) -> IER.

    ``a_m`` is A_M(DIMENSION_3, -3:3, 0:DIMENSION_M) in Fortran order, i.e. a
    C-contiguous array of shape (DIMENSION_M+1, 7, DIMENSION_3) (or (7, N) for
    one phase); ``b_m`` is B_M(DIMENSION_3, 0:DIMENSION_M) as (DIMENSION_M+1, N)
    (or (N,)).  VAR, A_M(:,:,M) and B_M(:,M) are updated in place.
    """
    L = lib()
    ier = C.c_int(0)
    vn = vname.encode()
    sw = sweep.encode()
    pcs = pc.encode()
    L.mfixgpu_solve_lin_eq_(vn, C.byref(C.c_int(vno)), _ptr(var), _ptr(a_m), _ptr(b_m), C.byref(C.c_int(m)),
                            C.byref(C.c_int(itmax)), C.byref(C.c_int(method)), sw, C.byref(C.c_double(tol1)), pcs,
                            C.byref(ier), len(vn), len(sw), len(pcs))
    return ier.value


def defer_lin_eq(vname: str, vno: int, var: np.ndarray, a_m: np.ndarray, b_m: np.ndarray, m: int, itmax: int,
                 method: int, sweep: str, tol1: float, pc: str) -> C.c_int:
    """mfixgpu_solve_lin_eq_defer_: SOLVE_LIN_EQ's arguments, queued for flush_lin_eq().
    Returns the IER cell (MFIXGPU_ERR_INCOMPLETE until the flush writes it); the
    arrays and the cell must stay alive and untouched until then."""
    L = lib()
    ier = C.c_int(0)
    vn, sw, pcs = vname.encode(), sweep.encode(), pc.encode()
    L.mfixgpu_solve_lin_eq_defer_(vn, C.byref(C.c_int(vno)), _ptr(var), _ptr(a_m), _ptr(b_m), C.byref(C.c_int(m)),
                                  C.byref(C.c_int(itmax)), C.byref(C.c_int(method)), sw, C.byref(C.c_double(tol1)),
                                  pcs, C.byref(ier), len(vn), len(sw), len(pcs))
    return ier


def flush_lin_eq() -> int:
    """mfixgpu_solve_lin_eq_flush: solve every deferred call; 0 or the first error code."""
    return lib().mfixgpu_solve_lin_eq_flush()


def pending_lin_eq() -> int:
    return lib().mfixgpu_solve_lin_eq_pending()


def last_stats() -> dict:
    s = Stats()
    lib().mfixgpu_last_stats(C.byref(s))
    return {k: getattr(s, k) for k, _ in Stats._fields_ if not k.startswith("pad")}


KERNEL_CLASSES = ("jline", "p_update", "matvec_alpha", "s_update", "matvec_omega", "xr_update", "outer_step",
                  "other_sweep")


def last_kernel_times() -> dict:
    """Per kernel class of the last solve (option time_kernels): (ms, launches)."""
    ms = (C.c_double * 16)()
    n = (C.c_longlong * 16)()
    k = lib().mfixgpu_last_kernel_times(ms, n, 16)
    return {KERNEL_CLASSES[q] if q < len(KERNEL_CLASSES) else str(q): (ms[q], n[q]) for q in range(k)}


def last_error() -> str:
    return lib().mfixgpu_last_error().decode()


def iter_tot(vno: int) -> int:
    return lib().mfixgpu_iter_tot(vno)


def reset_iter_tot() -> None:
    lib().mfixgpu_reset_iter_tot()


def set_option(name: str, value: float) -> int:
    return lib().mfixgpu_set_option(name.encode(), float(value))


def get_option(name: str) -> float:
    return lib().mfixgpu_get_option(name.encode())


def finalize() -> None:
    lib().mfixgpu_finalize()


def autotune_cache(path: str | None) -> int:
    """Read/write the J-line autotuner's choices from/to a JSON file."""
    return lib().mfixgpu_autotune_cache((path or "").encode())


def autotune_table() -> list[tuple[int, int, int]]:
    """(element bytes, line length, lanes per line) choices recorded so far."""
    n = lib().mfixgpu_autotune_table(None, 0)
    buf = (C.c_int * max(3 * n, 3))()
    n = lib().mfixgpu_autotune_table(buf, n)
    return [(buf[3 * q], buf[3 * q + 1], buf[3 * q + 2]) for q in range(n)]


def geom(imax2: int, jmax2: int, kmax2: int, do_k: int, cyclic: int = 0) -> Geom:
    return Geom(imax2, jmax2, kmax2, do_k, imax2 * jmax2 * kmax2, cyclic, 0)


def init_cyclic(cyclic_x: bool, cyclic_y: bool, cyclic_z: bool) -> int:
    """mfixgpu_init_cyclic: CYCLIC_X/Y/Z of the registered geometry."""
    return lib().mfixgpu_init_cyclic(C.byref(C.c_int(int(cyclic_x))), C.byref(C.c_int(int(cyclic_y))),
                                     C.byref(C.c_int(int(cyclic_z))))


def leq_matvec(g: Geom, a_dev: int, var_dev: int, avar_dev: int) -> int:
    """LEQ_MATVEC on device pointers (ints, e.g. torch.Tensor.data_ptr())."""
    return lib().mfixgpu_leq_matvec(C.byref(g), a_dev, var_dev, avar_dev)


def leq_msolve(g: Geom, b_dev: int, a_dev: int, var_dev: int, sweep: str = "RSRS", pc: str = "LINE") -> int:
    return lib().mfixgpu_leq_msolve(C.byref(g), b_dev, a_dev, var_dev, sweep.ljust(4)[:4].encode(),
                                    pc.ljust(4)[:4].encode())


def dot_product_par(r1_dev: int, r2_dev: int, n: int) -> float:
    out = C.c_double(0.0)
    rc = lib().mfixgpu_dot_product_par(r1_dev, r2_dev, n, C.byref(out))
    if rc:
        raise RuntimeError(f"mfixgpu_dot_product_par failed ({rc}): {last_error()}")
    return out.value


NOALLOC_MAX_N = 268435456  # MFIXGPU_NOALLOC_MAX_N


def dot_product_par_noalloc(r1_dev: int, r2_dev: int, n: int, out_dev: int, stream: int = 0) -> int:
    """mfixgpu_dot_product_par_noalloc: writes sum(r1*r2) to the device double at out_dev
    without allocating device memory.  Returns 0 or an error code."""
    return lib().mfixgpu_dot_product_par_noalloc(r1_dev, r2_dev, n, out_dev, stream or None)


@dataclass
class BatchResult:
    ier: int
    iterations: int
    outer_steps: int
    exit_kind: int
    rnorm0: float
    rnorm: float
    fp64_fallback: int = 0


def batch_solve(systems, sweep: str = "RSRS", pc: str = "LINE", precision: int = 0, on_device: bool = False,
                pointers=None):
    """mfixgpu_batch_solve over host :class:`mfix_b200.systems.System` objects (solved in
    place), or over device pointers given as ``pointers[q] = (a, b, x)`` with
    ``on_device=True``.  Returns (rc, [BatchResult...])."""
    arr = (SystemC * len(systems))()
    for q, s in enumerate(systems):
        arr[q].imax2, arr[q].jmax2, arr[q].kmax2, arr[q].do_k = s.imax2, s.jmax2, s.kmax2, s.do_k
        arr[q].dimension_3 = s.n
        if on_device:
            arr[q].a_m, arr[q].b_m, arr[q].var = pointers[q]
        else:
            arr[q].a_m, arr[q].b_m, arr[q].var = _ptr(s.a), _ptr(s.b), _ptr(s.x)
        arr[q].tol = s.tol
        arr[q].itmax = s.itmax
    rc = lib().mfixgpu_batch_solve(arr, len(systems), sweep.ljust(4)[:4].encode(), pc.ljust(4)[:4].encode(),
                                   int(precision), int(on_device))
    res = [BatchResult(arr[q].ier, arr[q].iterations, arr[q].outer_steps, arr[q].exit_kind, arr[q].rnorm0,
                       arr[q].rnorm, arr[q].fp64_fallback) for q in range(len(systems))]
    return rc, res


def solve_system(s, method: int = 2, sweep: str = "RSRS", pc: str = "LINE", vno: int = 1) -> int:
    """Drop-in solve of one :class:`mfix_b200.systems.System` (in place)."""
    rc = init_geometry(s.imax2, s.jmax2, s.kmax2, s.do_k, s.n, 0)
    cyc = getattr(s, "cyc", 0)
    if not rc and cyc:
        rc = init_cyclic(cyc & 1, cyc & 2, cyc & 4)
    if rc:
        return rc
    return solve_lin_eq("Test", vno, s.x, s.a, s.b, 0, s.itmax, method, sweep, s.tol, pc)


def _struct_dict(st) -> dict:
    out = {}
    for name, _ in st._fields_:
        if name.startswith("pad"):
            continue
        v = getattr(st, name)
        out[name] = list(v) if isinstance(v, C.Array) else v
    return out


class Server:
    """The request server (mfixgpu_server_*): continuous batching of solves.

    ``submit`` takes host arrays (or device pointers with ``on_device``) that
    must stay alive and untouched until the request is done; results come back
    as dicts with the IER fields and the server-clock times t_submit, t_admit,
    t_start and t_done."""

    def __init__(self, precision: int = 1, max_systems: int = 256, check_every: int = 4, hbm_budget: float = 0.0,
                 sweep: str = "RSRS", pc: str = "LINE", device: int = 0, inner_tol: float = 0.0):
        cfg = ServerConfigC(int(precision), int(max_systems), int(check_every), int(device), float(hbm_budget),
                            float(inner_tol), sweep.ljust(4)[:4].encode(), pc.ljust(4)[:4].encode())
        h = C.c_void_p()
        rc = lib().mfixgpu_server_create(C.byref(cfg), C.byref(h))
        if rc:
            raise RuntimeError(f"mfixgpu_server_create: {rc} ({last_error()})")
        self._h = h
        self._keep: dict[int, tuple] = {}

    def submit(self, s, zero_guess: bool = False, write_ab: bool = False, on_device: bool = False,
               pointers=None) -> int:
        """Queues System ``s`` (host arrays) or, with ``on_device``, the device
        pointers ``pointers = (a, b, x)``.  Returns the ticket (>= 0) or an error code."""
        c = SystemC()
        c.imax2, c.jmax2, c.kmax2, c.do_k = s.imax2, s.jmax2, s.kmax2, s.do_k
        c.dimension_3 = s.n
        if on_device:
            c.a_m, c.b_m, c.var = pointers
        else:
            c.a_m, c.b_m, c.var = _ptr(s.a), _ptr(s.b), _ptr(s.x)
        c.tol = s.tol
        c.itmax = s.itmax
        flags = (REQ_ZERO_GUESS if zero_guess else 0) | (REQ_WRITE_AB if write_ab else 0) | \
                (REQ_ON_DEVICE if on_device else 0)
        t = int(lib().mfixgpu_server_submit(self._h, C.byref(c), flags))
        if t >= 0:
            self._keep[t] = (s, pointers)
        return t

    def _done(self, t: int, rc: int, r: RequestC):
        if rc == 1:
            self._keep.pop(t, None)
            return _struct_dict(r)
        if rc == 0:
            return None
        raise KeyError(f"ticket {t}: {rc}")

    def poll(self, t: int):
        r = RequestC()
        return self._done(t, lib().mfixgpu_server_poll(self._h, t, C.byref(r)), r)

    def wait(self, t: int, timeout: float = -1.0):
        r = RequestC()
        return self._done(t, lib().mfixgpu_server_wait(self._h, t, float(timeout), C.byref(r)), r)

    def wait_any(self, timeout: float = -1.0):
        """(ticket, result) of a finished request nobody has collected, or None on timeout."""
        r = RequestC()
        t = C.c_longlong(-1)
        rc = lib().mfixgpu_server_wait_any(self._h, float(timeout), C.byref(t), C.byref(r))
        if rc != 1:
            return None
        self._keep.pop(t.value, None)
        return t.value, _struct_dict(r)

    def counters(self) -> dict:
        c = ServerCountersC()
        lib().mfixgpu_server_counters_get(self._h, C.byref(c))
        return _struct_dict(c)

    def cancel_queued(self) -> None:
        """Requests not yet admitted finish with IER_CANCELLED."""
        lib().mfixgpu_server_cancel_queued(self._h)

    def close(self) -> None:
        if self._h:
            lib().mfixgpu_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
