"""Seeded synthetic MFIX systems in the A_M / B_M layout.

Arrays follow the reference's Fortran storage: ``a`` has shape ``(7, N)`` with
``a[d + 3]`` the contiguous diagonal ``A_M(:, d)`` (so the buffer is exactly
``A_M(DIMENSION_3, -3:3)`` in column-major order); the cell index puts J
fastest, then I, then K (model/include/functions.inc:37-42), and the grid
carries the one-cell wall layer (model/set_max2.f:48-66).  Wall rows follow
INIT_AB_M (model/init_ab_m.f:20-78): ``A(0) = -1``, other diagonals 0, ``B = 0``.

Every random draw comes from a counter-based splitmix64 stream keyed by
(seed, tag, index), so any subset of a system can be regenerated and the
values do not depend on evaluation order.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_GOLD = 0x9E3779B97F4A7C15
_TAGK = 0xD1B54A32D192ED03
_OFF = 0x632BE59BD9B4E019
_MASK = (1 << 64) - 1


def _mix64(z: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def _mix64_int(z: int) -> int:
    z &= _MASK
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK
    return z ^ (z >> 31)


def uniform(seed: int, tag: int, idx) -> np.ndarray:
    """U[0,1) draws of stream (seed, tag) at counter positions ``idx``."""
    key = _mix64_int((seed * _GOLD + tag * _TAGK + _OFF) & _MASK)
    idx = np.asarray(idx, dtype=np.uint64)
    with np.errstate(over="ignore"):
        v = _mix64(np.uint64(key) + (idx + np.uint64(1)) * np.uint64(_GOLD))
    return (v >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


def normal(seed: int, tag: int, idx, sigma: float) -> np.ndarray:
    """N(0, sigma) by Box-Muller from streams (tag, tag+1)."""
    u1 = 1.0 - uniform(seed, tag, idx)  # (0, 1]
    u2 = uniform(seed, tag + 1, idx)
    return sigma * np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


@dataclass
class System:
    """One A_M / B_M / VAR triple on a box of (imax2, jmax2, kmax2) cells."""
    imax2: int
    jmax2: int
    kmax2: int
    do_k: int
    a: np.ndarray  # (7, n) float64
    b: np.ndarray  # (n,)
    x: np.ndarray  # (n,) initial guess
    tol: float = 1e-8
    itmax: int = 500
    kind: str = ""
    cyc: int = 0  # cyclic axes: 1 X (I), 2 Y (J), 4 Z (K)

    @property
    def n(self) -> int:
        return self.imax2 * self.jmax2 * self.kmax2

    def copy(self) -> "System":
        return System(self.imax2, self.jmax2, self.kmax2, self.do_k, self.a.copy(), self.b.copy(),
                      self.x.copy(), self.tol, self.itmax, self.kind, self.cyc)


def _grid(imax: int, jmax: int, kmax: int, do_k: bool):
    imax2, jmax2 = imax + 2, jmax + 2
    kmax2 = kmax + 2 if do_k else 1
    return imax2, jmax2, kmax2


def _interior(imax2, jmax2, kmax2, do_k):
    """Boolean [k, i, j] mask of interior (non wall-layer) cells."""
    k = np.arange(kmax2)[:, None, None]
    i = np.arange(imax2)[None, :, None]
    j = np.arange(jmax2)[None, None, :]
    m = (i >= 1) & (i <= imax2 - 2) & (j >= 1) & (j <= jmax2 - 2)
    if do_k:
        m = m & (k >= 1) & (k <= kmax2 - 2)
    return np.broadcast_to(m, (kmax2, imax2, jmax2))


def _assemble(imax2, jmax2, kmax2, do_k, face_fn, centre_factor, seed, b_tag):
    """Build A and B from a per-face coefficient function.

    face_fn(axis, low_idx, high_idx) -> (coef_in_low_row, coef_in_high_row) for
    the faces between interior cells along `axis` (0: I, 1: J, 2: K).
    """
    n = imax2 * jmax2 * kmax2
    shape = (kmax2, imax2, jmax2)
    a = np.zeros((7, n), dtype=np.float64)
    A = a.reshape(7, *shape)
    inter = _interior(imax2, jmax2, kmax2, do_k)
    flat = np.arange(n, dtype=np.int64).reshape(shape)
    # (axis, numpy axis of the [k,i,j] grid, diagonal index in low row, in high row)
    axes = [(0, 1, 1, -1), (1, 2, 2, -2)]
    if do_k:
        axes.append((2, 0, 3, -3))
    for axis, npax, d_low, d_high in axes:
        sl_lo = [slice(None)] * 3
        sl_hi = [slice(None)] * 3
        sl_lo[npax] = slice(0, shape[npax] - 1)
        sl_hi[npax] = slice(1, shape[npax])
        lo, hi = tuple(sl_lo), tuple(sl_hi)
        both = inter[lo] & inter[hi]  # faces touching the wall layer stay zero
        low_idx = flat[lo][both]
        high_idx = flat[hi][both]
        c_low, c_high = face_fn(axis, low_idx, high_idx)
        a[d_low + 3][low_idx] = c_low
        a[d_high + 3][high_idx] = c_high
    off = a[[0, 1, 2, 4, 5, 6]].sum(axis=0)
    wall = ~inter.reshape(-1)
    a[3] = -off * centre_factor
    a[:, wall] = 0.0
    a[3][wall] = -1.0
    b = 2.0 * uniform(seed, b_tag, np.arange(n)) - 1.0
    b[wall] = 0.0
    del A
    return a, b


def conv_diff(imax: int, jmax: int, kmax: int, seed: int = 0, do_k: bool = True, itmax: int = 500,
              tol: float = 1e-8) -> System:
    """3-D 7-point upwind convection-diffusion system (the 64^3 / 256^3 workloads).

    Per interior face between cells P (low) and Q (high): D ~ U[0.5, 1.5] and
    F ~ N(0, 0.5) (standard deviation 0.5); row P gets a_Q = D + max(-F, 0),
    row Q gets a_P = D + max(F, 0).  Faces touching the wall layer are zero;
    A(0) = -(sum of the remaining a_nb)(1 + 1e-3); B ~ U[-1, 1] on interior cells.
    """
    imax2, jmax2, kmax2 = _grid(imax, jmax, kmax, do_k)

    def face(axis, lo, hi):
        D = 0.5 + uniform(seed, 1 + 4 * axis, lo)
        F = normal(seed, 2 + 4 * axis, lo, 0.5)
        return D + np.maximum(-F, 0.0), D + np.maximum(F, 0.0)

    a, b = _assemble(imax2, jmax2, kmax2, do_k, face, 1.0 + 1e-3, seed, 20)
    return System(imax2, jmax2, kmax2, int(do_k), a, b, np.zeros(imax2 * jmax2 * kmax2), tol, itmax,
                  "conv_diff")


def diffusion_sym(imax: int, jmax: int, kmax: int, seed: int = 0, do_k: bool = True, delta: float = 1e-3,
                  itmax: int = 500, tol: float = 1e-8) -> System:
    """Symmetric 7-point diffusion, face coefficient D ~ U[0.5, 1.5], with one
    centre for every interior row: -(largest row sum)(1 + delta).  Dividing
    each row by its diagonal (LEQ_CG0's scaling, model/leq_cg.f:197-211) then
    keeps the operator symmetric, which conjugate gradients needs; rows with
    different diagonals would make the scaled operator non-symmetric."""
    imax2, jmax2, kmax2 = _grid(imax, jmax, kmax, do_k)

    def face(axis, lo, hi):
        c = 0.5 + uniform(seed, 70 + axis, lo)
        return c, c

    a, b = _assemble(imax2, jmax2, kmax2, do_k, face, 1.0, seed, 74)
    interior = _interior(imax2, jmax2, kmax2, do_k).reshape(-1)
    a[3][interior] = -(1.0 + delta) * np.max(-a[3][interior])
    return System(imax2, jmax2, kmax2, int(do_k), a, b, np.zeros(imax2 * jmax2 * kmax2), tol, itmax,
                  "diffusion_sym")


def void_fraction(imax2, jmax2, kmax2, seed, nspheres=40, rmin=6.0, rmax=20.0):
    """eps_g field: 0.4 background, spheres of eps_g = 0.95 (radius U[rmin, rmax],
    centres uniform over the interior)."""
    eps = np.full((kmax2, imax2, jmax2), 0.4)
    s = np.arange(nspheres)
    ci = 1.0 + uniform(seed, 30, s) * (imax2 - 2)
    cj = 1.0 + uniform(seed, 31, s) * (jmax2 - 2)
    ck = 1.0 + uniform(seed, 32, s) * (kmax2 - 2)
    rr = rmin + uniform(seed, 33, s) * (rmax - rmin)
    k = np.arange(kmax2)[:, None, None]
    i = np.arange(imax2)[None, :, None]
    j = np.arange(jmax2)[None, None, :]
    for q in range(nspheres):
        r2 = rr[q] * rr[q]
        klo, khi = int(max(0, np.floor(ck[q] - rr[q]))), int(min(kmax2, np.ceil(ck[q] + rr[q]) + 1))
        ilo, ihi = int(max(0, np.floor(ci[q] - rr[q]))), int(min(imax2, np.ceil(ci[q] + rr[q]) + 1))
        jlo, jhi = int(max(0, np.floor(cj[q] - rr[q]))), int(min(jmax2, np.ceil(cj[q] + rr[q]) + 1))
        sub = ((k[klo:khi] - ck[q]) ** 2 + (i[:, ilo:ihi] - ci[q]) ** 2 + (j[:, :, jlo:jhi] - cj[q]) ** 2) <= r2
        eps[klo:khi, ilo:ihi, jlo:jhi][sub] = 0.95
    return eps.reshape(-1)


def pressure_like(imax: int, jmax: int, kmax: int, seed: int = 0, nspheres: int = 40, rmin: float = 6.0,
                  rmax: float = 20.0, delta: float = 1e-6, itmax: int = 5000, tol: float = 1e-8) -> System:
    """Symmetric 7-point diffusion with face coefficient eps_f * D, D ~ U[0.5, 1.5],
    eps_f the arithmetic mean of the two cells' eps_g, centre -(sum)(1 + delta)
    (the 192x384x192 pressure-correction-like workload)."""
    imax2, jmax2, kmax2 = _grid(imax, jmax, kmax, True)
    eps = void_fraction(imax2, jmax2, kmax2, seed, nspheres, rmin, rmax)

    def face(axis, lo, hi):
        D = 0.5 + uniform(seed, 40 + axis, lo)
        c = 0.5 * (eps[lo] + eps[hi]) * D
        return c, c

    a, b = _assemble(imax2, jmax2, kmax2, True, face, 1.0 + delta, seed, 44)
    return System(imax2, jmax2, kmax2, 1, a, b, np.zeros(imax2 * jmax2 * kmax2), tol, itmax, "pressure_like")


def known_answer(imax: int, jmax: int, kmax: int, seed: int = 0, do_k: bool = True):
    """The recipe of model/test_lin_eq.f:63-117: off-diagonals U[0,1), A(0) =
    -70*max(u, 0.1), x_act = u + 1e-5, b = A x_act.  Coefficients that point
    out of the array are zeroed so that b = A x_act holds for the clamped
    neighbours of LEQ_MATVEC as well.  Returns (system, x_act)."""
    imax2, jmax2, kmax2 = _grid(imax, jmax, kmax, do_k)
    n = imax2 * jmax2 * kmax2
    idx = np.arange(n)
    a = np.zeros((7, n))
    for d in range(7):
        a[d] = uniform(seed, 50 + d, idx)
    a[3] = -np.maximum(uniform(seed, 57, idx), 0.1) * 70.0
    if not do_k:
        a[0] = 0.0
        a[6] = 0.0
    j = idx % jmax2
    i = (idx // jmax2) % imax2
    k = idx // (jmax2 * imax2)
    a[1][j == 0] = 0.0
    a[5][j == jmax2 - 1] = 0.0
    a[2][i == 0] = 0.0
    a[4][i == imax2 - 1] = 0.0
    if do_k:
        a[0][k == 0] = 0.0
        a[6][k == kmax2 - 1] = 0.0
    x_act = uniform(seed, 58, idx) + 1e-5
    b = matvec_np(imax2, jmax2, kmax2, do_k, a, x_act)
    return System(imax2, jmax2, kmax2, int(do_k), a, b, np.zeros(n), 1e-10, 500, "known_answer"), x_act


def neighbour_index(m: int, s: int, cyclic: bool) -> np.ndarray:
    """0-based index of each cell's neighbour s = -1 / +1 along an axis of extent m:
    clamped at the array edge (model/set_increments.f:80-109), or, along a cyclic
    axis, the interior cells 1..m-2 wrapping onto each other (IMAP_C(IMAX2) = IMIN1,
    IMAP_C(IMIN2) = IMAX1, model/dmp_modules/gridmap_mod.f:496-503)."""
    idx = np.arange(m)
    src = np.clip(idx + s, 0, m - 1)
    if cyclic and m >= 3:
        inner = (idx >= 1) & (idx <= m - 2)
        wrapped = 1 + (idx - 1 + s) % (m - 2)
        src = np.where(inner, wrapped, src)
    return src


def matvec_np(imax2, jmax2, kmax2, do_k, a, x, cyc: int = 0):
    """A*x with the neighbours of LEQ_MATVEC (numpy, any size); cyc: cyclic axes
    (1 I, 2 J, 4 K)."""
    shape = (kmax2, imax2, jmax2)
    X = x.reshape(shape)
    bit = {0: 4, 1: 1, 2: 2}  # numpy axis -> cyclic bit

    def shift(ax, s):
        return np.take(X, neighbour_index(shape[ax], s, bool(cyc & bit[ax])), axis=ax)

    A = a.reshape(7, *shape)
    y = A[1] * shift(2, -1) + A[2] * shift(1, -1) + A[3] * X + A[4] * shift(1, 1) + A[5] * shift(2, 1)
    if do_k:
        y = y + A[0] * shift(0, -1)
        y = y + A[6] * shift(0, 1)
    return y.reshape(-1)


def batch_sizes(count: int, seed: int, lo: int = 16, hi: int = 96):
    """Per-axis sizes drawn uniformly from lo..hi for `count` systems."""
    s = np.arange(count)
    out = []
    for ax in range(3):
        u = uniform(seed, 60 + ax, s)
        out.append(lo + np.minimum((u * (hi - lo + 1)).astype(np.int64), hi - lo))
    return [(int(out[0][q]), int(out[1][q]), int(out[2][q])) for q in range(count)]


def coefficient_contrast(sys: System) -> float:
    """max/min over interior rows of the nonzero off-diagonal coefficients."""
    off = sys.a[[0, 1, 2, 4, 5, 6]]
    nz = off[off > 0]
    return float(nz.max() / nz.min()) if nz.size else 1.0


def pressure_scaled(imax: int, jmax: int, kmax: int, seed: int = 0, itmax: int = 5000, tol: float = 1e-8) -> System:
    """The pressure-like recipe on a smaller box, its bubbles scaled with it:
    40 spheres of radius U[6, 20] on 192x384x192 interior cells become
    round(40 s^3) spheres (at least one) of radius U[6 s, 20 s] (at least
    U[1.5, 2.5]), s the cube root of the volume ratio."""
    s = (imax * jmax * kmax / (192.0 * 384.0 * 192.0)) ** (1.0 / 3.0)
    nsph = max(1, int(round(40 * s ** 3)))
    rmin = max(1.5, 6.0 * s)
    rmax = max(rmin + 1.0, 20.0 * s)
    return pressure_like(imax, jmax, kmax, seed=seed, nspheres=nsph, rmin=rmin, rmax=rmax, itmax=itmax, tol=tol)


def serve_mix(count: int, seed: int, lo: int = 24, hi: int = 160, pressure_share: float = 0.2,
              tols=(1e-6, 1e-8)):
    """Request mix of the serving workload: per-axis sizes log-uniform on
    [lo, hi], a `pressure_share` of pressure-like systems (the rest
    convection-diffusion), TOL drawn uniformly from `tols`.  Returns a list of
    (kind, (imax, jmax, kmax), tol, system_seed)."""
    q = np.arange(count)
    dims = []
    for ax in range(3):
        u = uniform(seed, 70 + ax, q)
        v = np.exp(np.log(lo) + u * (np.log(hi + 1) - np.log(lo)))
        dims.append(np.minimum(np.floor(v).astype(np.int64), hi))
    kind = uniform(seed, 73, q) < pressure_share
    tsel = np.minimum((uniform(seed, 74, q) * len(tols)).astype(np.int64), len(tols) - 1)
    return [("pressure_like" if kind[i] else "conv_diff", (int(dims[0][i]), int(dims[1][i]), int(dims[2][i])),
             float(tols[tsel[i]]), int(seed * 100003 + i)) for i in range(count)]


def make_request_system(kind: str, dims, tol: float, seed: int) -> System:
    if kind == "pressure_like":
        return pressure_scaled(*dims, seed=seed, tol=tol)
    return conv_diff(*dims, seed=seed, tol=tol)


@dataclass
class PPFields:
    """The fields SOLVE_PP_G assembles the gas pressure correction from, in MFIX's
    layouts (cell arrays of DIMENSION_3; D_E/D_N/D_T with MMAX+1 phases, the
    solids arrays with MMAX phases, phase-major)."""
    imax2: int
    jmax2: int
    kmax2: int
    do_k: int
    flag: np.ndarray
    rop_ge: np.ndarray
    rop_gn: np.ndarray
    rop_gt: np.ndarray | None
    ayz: np.ndarray
    axz: np.ndarray
    axy: np.ndarray | None
    u_g: np.ndarray
    v_g: np.ndarray
    w_g: np.ndarray | None
    rop_g: np.ndarray
    rop_go: np.ndarray
    vol: np.ndarray
    sum_r_g: np.ndarray
    d_e: np.ndarray
    d_n: np.ndarray
    d_t: np.ndarray | None
    mmax: int
    close_packed: np.ndarray
    rop_se: np.ndarray | None
    rop_sn: np.ndarray | None
    rop_st: np.ndarray | None
    u_s: np.ndarray | None
    v_s: np.ndarray | None
    w_s: np.ndarray | None
    rop_s: np.ndarray | None
    rop_so: np.ndarray | None
    sum_r_s: np.ndarray | None
    odt: float
    ijk_p_g: int

    @property
    def n(self) -> int:
        return self.imax2 * self.jmax2 * self.kmax2


FLAG_FLUID, FLAG_P_OUTFLOW, FLAG_WALL = 1, 11, 100  # MFIX FLAG values (FLUID_AT, P_FLOW_AT, a wall)


def pp_fields(imax: int, jmax: int, kmax: int, seed: int = 0, do_k: bool = True, mmax: int = 1,
              close_packed=(0,), outflow: bool = True, obstacle: bool = True, ijk_p_g: int = 0,
              dt: float = 0.01) -> PPFields:
    """Seeded pressure-correction fields on a box with its wall layer: face
    densities and areas, velocities, bulk densities, volumes, mass sources and
    D coefficients; a pressure-outflow patch (FLAG 11) on the north wall, an
    internal obstacle (wall cells) and `mmax` solids phases, close packed as
    `close_packed` says.  ijk_p_g: 1-based reference cell (0: none)."""
    imax2, jmax2, kmax2 = imax + 2, jmax + 2, (kmax + 2 if do_k else 1)
    n = imax2 * jmax2 * kmax2
    idx = np.arange(n, dtype=np.uint64)
    u = lambda tag, lo, hi, m=1: lo + (hi - lo) * uniform(seed, tag, np.arange(m * n, dtype=np.uint64))
    j, i, k = np.meshgrid(np.arange(jmax2), np.arange(imax2), np.arange(kmax2), indexing="ij")
    j = j.transpose(2, 1, 0).ravel()  # J fastest, then I, then K
    i = i.transpose(2, 1, 0).ravel()
    k = k.transpose(2, 1, 0).ravel()
    flag = np.full(n, FLAG_FLUID, dtype=np.int32)
    wall = (i == 0) | (i == imax2 - 1) | (j == 0) | (j == jmax2 - 1)
    if do_k:
        wall |= (k == 0) | (k == kmax2 - 1)
    flag[wall] = FLAG_WALL
    if outflow:  # a pressure-outflow patch on the north wall
        patch = (j == jmax2 - 1) & (i >= imax2 // 3) & (i < 2 * imax2 // 3)
        if do_k:
            patch &= (k >= kmax2 // 3) & (k < 2 * kmax2 // 3)
        flag[patch] = FLAG_P_OUTFLOW
    if obstacle:  # a block of wall cells inside
        ob = (i >= imax2 // 2 - 1) & (i <= imax2 // 2) & (j >= jmax2 // 3) & (j <= jmax2 // 3 + 1)
        if do_k:
            ob &= (k >= kmax2 // 2 - 1) & (k <= kmax2 // 2)
        flag[ob] = FLAG_WALL
    del idx
    cp = np.array(list(close_packed)[:mmax] + [0] * max(0, mmax - len(close_packed)), dtype=np.int32)
    sol = mmax > 0
    return PPFields(
        imax2, jmax2, kmax2, 1 if do_k else 0, flag,
        rop_ge=u(300, 0.5, 1.5), rop_gn=u(301, 0.5, 1.5), rop_gt=u(302, 0.5, 1.5) if do_k else None,
        ayz=u(303, 0.8, 1.2), axz=u(304, 0.8, 1.2), axy=u(305, 0.8, 1.2) if do_k else None,
        u_g=u(306, -1.0, 1.0), v_g=u(307, -1.0, 1.0), w_g=u(308, -1.0, 1.0) if do_k else None,
        rop_g=u(309, 0.9, 1.1), rop_go=u(310, 0.9, 1.1), vol=u(311, 0.9, 1.1), sum_r_g=u(312, -0.01, 0.01),
        d_e=u(313, 0.1, 1.0, mmax + 1), d_n=u(314, 0.1, 1.0, mmax + 1),
        d_t=u(315, 0.1, 1.0, mmax + 1) if do_k else None,
        mmax=mmax, close_packed=cp,
        rop_se=u(316, 0.1, 0.5, mmax) if sol else None, rop_sn=u(317, 0.1, 0.5, mmax) if sol else None,
        rop_st=u(318, 0.1, 0.5, mmax) if sol and do_k else None,
        u_s=u(319, -0.5, 0.5, mmax) if sol else None, v_s=u(320, -0.5, 0.5, mmax) if sol else None,
        w_s=u(321, -0.5, 0.5, mmax) if sol and do_k else None,
        rop_s=u(322, 0.1, 0.3, mmax) if sol else None, rop_so=u(323, 0.1, 0.3, mmax) if sol else None,
        sum_r_s=u(324, -0.001, 0.001, mmax) if sol else None,
        odt=1.0 / dt, ijk_p_g=int(ijk_p_g))


def conv_diff_cyclic(imax: int, jmax: int, kmax: int, seed: int = 0, cyc: int = 1, do_k: bool = True,
                     itmax: int = 500, tol: float = 1e-8) -> System:
    """conv_diff with periodic faces along the cyclic axes `cyc` (1 I, 2 J, 4 K):
    the face between the last and the first interior cell of each line along
    such an axis gets the same upwind coefficients as any interior face (row of
    the last cell: its + diagonal; row of the first: its - diagonal), as the
    neighbour increments of a cyclic run (model/set_increments.f:73-113) couple
    them.  The centre is recomputed with the (1 + 1e-3) excess."""
    s = conv_diff(imax, jmax, kmax, seed=seed, do_k=do_k, itmax=itmax, tol=tol)
    s.cyc = cyc
    imax2, jmax2, kmax2 = s.imax2, s.jmax2, s.kmax2
    shape = (kmax2, imax2, jmax2)
    a = s.a
    inter = _interior(imax2, jmax2, kmax2, do_k)
    flat = np.arange(s.n, dtype=np.int64).reshape(shape)
    axes = [(0, 1, 1, -1, 1), (1, 2, 2, -2, 2)]
    if do_k:
        axes.append((2, 0, 3, -3, 4))
    for axis, npax, d_low, d_high, bit in axes:
        if not (cyc & bit) or shape[npax] < 4:
            continue
        last = [slice(None)] * 3
        first = [slice(None)] * 3
        last[npax] = shape[npax] - 2
        first[npax] = 1
        m_last, m_first = inter[tuple(last)], inter[tuple(first)]
        lo = flat[tuple(last)][m_last]
        hi = flat[tuple(first)][m_first]
        D = 0.5 + uniform(seed, 60 + 4 * axis, lo)
        F = normal(seed, 61 + 4 * axis, lo, 0.5)
        a[d_low + 3][lo] = D + np.maximum(-F, 0.0)
        a[d_high + 3][hi] = D + np.maximum(F, 0.0)
    wall = ~inter.reshape(-1)
    off = a[[0, 1, 2, 4, 5, 6]].sum(axis=0)
    a[3] = np.where(wall, -1.0, -off * (1.0 + 1e-3))
    s.kind = "conv_diff_cyclic"
    return s
