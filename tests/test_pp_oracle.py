"""CPU pin of the oracle's pressure-correction assembly.

An independent numpy restatement of CONV_PP_G (model/conv_pp_g.f:33-182) and
SOURCE_PP_G (model/source_pp_g.f:18-214) for an incompressible run on a
Cartesian grid, every term in the reference's left-to-right order (numpy's
elementwise operations round each product and sum, as the oracle compiled
without FMA contraction does), against oracle.conv_source_pp_g, bit for bit:
gas and solids phases, close-packed phases skipped, wall and obstacle cells,
the links to pressure-outflow cells cut, the reference cell IJK_P_G.
"""
import numpy as np
import pytest

import oracle as O
from mfix_b200 import systems as S

SMALL_NUMBER = 1.0e-15


def _np_conv_source(f):
    n, J, I = f.n, f.jmax2, f.imax2
    p = np.arange(n)
    j, i, k = p % J, (p // J) % I, p // (J * I)
    # clamped neighbours (model/set_increments.f:80-109)
    im = np.where(i > 0, p - J, p)
    ip = np.where(i < I - 1, p + J, p)
    jm = np.where(j > 0, p - 1, p)
    jp = np.where(j < J - 1, p + 1, p)
    if f.do_k:
        km = np.where(k > 0, p - J * I, p)
        kp = np.where(k < f.kmax2 - 1, p + J * I, p)
    fluid = f.flag == 1
    pflow = (f.flag == 10) | (f.flag == 11)
    zero = np.zeros(n)

    def ph(arr, m):  # phase m's slice of a (phases * n) array
        return arr[m * n:(m + 1) * n]

    # CONV_PP_G, gas: each face coefficient from the cell below the face
    ae = f.rop_ge * f.ayz
    aw = f.rop_ge[im] * f.ayz[im]
    an = f.rop_gn * f.axz
    as_ = f.rop_gn[jm] * f.axz[jm]
    at = f.rop_gt * f.axy if f.do_k else zero.copy()
    ab = f.rop_gt[km] * f.axy[km] if f.do_k else zero.copy()
    # SOURCE_PP_G, gas (:87-106)
    bma = (f.rop_g - f.rop_go) * f.vol * f.odt
    bme = ae * f.u_g
    bmw = aw * f.u_g[im]
    bmn = an * f.v_g
    bms = as_ * f.v_g[jm]
    bmt = at * f.w_g if f.do_k else zero
    bmb = ab * f.w_g[km] if f.do_k else zero
    bmr = f.sum_r_g * f.vol
    b = -((-(bma + bme - bmw + bmn - bms + bmt - bmb)) + bmr)
    bmax = np.maximum.reduce([np.abs(v) for v in (bma, bme, bmw, bmn, bms, bmt, bmb, bmr)])
    ae = ae * ph(f.d_e, 0)
    aw = aw * ph(f.d_e, 0)[im]
    an = an * ph(f.d_n, 0)
    as_ = as_ * ph(f.d_n, 0)[jm]
    if f.do_k:
        at = at * ph(f.d_t, 0)
        ab = ab * ph(f.d_t, 0)[km]
    # solids phases that do not become close packed (:117-145)
    for m in range(1, f.mmax + 1):
        if f.close_packed[m - 1]:
            continue
        se = ph(f.rop_se, m - 1) * f.ayz
        sw = ph(f.rop_se, m - 1)[im] * f.ayz[im]
        sn = ph(f.rop_sn, m - 1) * f.axz
        ss = ph(f.rop_sn, m - 1)[jm] * f.axz[jm]
        t = (ph(f.rop_s, m - 1) - ph(f.rop_so, m - 1)) * f.vol * f.odt
        t = t + se * ph(f.u_s, m - 1) - sw * ph(f.u_s, m - 1)[im] + sn * ph(f.v_s, m - 1) - ss * ph(f.v_s, m - 1)[jm]
        if f.do_k:
            st = ph(f.rop_st, m - 1) * f.axy
            sb = ph(f.rop_st, m - 1)[km] * f.axy[km]
            t = t + st * ph(f.w_s, m - 1) - sb * ph(f.w_s, m - 1)[km]
        b = b - ((-t) + ph(f.sum_r_s, m - 1) * f.vol)
        ae = ae + se * ph(f.d_e, m)
        aw = aw + sw * ph(f.d_e, m)[im]
        an = an + sn * ph(f.d_n, m)
        as_ = as_ + ss * ph(f.d_n, m)[jm]
        if f.do_k:
            at = at + st * ph(f.d_t, m)
            ab = ab + sb * ph(f.d_t, m)[km]
    ac = -(ae + aw + an + as_ + at + ab)
    small = (np.abs(ac) < SMALL_NUMBER) & (np.abs(b) < SMALL_NUMBER)
    ac = np.where(small, -1.0, ac)
    b = np.where(small, 0.0, b)
    # links to pressure-flow cells cut (:224-243)
    aw = np.where(pflow[im], 0.0, aw)
    ae = np.where(pflow[ip], 0.0, ae)
    as_ = np.where(pflow[jm], 0.0, as_)
    an = np.where(pflow[jp], 0.0, an)
    if f.do_k:
        ab = np.where(pflow[km], 0.0, ab)
        at = np.where(pflow[kp], 0.0, at)
    a = np.stack([ab, as_, aw, ac, ae, an, at])
    # cells outside the fluid: identity rows (:187-199)
    a[:, ~fluid] = 0.0
    a[3, ~fluid] = -1.0
    b = np.where(fluid, b, 0.0)
    bmax = np.where(fluid, bmax, 0.0)
    # the reference cell of an incompressible run (:247-251)
    if f.ijk_p_g >= 1:
        a[:, f.ijk_p_g - 1] = 0.0
        a[3, f.ijk_p_g - 1] = -1.0
        b[f.ijk_p_g - 1] = 0.0
    return a, b, bmax


CASES = [
    ("3d_one_phase", dict(imax=12, jmax=10, kmax=8, seed=1, mmax=1)),
    ("3d_two_phases_one_packed", dict(imax=10, jmax=9, kmax=7, seed=2, mmax=2, close_packed=(0, 1))),
    ("3d_gas_only_ref_cell", dict(imax=9, jmax=11, kmax=6, seed=3, mmax=0, ijk_p_g=200)),
    ("2d_one_phase", dict(imax=20, jmax=14, kmax=1, seed=4, do_k=False, mmax=1)),
    ("3d_no_outflow", dict(imax=8, jmax=8, kmax=8, seed=5, mmax=1, outflow=False)),
]


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_oracle_assembly_matches_numpy(name, kw):
    f = S.pp_fields(**kw)
    a_c, b_c, m_c = O.conv_source_pp_g(f)
    a_n, b_n, m_n = _np_conv_source(f)
    assert np.array_equal(a_c, a_n)
    assert np.array_equal(b_c, b_n)
    assert np.array_equal(m_c, m_n)
    fl = f.flag == 1
    assert fl.any() and (~fl).any()
