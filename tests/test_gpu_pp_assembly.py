"""The gas pressure-correction system assembled on the device.

CONV_PP_G + SOURCE_PP_G (model/conv_pp_g.f:33-182, model/source_pp_g.f:18-214)
through mfixgpu_conv_source_pp_g against the oracle's C restatement of the same
routines: A_M(:,:,0), B_M(:,0) and B_MMAX(:,0) bit for bit, in 3-D and 2-D, with
solids phases (one close packed), a pressure-outflow patch, an internal
obstacle and a reference cell, from host arrays and from device arrays.
SOLVE_PP_G through mfixgpu_solve_pp_g_ against the oracle's assembly, its
CALC_RESID_PP and its LEQ_BICGS: the same IER, RESG to rounding, PP_G within
the solver tolerance, ITER_TOT(1) accounting.
"""
import numpy as np
import pytest

import oracle as O
from mfix_b200 import leq
from mfix_b200 import systems as S

pytestmark = pytest.mark.gpu

CASES = [
    ("3d_two_solids", dict(imax=14, jmax=17, kmax=11, seed=3, mmax=2, close_packed=(0, 1))),
    ("2d_one_solid", dict(imax=30, jmax=25, kmax=1, seed=4, do_k=False, mmax=1)),
    ("3d_gas_ref_cell", dict(imax=12, jmax=10, kmax=13, seed=5, mmax=0, outflow=False, ijk_p_g=500)),
]


def _geom(f):
    assert leq.init_geometry(f.imax2, f.jmax2, f.kmax2, f.do_k, f.n, max(f.mmax, 1)) == 0


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_assembly_matches_oracle_bitwise(name, kw):
    f = S.pp_fields(**kw)
    a_ref, b_ref, bm_ref = O.conv_source_pp_g(f)
    _geom(f)
    a, b, bm = np.full((7, f.n), np.nan), np.full(f.n, np.nan), np.full(f.n, np.nan)
    assert leq.conv_source_pp_g(f, a, b, bm) == 0, leq.last_error()
    assert np.array_equal(a, a_ref)
    assert np.array_equal(b, b_ref)
    assert np.array_equal(bm, bm_ref)
    fl = f.flag == 1
    assert np.all(a[3][~fl] == -1.0) and np.all(b[~fl] == 0.0)  # identity rows outside the fluid


def test_assembly_from_device_arrays(cuda):
    f = S.pp_fields(imax=16, jmax=12, kmax=9, seed=7, mmax=1)
    a_ref, b_ref, bm_ref = O.conv_source_pp_g(f)
    _geom(f)
    dev = {name: cuda.from_numpy(getattr(f, name)).cuda() for name in leq.PP_ARRAYS
           if getattr(f, name) is not None}
    ptrs = {name: t.data_ptr() for name, t in dev.items()}
    a = cuda.empty((7, f.n), dtype=cuda.float64, device="cuda")
    b = cuda.empty(f.n, dtype=cuda.float64, device="cuda")
    bm = cuda.empty(f.n, dtype=cuda.float64, device="cuda")
    assert leq.conv_source_pp_g(f, a.data_ptr(), b.data_ptr(), bm.data_ptr(), device_ptrs=ptrs) == 0, \
        leq.last_error()
    cuda.cuda.synchronize()
    assert np.array_equal(a.cpu().numpy(), a_ref)
    assert np.array_equal(b.cpu().numpy(), b_ref)
    assert np.array_equal(bm.cpu().numpy(), bm_ref)


@pytest.mark.parametrize("normg", [0.0, 2.5])
@pytest.mark.parametrize("name,kw", CASES[:2], ids=[c[0] for c in CASES[:2]])
def test_solve_pp_g_matches_oracle(name, kw, normg):
    f = S.pp_fields(**kw)
    a_ref, b_ref, bm_ref = O.conv_source_pp_g(f)
    norm = normg if normg != 0.0 else O.calc_resid_pp(f, bm_ref, 1.0) / 10.0  # model/solve_pp_g.f:94-101
    resg_ref = O.calc_resid_pp(f, b_ref, norm)
    ref = S.System(f.imax2, f.jmax2, f.kmax2, f.do_k, a_ref.copy(), b_ref.copy(), np.zeros(f.n), tol=1e-8,
                   itmax=500)
    st = O.leq_bicgs(ref)
    _geom(f)
    leq.reset_iter_tot()
    pp = np.full(f.n, 7.0)  # SOLVE_PP_G starts from PP_G = 0 whatever it held
    ier, resg = leq.solve_pp_g(f, normg, pp, itmax=500, tol=1e-8)
    assert ier == st["ier"] == 0, leq.last_error()
    assert abs(resg - resg_ref) <= 1e-12 * abs(resg_ref)
    assert np.linalg.norm(pp - ref.x) <= 1e-6 * np.linalg.norm(ref.x)
    assert leq.iter_tot(1) == leq.last_stats()["iter_tot_add"] > 0
