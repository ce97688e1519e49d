"""CPU checks of the seeded generators (the synthetic workloads' shapes and values)."""
import numpy as np

from mfix_b200 import systems as S


def _walls(s):
    idx = np.arange(s.n)
    j = idx % s.jmax2
    i = (idx // s.jmax2) % s.imax2
    k = idx // (s.jmax2 * s.imax2)
    w = (i == 0) | (i == s.imax2 - 1) | (j == 0) | (j == s.jmax2 - 1)
    if s.do_k:
        w |= (k == 0) | (k == s.kmax2 - 1)
    return w


def test_conv_diff_layout_and_walls():
    s = S.conv_diff(6, 7, 5, seed=0)
    assert (s.imax2, s.jmax2, s.kmax2) == (8, 9, 7) and s.a.shape == (7, s.n)
    w = _walls(s)
    assert np.all(s.a[3][w] == -1.0) and np.all(s.a[[0, 1, 2, 4, 5, 6]][:, w] == 0.0) and np.all(s.b[w] == 0.0)
    off = s.a[[0, 1, 2, 4, 5, 6]][:, ~w].sum(axis=0)
    np.testing.assert_allclose(-s.a[3][~w], off * (1 + 1e-3), rtol=1e-15)
    assert np.all(s.a[[0, 1, 2, 4, 5, 6]] >= 0.0)
    assert np.all(np.abs(s.b[~w]) <= 1.0)


def test_conv_diff_upwind_faces():
    s = S.conv_diff(5, 5, 5, seed=1)
    # face between P and its J neighbour Q: a_Q(P) - a_P(Q) = max(-F,0) - max(F,0) = -F
    p = 2 + 2 * s.jmax2 + 2 * s.jmax2 * s.imax2
    q = p + 1
    d_sum = s.a[5][p] + s.a[1][q]
    assert d_sum >= 1.0  # 2D + |F| with D >= 0.5


def test_seeded_and_deterministic():
    a = S.conv_diff(6, 6, 6, seed=3)
    b = S.conv_diff(6, 6, 6, seed=3)
    c = S.conv_diff(6, 6, 6, seed=4)
    assert np.array_equal(a.a, b.a) and np.array_equal(a.b, b.b)
    assert not np.array_equal(a.a, c.a)


def test_pressure_like_symmetric():
    s = S.pressure_like(10, 12, 9, seed=2, nspheres=3, rmin=2, rmax=4)
    c1, c2 = s.jmax2, s.jmax2 * s.imax2
    for d, off in ((2, 1), (1, c1), (3, c2)):  # J, I, K
        lo = np.arange(s.n - off)
        np.testing.assert_array_equal(s.a[d + 3][lo], s.a[-d + 3][lo + off])
    assert S.coefficient_contrast(s) > 2.0


def test_2d_system():
    s = S.conv_diff(9, 7, 1, seed=5, do_k=False)
    assert s.kmax2 == 1 and s.do_k == 0
    assert not s.a[0].any() and not s.a[6].any()


def test_known_answer_consistent():
    s, x = S.known_answer(5, 6, 4, seed=6)
    np.testing.assert_allclose(S.matvec_np(s.imax2, s.jmax2, s.kmax2, s.do_k, s.a, x), s.b, rtol=1e-14)


def test_batch_sizes_range():
    sz = S.batch_sizes(512, seed=0)
    arr = np.array(sz)
    assert arr.min() >= 16 and arr.max() <= 96 and len(set(sz)) > 400


def test_uniform_stream_matches_oracle():
    import oracle as O

    idx = np.array([0, 1, 17, 10**9])
    got = S.uniform(0x5EED, 0xA1, idx)
    for q, v in zip(idx, got):
        assert O.uniform(0x5EED, 0xA1, int(q)) == v


def test_diffusion_sym_scaled_operator_is_symmetric():
    """One interior diagonal: dividing each row by its diagonal (LEQ_CG0's
    scaling) keeps the operator symmetric, which conjugate gradients needs."""
    s = S.diffusion_sym(7, 9, 6, seed=2)
    a = s.a / s.a[3]
    n = s.n
    rng = np.random.default_rng(0)
    u, v = rng.standard_normal(n), rng.standard_normal(n)
    interior = s.a[3] != -1.0  # wall rows are identity rows, decoupled from the interior
    u[~interior] = 0.0
    v[~interior] = 0.0
    Au = S.matvec_np(s.imax2, s.jmax2, s.kmax2, s.do_k, a, u)
    Av = S.matvec_np(s.imax2, s.jmax2, s.kmax2, s.do_k, a, v)
    assert abs(v @ Au - u @ Av) <= 1e-12 * abs(v @ Au)
    assert np.allclose(s.a[3][interior], s.a[3][interior][0])
