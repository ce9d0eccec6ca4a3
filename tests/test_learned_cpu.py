"""Host side of the learned preconditioner: BF16 rounding, the reference
convolution (the oracle of the device kernels) against finite differences, the
cosine loss gradient and the regular-domain lattice."""
import numpy as np

from hirensi_b200 import learned as Lr
from hirensi_b200.mesh import box_mesh


def test_bf16_round_to_nearest_even():
    vals = np.array([1.0, 1.00390625, 1.01171875, -3.140625, 1e-30, 65504.0], dtype=np.float32)
    r = Lr.round_bf16(vals)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: rounds to the even mantissa (1.0)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.015625 and r[3] == -3.140625
    assert abs(r[4] - 1e-30) / 1e-30 < 2 ** -8 and r[5] == 65536.0


def test_reference_convolution_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((3, 4, 5, 6))
    w = rng.standard_normal((2, 3, 27)) * 0.3
    b = rng.standard_normal(2) * 0.1
    for relu in (0, 1):
        y = Lr.conv_ref(x, w, b, relu)
        gy = rng.standard_normal(y.shape)
        gx, gw, gb = Lr.conv_ref_backward(x, w, y, relu, gy)
        f = lambda xx, ww, bb: float((Lr.conv_ref(xx, ww, bb, relu) * gy).sum())
        eps = 1e-6
        for idx in [(0, 1, 2, 3), (2, 3, 4, 5), (1, 0, 0, 0)]:
            xp = x.copy(); xp[idx] += eps
            xm = x.copy(); xm[idx] -= eps
            assert abs((f(xp, w, b) - f(xm, w, b)) / (2 * eps) - gx[idx]) < 1e-6
        for idx in [(0, 1, 13), (1, 2, 0), (1, 0, 26)]:
            wp = w.copy(); wp[idx] += eps
            wm = w.copy(); wm[idx] -= eps
            assert abs((f(x, wp, b) - f(x, wm, b)) / (2 * eps) - gw[idx]) < 1e-6
        bp = b.copy(); bp[1] += eps
        bm = b.copy(); bm[1] -= eps
        assert abs((f(x, w, bp) - f(x, w, bm)) / (2 * eps) - gb[1]) < 1e-6


def test_cosine_loss_gradient():
    rng = np.random.default_rng(1)
    a, t = rng.standard_normal(50), rng.standard_normal(50)
    L, g = Lr.cosine_loss(a, t)
    assert 0.0 <= L <= 1.0
    eps = 1e-7
    for i in (0, 17, 49):
        ap = a.copy(); ap[i] += eps
        am = a.copy(); am[i] -= eps
        assert abs((Lr.cosine_loss(ap, t)[0] - Lr.cosine_loss(am, t)[0]) / (2 * eps) - g[i]) < 1e-6
    # scale invariance
    assert abs(Lr.cosine_loss(3.7 * a, t)[0] - L) < 1e-12
    assert Lr.cosine_loss(t, t)[0] < 1e-12


def test_lattice_of_box_mesh():
    m = box_mesh(4, 3, 2, 2.5, 1)
    lat = Lr.Lattice.of(m)
    assert lat.shape == (5, 7, 9)
    v = np.arange(m.nj, dtype=np.float64)
    back = lat.from_grid(lat.to_grid(v), m.nj)
    assert np.array_equal(back[m.store_nodes], v[m.store_nodes])
    x = Lr.features(lat, v, -v, np.ones(m.nstore // 3), np.full(m.nj, 200.0))
    assert x.shape == (4, 5, 7, 9)
    assert np.abs(x[0]).max() == 1.0 and np.allclose(x[3], 0.5)


def test_features_with_pseudo_hessian_channels():
    from hirensi_b200.learned import Lattice, features
    from hirensi_b200.mesh import box_mesh
    m = box_mesh(2, 2, 1, 2.5, 1)
    lat = Lattice.of(m)
    rng = np.random.default_rng(0)
    nj = m.nj
    g_l, g_m, vs = rng.standard_normal(nj), rng.standard_normal(nj), 200.0 + rng.random(nj)
    il = rng.random(len(m.store_nodes)) + 0.1
    x4 = features(lat, g_l, g_m, il, vs)
    x6 = features(lat, g_l, g_m, il, vs, (rng.random(nj) + 1e-3, rng.random(nj) + 1e-3))
    assert x4.shape == (4,) + lat.shape and x6.shape == (6,) + lat.shape
    assert np.array_equal(x6[:4], x4)
    for c in (4, 5):
        assert abs(x6[c].mean()) < 1e-9 and abs(x6[c].std() - 1.0) < 1e-9
