"""Structural checks of the oracle's element-level restatement (CPU)."""
import numpy as np
import pytest

import oracle as O
from hirensi_b200.mesh import LOCAL_IJK, box_mesh, default_pml_param

G = [-1.0, 0.0, 1.0]


def box_xt(h=(2.0, 3.0, 1.5), origin=(0.0, 0.0, -1.5), shear=0.0):
    """Nodal coordinates XT[3][27] of a (possibly sheared) hexahedron."""
    xt = np.zeros((3, 27))
    for i, (a, b, c) in enumerate(LOCAL_IJK):
        x = origin[0] + 0.5 * h[0] * a + shear * 0.5 * h[2] * c
        y = origin[1] + 0.5 * h[1] * b
        z = origin[2] + 0.5 * h[2] * c
        xt[:, i] = (x, y, z)
    return xt


def test_gll_rule():
    x, w = [-1.0, 0.0, 1.0], [1 / 3, 4 / 3, 1 / 3]
    assert abs(sum(w) - 2.0) < 1e-15 and x[1] == 0.0


@pytest.mark.parametrize("pt", [(0.1, -0.3, 0.7), (-0.9, 0.2, 0.05), (0.5, 0.5, -0.5)])
def test_shape_partition_of_unity(pt):
    fn, d = O.shape_3_27(*pt)
    assert abs(fn.sum() - 1.0) < 1e-14
    assert np.all(np.abs(d.sum(axis=0)) < 1e-14)
    # reproduces linear and quadratic fields
    xi = np.array([[G[a], G[b], G[c]] for a, b, c in LOCAL_IJK])
    assert abs(fn @ xi[:, 0] - pt[0]) < 1e-14
    assert abs(fn @ (xi[:, 1] ** 2) - pt[1] ** 2) < 1e-14
    assert abs(d[:, 2] @ (xi[:, 2] ** 2) - 2 * pt[2]) < 1e-13


def test_shape_kronecker_at_gll_nodes():
    for i, (a, b, c) in enumerate(LOCAL_IJK):
        fn, _ = O.shape_3_27(G[a], G[b], G[c])
        e = np.zeros(27)
        e[i] = 1.0
        assert np.array_equal(fn, e)


def _rigid_modes(xt):
    modes = []
    for d in range(3):
        v = np.zeros((3, 27))
        v[d] = 1.0
        modes.append(v.reshape(-1))
    x, y, z = xt
    for a, b in [(0, 1), (1, 2), (0, 2)]:
        v = np.zeros((3, 27))
        v[a] = -xt[b]
        v[b] = xt[a]
        modes.append(v.reshape(-1))
    return modes


@pytest.mark.parametrize("shear", [0.0, 0.3])
def test_element_k_symmetric_with_rigid_null_space(shear):
    xt = box_xt(shear=shear)
    lam = np.linspace(100.0, 160.0, 27)
    mu = np.linspace(80.0, 90.0, 27)
    ek = O.element_k(xt, lam, mu)
    assert np.array_equal(ek, ek.T)
    scale = np.abs(ek).max()
    for v in _rigid_modes(xt):
        assert np.abs(ek @ v).max() < 1e-12 * scale * np.abs(v).max()
    # positive semi-definite with exactly 6 zero modes
    w = np.linalg.eigvalsh(ek)
    assert np.sum(np.abs(w) < 1e-9 * w.max()) == 6
    assert w.min() > -1e-9 * w.max()


def test_element_mass_is_diagonal_and_integrates_volume():
    h = (2.0, 3.0, 1.5)
    xt = box_xt(h=h)
    p = default_pml_param(((-10, 10), (-10, 10), (-10, 0)), 3.0)
    em = O.element_m(xt, 2e-3, p, 201)
    assert np.count_nonzero(em - np.diag(np.diag(em))) == 0
    assert abs(np.diag(em).sum() - 3 * 2e-3 * np.prod(h)) < 1e-15


def test_pml_finder_profile_and_top_zone():
    p = default_pml_param(((-20, 20), (-20, 20), (-20, 0)), 7.5, alpha0=5.0, beta0=400.0)
    inner = O.pml_finder([0.0, 0.0, -5.0], p)
    assert np.array_equal(inner[:6], [1, 1, 1, 0, 0, 0])
    assert inner[6] == 1.0 and inner[7] == 0.0 and inner[8] == 0.0 and inner[9] == 0.0
    x = 20.0 + 3.75   # half-way through the x+ layer
    ab = O.pml_finder([x, 0.0, -5.0], p)
    assert abs(ab[0] - (1 + 5.0 * 0.25)) < 1e-15 and abs(ab[3] - 400.0 * 0.25) < 1e-13
    corner = O.pml_finder([-27.5, 27.5, -27.5], p)
    assert np.allclose(corner[:3], 6.0) and np.allclose(corner[3:6], 400.0)
    assert abs(corner[9] - 400.0 ** 3) < 1e-6 and np.all(corner[10:] == 0.0)
    p_top = p.copy()
    p_top[4, 3] = -1.0
    with pytest.raises(ValueError):
        O.pml_finder([0.0, 0.0, 0.0], p_top)


def test_en_diagonal_and_ea_structural_zeros():
    p = default_pml_param(((-2, 2), (-2, 2), (-2, 0)), 3.0)
    xt = box_xt(h=(2.0, 2.0, 2.0), origin=(2.0, 0.0, -2.0))   # in the x+ layer
    for f in (301, 302, 303, 304):
        en = O.element_en(xt, p, f)
        assert np.count_nonzero(en - np.diag(np.diag(en))) == 0
    lam = np.full(27, 160.0)
    mu = np.full(27, 80.0)
    for f in range(101, 107):
        ea = O.element_ea(xt, lam, mu, p, f)
        assert np.all(ea[0:27, 135:162] == 0) and np.all(ea[27:54, 108:135] == 0) and np.all(ea[54:81, 81:108] == 0)
    assert np.abs(O.element_ea(xt, lam, mu, p, 101)).max() > 0


def test_surface_traction_integrates_face_area():
    xt = box_xt(h=(2.0, 3.0, 1.5), origin=(0.0, 0.0, -1.5))
    efs = O.element_fs(xt, 5)
    assert abs(efs[54:81].sum() - 6.0) < 1e-14 and np.all(efs[:54] == 0.0)
    with pytest.raises(ValueError):
        O.element_fs(box_xt(origin=(0.0, 0.0, -5.0)), 5)


@pytest.mark.parametrize("eps", [np.diag([1.0, 0.0, 0.0]),
                                 np.array([[0.3, -0.2, 0.5], [-0.2, -0.7, 0.1], [0.5, 0.1, 0.4]])])
def test_element_k_patch_test_gives_exact_boundary_tractions(eps):
    """Uniform strain eps on an affine box with uniform lam, mu: K u equals the
    consistent boundary forces of the stress sig = lam tr(eps) I + 2 mu eps, that
    is F_I = sum over the faces f holding node I of (int_f N_I dA) sig n_f, with
    int_f N_I dA = W_a W_b area_f / 4 for the GLL weights W = (1/3, 4/3, 1/3).
    The 3-point GLL rule integrates grad N_I . sig exactly here, so the identity
    holds to rounding.  A swap of the roles of lam and mu breaks it."""
    h = (2.0, 3.0, 1.5)
    xt = box_xt(h=h)
    lam0, mu0 = 130.0, 85.0
    ek = O.element_k(xt, np.full(27, lam0), np.full(27, mu0))
    u = (eps @ xt).reshape(-1)                      # u_c(x) = sum_k eps_ck x_k at every node
    sig = lam0 * np.trace(eps) * np.eye(3) + 2.0 * mu0 * eps
    W = np.array([1.0, 4.0, 1.0]) / 3.0
    area = [h[1] * h[2], h[0] * h[2], h[0] * h[1]]  # faces normal to x, y, z
    f_ref = np.zeros((3, 27))
    for i, ijk in enumerate(LOCAL_IJK):
        for ax in range(3):
            if ijk[ax] == 1:
                continue
            n = np.zeros(3)
            n[ax] = 1.0 if ijk[ax] == 2 else -1.0
            a, b = [ijk[k] for k in range(3) if k != ax]
            f_ref[:, i] += W[a] * W[b] * area[ax] / 4.0 * (sig @ n)
    f = ek @ u
    scale = np.abs(f_ref).max()
    assert np.abs(f - f_ref.reshape(-1)).max() < 1e-12 * scale
    centre = [i for i, ijk in enumerate(LOCAL_IJK) if tuple(ijk) == (1, 1, 1)][0]
    assert np.abs(f.reshape(3, 27)[:, centre]).max() < 1e-12 * scale


def test_tv_regularization_is_the_gradient_of_the_tv_functional():
    """Known answer of the TV term: per node it is the derivative of
    T(m) = sum over regular-domain elements and GLL points of w detJ sqrt(|grad m|^2 + eps)
    with eps = 0.01.  T is evaluated here independently (axis-aligned boxes: grad N =
    dN/dxi * 2/h, detJ = (h/2)^3) and differenced centrally at a few nodes."""
    from problems import RHO
    mesh = box_mesh(3, 3, 2, 2.5, 1)
    om = O.OracleMesh(mesh, RHO)
    rng = np.random.default_rng(5)
    x, y, z = mesh.xyz.T
    mu = 100.0 + 20.0 * np.sin(0.3 * x) * np.cos(0.2 * y) + 5.0 * z + rng.uniform(-1, 1, mesh.nj)
    lam = 2.0 * mu
    _, reg_mu, _, _ = O.tv_reg(om, lam, mu)
    h = mesh.h
    W = [1.0 / 3.0, 4.0 / 3.0, 1.0 / 3.0]
    pts = [(a, b, c) for c in range(3) for b in range(3) for a in range(3)]
    dN = {q: O.shape_3_27(G[q[0]], G[q[1]], G[q[2]])[1] * (2.0 / h) for q in pts}
    rd = np.nonzero(mesh.mtel == 1)[0]

    def T(m):
        tot = 0.0
        for e in rd:
            me = m[mesh.inod[e]]
            for q in pts:
                g = dN[q].T @ me
                tot += W[q[0]] * W[q[1]] * W[q[2]] * (h / 2.0) ** 3 * np.sqrt(g @ g + 0.01)
        return tot

    nodes = np.unique(mesh.inod[rd])
    for k in rng.choice(nodes, 5, replace=False):
        d = 1e-3
        mp, mm = mu.copy(), mu.copy()
        mp[k] += d
        mm[k] -= d
        fd = (T(mp) - T(mm)) / (2 * d)
        assert abs(fd - reg_mu[k]) <= 1e-6 * max(abs(reg_mu[k]), 1e-3)


@pytest.mark.parametrize("shear", [0.0, 0.3])
def test_element_gradient_is_the_derivative_of_the_stiffness_form(shear):
    """Known answer tying the control kernel (ELEMENT_g_3D) to ELEMENT_K_3D: the
    adjoint-state gradient of a parameter of K is u^T (dK/dm_i) p.  EK is linear in
    the nodal lam and mu, so a unit difference of EK gives dK/dm_i exactly, and
    element_g must equal u^T (EK(m + e_i) - EK(m)) p for every node i."""
    xt = box_xt(shear=shear)
    rng = np.random.default_rng(11)
    lam = rng.uniform(100.0, 160.0, 27)
    mu = rng.uniform(60.0, 90.0, 27)
    eu = rng.standard_normal(81)
    ep = rng.standard_normal(81)
    gm, gl = O.element_g(xt, eu, ep)
    k0 = O.element_k(xt, lam, mu)
    for i in range(27):
        e = np.zeros(27)
        e[i] = 1.0
        dkm = O.element_k(xt, lam, mu + e) - k0
        dkl = O.element_k(xt, lam + e, mu) - k0
        assert abs(eu @ dkm @ ep - gm[i]) <= 1e-9 * np.abs(gm).max()
        assert abs(eu @ dkl @ ep - gl[i]) <= 1e-9 * np.abs(gl).max()
    # the (lam + 2 mu, mu) parameterization: d/dmu at fixed lam + 2 mu = d/dmu - 2 d/dlam
    gm2, gl2 = O.element_g(xt, eu, ep, lambda_2mu=True)
    assert np.abs(gm2 - (gm - 2.0 * gl)).max() <= 1e-12 * np.abs(gm).max()
    assert np.array_equal(gl2, gl)


@pytest.mark.parametrize("shear", [0.0, 0.3])
def test_pml_without_stretching_reduces_to_the_elastic_stiffness(shear):
    """Known answer of the mixed displacement-stress PML element: with alpha = 1 and
    beta = 0 (no stretching, no attenuation) the stress rows N_a s' = -EA_upper^T u'
    can be eliminated, and the displacement rows then carry EA_lower N_a^-1 EA_upper^T,
    which must be the elastic stiffness EK of the same element and material.  This
    ties the EA blocks of kind e (upper: strain weights 1, 0, 1, 1; lower: lam + 2 mu,
    lam, 2 mu) and the EN weights (1, 1, 1, 2, 2, 2) to ELEMENT_K_3D."""
    xt = box_xt(origin=(12.0, 0.0, -1.5), shear=shear)     # inside the x+ PML zone
    p = default_pml_param(((-10, 10), (-10, 10), (-10, 0)), 3.0, alpha0=0.0, beta0=0.0)
    rng = np.random.default_rng(1)
    lam = rng.uniform(100.0, 160.0, 27)
    mu = rng.uniform(60.0, 90.0, 27)
    upper = O.element_ea(xt, lam, mu, p, 101)
    lower = O.element_ea(xt, lam, mu, p, 104)
    na = O.element_en(xt, p, 301)
    assert np.count_nonzero(na - np.diag(np.diag(na))) == 0
    k_eff = lower @ np.diag(1.0 / np.diag(na)) @ upper.T
    ek = O.element_k(xt, lam, mu)
    assert np.abs(k_eff - ek).max() <= 1e-13 * np.abs(ek).max()


@pytest.mark.parametrize("fr", [5.0, 15.0, 60.0])
def test_time_function_ricker_known_values(fr):
    """TIME_FUNCTION case 2 (S4/IO.F90:608-621): with u = 2 pi fr t - 3 sqrt(6) the
    normalized wavelet starts at 0 (u^2 = 54 cancels the 13 e^-13.5 offset), peaks at
    -1 at u = 0, is symmetric about that centre, is 0 from t = 6 sqrt(6) / (2 pi fr) on,
    and is minus a Ricker wavelet of peak frequency fr up to the offset."""
    w = 2.0 * np.pi * fr
    tc, tmax = 3.0 * np.sqrt(6.0) / w, 6.0 * np.sqrt(6.0) / w
    off = 13.0 * np.exp(-13.5)
    assert abs(O.time_function(0.0, 2, fr)) < 1e-15
    assert abs(O.time_function(tc, 2, fr) + 1.0) < 1e-15
    assert O.time_function(tmax, 2, fr) == 0.0 and O.time_function(2 * tmax, 2, fr) == 0.0
    for tau in (0.1 * tc, 0.37 * tc, 0.8 * tc):
        a, b = O.time_function(tc - tau, 2, fr), O.time_function(tc + tau, 2, fr)
        assert abs(a - b) < 1e-14
        ricker = (1.0 - 2.0 * (np.pi * fr * tau) ** 2) * np.exp(-((np.pi * fr * tau) ** 2))
        assert abs(a - (-0.5 * ricker - off) / (0.5 + off)) < 1e-14


def test_time_function_gaussian_and_table_layout():
    """Case 3 is exp(-(t - 0.06)^2 / 0.0004); the per-step table holds the values at
    T, T + dt and T + dt/2 (the three calls of the RK4 step)."""
    assert O.time_function(0.06, 3) == 1.0
    assert abs(O.time_function(0.08, 3) - np.exp(-1.0)) < 1e-15
    dt = 1e-3
    tab = O.time_table(10, dt, 2, 15.0)
    for i in range(11):
        T = i * dt
        assert tab[i, 0] == O.time_function(T, 2, 15.0)
        assert tab[i, 1] == O.time_function(T + dt, 2, 15.0)
        assert tab[i, 2] == O.time_function(T + 0.5 * dt, 2, 15.0)
    assert np.array_equal(tab[1:, 0], tab[:-1, 1])
