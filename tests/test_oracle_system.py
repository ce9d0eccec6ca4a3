"""Algebraic checks of the oracle's assembled operator and time loops (CPU).

* dot-product test of every per-step operator: with A = -M^-1 X (forward) and
  A' = the adjoint-scaled operator, <M A x, y> = +-<M x, A'^T y> (+ for K,
  - for the first-order terms C and G, whose sign the OtD adjoint flips);
* linearity of the forward loop in the source (bit exact for a factor 2);
* the finite-difference gradient check of S4/Gradient_check.F90 (relative
  perturbation 1e-4 of one nodal mu or lambda, compared with the sign-flipped
  gradient before the gradient-mass scaling) at 10 random regular-domain nodes.
  The OtD gradient is not the exact derivative of the discrete misfit, so on
  this coarse 300-step problem the two agree to a few percent (direction cosine
  above 0.999), not to the 2e-4 the reference reports for its fine mesh.
"""
import numpy as np
import pytest

import oracle as O
from problems import RHO, oracle_forward, tiny, traces_from_history


@pytest.fixture(scope="module")
def prob():
    p = tiny(nshot=1, nstep=300, nx=4, ny=4, nz=2, npml=1, fr=60.0)
    om, S, hist = oracle_forward(p, p["lam"], p["mu"])
    return p, om, S, hist


def test_operator_shapes(prob):
    p, om, S, _ = prob
    for w in range(3):
        ia, ja, a = S.csr(w)
        assert ia[0] == 0 and ia[-1] == a.size and np.all(np.diff(ia) >= 0)
        # entries whose element contributions cancel stay stored as explicit zeros
        assert np.count_nonzero(a) > 0.8 * a.size
        for i in range(0, p["mesh"].neq, 97):   # sorted unique columns
            assert np.all(np.diff(ja[ia[i]:ia[i + 1]]) > 0)
    dm, _ = S.vectors()
    assert np.all(dm > 0)


def test_regular_domain_stiffness_is_symmetric(prob):
    p, om, S, _ = prob
    m = p["mesh"]
    ia, ja, a = S.csr(1)
    K = np.zeros((m.neq, m.neq))
    for i in range(m.neq):
        K[i, ja[ia[i]:ia[i + 1]]] = a[ia[i]:ia[i + 1]]
    rd_nodes = np.nonzero(m.node_mat_id == 0)[0]
    eq = m.ID[rd_nodes, :3].ravel()
    sub = K[np.ix_(eq, eq)]
    assert np.array_equal(sub, sub.T)


@pytest.mark.parametrize("which", [0, 1, 2])
def test_dot_product_adjoint_operator(prob, which):
    p, om, S, _ = prob
    rng = np.random.default_rng(which)
    dm, _ = S.vectors()
    x = rng.standard_normal(p["mesh"].neq)
    y = rng.standard_normal(p["mesh"].neq)
    lhs = float((dm * S.apply(which, x)) @ y)
    rhs = float((dm * x) @ S.apply(which, y, transpose_adjoint=True))
    # the adjoint keeps -K but flips C and G (S4/Solver_PETSc_Explicit.F90:1219-1223)
    sign = 1.0 if which == 1 else -1.0
    assert abs(lhs - sign * rhs) <= 1e-12 * max(abs(lhs), 1e-300)


def test_forward_is_linear_in_the_source(prob):
    p, om, S, hist = prob
    b = np.zeros(p["mesh"].neq)
    b[p["src_eq"][0]] = 2.0
    u2 = S.forward(b, p["ftab"][0], p["nstep"], p["dt"], p["mesh"].store_eq)
    assert np.array_equal(u2, 2.0 * hist[0])


def test_misfit_vanishes_on_own_data(prob):
    p, om, S, hist = prob
    dis = traces_from_history(p, hist[0])
    assert O.misfit(p["nstep"], p["dt"], p["eqdis"], p["eqdis_map"], hist[0], dis) == 0.0
    J = O.misfit(p["nstep"], p["dt"], p["eqdis"], p["eqdis_map"], hist[0], 0.0 * dis)
    ref = 0.5 * p["dt"] * float((dis[:, 1:] ** 2).sum())
    assert abs(J - ref) <= 1e-12 * ref


def test_finite_difference_gradient(prob):
    p, om, S, hist = prob
    m = p["mesh"]
    _, _, ht = oracle_forward(p, p["lam_t"], p["mu_t"])
    dis = traces_from_history(p, ht[0])

    def J(lam, mu):
        _, _, h = oracle_forward(p, lam, mu)
        return O.misfit(p["nstep"], p["dt"], p["eqdis"], p["eqdis_map"], h[0], dis)

    lam, mu = p["lam"], p["mu"]
    J0 = J(lam, mu)
    pk = S.adjoint(p["nstep"], p["dt"], m.store_eq, hist[0], p["eqdis"], p["eqdis_map"], dis)
    gl, gm = O.control(om, p["nstep"], p["dt"], m.store_eq, hist[0], pk)
    g = {"lam": -gl, "mu": -gm}   # S4/Program_Main.F90:412-413
    rd = np.nonzero(m.node_mat_id == 0)[0]
    nodes = np.random.default_rng(0).choice(rd, 10, replace=False)
    fd, adj = [], []
    eps = 1.0e-4
    for k in nodes:
        for name in ("mu", "lam"):
            l2, m2 = lam.copy(), mu.copy()
            arr = m2 if name == "mu" else l2
            base = arr[k]
            arr[k] = base * (1.0 + eps)
            fd.append((J(l2, m2) - J0) / (base * eps))
            adj.append(g[name][k])
    fd, adj = np.array(fd), np.array(adj)
    cos = float(fd @ adj / (np.linalg.norm(fd) * np.linalg.norm(adj)))
    assert cos > 0.999
    big = np.abs(fd) > 0.1 * np.abs(fd).max()
    assert np.median(np.abs(fd[big] - adj[big]) / np.abs(fd[big])) < 0.1


def test_forward_is_fourth_order_in_dt():
    """Known answer of the integrator: the displacement at a fixed time from steps
    dt, dt/2, dt/4 (the source sampled at t, t + dt/2, t + dt each step) differs by
    amounts whose ratio is 2^4 = 16, as for classical RK4 on the semi-discrete
    system with its C (damping) and G (integral) terms."""
    p = tiny(nshot=1, nstep=300)
    om = O.OracleMesh(p["mesh"], RHO)
    S = O.OracleSystem.assemble(om, p["lam"], p["mu"])
    b = np.zeros(p["mesh"].neq)
    b[p["src_eq"][0]] = 1.0
    T = 0.024
    end = {}
    for dt in (2e-4, 1e-4, 5e-5):
        n = int(round(T / dt))
        end[dt] = S.forward(b, O.time_table(n, dt, 2, 60.0), n, dt, p["mesh"].store_eq)[-1]
    assert np.abs(end[5e-5]).max() > 0
    e1 = np.linalg.norm(end[2e-4] - end[1e-4])
    e2 = np.linalg.norm(end[1e-4] - end[5e-5])
    assert 14.0 < e1 / e2 < 18.0


@pytest.mark.parametrize("alpha0", [0.0, 5.0])
def test_pml_without_attenuation_keeps_only_the_stretching_coupling(alpha0):
    """Known answer of the mixed displacement-stress PML: with beta0 = 0 the
    coefficients b, c, d and the weights of the p and w kinds vanish (each holds a
    factor beta).  So G has no entries, K is the regular-domain stiffness alone
    (no stress DOF, no displacement row of a node outside the regular domain), and
    C couples displacements and stresses only, through the alpha-only weights of
    kind e.  K does not depend on alpha0."""
    from hirensi_b200.mesh import box_mesh
    from problems import layered
    m = box_mesh(4, 4, 2, 2.5, 1, alpha0=alpha0, beta0=0.0)
    lam, mu = layered(m)
    S = O.OracleSystem.assemble(O.OracleMesh(m, RHO), lam, mu)
    stress = np.zeros(m.neq, bool)
    e = m.ID[:, 3:9]
    stress[e[e >= 0]] = True
    rd_nodes = np.unique(m.inod[m.mtel == 1])
    in_rd = np.zeros(m.neq, bool)
    u = m.ID[rd_nodes, 0:3]
    in_rd[u[u >= 0]] = True

    def blocks(which):
        ia, ja, a = S.csr(which)
        rows = np.repeat(np.arange(m.neq), np.diff(ia))
        nz = a != 0
        return rows[nz], ja[nz], a[nz]

    r, c, _ = blocks(2)
    assert r.size == 0
    r, c, kv = blocks(1)
    assert r.size > 0 and not stress[r].any() and not stress[c].any()
    assert in_rd[r].all() and in_rd[c].all()
    r, c, _ = blocks(0)
    assert r.size > 0
    assert np.all(stress[r] != stress[c])
    # the regular-domain stiffness is the same for any alpha0
    m0 = box_mesh(4, 4, 2, 2.5, 1, alpha0=0.0, beta0=0.0)
    S0 = O.OracleSystem.assemble(O.OracleMesh(m0, RHO), lam, mu)
    ia0, ja0, a0 = S0.csr(1)
    ia1, ja1, a1 = S.csr(1)
    assert np.array_equal(ia0, ia1) and np.array_equal(ja0, ja1) and np.array_equal(a0, a1)


def test_misfit_formula_with_duplicate_receivers():
    """Compute_Misfit: J = sum over n = 1..NSTEP of dt/2 |r_n|^2, where r_n is
    assembled into the equation vector, so receivers that share an equation add
    before squaring; step 0 does not count."""
    rng = np.random.default_rng(2)
    nstep, dt, nstore = 12, 1e-3, 9
    eqdis = np.array([5, 7, 5, 11, 7, 3], np.int32)           # equations 5 and 7 twice
    eqdis_map = np.array([0, 4, 0, 8, 4, 2], np.int32)        # their positions in U_Store
    u = rng.standard_normal((nstep + 1, nstore))
    d = rng.standard_normal((len(eqdis), nstep + 1))
    J = O.misfit(nstep, dt, eqdis, eqdis_map, u, d)
    ref = 0.0
    for n in range(1, nstep + 1):
        r = {}
        for q, e in enumerate(eqdis):
            r[e] = r.get(e, 0.0) + u[n, eqdis_map[q]] - d[q, n]
        ref += 0.5 * dt * sum(v * v for v in r.values())
    assert abs(J - ref) <= 1e-14 * ref
    d0 = d.copy()
    d0[:, 0] += 100.0
    assert O.misfit(nstep, dt, eqdis, eqdis_map, u, d0) == J
