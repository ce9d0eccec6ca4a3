"""GPU parity at the benchmark configurations' own sizes, through the C ABI.

* Forward-only configuration: 16x16x8 27-node hexahedra (2.5 m) + 3-element PML,
  3-layer model, one vertical Ricker force (15 Hz) at the surface centre, 2000
  steps at dt = 1e-4, 5x5 surface receivers.  The device-assembled operator's
  histories and seismograms against the FP64 oracle: FP64 stepping <= 1e-10,
  FP32 stepping <= 1e-4 (relative L2).
* Inversion configuration, one shot (the shot at (-10, -10)), 2000 steps: misfit
  and raw gradient of the initial (linear Vs) model against data of the true
  model (layers + Gaussian anomaly), against the oracle's forward, adjoint and
  control (S4/Solver_PETSc_Explicit.F90:660-1522): FP64 <= 1e-10, FP32 gradient
  <= 1e-3.
* The dot-product test of the device's per-step operators on random vectors:
  <M A x, y> = +-<M x, A'^T y> (S4/Solver_PETSc_Explicit.F90:1219-1229), and the
  device operator equals the oracle's.
* The finite-difference gradient check of S4/Gradient_check.F90:22-35 (mu) and
  :123-135 (lambda) on the inversion configuration (4 shots, 2000 steps), all
  through hrn_assemble / hrn_forward / hrn_misfit / hrn_adjoint_gradient: a
  relative perturbation of 1e-4 of one nodal value at 10 random regular-domain
  nodes, compared with the sign-flipped gradient before the gradient-mass scaling.

The oracle runs with every host thread (its results do not depend on the count).
"""
import os

import numpy as np
import pytest

import oracle as O
from problems import rel_l2

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 1e-4
TOL32_GRAD = 1e-3
NT = os.cpu_count() or 1


def _solver(prob, precision, lam, mu):
    from hirensi_b200.configs import RHO
    from hirensi_b200.solver import Solver
    s = Solver(precision)
    s.set_mesh(prob.mesh, RHO)
    s.assemble(lam, mu)
    s.set_history(prob.mesh.store_eq)
    s.set_shots(prob.nstep, prob.dt, prob.src_eq, prob.src_b, prob.ftab)
    s.set_receivers(prob.eqdis, prob.eqdis_map)
    return s


def _oracle_history(prob, lam, mu, shot=0):
    from hirensi_b200.configs import RHO
    om = O.OracleMesh(prob.mesh, RHO)
    S = O.OracleSystem.assemble(om, lam, mu)
    b = np.zeros(prob.mesh.neq)
    b[prob.src_eq[shot]] = 1.0
    u = S.forward(b, prob.ftab[shot], prob.nstep, prob.dt, prob.mesh.store_eq, nthreads=NT)
    return om, S, u


# -- forward-only configuration ------------------------------------------------------

@pytest.fixture(scope="module")
def forward_case():
    from hirensi_b200.configs import forward_config
    prob = forward_config()
    _, _, u = _oracle_history(prob, prob.lam_true, prob.mu_true)
    return prob, u


@pytest.mark.parametrize("precision,tol", [("fp64", TOL64), ("fp32", TOL32)])
def test_forward_configuration_seismograms(gpu_lib, forward_case, precision, tol):
    prob, u_ref = forward_case
    assert prob.nstep == 2000 and prob.mesh.nel == 5324 and prob.eqdis.size == 75
    with _solver(prob, precision, prob.lam_true, prob.mu_true) as s:
        s.forward()
        u = s.history(0)
        tr = s.traces()[0]
    tr_ref = np.ascontiguousarray(u_ref[:, prob.eqdis_map].T)
    assert np.abs(tr_ref).max() > 0
    e_hist, e_tr = rel_l2(u, u_ref), rel_l2(tr, tr_ref)
    print(f"forward configuration {precision}: history {e_hist:.2e}, seismograms {e_tr:.2e}")
    assert e_hist < tol and e_tr < tol


# -- inversion configuration, one shot ------------------------------------------------

@pytest.fixture(scope="module")
def gradient_case():
    from hirensi_b200.configs import inversion_config
    prob = inversion_config(shots=((-10.0, -10.0),))
    _, _, u_t = _oracle_history(prob, prob.lam_true, prob.mu_true)
    dis = np.ascontiguousarray(u_t[:, prob.eqdis_map].T)
    del u_t
    om, S, u = _oracle_history(prob, prob.lam0, prob.mu0)
    store = prob.mesh.store_eq
    J = O.misfit(prob.nstep, prob.dt, prob.eqdis, prob.eqdis_map, u, dis)
    p = S.adjoint(prob.nstep, prob.dt, store, u, prob.eqdis, prob.eqdis_map, dis, nthreads=NT)
    gl, gm = O.control(om, prob.nstep, prob.dt, store, u, p, nthreads=NT)
    return prob, dis, J, gl, gm


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_inversion_configuration_misfit_and_gradient(gpu_lib, gradient_case, precision):
    prob, dis, J_ref, gl_ref, gm_ref = gradient_case
    with _solver(prob, precision, prob.lam0, prob.mu0) as s:
        s.forward()
        J = s.misfit(dis[None])
        gl, gm = s.adjoint_gradient(dis[None])
    assert J_ref > 0 and np.abs(gm_ref).max() > 0
    e_j, e_l, e_m = abs(J - J_ref) / J_ref, rel_l2(gl, gl_ref), rel_l2(gm, gm_ref)
    print(f"inversion configuration {precision}: misfit {e_j:.2e}, g_lambda {e_l:.2e}, g_mu {e_m:.2e}")
    if precision == "fp64":
        assert e_j < TOL64 and e_l < TOL64 and e_m < TOL64
    else:
        assert e_j < TOL32 and e_l < TOL32_GRAD and e_m < TOL32_GRAD


# -- dot-product test of the device operator ----------------------------------------------

@pytest.mark.parametrize("which", [0, 1, 2])
def test_device_operator_dot_product(gpu_lib, which):
    from hirensi_b200.configs import RHO, forward_config
    prob = forward_config(nstep=10)
    m = prob.mesh
    om = O.OracleMesh(m, RHO)
    S = O.OracleSystem.assemble(om, prob.lam_true, prob.mu_true)
    rng = np.random.default_rng(10 + which)
    x = rng.standard_normal(m.neq)
    y = rng.standard_normal(m.neq)
    with _solver(prob, "fp64", prob.lam_true, prob.mu_true) as s:
        dm = s.diag_m()
        ax = s.apply_operator(which, x)
        aty = s.apply_operator(which, y, adjoint=True)
    # the device operator is the oracle's (assembly order differs: colour order)
    assert rel_l2(ax, S.apply(which, x)) < 1e-12
    assert rel_l2(aty, S.apply(which, y, transpose_adjoint=True)) < 1e-12
    lhs = float((dm * ax) @ y)
    rhs = float((dm * x) @ aty)
    sign = 1.0 if which == 1 else -1.0   # the OtD adjoint flips C and G, keeps K
    assert abs(lhs) > 0
    assert abs(lhs - sign * rhs) <= 1e-12 * abs(lhs)


# -- finite-difference gradient check through the GPU path ------------------------------------

def test_gradient_check_finite_differences(gpu_lib):
    from hirensi_b200.configs import inversion_config
    prob = inversion_config()
    m = prob.mesh
    with _solver(prob, "fp64", prob.lam_true, prob.mu_true) as s:
        s.forward()
        dis = s.traces()
        s.set_data(dis)
        s.assemble(prob.lam0, prob.mu0)
        s.forward()
        J0 = s.misfit(None)
        gl, gm = s.adjoint_gradient(None)
        g = {"lam": -gl, "mu": -gm}          # S4/Program_Main.F90:412-413, before iMg
        rd = np.nonzero((m.node_mat_id == 0) & (m.xyz[:, 2] > -12.0))[0]
        nodes = np.random.default_rng(0).choice(rd, 10, replace=False)
        eps = 1.0e-4
        rows = []
        for k in nodes:
            for name in ("mu", "lam"):
                lam, mu = prob.lam0.copy(), prob.mu0.copy()
                arr = mu if name == "mu" else lam
                base = arr[k]
                arr[k] = base * (1.0 + eps)
                s.assemble(lam, mu)
                s.forward()
                fd = (s.misfit(None) - J0) / (base * eps)
                rows.append((int(k), name, fd, g[name][k]))
    fd = np.array([r[2] for r in rows])
    adj = np.array([r[3] for r in rows])
    rel = np.abs(fd - adj) / np.abs(fd)
    for (k, name, f, a), e in zip(rows, rel):
        print(f"node {k:6d} {name:3s}: FD {f:+.6e}  adjoint {a:+.6e}  rel {e:.2e}")
    cos = float(fd @ adj / (np.linalg.norm(fd) * np.linalg.norm(adj)))
    print(f"cosine {cos:.8f}, median rel {np.median(rel):.2e}, max rel {rel.max():.2e}")
    assert np.all(np.sign(fd) == np.sign(adj))
    assert cos > 0.9999
    assert np.median(rel) < 1e-2
