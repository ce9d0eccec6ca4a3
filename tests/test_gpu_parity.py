"""GPU parity of the CUDA time loops against the FP64 oracle (through the C ABI).

Tolerances (relative L2 over the whole compared array): FP64 stepping 1e-10
for histories, seismograms, misfit and gradients; FP32 stepping 1e-4 for
histories and seismograms and 1e-3 for gradients (a correlation of two FP32
wavefields), all against the FP64 oracle.
"""
import numpy as np
import pytest

import oracle as O
from problems import RHO, oracle_forward, rel_l2, tiny, traces_from_history

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 1e-4
TOL32_GRAD = 1e-3


def _solver(p, om_sys, precision="fp64"):
    from hirensi_b200.solver import Solver
    s = Solver(precision)
    mats = [om_sys.csr(w) for w in range(3)]
    dm, _ = om_sys.vectors()
    s.set_operator_csr(mats[0], mats[1], mats[2], dm)
    s.set_mesh(p["mesh"], RHO)
    s.set_history(p["mesh"].store_eq)
    s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
    s.set_receivers(p["eqdis"], p["eqdis_map"])
    return s


@pytest.mark.parametrize("nshot", [1, 3])
def test_forward_fp64_matches_oracle(gpu_lib, nshot):
    p = tiny(nshot=nshot, nstep=300)
    om, S, hist = oracle_forward(p, p["lam"], p["mu"])
    with _solver(p, S) as s:
        s.forward()
        for k in range(nshot):
            u = s.history(k)
            assert np.abs(hist[k]).max() > 0
            assert rel_l2(u, hist[k]) < TOL64
        tr = s.traces()
        for k in range(nshot):
            assert rel_l2(tr[k], traces_from_history(p, hist[k])) < TOL64


def test_forward_fp32_within_1e4(gpu_lib):
    p = tiny(nshot=2, nstep=300)
    om, S, hist = oracle_forward(p, p["lam"], p["mu"])
    with _solver(p, S, "fp32") as s:
        s.forward()
        for k in range(2):
            assert rel_l2(s.history(k), hist[k]) < TOL32


def test_adjoint_gradient_and_misfit_fp64(gpu_lib):
    p = tiny(nshot=2, nstep=200)
    # measured data from the true model, synthetics from the layered start model
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    om, S, hist = oracle_forward(p, p["lam"], p["mu"])
    dis = np.stack([traces_from_history(p, h) for h in hist_t])
    store = p["mesh"].store_eq
    J_ref = sum(O.misfit(p["nstep"], p["dt"], p["eqdis"], p["eqdis_map"], hist[k], dis[k]) for k in range(2))
    g_ref_l = np.zeros(p["mesh"].nj)
    g_ref_m = np.zeros(p["mesh"].nj)
    p_ref = []
    for k in range(2):
        pk = S.adjoint(p["nstep"], p["dt"], store, hist[k], p["eqdis"], p["eqdis_map"], dis[k])
        p_ref.append(pk)
        gl, gm = O.control(om, p["nstep"], p["dt"], store, hist[k], pk)
        g_ref_l += gl
        g_ref_m += gm
    with _solver(p, S) as s:
        s.forward()
        J = s.misfit(dis)
        assert J > 0
        assert abs(J - J_ref) <= TOL64 * abs(J_ref)
        gl, gm = s.adjoint_gradient(dis, keep_p=True)
        for k in range(2):
            assert rel_l2(s.adjoint_history(k)[1:], p_ref[k][1:]) < TOL64
        assert np.abs(g_ref_m).max() > 0
        assert rel_l2(gl, g_ref_l) < TOL64
        assert rel_l2(gm, g_ref_m) < TOL64


def test_gradient_fp32_within_1e4(gpu_lib):
    p = tiny(nshot=1, nstep=200)
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    om, S, hist = oracle_forward(p, p["lam"], p["mu"])
    dis = traces_from_history(p, hist_t[0])[None]
    pk = S.adjoint(p["nstep"], p["dt"], p["mesh"].store_eq, hist[0], p["eqdis"], p["eqdis_map"], dis[0])
    gl_ref, gm_ref = O.control(om, p["nstep"], p["dt"], p["mesh"].store_eq, hist[0], pk)
    with _solver(p, S, "fp32") as s:
        s.forward()
        gl, gm = s.adjoint_gradient(dis)
        assert rel_l2(gl, gl_ref) < TOL32_GRAD
        assert rel_l2(gm, gm_ref) < TOL32_GRAD


@pytest.mark.parametrize("variant", [40, 80, 160, 41, 81, 161, 42, 43, 82, 83, 44, 45, 84, 85, 46, 86, 47, 87])
def test_every_stage_kernel_variant_matches_oracle(gpu_lib, variant):
    p = tiny(nshot=2, nstep=120)
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    om, S, hist = oracle_forward(p, p["lam"], p["mu"])
    dis = np.stack([traces_from_history(p, h) for h in hist_t])
    pk = S.adjoint(p["nstep"], p["dt"], p["mesh"].store_eq, hist[0], p["eqdis"], p["eqdis_map"], dis[0])
    with _solver(p, S) as s:
        s.set_variant(variant, variant)
        s.forward()
        assert s.variant() == (variant, variant)
        for k in range(2):
            assert rel_l2(s.history(k), hist[k]) < TOL64
        s.adjoint_gradient(dis, keep_p=True)
        assert rel_l2(s.adjoint_history(0)[1:], pk[1:]) < TOL64


def test_receivers_sharing_equations_fp64(gpu_lib):
    """Receivers listed twice (the same equations with different measured data): the
    residuals of one equation add before the misfit squares them and before the
    adjoint source takes them, as the reference assembles them into one vector."""
    p = tiny(nshot=2, nstep=150)
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    om, S, hist = oracle_forward(p, p["lam"], p["mu"])
    dis1 = np.stack([traces_from_history(p, h) for h in hist_t])
    eqdis = np.concatenate([p["eqdis"], p["eqdis"][:6]])
    emap = np.concatenate([p["eqdis_map"], p["eqdis_map"][:6]])
    rng = np.random.default_rng(4)
    extra = dis1[:, :6] * (1.0 + 0.1 * rng.standard_normal(dis1[:, :6].shape))
    dis = np.ascontiguousarray(np.concatenate([dis1, extra], axis=1))
    store = p["mesh"].store_eq
    J_ref = sum(O.misfit(p["nstep"], p["dt"], eqdis, emap, hist[k], dis[k]) for k in range(2))
    g_ref_l = np.zeros(p["mesh"].nj)
    g_ref_m = np.zeros(p["mesh"].nj)
    for k in range(2):
        pk = S.adjoint(p["nstep"], p["dt"], store, hist[k], eqdis, emap, dis[k])
        gl, gm = O.control(om, p["nstep"], p["dt"], store, hist[k], pk)
        g_ref_l += gl
        g_ref_m += gm
    with _solver(p, S) as s:
        s.set_receivers(eqdis, emap)
        s.forward()
        J = s.misfit(dis)
        assert J > 0 and abs(J - J_ref) <= TOL64 * J_ref
        gl, gm = s.adjoint_gradient(dis)
        assert np.abs(g_ref_m).max() > 0
        assert rel_l2(gl, g_ref_l) < TOL64
        assert rel_l2(gm, g_ref_m) < TOL64
