"""Matrix-free stage variants against the FP64 oracle, with the operator assembled
on the device from the mesh.

Even variants (90, 92, 94) write each element's contribution to a slot and sum
the slots of a row in ascending element order (reproducible run to run); odd
variants (91, 93, 95) add the contributions atomically.  90/91 take one shot per
thread, 92/93 two, 94/95 four (FP32 only); 100-105 are the same with the stage
inputs rebuilt from x and kb instead of materialized by the previous stage.  Tolerances as in the CSR parity tests: FP64 1e-10
relative L2 for histories, adjoint histories and gradients; FP32 1e-4 for
histories and 1e-3 for gradients.
"""
import numpy as np
import pytest

import oracle as O
from problems import RHO, oracle_forward, rel_l2, tiny, traces_from_history

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 1e-4
TOL32_GRAD = 1e-3


def _solver(p, precision="fp64"):
    from hirensi_b200.solver import Solver
    s = Solver(precision)
    s.set_mesh(p["mesh"], RHO)
    s.assemble(p["lam"], p["mu"])
    s.set_history(p["mesh"].store_eq)
    s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
    s.set_receivers(p["eqdis"], p["eqdis_map"])
    return s


def _oracle_adjoint(p, om, S, hist, dis):
    gl = np.zeros(p["mesh"].nj)
    gm = np.zeros(p["mesh"].nj)
    padj = []
    for k in range(p["nshot"]):
        pk = S.adjoint(p["nstep"], p["dt"], p["mesh"].store_eq, hist[k], p["eqdis"], p["eqdis_map"], dis[k])
        padj.append(pk)
        a, b = O.control(om, p["nstep"], p["dt"], p["mesh"].store_eq, hist[k], pk)
        gl += a
        gm += b
    return padj, gl, gm


@pytest.mark.parametrize("variant,nshot", [(90, 1), (91, 1), (90, 3), (91, 3), (92, 2), (93, 4),
                                           (100, 1), (101, 3), (102, 2), (103, 4)])
def test_matrix_free_fp64_matches_oracle(gpu_lib, variant, nshot):
    p = tiny(nshot=nshot, nstep=150)
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    om, S, hist = oracle_forward(p, p["lam"], p["mu"])
    dis = np.stack([traces_from_history(p, h) for h in hist_t])
    padj, gl_ref, gm_ref = _oracle_adjoint(p, om, S, hist, dis)
    with _solver(p) as s:
        s.set_variant(variant, variant)
        s.forward()
        assert s.variant() == (variant, variant)
        for k in range(nshot):
            assert np.abs(hist[k]).max() > 0
            assert rel_l2(s.history(k), hist[k]) < TOL64
        gl, gm = s.adjoint_gradient(dis, keep_p=True)
        for k in range(nshot):
            assert rel_l2(s.adjoint_history(k)[1:], padj[k][1:]) < TOL64
        assert np.abs(gm_ref).max() > 0
        assert rel_l2(gl, gl_ref) < TOL64
        assert rel_l2(gm, gm_ref) < TOL64


@pytest.mark.parametrize("variant", [90, 91, 92, 93, 94, 95, 100, 101, 102, 103, 104, 105])
def test_matrix_free_fp32_within_bars(gpu_lib, variant):
    p = tiny(nshot=4, nstep=150)
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    om, S, hist = oracle_forward(p, p["lam"], p["mu"])
    dis = np.stack([traces_from_history(p, h) for h in hist_t])
    _, gl_ref, gm_ref = _oracle_adjoint(p, om, S, hist, dis)
    with _solver(p, "fp32") as s:
        s.set_variant(variant, variant)
        s.forward()
        for k in range(4):
            assert rel_l2(s.history(k), hist[k]) < TOL32
        gl, gm = s.adjoint_gradient(dis)
        assert rel_l2(gl, gl_ref) < TOL32_GRAD
        assert rel_l2(gm, gm_ref) < TOL32_GRAD


def test_element_slot_variant_is_reproducible(gpu_lib):
    p = tiny(nshot=2, nstep=100)
    with _solver(p) as s:
        s.set_variant(90, 90)
        s.forward()
        h1 = [s.history(k) for k in range(2)]
        s.forward()
        for k in range(2):
            assert np.array_equal(s.history(k), h1[k])


def test_matrix_free_variant_must_fit_shots_and_precision(gpu_lib):
    from hirensi_b200.solver import HrnError
    p = tiny(nshot=3, nstep=20)
    with _solver(p) as s:
        s.set_variant(92, 92)   # two shots per thread: 3 shots do not divide
        with pytest.raises(HrnError):
            s.forward()
    p = tiny(nshot=4, nstep=20)
    with _solver(p) as s:
        s.set_variant(94, 94)   # four shots per thread: FP32 only
        with pytest.raises(HrnError):
            s.forward()


def test_matrix_free_needs_an_assembled_operator(gpu_lib):
    from hirensi_b200.solver import HrnError, Solver
    p = tiny(nshot=1, nstep=20)
    _, S, _ = oracle_forward(p, p["lam"], p["mu"])
    s = Solver("fp64")
    mats = [S.csr(w) for w in range(3)]
    dm, _ = S.vectors()
    s.set_operator_csr(mats[0], mats[1], mats[2], dm)
    s.set_mesh(p["mesh"], RHO)
    s.set_history(p["mesh"].store_eq)
    s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
    s.set_receivers(p["eqdis"], p["eqdis_map"])
    s.set_variant(90, 90)
    with pytest.raises(HrnError):
        s.forward()
    s.close()


def test_operator_without_csr_equals_assembled_operator(gpu_lib):
    """hrn_set_operator_mode(matrix-free): only DIAG_M is assembled and the element
    kernels apply C, K, G; results equal those of the same variant on the fully
    assembled operator bit for bit (slot variant), and the tuner picks a matrix-free
    variant."""
    from hirensi_b200.capi import HrnError
    from hirensi_b200.solver import Solver
    p = tiny(nshot=2, nstep=120)
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    dis = np.stack([traces_from_history(p, h) for h in hist_t])
    out = []
    for mf in (False, True):
        with Solver("fp64") as s:
            s.set_mesh(p["mesh"], RHO)
            s.set_operator_mode(mf)
            s.assemble(p["lam"], p["mu"])
            s.set_history(p["mesh"].store_eq)
            s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
            s.set_receivers(p["eqdis"], p["eqdis_map"])
            s.set_variant(92, 92)
            s.forward()
            gl, gm = s.adjoint_gradient(dis)
            out.append(([s.history(k) for k in range(2)], gl, gm, s.diag_m()))
            if mf:
                assert s.operator_nnz(1) == 0
                s.set_variant(41, 41)
                with pytest.raises(HrnError):
                    s.forward()
                s.set_variant(0, 0)
                s.forward()
                assert 90 <= s.variant()[0] <= 105
    for k in range(2):
        assert np.array_equal(out[0][0][k], out[1][0][k])
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])
    assert np.array_equal(out[0][3], out[1][3])


def test_split_element_launches_on_a_larger_mesh(gpu_lib):
    """24 x 24 x 12 elements + PML 2 (10,976 elements): the element grids of the
    FP64 2-shot-per-thread and the FP32 1-shot-per-thread variants exceed 16
    blocks per SM, so the PML and regular-domain elements run as separate
    launches.  FP64 results equal the CSR kernel's to rounding (another
    summation order), FP32 results stay within the FP32 bar."""
    from hirensi_b200.solver import Solver
    p = tiny(nshot=4, nstep=30, nx=24, ny=24, nz=12, npml=2)
    assert p["mesh"].inod.shape[0] == 28 * 28 * 14

    def run(precision, variant):
        with Solver(precision) as s:
            s.set_mesh(p["mesh"], RHO)
            s.assemble(p["lam"], p["mu"])
            s.set_history(p["mesh"].store_eq)
            s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
            s.set_receivers(p["eqdis"], p["eqdis_map"])
            s.set_variant(variant, variant)
            s.forward()
            return [s.history(k) for k in range(4)]

    ref = run("fp64", 41)
    assert np.abs(ref[0]).max() > 0
    for v in (92, 93):
        h = run("fp64", v)
        for k in range(4):
            assert rel_l2(h[k], ref[k]) < 1e-12
    for v in (90, 91):
        h = run("fp32", v)
        for k in range(4):
            assert rel_l2(h[k], ref[k]) < 1e-4
