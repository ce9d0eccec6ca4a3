"""Device assembly of C, K, G and DIAG_M against the oracle's ASSEM_* restatement."""
import numpy as np
import pytest

import oracle as O
from problems import RHO, oracle_forward, rel_l2, tiny

pytestmark = pytest.mark.gpu


def _assembled(p, lam, mu, precision="fp64", solver=None):
    from hirensi_b200.solver import Solver
    s = solver or Solver(precision)
    if solver is None:
        s.set_mesh(p["mesh"], RHO)
    s.assemble(lam, mu)
    return s


@pytest.mark.parametrize("npml", [1, 2])
def test_pattern_and_values_match_oracle(gpu_lib, npml):
    p = tiny(nx=4, ny=2, nz=2, npml=npml)
    om = O.OracleMesh(p["mesh"], RHO)
    S = O.OracleSystem.assemble(om, p["lam_t"], p["mu_t"])
    with _assembled(p, p["lam_t"], p["mu_t"]) as s:
        for w in range(3):
            ia_r, ja_r, a_r = S.csr(w)
            ia, ja, a = s.operator_csr(w)
            # same stored entries as PETSc with MAT_IGNORE_ZERO_ENTRIES
            assert np.array_equal(ia, ia_r), w
            assert np.array_equal(ja, ja_r), w
            # element arithmetic is identical; only the order of the cross-element sum
            # differs, so entries that cancel to round-off may differ in their residue
            assert np.max(np.abs(a - a_r)) <= 1e-14 * np.abs(a_r).max(), w
            big = np.abs(a_r) > 1e-8 * np.abs(a_r).max()
            assert np.max(np.abs(a - a_r)[big] / np.abs(a_r)[big]) < 1e-13, w
        dm_r, _ = S.vectors()
        assert np.max(np.abs(s.diag_m() - dm_r) / dm_r) < 1e-14


def test_reassembly_keeps_pattern(gpu_lib):
    p = tiny(nx=4, ny=4, nz=2, npml=1)
    om = O.OracleMesh(p["mesh"], RHO)
    with _assembled(p, p["lam"], p["mu"]) as s:
        s.assemble(p["lam_t"], p["mu_t"])
        S = O.OracleSystem.assemble(om, p["lam_t"], p["mu_t"])
        for w in range(3):
            ia_r, ja_r, a_r = S.csr(w)
            ia, ja, a = s.operator_csr(w)
            assert np.array_equal(ja, ja_r)
            assert rel_l2(a, a_r) < 1e-14


def test_forward_through_device_assembly(gpu_lib):
    p = tiny(nshot=2, nstep=250)
    _, _, hist = oracle_forward(p, p["lam_t"], p["mu_t"])
    with _assembled(p, p["lam_t"], p["mu_t"]) as s:
        s.set_history(p["mesh"].store_eq)
        s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
        s.set_receivers(p["eqdis"], p["eqdis_map"])
        s.forward()
        for k in range(2):
            assert rel_l2(s.history(k), hist[k]) < 1e-10
