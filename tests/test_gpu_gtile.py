"""Staged-gather stage kernels (variants 44-47, 84-87) through the C ABI.

The rows are cut into compact tiles whose gathered stage inputs are loaded once
into shared memory.  Entries keep their order inside a row, so with the same
lane count and stage-input mode the row sums are those of the row-parallel
kernel: 44 = 40, 45 = 41, 84 = 80, 85 = 81 bit for bit; 46 and 86 stage the same
records by bulk copies of runs of consecutive columns, so 46 = 41 and 86 = 81; 47 and 87
run the same sums and epilogue in persistent CTAs whose producer warp moves each tile's
data by bulk copies while the consumer warps work on the previous tile, so 47 = 41 and
87 = 81.  Parity against the FP64
oracle uses the bars of the other stage kernels (1e-10 FP64, 1e-4 FP32).
"""
import numpy as np
import pytest

from problems import RHO, oracle_forward, rel_l2, tiny, traces_from_history

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 1e-4
PAIRS = [(44, 40), (45, 41), (84, 80), (85, 81)]


def _csr_solver(p, om_sys, precision="fp64", mesh=True):
    from hirensi_b200.solver import Solver
    s = Solver(precision)
    mats = [om_sys.csr(w) for w in range(3)]
    dm, _ = om_sys.vectors()
    s.set_operator_csr(mats[0], mats[1], mats[2], dm)
    if mesh:
        s.set_mesh(p["mesh"], RHO)
    s.set_history(p["mesh"].store_eq)
    s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
    s.set_receivers(p["eqdis"], p["eqdis_map"])
    return s


def _assembled_solver(p, lam, mu, precision="fp64"):
    from hirensi_b200.solver import Solver
    s = Solver(precision)
    s.set_mesh(p["mesh"], RHO)
    s.assemble(lam, mu)
    s.set_history(p["mesh"].store_eq)
    s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
    s.set_receivers(p["eqdis"], p["eqdis_map"])
    return s


@pytest.mark.parametrize("variant,row_parallel", PAIRS)
def test_staged_tiles_equal_row_parallel_kernel(gpu_lib, variant, row_parallel):
    p = tiny(nshot=3, nstep=150)
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    dis = np.stack([traces_from_history(p, h) for h in hist_t])
    out = {}
    for v in (variant, row_parallel):
        with _assembled_solver(p, p["lam"], p["mu"]) as s:
            s.set_variant(v, v)
            s.forward()
            assert s.variant() == (v, v)
            gl, gm = s.adjoint_gradient(dis, keep_p=True)
            out[v] = ([s.history(k) for k in range(3)], [s.adjoint_history(k) for k in range(3)])
    for k in range(3):
        assert np.array_equal(out[variant][0][k], out[row_parallel][0][k])
        assert np.array_equal(out[variant][1][k], out[row_parallel][1][k])


@pytest.mark.parametrize("mesh", [True, False])
def test_staged_tiles_fp64_match_oracle(gpu_lib, mesh):
    """With the mesh the tiles follow a Morton curve of the nodes; without it
    they are runs of consecutive rows."""
    p = tiny(nshot=2, nstep=200)
    om, S, hist = oracle_forward(p, p["lam"], p["mu"])
    with _csr_solver(p, S, mesh=mesh) as s:
        s.set_variant(45, 45)
        s.forward()
        for k in range(2):
            assert np.abs(hist[k]).max() > 0
            assert rel_l2(s.history(k), hist[k]) < TOL64


@pytest.mark.parametrize("nshot,variant", [(4, 45), (8, 44), (8, 85)])
def test_staged_tiles_fp32_within_bars(gpu_lib, nshot, variant):
    p = tiny(nshot=nshot, nstep=200)
    om, S, hist = oracle_forward(p, p["lam"], p["mu"])
    with _csr_solver(p, S, "fp32") as s:
        s.set_variant(variant, variant)
        s.forward()
        for k in range(nshot):
            assert rel_l2(s.history(k), hist[k]) < TOL32


def test_staged_tiles_follow_reassembly(gpu_lib):
    """A new model rescales the operator; the tile-ordered values follow it."""
    p = tiny(nshot=2, nstep=150)
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    with _assembled_solver(p, p["lam"], p["mu"]) as s:
        s.set_variant(45, 45)
        s.forward()
        s.assemble(p["lam_t"], p["mu_t"])
        s.forward()
        for k in range(2):
            assert rel_l2(s.history(k), hist_t[k]) < TOL64


def test_staged_tiles_split_to_fit_shared_memory(gpu_lib):
    """Eight FP64 shots make 64-byte records, so the larger tiles of the
    16 x 16 x 8 mesh are halved until their staged set fits; results still equal
    the row-parallel kernel's."""
    from hirensi_b200 import configs
    shots = [(x, y) for x in (-15.0, -5.0, 5.0, 15.0) for y in (-10.0, 10.0)]
    prob = configs.inversion_config(nstep=12, shots=shots)
    m = prob.mesh
    nshot = prob.nshot
    assert nshot == 8
    hists = {}
    for v in (85, 81):
        from hirensi_b200.solver import Solver
        with Solver("fp64") as s:
            s.set_mesh(m, RHO)
            s.assemble(prob.lam0, prob.mu0)
            s.set_history(m.store_eq)
            s.set_shots(prob.nstep, prob.dt, prob.src_eq, prob.src_b, prob.ftab)
            s.set_receivers(prob.eqdis, prob.eqdis_map)
            s.set_variant(v, v)
            s.forward()
            hists[v] = [s.history(k) for k in range(nshot)]
    for k in range(nshot):
        assert np.abs(hists[81][k]).max() > 0
        assert np.array_equal(hists[85][k], hists[81][k])


@pytest.mark.parametrize("nshot,precision", [(5, "fp64"), (6, "fp64"), (7, "fp32"), (6, "fp32")])
def test_staged_tiles_odd_shot_counts(gpu_lib, nshot, precision):
    """Shot counts whose records take the scalar and 2-wide shared-memory paths."""
    p = tiny(nshot=nshot, nstep=60)
    out = {}
    for v in (45, 41):
        with _assembled_solver(p, p["lam"], p["mu"], precision) as s:
            s.set_variant(v, v)
            s.forward()
            out[v] = [s.history(k) for k in range(nshot)]
    for k in range(nshot):
        assert np.abs(out[41][k]).max() > 0
        assert np.array_equal(out[45][k], out[41][k])


@pytest.mark.parametrize("nshot,precision,variant,row_parallel",
                         [(2, "fp64", 46, 41), (4, "fp64", 86, 81), (4, "fp32", 46, 41), (8, "fp32", 86, 81),
                          (2, "fp64", 47, 41), (4, "fp64", 47, 41), (4, "fp64", 87, 81), (4, "fp32", 47, 41),
                          (8, "fp32", 87, 81)])
def test_bulk_copied_runs_equal_row_parallel_kernel(gpu_lib, nshot, precision, variant, row_parallel):
    """Records of a multiple of 16 bytes moved by one bulk copy per run of
    consecutive columns: histories and adjoint histories equal the row-parallel
    kernel's bit for bit, in every stage (stage 1 copies from the state, stages
    2-4 from the materialized inputs)."""
    p = tiny(nshot=nshot, nstep=120)
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    dis = np.stack([traces_from_history(p, h) for h in hist_t])
    out = {}
    for v in (variant, row_parallel):
        with _assembled_solver(p, p["lam"], p["mu"], precision) as s:
            s.set_variant(v, v)
            s.forward()
            assert s.variant() == (v, v)
            s.adjoint_gradient(dis, keep_p=True)
            out[v] = ([s.history(k) for k in range(nshot)], [s.adjoint_history(k) for k in range(nshot)])
    for k in range(nshot):
        assert np.abs(out[row_parallel][0][k]).max() > 0
        assert np.array_equal(out[variant][0][k], out[row_parallel][0][k])
        assert np.array_equal(out[variant][1][k], out[row_parallel][1][k])


@pytest.mark.parametrize("variant", [86, 87])
def test_bulk_copied_runs_on_split_tiles(gpu_lib, variant):
    """Eight FP64 shots (64-byte records) on the 16 x 16 x 8 mesh: halved tiles, runs
    of 64-byte records; equal to the row-parallel kernel."""
    from hirensi_b200 import configs
    from hirensi_b200.solver import Solver
    shots = [(x, y) for x in (-15.0, -5.0, 5.0, 15.0) for y in (-10.0, 10.0)]
    prob = configs.inversion_config(nstep=12, shots=shots)
    m = prob.mesh
    hists = {}
    for v in (variant, 81):
        with Solver("fp64") as s:
            s.set_mesh(m, RHO)
            s.assemble(prob.lam0, prob.mu0)
            s.set_history(m.store_eq)
            s.set_shots(prob.nstep, prob.dt, prob.src_eq, prob.src_b, prob.ftab)
            s.set_receivers(prob.eqdis, prob.eqdis_map)
            s.set_variant(v, v)
            s.forward()
            hists[v] = [s.history(k) for k in range(prob.nshot)]
    for k in range(prob.nshot):
        assert np.abs(hists[81][k]).max() > 0
        assert np.array_equal(hists[variant][k], hists[81][k])


def test_bulk_copied_runs_refuse_unaligned_records(gpu_lib):
    """Three FP64 shots make 24-byte records, which a bulk copy cannot move: the
    forward fails with HRN_EARG and the tuner never picks 46 / 86 for them."""
    from hirensi_b200.capi import HrnError
    p = tiny(nshot=3, nstep=20)
    with _assembled_solver(p, p["lam"], p["mu"]) as s:
        s.set_variant(46, 46)
        with pytest.raises(HrnError) as ei:
            s.forward()
        assert ei.value.code == 1
    with _assembled_solver(p, p["lam"], p["mu"]) as s:
        s.forward()
        assert s.variant()[0] not in (46, 86)


def test_pipelined_tiles_with_checkpointed_adjoint(gpu_lib):
    """Variant 47 in the checkpointed adjoint, whose recomputed forward segments and
    adjoint steps both run the pipelined tiles: the gradient equals variant 41's."""
    p = tiny(nshot=4, nstep=90)
    _, _, hist_t = oracle_forward(p, p["lam_t"], p["mu_t"])
    dis = np.stack([traces_from_history(p, h) for h in hist_t])
    g = {}
    for v in (47, 41):
        with _assembled_solver(p, p["lam"], p["mu"]) as s:
            s.set_variant(v, v)
            s.set_checkpointing(20)
            s.forward()
            g[v] = s.adjoint_gradient(dis)
    assert np.abs(g[41][1]).max() > 0
    assert np.array_equal(g[47][0], g[41][0]) and np.array_equal(g[47][1], g[41][1])
