"""Device kernels of the learned preconditioner against the host oracle: the BF16
3-D convolution forward and backward on the tensor cores (FP32 accumulation), the
source illumination of the forward history, and a few training steps lowering the
loss."""
import ctypes as C

import numpy as np
import pytest

from hirensi_b200 import learned as Lr
from problems import RHO, tiny

pytestmark = pytest.mark.gpu


def _bits(t, a):
    return t.from_numpy(Lr.to_bf16_bits(a).view(np.int16).ravel()).cuda()


def _last(a):
    """[c, nz, ny, nx] -> channels-last [V, 16] with the channels past c zero."""
    c = a.shape[0]
    out = np.zeros((a[0].size, 16), dtype=a.dtype)
    out[:, :c] = a.reshape(c, -1).T
    return out


def _first(a, c, shape):
    """channels-last [V, 16] -> [c, nz, ny, nx]."""
    return np.ascontiguousarray(a.reshape(-1, 16)[:, :c].T).reshape((c,) + shape)


@pytest.mark.parametrize("cin,cout,shape,relu", [(4, 16, (5, 7, 9), 1), (16, 16, (6, 5, 8), 1), (16, 2, (4, 6, 5), 0),
                                                 (6, 16, (17, 33, 33), 1), (16, 16, (3, 40, 47), 1),
                                                 (16, 16, (1, 1, 300), 1), (4, 16, (2, 1, 3), 0), (16, 2, (1, 9, 1), 1)])
def test_conv3d_kernels_match_oracle(gpu_lib, cin, cout, shape, relu):
    """The tensor-core layers against the numpy oracle: the forward within one BF16
    rounding of the FP64 result; the gradients at FP32-accumulation accuracy against
    the oracle fed the same BF16-rounded masked gy (the tensor-core operand); gb from
    the FP32 gy.  The shapes include tiles cut by the grid's end, more than one
    weight-gradient voxel chunk, and grids one voxel thin along one or two axes (the
    padded copy's border on both sides of every tap)."""
    import torch
    rng = np.random.default_rng(cin * 100 + cout)
    x = Lr.round_bf16(rng.standard_normal((cin,) + shape))
    w = Lr.round_bf16(rng.standard_normal((cout, cin, 27)) * 0.2)
    b = (rng.standard_normal(cout) * 0.1).astype(np.float32).astype(np.float64)
    V = int(np.prod(shape))
    xd, wd = _bits(torch, _last(x)), _bits(torch, w)
    bd = torch.from_numpy(b.astype(np.float32)).cuda()
    yd = torch.full((16 * V,), 0x7FC0, dtype=torch.int16, device="cuda")   # NaN bits: every channel is written
    nz, ny, nx = shape
    rc = gpu_lib.hrn_cnn_conv3d_forward(cin, cout, nz, ny, nx, C.c_void_p(xd.data_ptr()), C.c_void_p(wd.data_ptr()),
                                        C.c_void_p(bd.data_ptr()), relu, C.c_void_p(yd.data_ptr()), None)
    assert rc == 0
    yl = Lr.from_bf16_bits(yd.cpu().numpy().view(np.uint16)).astype(np.float64).reshape(V, 16)
    assert np.all(yl[:, cout:] == 0.0)
    y = _first(yl, cout, shape)
    yr = Lr.conv_ref(x, w, b, relu)
    # BF16 output: within one rounding of the FP64 result
    assert np.all(np.abs(y - yr) <= 2.0 ** -7 * np.abs(yr) + 1e-6)
    gy = rng.standard_normal(y.shape).astype(np.float32).astype(np.float64)
    gyd = torch.from_numpy(_last(gy).astype(np.float32).ravel()).cuda()
    gx = torch.full((16 * V,), float("nan"), dtype=torch.float32, device="cuda")
    gw = torch.zeros(cout * cin * 27, dtype=torch.float32, device="cuda")
    gb = torch.zeros(cout, dtype=torch.float32, device="cuda")
    rc = gpu_lib.hrn_cnn_conv3d_backward(cin, cout, nz, ny, nx, C.c_void_p(xd.data_ptr()), C.c_void_p(wd.data_ptr()),
                                         C.c_void_p(yd.data_ptr()), relu, C.c_void_p(gyd.data_ptr()),
                                         C.c_void_p(gx.data_ptr()), C.c_void_p(gw.data_ptr()), C.c_void_p(gb.data_ptr()), None)
    assert rc == 0
    gxl = gx.cpu().numpy().reshape(V, 16)
    assert np.all(gxl[:, cin:] == 0.0)
    gxr, gwr, _ = Lr.conv_ref_backward(x, w, y, relu, Lr.round_bf16(gy * ((y > 0) if relu else 1.0)))
    _, _, gbr = Lr.conv_ref_backward(x, w, y, relu, gy)
    rel = lambda a, r: np.linalg.norm(a.ravel() - r.ravel()) / np.linalg.norm(r.ravel())
    assert rel(_first(gxl, cin, shape), gxr) < 1e-5
    assert rel(gw.cpu().numpy().reshape(cout, cin, 27), gwr) < 1e-5
    assert rel(gb.cpu().numpy(), gbr) < 1e-5
    # invalid sizes are refused without a launch
    assert gpu_lib.hrn_cnn_conv3d_forward(17, cout, nz, ny, nx, C.c_void_p(xd.data_ptr()), C.c_void_p(wd.data_ptr()),
                                          C.c_void_p(bd.data_ptr()), relu, C.c_void_p(yd.data_ptr()), None) == 1


def test_illumination_matches_history(gpu_lib):
    import torch
    from hirensi_b200.solver import Solver
    p = tiny(nshot=2, nstep=40)
    with Solver("fp64") as s:
        s.set_mesh(p["mesh"], RHO)
        s.assemble(p["lam"], p["mu"])
        s.set_history(p["mesh"].store_eq)
        s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
        s.set_receivers(p["eqdis"], p["eqdis_map"])
        s.forward()
        out = torch.zeros(s.nstore // 3, dtype=torch.float64, device="cuda")
        assert gpu_lib.hrn_illumination(s.h, C.c_void_p(out.data_ptr())) == 0
        ref = sum((s.history(k) ** 2).reshape(p["nstep"] + 1, -1, 3).sum(axis=(0, 2)) for k in range(2))
    got = out.cpu().numpy()
    assert ref.max() > 0
    assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)


def test_training_steps_lower_the_loss(gpu_lib):
    rng = np.random.default_rng(3)
    shape = (5, 7, 9)
    dnet = Lr.DeviceNet(Lr.Net(seed=1), shape)
    samples = []
    for _ in range(3):
        x = rng.standard_normal((4,) + shape)
        q = rng.standard_normal((2,) + shape)
        dm = q * np.exp(0.5 * x[2:4])          # a target reachable by a positive scale
        samples.append((x, q, dm))
    hist = Lr.train(dnet, samples, epochs=25, lr=1e-2)
    assert hist[-1] < hist[0]


def test_trained_network_beats_plain_and_unit_scale_on_held_out_models(gpu_lib):
    import os
    from hirensi_b200.configs import inversion_config
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    # the network with the pseudo-Hessian inputs, as bench.py uses it
    weights = os.path.join(root, "hirensi_b200", "data", "precond_cnn6_16x16x8.npz")
    runner = Lr._Runner(inversion_config(nstep=2000), "fp32")
    dnet = Lr.DeviceNet(Lr.Net.load(weights), runner.lat.shape)
    rows = Lr.fwi_gain(runner, dnet, [5000, 5001], n_iter=5)
    for r in rows:
        # held-out seeds (training used 1000..1047): the network's direction must do
        # clearly better than the plain L-BFGS path and than the unscaled gradient
        assert r["learned_reduction"] > 2.0 * r["plain_reduction"]
        assert r["learned_reduction"] > 2.0 * r["unit_scale_reduction"]
        assert r["learned_accepted"] >= 3
