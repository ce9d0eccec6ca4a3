"""Learned gradient preconditioner of the inversion.

A small 3-D CNN looks at the gradient, the source illumination, the current
shear-wave speed and (in the 6-input form) the diagonal pseudo-Hessian on the
regular-domain node lattice, and returns a positive
diagonal scale D for each of the lambda and mu gradients.  The inversion tries
the scaled steepest-descent direction -D * g first.  Its Armijo line search on
the true misfit accepts it, or the iteration falls back to the plain L-BFGS
direction (``hirensi_b200.inversion.FWI``).

* Network: four 3x3x3 convolutions (4 or 6 -> 16 -> 16 -> 16 -> 2 channels, ReLU
  between), BF16 weights and activations with FP32 accumulation, run by the
  library's own kernels (hrn_cnn_conv3d_forward / _backward).  D = exp(clip(z, -4, 4)).
* Loss of one sample: sum over lambda, mu of 1 - cos^2(D * q, dm), where q = -g
  is the scaled gradient the inversion steps along and dm = m_true - m.  It is
  scale-invariant, because the inversion caps the step length itself.
* Data: seeded random layered models with an anomaly, whose gradients the
  library computes.  Samples come from the starting model and from the iterates
  of a short plain inversion (its accepted L-BFGS steps).
* Training: Adam on FP32 master weights, gradients from the backward kernels.

The voxel grid is the node lattice of the regular domain of a box mesh
((2nx+1) x (2ny+1) x (2nz+1)): one voxel per stored node.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

CH = (4, 16, 16, 16, 2)       # channels of the five activations (4-input form)
ZCLIP = 4.0


# ---------------------------------------------------------------------------
# BF16 <-> FP32 on the host (round to nearest even, as __float2bfloat16_rn)

def to_bf16_bits(a: np.ndarray) -> np.ndarray:
    f = np.ascontiguousarray(a, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    r = (b + 0x7FFF + ((b >> 16) & 1)) >> 16
    return r.astype(np.uint16)


def from_bf16_bits(h: np.ndarray) -> np.ndarray:
    return (np.asarray(h, dtype=np.uint32) << 16).view(np.float32)


def round_bf16(a: np.ndarray) -> np.ndarray:
    return from_bf16_bits(to_bf16_bits(a)).astype(np.float64)


# ---------------------------------------------------------------------------
# reference convolution (numpy, float64 on BF16-rounded inputs): the oracle of
# the device kernels

def _shift(x: np.ndarray, dz: int, dy: int, dx: int) -> np.ndarray:
    """x[..., z + dz, y + dy, x + dx] with zeros outside."""
    out = np.zeros_like(x)
    nz, ny, nx = x.shape[-3:]

    def sl(d, n):
        return slice(max(0, -d), n - max(0, d)), slice(max(0, d), n - max(0, -d))

    (oz, iz), (oy, iy), (ox, ix) = sl(dz, nz), sl(dy, ny), sl(dx, nx)
    out[..., oz, oy, ox] = x[..., iz, iy, ix]
    return out


def conv_ref(x, w, b, relu):
    """x [cin, nz, ny, nx], w [cout, cin, 27], b [cout] -> y [cout, nz, ny, nx]."""
    cout = w.shape[0]
    y = np.zeros((cout,) + x.shape[1:])
    for k in range(27):
        xs = _shift(x, k // 9 - 1, (k // 3) % 3 - 1, k % 3 - 1)
        y += np.einsum("oc,czyx->ozyx", w[:, :, k], xs)
    y += b[:, None, None, None]
    return np.maximum(y, 0.0) if relu else y


def conv_ref_backward(x, w, y, relu, gy):
    gz = gy * (y > 0) if relu else gy
    gx = np.zeros_like(x)
    gw = np.zeros_like(w)
    for k in range(27):
        dz, dy, dx = k // 9 - 1, (k // 3) % 3 - 1, k % 3 - 1
        xs = _shift(x, dz, dy, dx)
        gw[:, :, k] = np.einsum("ozyx,czyx->oc", gz, xs)
        gx += _shift(np.einsum("oc,ozyx->czyx", w[:, :, k], gz), -dz, -dy, -dx)
    return gx, gw, gz.sum(axis=(1, 2, 3))


# ---------------------------------------------------------------------------
# lattice of the regular domain

@dataclasses.dataclass
class Lattice:
    shape: tuple          # (nz, ny, nx) voxels
    store_to_voxel: np.ndarray   # [nstore/3] voxel of each stored node (history order)
    store_nodes: np.ndarray      # [nstore/3] node id of each stored node

    @staticmethod
    def of(mesh) -> "Lattice":
        nodes = np.asarray(mesh.store_nodes)
        x = mesh.xyz[nodes]
        s = 0.5 * mesh.h
        lo = x.min(axis=0)
        idx = np.rint((x - lo) / s).astype(np.int64)
        nx, ny, nz = (idx.max(axis=0) + 1).tolist()
        vox = (idx[:, 2] * ny + idx[:, 1]) * nx + idx[:, 0]
        if np.unique(vox).size != vox.size or vox.size != nx * ny * nz:
            raise ValueError("the stored nodes do not fill a lattice")
        return Lattice((nz, ny, nx), vox, nodes)

    def to_grid(self, node_values: np.ndarray) -> np.ndarray:
        g = np.zeros(int(np.prod(self.shape)))
        g[self.store_to_voxel] = node_values[self.store_nodes]
        return g.reshape(self.shape)

    def from_grid(self, grid: np.ndarray, nj: int) -> np.ndarray:
        out = np.zeros(nj)
        out[self.store_nodes] = np.asarray(grid).reshape(-1)[self.store_to_voxel]
        return out


def features(lat: Lattice, g_l, g_m, illum_store, vs, ph=None) -> np.ndarray:
    """Input channels [4 or 6, nz, ny, nx]: the two gradients scaled to unit max, the
    log illumination standardized, the shear-wave speed / 400, and with ph = (H_lambda,
    H_mu) [nj] the log pseudo-Hessian diagonals standardized."""
    def unit(v):
        m = np.abs(v).max()
        return v / m if m > 0 else v

    def log_std(v):
        v = np.asarray(v, dtype=np.float64)
        v = np.log(np.maximum(v, 0.0) + 1e-300 + np.max(v) * 1e-12)
        return (v - v.mean()) / (v.std() + 1e-12)

    il = np.zeros(int(np.prod(lat.shape)))
    il[lat.store_to_voxel] = log_std(illum_store)
    ch = [unit(lat.to_grid(g_l)), unit(lat.to_grid(g_m)), il.reshape(lat.shape), lat.to_grid(vs) / 400.0]
    if ph is not None:
        for h in ph:
            g = np.zeros(int(np.prod(lat.shape)))
            g[lat.store_to_voxel] = log_std(np.asarray(h)[lat.store_nodes])
            ch.append(g.reshape(lat.shape))
    return np.stack(ch)


def cosine_loss(a: np.ndarray, t: np.ndarray):
    """L = 1 - cos^2(a, t) and dL/da."""
    at = float(a.ravel() @ t.ravel())
    aa = float(a.ravel() @ a.ravel())
    tt = float(t.ravel() @ t.ravel())
    if aa == 0.0 or tt == 0.0:
        return 1.0, np.zeros_like(a)
    L = 1.0 - at * at / (aa * tt)
    grad = -2.0 * at / (aa * tt) * (t - (at / aa) * a)
    return L, grad


# ---------------------------------------------------------------------------
# the network on the device kernels

class Net:
    def __init__(self, seed: int = 0, weights: dict | None = None, inputs: int = 4):
        if weights is not None:
            inputs = int(np.asarray(weights["w0"]).shape[1])
        if inputs not in (4, 6):
            raise ValueError("the network takes 4 or 6 input channels")
        self.ch = (inputs,) + CH[1:]
        rng = np.random.default_rng(seed)
        self.w, self.b = [], []
        for i in range(4):
            cin, cout = self.ch[i], self.ch[i + 1]
            std = np.sqrt(2.0 / (cin * 27)) * (0.1 if i == 3 else 1.0)
            self.w.append(rng.standard_normal((cout, cin, 27)).astype(np.float32) * np.float32(std))
            self.b.append(np.zeros(cout, dtype=np.float32))
        if weights is not None:
            self.w = [np.asarray(weights[f"w{i}"], dtype=np.float32) for i in range(4)]
            self.b = [np.asarray(weights[f"b{i}"], dtype=np.float32) for i in range(4)]

    def state(self) -> dict:
        d = {f"w{i}": self.w[i] for i in range(4)}
        d.update({f"b{i}": self.b[i] for i in range(4)})
        return d

    def save(self, path: str):
        np.savez(path, **self.state())

    @staticmethod
    def load(path: str) -> "Net":
        with np.load(path) as d:
            return Net(weights={k: d[k] for k in d.files})


class DeviceNet:
    """Forward and backward passes of a Net through libhirensi_b200.so."""

    def __init__(self, net: Net, shape: tuple, device=None):
        import torch
        from . import capi
        self.torch = torch
        self.L = capi.load()
        self.net = net
        self.shape = shape
        self.dev = device or torch.device("cuda", torch.cuda.current_device())
        self.stream = torch.cuda.current_stream(self.dev).cuda_stream
        V = int(np.prod(shape))
        self.V = V
        self.ch = net.ch
        # channels-last activations with a channel stride of 16 ([V][16] BF16 bits); the
        # channels past a layer's count stay zero
        self.act = [torch.zeros(16 * V, dtype=torch.int16, device=self.dev) for _ in self.ch]
        self.sync_weights()

    def _ck(self, rc):
        if rc != 0:
            raise RuntimeError(f"hirensi_b200 CNN kernel error {rc}")

    def sync_weights(self):
        t = self.torch
        self.wd = [t.from_numpy(to_bf16_bits(w).view(np.int16)).to(self.dev) for w in self.net.w]
        self.bd = [t.from_numpy(b).to(self.dev) for b in self.net.b]

    def forward(self, x: np.ndarray) -> np.ndarray:
        """x [inputs, nz, ny, nx] -> z [2, nz, ny, nx] (the network's last activation)."""
        t = self.torch
        CH = self.ch
        nz, ny, nx = self.shape
        xl = np.zeros((self.V, 16))
        xl[:, :CH[0]] = np.asarray(x).reshape(CH[0], self.V).T
        self.act[0].copy_(t.from_numpy(to_bf16_bits(xl).view(np.int16).ravel()))
        for i in range(4):
            self._ck(self.L.hrn_cnn_conv3d_forward(CH[i], CH[i + 1], nz, ny, nx, C.c_void_p(self.act[i].data_ptr()),
                                                   C.c_void_p(self.wd[i].data_ptr()), C.c_void_p(self.bd[i].data_ptr()),
                                                   int(i < 3), C.c_void_p(self.act[i + 1].data_ptr()), C.c_void_p(self.stream)))
        z = self.act[4].cpu().numpy().view(np.uint16).reshape(self.V, 16)[:, :CH[4]]
        return from_bf16_bits(np.ascontiguousarray(z.T)).astype(np.float64).reshape((CH[4],) + self.shape)

    def backward(self, gz: np.ndarray):
        """Weight and bias gradients for dL/dz = gz (after a forward of the same input)."""
        t = self.torch
        CH = self.ch
        nz, ny, nx = self.shape
        gl = np.zeros((self.V, 16), dtype=np.float32)
        gl[:, :CH[4]] = np.asarray(gz, dtype=np.float32).reshape(CH[4], self.V).T
        gy = t.from_numpy(gl.ravel()).to(self.dev)
        gws, gbs = [None] * 4, [None] * 4
        for i in range(3, -1, -1):
            gw = t.zeros(CH[i + 1] * CH[i] * 27, dtype=t.float32, device=self.dev)
            gb = t.zeros(CH[i + 1], dtype=t.float32, device=self.dev)
            gx = t.zeros(16 * self.V, dtype=t.float32, device=self.dev) if i > 0 else None
            self._ck(self.L.hrn_cnn_conv3d_backward(CH[i], CH[i + 1], nz, ny, nx, C.c_void_p(self.act[i].data_ptr()),
                                                    C.c_void_p(self.wd[i].data_ptr()), C.c_void_p(self.act[i + 1].data_ptr()),
                                                    int(i < 3), C.c_void_p(gy.data_ptr()),
                                                    C.c_void_p(gx.data_ptr() if gx is not None else 0),
                                                    C.c_void_p(gw.data_ptr()), C.c_void_p(gb.data_ptr()), C.c_void_p(self.stream)))
            gws[i] = gw.cpu().numpy().reshape(CH[i + 1], CH[i], 27)
            gbs[i] = gb.cpu().numpy()
            gy = gx
        return gws, gbs


def conv_bench(shape, reps: int = 20, inputs: int = 6, seed: int = 0) -> dict:
    """Device time of the network's convolutions on a lattice of `shape` (nz, ny, nx):
    the four forward layers, then the four backward layers (data and weight
    gradients), each timed over `reps` back-to-back passes with CUDA events on the
    network's stream, activations resident on the device.  The calls go through the C
    ABI, and each one reads its kernels' error flag back (a stream synchronization),
    so the times include that round trip.  The tensor cores run every
    layer at 16 input and 16 output channels; `tflops_mma` counts those MMAs,
    `tflops_useful` only the layers' real channel counts."""
    import torch
    net = Net(seed=seed, inputs=inputs)
    dn = DeviceNet(net, tuple(shape))
    rng = np.random.default_rng(seed)
    dn.forward(rng.standard_normal((net.ch[0],) + tuple(shape)))        # activations of a real input
    nz, ny, nx = shape
    V = dn.V
    CH = net.ch
    t = torch
    gy = [t.from_numpy(rng.standard_normal(16 * V).astype(np.float32)).to(dn.dev) for _ in range(4)]
    gx = [t.zeros(16 * V, dtype=t.float32, device=dn.dev) for _ in range(4)]
    gw = [t.zeros(CH[i + 1] * CH[i] * 27, dtype=t.float32, device=dn.dev) for i in range(4)]
    gb = [t.zeros(CH[i + 1], dtype=t.float32, device=dn.dev) for i in range(4)]
    stream = torch.cuda.ExternalStream(dn.stream) if dn.stream else torch.cuda.current_stream(dn.dev)

    def fwd():
        for i in range(4):
            dn._ck(dn.L.hrn_cnn_conv3d_forward(CH[i], CH[i + 1], nz, ny, nx, C.c_void_p(dn.act[i].data_ptr()),
                                               C.c_void_p(dn.wd[i].data_ptr()), C.c_void_p(dn.bd[i].data_ptr()),
                                               int(i < 3), C.c_void_p(dn.act[i + 1].data_ptr()), C.c_void_p(dn.stream)))

    def bwd():
        for i in range(3, -1, -1):
            dn._ck(dn.L.hrn_cnn_conv3d_backward(CH[i], CH[i + 1], nz, ny, nx, C.c_void_p(dn.act[i].data_ptr()),
                                                C.c_void_p(dn.wd[i].data_ptr()), C.c_void_p(dn.act[i + 1].data_ptr()),
                                                int(i < 3), C.c_void_p(gy[i].data_ptr()),
                                                C.c_void_p(gx[i].data_ptr() if i > 0 else 0),
                                                C.c_void_p(gw[i].data_ptr()), C.c_void_p(gb[i].data_ptr()),
                                                C.c_void_p(dn.stream)))

    out = {"shape": list(shape), "voxels": V, "channels": list(CH), "reps": reps}
    for name, fn, passes in (("forward", fwd, [1, 1, 1, 1]), ("backward", bwd, [1, 2, 2, 2])):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        # backward: the weight gradient of every layer, the data gradient of layers 1-3
        useful = sum(2.0 * V * 27 * CH[i] * CH[i + 1] * passes[i] for i in range(4))
        mma = sum(2.0 * V * 27 * 16 * 16 * passes[i] for i in range(4))
        out[name] = {"ms": ms, "tflops_useful": useful / (ms * 1e-3) / 1e12, "tflops_mma": mma / (ms * 1e-3) / 1e12}
    return out


def scale_from_z(z: np.ndarray) -> np.ndarray:
    return np.exp(np.clip(z, -ZCLIP, ZCLIP))


def sample_loss(dnet: DeviceNet, x, q, dm):
    """Loss of one sample and its gradients.  q, dm: [2, nz, ny, nx]."""
    z = dnet.forward(x)
    D = scale_from_z(z)
    L = 0.0
    gz = np.zeros_like(z)
    for c in range(2):
        a = D[c] * q[c]
        Lc, ga = cosine_loss(a, dm[c])
        L += Lc
        inside = np.abs(z[c]) < ZCLIP
        gz[c] = ga * a * inside          # d a / d z = a inside the clip
    gws, gbs = dnet.backward(gz)
    return L, gws, gbs


class Adam:
    def __init__(self, params, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.p, self.lr, self.b1, self.b2, self.eps = params, lr, b1, b2, eps
        self.m = [np.zeros_like(x) for x in params]
        self.v = [np.zeros_like(x) for x in params]
        self.t = 0

    def step(self, grads):
        self.t += 1
        for i, (p, g) in enumerate(zip(self.p, grads)):
            self.m[i] = self.b1 * self.m[i] + (1 - self.b1) * g
            self.v[i] = self.b2 * self.v[i] + (1 - self.b2) * g * g
            mh = self.m[i] / (1 - self.b1 ** self.t)
            vh = self.v[i] / (1 - self.b2 ** self.t)
            p -= (self.lr * mh / (np.sqrt(vh) + self.eps)).astype(p.dtype)


def train(dnet: DeviceNet, samples, epochs: int = 40, lr: float = 2e-3, log=None):
    """samples: list of (x, q, dm).  Full-batch Adam; returns the loss history."""
    net = dnet.net
    opt = Adam(net.w + net.b, lr=lr)
    hist = []
    for ep in range(epochs):
        tot = 0.0
        gw = [np.zeros_like(w) for w in net.w]
        gb = [np.zeros_like(b) for b in net.b]
        for x, q, dm in samples:
            L, gws, gbs = sample_loss(dnet, x, q, dm)
            tot += L
            for i in range(4):
                gw[i] += gws[i] / len(samples)
                gb[i] += gbs[i] / len(samples)
        opt.step(gw + gb)
        dnet.sync_weights()
        hist.append(tot / len(samples))
        if log:
            log(ep, hist[-1])
    return hist


def evaluate(dnet: DeviceNet, samples) -> tuple[float, float]:
    """Mean loss of the network and of the unscaled direction (D = 1) on samples."""
    ln, l1 = 0.0, 0.0
    for x, q, dm in samples:
        D = scale_from_z(dnet.forward(x))
        for c in range(2):
            ln += cosine_loss(D[c] * q[c], dm[c])[0]
            l1 += cosine_loss(q[c], dm[c])[0]
    return ln / len(samples), l1 / len(samples)


class LearnedPreconditioner:
    """Proposal hook of FWI: scaled steepest-descent direction from the network."""

    def __init__(self, dnet: DeviceNet, mesh, rho: float):
        self.dnet = dnet
        self.lat = Lattice.of(mesh)
        self.mesh = mesh
        self.rho = rho

    def direction(self, backend, g_l, g_m, lam, mu):
        """p = -D * g (host round trip of the small grids); returns device/host vectors
        of the backend."""
        gl, gm = backend.host(g_l), backend.host(g_m)
        il = backend.illumination()
        vs = np.sqrt(np.maximum(backend.host(mu), 0.0) / self.rho)
        ph = backend.pseudo_hessian() if self.dnet.ch[0] == 6 else None
        x = features(self.lat, gl, gm, il, vs, ph)
        D = scale_from_z(self.dnet.forward(x))
        nj = self.mesh.nj
        pl = -self.lat.from_grid(D[0], nj) * gl
        pm = -self.lat.from_grid(D[1], nj) * gm
        return backend.vec(pl), backend.vec(pm)


# ---------------------------------------------------------------------------
# training data from the solver, training, evaluation

def random_true_model(prob, rng):
    """A model of the inversion configuration's distribution: three layers with
    Vs 200 / 300 / 400 m/s (each +-10 %, interfaces at 7.5 and 15 m +-2 m) and a
    Gaussian Vs anomaly of +-20..40 % (radius 3..7 m) at a random position in the
    regular domain.  Lengths are those of the configuration's 20 m deep box and
    scale with the depth of a deeper one (the training mesh: 50 m, factor 2.5)."""
    from .configs import extend_into_pml, layered_vs, vs_to_lame
    m = prob.mesh
    (x0, x1), (y0, y1), (z0, _) = m.rd_box
    f = -z0 / 20.0
    vs_l = np.array([200.0, 300.0, 400.0]) * (1.0 + rng.uniform(-0.1, 0.1, 3))
    vs = layered_vs(m, tuple(vs_l), (f * (-7.5 + rng.uniform(-2, 2)), f * (-15.0 + rng.uniform(-2, 2))))
    c = np.array([rng.uniform(0.7 * x0, 0.7 * x1), rng.uniform(0.7 * y0, 0.7 * y1), rng.uniform(0.8 * z0, 0.2 * z0)])
    r = f * rng.uniform(3.0, 7.0)
    amp = rng.choice([-1.0, 1.0]) * rng.uniform(0.2, 0.4)
    d2 = ((m.xyz - c) ** 2).sum(axis=1)
    vs = extend_into_pml(m, vs * (1.0 + amp * np.exp(-d2 / (r * r))))
    return vs_to_lame(vs)


class _Runner:
    """One solver + device backend for many models of one configuration."""

    def __init__(self, prob, precision="fp32"):
        import torch
        from .configs import RHO
        from .inversion import DeviceBackend
        from .solver import Solver
        self.torch = torch
        self.prob = prob
        m = prob.mesh
        s = Solver(precision)
        s.set_mesh(m, RHO)
        s.assemble(prob.lam0, prob.mu0)
        s.set_history(m.store_eq)
        s.set_shots(prob.nstep, prob.dt, prob.src_eq, prob.src_b, prob.ftab)
        s.set_receivers(prob.eqdis, prob.eqdis_map)
        self.s = s
        self.b = DeviceBackend(s, m)
        self.lat = Lattice.of(m)
        self.rho = RHO

    def set_true(self, lam_t, mu_t):
        self.s.assemble(lam_t, mu_t)
        self.s.forward()
        dis = self.s.traces()
        self.dis_dev = self.torch.from_numpy(dis).cuda()
        self.s.set_data(device_ptr=self.dis_dev.data_ptr())

    def fwi(self, n_iter, cfg=None, preconditioner=None, observer=None, target_reduction=None):
        from .inversion import FWI, ArmijoFailure
        cfg = cfg or default_inversion_config()
        f = FWI(self.b, cfg, preconditioner=preconditioner)
        try:
            f.run(self.prob.lam0, self.prob.mu0, n_iter=n_iter, observer=observer, target_reduction=target_reduction)
        except ArmijoFailure:
            pass   # the iterations done so far stand
        return f.hist


def default_inversion_config():
    from .inversion import InversionConfig
    return InversionConfig(m_lbfgs=5, bounds_lambda=(10.0, 2000.0), bounds_mu=(10.0, 1000.0))


def study_inversion_config(fac: float = 20.0, tv: bool = False):
    """The inversion settings of the time-to-misfit comparison (bench.py's FWI legs):
    L-BFGS memory 5, the reference's step rules with the lambda bias, Fac_Max_Update
    `fac`, no TV regularization unless `tv` (with it the plain path stalls)."""
    from .inversion import InversionConfig
    return InversionConfig(m_lbfgs=5, bounds_lambda=(10.0, 2000.0), bounds_mu=(10.0, 1000.0),
                           fac_max_update_lambda=fac, fac_max_update_mu=fac, regularization="TV" if tv else None)


def _to_targets(h, targets):
    """Iterations and wall time at which the misfit first fell by each target fraction."""
    J0 = h[0]["misfit"]
    out = {}
    for r in targets:
        hit = next((x for x in h if x["misfit"] <= (1.0 - r) * J0), None)
        out[f"{int(round(r * 100))}pct"] = None if hit is None else {"iterations": hit["iter"], "wall_s": hit["wall_s"]}
    return out


def time_to_targets(runner: _Runner, dnet: DeviceNet, seeds, cap: int = 30, targets=(0.5, 0.9), cfg=None,
                    unit_scale_seeds=(), on_row=None):
    """Per held-out model: iterations and wall time to each misfit-reduction target for
    plain L-BFGS and for the network's proposals (and the unit-scale ablation on
    `unit_scale_seeds`), each run stopped at the last target or after `cap` iterations.
    on_row(rows), if given, sees the rows so far after each model."""
    cfg = cfg or study_inversion_config()
    pre = LearnedPreconditioner(dnet, runner.prob.mesh, runner.rho)
    rows = []
    for sd in seeds:
        rng = np.random.default_rng(int(sd))
        lam_t, mu_t = random_true_model(runner.prob, rng)
        runner.set_true(lam_t, mu_t)
        row = {"seed": int(sd)}
        runs = [("plain", None), ("learned", pre)]
        if int(sd) in set(int(x) for x in unit_scale_seeds):
            runs.append(("unit_scale", UnitScale()))
        for name, p in runs:
            h = runner.fwi(cap, cfg=cfg, preconditioner=p, target_reduction=max(targets))
            row[name] = {"reduction": 1.0 - h[-1]["misfit"] / h[0]["misfit"], "iterations": len(h) - 1,
                         "wall_s": h[-1]["wall_s"], **_to_targets(h, targets)}
            if p is not None:
                row[name]["accepted"] = int(sum(1 for x in h[1:] if x.get("learned")))
        rows.append(row)
        if on_row:
            on_row(rows)
    return rows


def generate_samples(runner: _Runner, seeds, iters: int = 3, log=None, inputs: int = 4, budget_s=None):
    """(x, q, dm) of the first `iters` iterations of a plain inversion of each seeded model;
    with budget_s, no further model is started once that many seconds have passed."""
    import time
    out = []
    t0 = time.perf_counter()
    for sd in seeds:
        if budget_s is not None and time.perf_counter() - t0 > budget_s:
            break
        rng = np.random.default_rng(int(sd))
        lam_t, mu_t = random_true_model(runner.prob, rng)
        runner.set_true(lam_t, mu_t)

        def obs(it, lam, mu, g_l, g_m):
            b = runner.b
            gl, gm = b.host(g_l), b.host(g_m)
            lh, mh = b.host(lam), b.host(mu)
            vs = np.sqrt(np.maximum(mh, 0.0) / runner.rho)
            x = features(runner.lat, gl, gm, b.illumination(), vs, b.pseudo_hessian() if inputs == 6 else None)
            q = np.stack([runner.lat.to_grid(-gl), runner.lat.to_grid(-gm)])
            dm = np.stack([runner.lat.to_grid(lam_t - lh), runner.lat.to_grid(mu_t - mh)])
            out.append((x, q, dm))

        runner.fwi(iters, observer=obs)
        if log:
            log(f"model seed {sd}: {len(out)} samples")
    return out


class UnitScale:
    """The proposal with D = 1 (the scaled gradient itself): the ablation of the network."""

    def direction(self, backend, g_l, g_m, lam, mu):
        return backend.vec(-backend.host(g_l)), backend.vec(-backend.host(g_m))


def fwi_gain(runner: _Runner, dnet: DeviceNet, seeds, n_iter: int = 10):
    """Misfit reduction and wall time of n_iter iterations with and without the
    network on each seeded model."""
    rows = []
    pre = LearnedPreconditioner(dnet, runner.prob.mesh, runner.rho)
    for sd in seeds:
        rng = np.random.default_rng(int(sd))
        lam_t, mu_t = random_true_model(runner.prob, rng)
        runner.set_true(lam_t, mu_t)
        h0 = runner.fwi(n_iter)
        h1 = runner.fwi(n_iter, preconditioner=pre)
        h2 = runner.fwi(n_iter, preconditioner=UnitScale())
        rows.append({"seed": int(sd), "plain_reduction": 1.0 - h0[-1]["misfit"] / h0[0]["misfit"],
                     "learned_reduction": 1.0 - h1[-1]["misfit"] / h1[0]["misfit"],
                     "unit_scale_reduction": 1.0 - h2[-1]["misfit"] / h2[0]["misfit"],
                     "plain_s": h0[-1]["wall_s"], "learned_s": h1[-1]["wall_s"], "unit_scale_s": h2[-1]["wall_s"],
                     "plain_iters": len(h0) - 1, "learned_iters": len(h1) - 1,
                     "learned_accepted": int(sum(1 for h in h1[1:] if h.get("learned"))),
                     "unit_scale_accepted": int(sum(1 for h in h2[1:] if h.get("learned")))})
    return rows


def main(argv=None):
    import argparse
    import json
    import time
    import torch
    from .configs import inversion_config, training_config
    ap = argparse.ArgumentParser(description="train the learned gradient preconditioner on solver-generated data")
    ap.add_argument("--out", help="weights file of a training run (.npz); a .json summary is written beside it")
    ap.add_argument("--models", type=int, default=48)
    ap.add_argument("--eval-models", type=int, default=6)
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--nstep", type=int, default=2000)
    ap.add_argument("--fwi-iters", type=int, default=10, help="iterations of the after-training comparison (0: none)")
    ap.add_argument("--eval-only", help="skip training: evaluate these weights")
    ap.add_argument("--inputs", type=int, choices=[4, 6], default=6,
                    help="input channels: 4 = gradients, illumination, Vs; 6 = also the pseudo-Hessian diagonals")
    ap.add_argument("--study", help="held-out study of these weights: time to 50 %% and 90 %% misfit reduction "
                                    "(writes a .json beside the weights with the suffix _study)")
    ap.add_argument("--study-models", type=int, default=32)
    ap.add_argument("--study-cap", type=int, default=30)
    ap.add_argument("--fac", type=float, default=20.0, help="Fac_Max_Update of the study's inversions")
    ap.add_argument("--mesh", choices=["16x16x8", "40x40x20"], default="16x16x8",
                    help="16x16x8: the inversion configuration (4 shots); 40x40x20: the training mesh of the "
                         "learned-preconditioner configuration (8 shots, configs.training_config)")
    ap.add_argument("--unit-scale-models", type=int, default=8, help="held-out models that also run the D = 1 ablation")
    ap.add_argument("--study-out", help="summary file of --study (default: beside the weights, suffix _study)")
    ap.add_argument("--data-budget-s", type=float, help="start no further training model after this many seconds")
    ap.add_argument("--conv-bench", help="only time the convolutions on a lattice NZxNYxNX (e.g. 41x81x81)")
    a = ap.parse_args(argv)
    t0 = time.time()
    if a.conv_bench:
        print(json.dumps(conv_bench(tuple(int(v) for v in a.conv_bench.split("x")), inputs=a.inputs)), flush=True)
        return
    prob = inversion_config(nstep=a.nstep) if a.mesh == "16x16x8" else training_config(nstep=a.nstep)
    runner = _Runner(prob, "fp32")
    if a.study:
        dnet = DeviceNet(Net.load(a.study), runner.lat.shape)
        seeds = list(range(5000, 5000 + a.study_models))
        out = a.study_out or a.study.replace(".npz", "_study.json")

        def summarize(rows):
            def med(key, tgt, field):
                v = [r[key][tgt][field] for r in rows if r[key].get(tgt)]
                return (float(np.median(v)) if v else None), len(v)
            summary = {"models": len(rows), "cap": a.study_cap, "fac_max_update": a.fac, "precision": "fp32",
                       "mesh": f"{prob.name}, {len(prob.src_eq)} shots, {prob.nstep} steps",
                       "lattice": list(runner.lat.shape)}
            for key in ("plain", "learned"):
                for tgt in ("50pct", "90pct"):
                    (mi, n), (mw, _) = med(key, tgt, "iterations"), med(key, tgt, "wall_s")
                    summary[f"{key}_{tgt}"] = {"reached": n, "median_iterations": mi, "median_wall_s": mw}
            for tgt in ("50pct", "90pct"):
                both = [r for r in rows if r["plain"].get(tgt) and r["learned"].get(tgt)]
                summary[f"median_speedup_to_{tgt}"] = (
                    float(np.median([r["plain"][tgt]["wall_s"] / r["learned"][tgt]["wall_s"] for r in both]))
                    if both else None)
            summary["rows"] = rows
            with open(out, "w") as f:
                json.dump(summary, f, indent=1)
            return summary

        rows = time_to_targets(runner, dnet, seeds, cap=a.study_cap, cfg=study_inversion_config(a.fac),
                               unit_scale_seeds=seeds[:a.unit_scale_models], on_row=summarize)
        summary = summarize(rows)
        print(json.dumps({k: v for k, v in summary.items() if k != "rows"}), flush=True)
        return
    if a.eval_only:
        dnet = DeviceNet(Net.load(a.eval_only), runner.lat.shape)
        for g in fwi_gain(runner, dnet, range(5000, 5000 + a.eval_models), a.fwi_iters):
            print(g, flush=True)
        return
    if not a.out:
        ap.error("training needs --out")
    train_s = generate_samples(runner, range(1000, 1000 + a.models), a.iters, inputs=a.inputs,
                               budget_s=a.data_budget_s, log=lambda m: print(m, flush=True))
    eval_s = generate_samples(runner, range(5000, 5000 + a.eval_models), a.iters, inputs=a.inputs)
    t_data = time.time() - t0
    dnet = DeviceNet(Net(seed=0, inputs=a.inputs), runner.lat.shape)
    hist = train(dnet, train_s, epochs=a.epochs, lr=a.lr, log=lambda ep, L: print(f"epoch {ep} loss {L:.4f}", flush=True))
    t_train = time.time() - t0 - t_data
    ev_net, ev_one = evaluate(dnet, eval_s)
    dnet.net.save(a.out)
    gains = fwi_gain(runner, dnet, range(5000, 5000 + a.eval_models), a.fwi_iters) if a.fwi_iters > 0 else []
    summary = {"train_samples": len(train_s), "eval_samples": len(eval_s), "epochs": a.epochs,
               "loss_first_epoch": hist[0], "loss_last_epoch": hist[-1], "eval_loss_network": ev_net,
               "eval_loss_unscaled_gradient": ev_one, "fwi": gains, "data_s": t_data, "train_s": t_train,
               "nstep": a.nstep, "shape": list(runner.lat.shape), "inputs": a.inputs,
               "mesh": f"{prob.name}, {len(prob.src_eq)} shots, {prob.nstep} steps"}
    with open(a.out.replace(".npz", ".json"), "w") as f:
        json.dump(summary, f, indent=1)
    print(json.dumps({k: v for k, v in summary.items() if k != "fwi"}), flush=True)
    for g in gains:
        print(g, flush=True)


if __name__ == "__main__":
    main()
