"""Oracle backend of hirensi_b200.inversion.FWI (numpy vectors, the CPU
restatement for assembly, time loops, gradient, TV and L-BFGS), and the oracle
primitives that drive oracle.inversion_loop, the independent restatement of the
reference's step and line-search rules."""
import numpy as np

import oracle as O
from problems import RHO


class OracleBackend:
    def __init__(self, mesh, shots, nstep, dt, eqdis, eqdis_map, dis):
        self.mesh = mesh
        self.n = mesh.nj
        self.om = O.OracleMesh(mesh, RHO)
        self.shots = shots          # list of (b vector [neq], ftab [nstep+1, 3])
        self.nstep, self.dt = nstep, dt
        self.eqdis, self.eqdis_map, self.dis = eqdis, eqdis_map, dis
        self.S = None
        self.hist = None

    def zeros(self):
        return np.zeros(self.n)

    def vec(self, host):
        return np.array(host, dtype=np.float64)

    def host(self, v):
        return v

    def copy(self, src, dst):
        dst[:] = src

    def axpby(self, a, x, b, y, z):
        z[:] = a * x + b * y if y is not None else a * x

    def mul(self, x, y, z):
        z[:] = x * y

    def dot(self, x, y):
        return float(x @ y)

    def norm2(self, x):
        return float(np.sqrt(x @ x))

    def norminf(self, x):
        return float(np.abs(x).max())

    def clip(self, x, lo, hi):
        np.clip(x, lo, hi, out=x)

    def extend(self, x):
        x[:] = x[self.mesh.extend_to]

    def gradient_mass_inverse(self):
        return O.inverse_gradient_mass(O.rmg(self.om))

    def tv(self, lam, mu, reg_l, reg_m):
        rl, rm, cl, cm = O.tv_reg(self.om, lam, mu)
        reg_l[:] = rl
        reg_m[:] = rm
        return cl, cm

    def lbfgs_setup(self, m, restriction):
        self.lb = O.LBFGSCoupled(self.n, m, restriction)

    def lbfgs_direction(self, it, it0, g_l, g_m, g_l_pre, g_m_pre, lam, mu, lam_pre, mu_pre, p_l, p_m):
        a, b = self.lb.direction(it, it0, g_l, g_m, g_l_pre, g_m_pre, lam, mu, lam_pre, mu_pre)
        p_l[:] = a
        p_m[:] = b

    def forward(self, lam, mu):
        self.S = O.OracleSystem.assemble(self.om, lam, mu)
        self.hist = [self.S.forward(b, ft, self.nstep, self.dt, self.mesh.store_eq) for b, ft in self.shots]
        return sum(O.misfit(self.nstep, self.dt, self.eqdis, self.eqdis_map, h, d) for h, d in zip(self.hist, self.dis))

    def gradient(self, g_l, g_m):
        g_l[:] = 0.0
        g_m[:] = 0.0
        for h, d in zip(self.hist, self.dis):
            pk = self.S.adjoint(self.nstep, self.dt, self.mesh.store_eq, h, self.eqdis, self.eqdis_map, d)
            a, b = O.control(self.om, self.nstep, self.dt, self.mesh.store_eq, h, pk)
            g_l += a
            g_m += b


def loop_primitives(be: OracleBackend):
    """evaluate / gradient / tv callables of oracle.inversion_loop over the oracle's
    forward, misfit, adjoint, control and TV, plus img, restriction and the
    extension map of the backend's mesh."""
    def evaluate(lam, mu):
        return be.forward(lam, mu)

    def gradient():
        gl, gm = np.zeros(be.n), np.zeros(be.n)
        be.gradient(gl, gm)
        return gl, gm

    def tv(lam, mu):
        return O.tv_reg(be.om, lam, mu)

    img, restriction = O.inverse_gradient_mass(O.rmg(be.om))
    return evaluate, gradient, tv, img, restriction, be.mesh.extend_to
