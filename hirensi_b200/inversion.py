"""Full-waveform inversion loop of S4/Program_Main.F90:379-921.

``FWI`` keeps the reference driver's control flow on the host:

* adjoint gradient, sign flip, TV regularization with the adaptive factor, and
  gradient-mass scaling;
* coupled L-BFGS direction, descent check, step capping, and the lambda-bias rule
  (including its integer-division weight);
* PML extension, material bounds, and Armijo backtracking.

Every vector operation runs through a backend.  ``DeviceBackend`` keeps all
nodal vectors on the GPU and uses libhirensi_b200.so's kernels.  The host only
receives scalars: dots, norms and misfits.

Configuration defaults are the reference's (S4/Adjustments.F90:137-183), except
that the material bounds are arguments: the reference's [50, 166] would clip
the layered models of the benchmark configurations.
"""
from __future__ import annotations

import dataclasses
import time

import numpy as np


@dataclasses.dataclass
class InversionConfig:
    m_lbfgs: int = 15                 # M_LBFGS
    fac_max_update_lambda: float = 5.0
    fac_max_update_mu: float = 5.0
    bounds_lambda: tuple = (50.0, 166.0)
    bounds_mu: tuple = (50.0, 166.0)
    regularization: str | None = "TV"   # 'TV' or None
    reg_factor: float = 0.3           # Regularization_factor_continuation
    bias_lambda: bool = True          # Bias_Lambda_search = 'Yes'
    n_iter_bias: int = 50
    armijo_c: float = 1.0e-4
    armijo_rho: float = 0.5
    iter_begin: int = 1
    search: str = "LBFGS"             # 'LBFGS' or 'SD'
    # line search of a preconditioner's proposal (no reference counterpart): 'wolfe' =
    # Armijo and the weak curvature condition, expanding a too-short step; 'armijo' =
    # one sufficient-decrease test
    proposal_search: str = "wolfe"
    wolfe_c2: float = 0.9
    wolfe_expansions: int = 2


class ArmijoFailure(RuntimeError):
    """Ten backtracking steps without sufficient decrease (the reference STOPs)."""


class FWI:
    """preconditioner: optional object with ``direction(backend, g_l, g_m, lam, mu)``
    returning a proposed update direction (``hirensi_b200.learned.LearnedPreconditioner``).
    Each iteration tries it first with a line search on the true misfit in FP64
    (``cfg.proposal_search``):

    * the first trial takes the step that moves no node by more than Fac_Max_Update;
    * a trial must pass the Armijo test J(m + s) <= J(m) + c1 g.s; if the first does
      not, the model is restored and the iteration takes the reference's L-BFGS path
      unchanged;
    * with 'wolfe', a trial that passes also needs the weak curvature condition
      g(m + s).s >= c2 g.s, with the gradient at the trial point (the next iteration's
      gradient, kept for it).  A trial that fails it has stopped short of the
      curvature, and the step doubles, at most ``wolfe_expansions`` times.  If a
      doubled step fails the Armijo test, the last trial that passed it stands.

    g is the gradient of the iteration as the reference forms it (sign flip, TV when on,
    gradient-mass scaling), and the trial's gradient gets the same treatment without the
    TV term."""

    def __init__(self, backend, cfg: InversionConfig, preconditioner=None):
        self.b = backend
        self.cfg = cfg
        self.pre = preconditioner

    def run(self, lam0, mu0, n_iter: int, target_reduction: float | None = None, log=None, observer=None):
        """observer(it, lam, mu, g_l, g_m), if given, sees each iteration's scaled
        gradient before the direction is chosen."""
        b, cfg = self.b, self.cfg
        n = b.n
        solves = {"forward": 0, "adjoint": 0}    # forward runs and adjoint runs with the gradient

        def fwd(lam_, mu_):
            solves["forward"] += 1
            return b.forward(lam_, mu_)

        def grad(gl_, gm_):
            solves["adjoint"] += 1
            b.gradient(gl_, gm_)
        lam, mu = b.vec(lam0), b.vec(mu0)
        lam_pre, mu_pre = b.zeros(), b.zeros()
        g_l, g_m, g_l_pre, g_m_pre = b.zeros(), b.zeros(), b.zeros(), b.zeros()
        p_l, p_m = b.zeros(), b.zeros()
        reg_l, reg_m = b.zeros(), b.zeros()
        tmp = b.zeros()
        raw_l, raw_m = b.zeros(), b.zeros()      # raw gradient of a proposal's trial point
        keep_l, keep_m = b.zeros(), b.zeros()    # the same, kept while the step doubles
        have_raw = False
        img, restriction = b.gradient_mass_inverse()
        b.lbfgs_setup(cfg.m_lbfgs, restriction)
        fac_l, fac_m = cfg.fac_max_update_lambda, cfg.fac_max_update_mu
        t0 = time.perf_counter()
        J = fwd(lam, mu)
        J0 = J
        hist = [dict(iter=0, misfit=J, cost=J, reg_lambda=0.0, reg_mu=0.0, g_lambda=0.0, g_mu=0.0, armijo=0,
                     wall_s=time.perf_counter() - t0, forward_solves=1, adjoint_solves=0)]
        self.hist = hist   # kept up to date, also when an ArmijoFailure ends the run
        if log:
            log(hist[-1])

        def update(a_l, a_m, it):
            if cfg.bias_lambda and it < cfg.n_iter_bias:
                pm_n = b.norm2(p_m)
                pl_n = b.norm2(p_l)
                W = 1.0 - float(it // cfg.n_iter_bias)
                fb_mu = W * pl_n / pm_n * a_l
                fb_lam = (1.0 - W) * pl_n * a_l
                b.axpby(fb_mu, p_m, fb_lam, p_l, tmp)
                b.axpby(1.0, lam_pre, 1.0, tmp, lam)
            else:
                b.axpby(a_l, p_l, 1.0, lam_pre, lam)
            b.axpby(a_m, p_m, 1.0, mu_pre, mu)
            b.extend(lam)
            b.extend(mu)
            b.clip(lam, *cfg.bounds_lambda)
            b.clip(mu, *cfg.bounds_mu)

        for it in range(cfg.iter_begin, cfg.iter_begin + n_iter):
            J_pre = J
            b.copy(g_l, g_l_pre)
            b.copy(g_m, g_m_pre)
            if have_raw:                         # computed by the proposal's line search
                b.copy(raw_l, g_l)
                b.copy(raw_m, g_m)
                have_raw = False
            else:
                grad(g_l, g_m)             # raw accumulated gradient of the current forward
            b.axpby(-1.0, g_l, 0.0, None, g_l)   # :412-413
            b.axpby(-1.0, g_m, 0.0, None, g_m)
            cost_rl = cost_rm = 0.0
            if cfg.regularization == "TV":
                cl, cm = b.tv(lam, mu, reg_l, reg_m)
                fl = cfg.reg_factor * b.norm2(g_l) / b.norm2(reg_l)
                fm = cfg.reg_factor * b.norm2(g_m) / b.norm2(reg_m)
                b.axpby(fl, reg_l, 0.0, None, reg_l)
                b.axpby(fm, reg_m, 0.0, None, reg_m)
                if it != 1:
                    b.axpby(1.0, g_l, 1.0, reg_l, g_l)
                    b.axpby(1.0, g_m, 1.0, reg_m, g_m)
                cost_rl, cost_rm = cl * fl, cm * fm
            if it == 1:
                cost_rl = cost_rm = 0.0
            b.mul(g_l, img, g_l)                 # :454-455
            b.mul(g_m, img, g_m)
            if observer is not None:
                observer(it, lam, mu, g_l, g_m)
            if cfg.search == "LBFGS":
                b.lbfgs_direction(it, cfg.iter_begin, g_l, g_m, g_l_pre, g_m_pre, lam, mu, lam_pre, mu_pre, p_l, p_m)
            else:
                b.axpby(-1.0, g_l, 0.0, None, p_l)
                b.axpby(-1.0, g_m, 0.0, None, p_m)
            b.copy(lam, lam_pre)
            b.copy(mu, mu_pre)
            # descent check (:529-556)
            gp_l = b.dot(g_l, p_l)
            chk_l = gp_l > 0
            if chk_l:
                b.axpby(-1.0, g_l, 0.0, None, p_l)
                gp_l = b.dot(g_l, p_l)
            gp_m = b.dot(g_m, p_m)
            chk_m = gp_m > 0
            if chk_m:
                b.axpby(-1.0, g_m, 0.0, None, p_m)
                gp_m = b.dot(g_m, p_m)
            # step size (:558-593)
            pl_max, pm_max = b.norminf(p_l), b.norminf(p_m)
            a_l, a_m = fac_l / pl_max, fac_m / pm_max
            a_l_sd, a_m_sd = a_l, a_m
            if cfg.search == "LBFGS" and it != cfg.iter_begin:
                a_l = a_m = 1.0
                if pl_max > fac_l:
                    a_l = fac_l / pl_max
                if pm_max > fac_m:
                    a_m = fac_m / pm_max
            if chk_l and cfg.search == "LBFGS":
                a_l = a_l_sd
            if chk_m and cfg.search == "LBFGS":
                a_m = a_m_sd
            learned = False
            search = {}
            if self.pre is not None:
                q_l, q_m = self.pre.direction(b, g_l, g_m, lam, mu)
                gq_l, gq_m = b.dot(g_l, q_l), b.dot(g_m, q_m)
                if gq_l < 0.0 and gq_m < 0.0:
                    al = fac_l / b.norminf(q_l)
                    am = fac_m / b.norminf(q_m)

                    def place(scale):
                        b.axpby(scale * al, q_l, 1.0, lam_pre, lam)
                        b.axpby(scale * am, q_m, 1.0, mu_pre, mu)
                        b.extend(lam)
                        b.extend(mu)
                        b.clip(lam, *cfg.bounds_lambda)
                        b.clip(mu, *cfg.bounds_mu)

                    wolfe = cfg.proposal_search == "wolfe"
                    slope0 = al * gq_l + am * gq_m            # g.s of the first trial (< 0)
                    best = None                               # (scale, J, curvature met)
                    trials = 0
                    for k in range(cfg.wolfe_expansions + 1 if wolfe else 1):
                        scale = float(2 ** k)
                        place(scale)
                        J_try = fwd(lam, mu)
                        trials += 1
                        if J_try > J_pre + cfg.armijo_c * scale * slope0:   # sufficient decrease
                            break
                        if not wolfe:
                            best = (scale, J_try, None)
                            break
                        grad(raw_l, raw_m)              # the trial point's gradient
                        b.axpby(-1.0, raw_l, 0.0, None, tmp)
                        b.mul(tmp, img, tmp)
                        d_l = b.dot(tmp, q_l)
                        b.axpby(-1.0, raw_m, 0.0, None, tmp)
                        b.mul(tmp, img, tmp)
                        d_m = b.dot(tmp, q_m)
                        curv = scale * (al * d_l + am * d_m) >= cfg.wolfe_c2 * scale * slope0
                        best = (scale, J_try, curv)
                        if curv:
                            break
                        b.copy(raw_l, keep_l)
                        b.copy(raw_m, keep_m)
                    if best is not None:
                        scale, J_best, curv = best
                        if scale != float(2 ** (trials - 1)):
                            # a doubled step failed the Armijo test: back to the last trial that
                            # passed it, with its forward state for the next iteration's inputs
                            place(scale)
                            J_best = fwd(lam, mu)
                            b.copy(keep_l, raw_l)
                            b.copy(keep_m, raw_m)
                        learned, J, a_l, a_m = True, J_best, scale * al, scale * am
                        have_raw = wolfe
                        search = {"trials": trials, "scale": scale}
                        if wolfe:
                            search["curvature"] = bool(curv)
                    else:
                        search = {"trials": trials}
            if learned:
                count = 0
                rec_extra = {"learned": True, "search": search}
            else:
                rec_extra = {"learned": False, "search": search} if self.pre is not None else {}
                update(a_l, a_m, it)
                J = fwd(lam, mu)
            armijo = cfg.armijo_c * abs(a_m) * gp_m + cfg.armijo_c * abs(a_l) * gp_l
            count = 0
            while not learned and J > J_pre + armijo:            # :737-896
                count += 1
                if count == 3:
                    fac_l /= 6.0
                    fac_m /= 6.0
                a_l *= cfg.armijo_rho
                a_m *= cfg.armijo_rho
                if count == 9:
                    a_l, a_m = -a_l, -a_m
                update(a_l, a_m, it)
                J = fwd(lam, mu)
                armijo = cfg.armijo_c * abs(a_m) * gp_m + cfg.armijo_c * abs(a_l) * gp_l
                if count == 10:
                    raise ArmijoFailure(f"Armijo condition failure at iteration {it}")
            rec = dict(iter=it, misfit=J, cost=J + cost_rl + cost_rm, reg_lambda=cost_rl, reg_mu=cost_rm,
                       g_lambda=b.norm2(g_l), g_mu=b.norm2(g_m), armijo=count, alpha_lambda=a_l, alpha_mu=a_m,
                       wall_s=time.perf_counter() - t0, forward_solves=solves["forward"],
                       adjoint_solves=solves["adjoint"], **rec_extra)
            hist.append(rec)
            if log:
                log(rec)
            if target_reduction is not None and J <= (1.0 - target_reduction) * J0:
                break
        self.lam, self.mu = lam, mu
        return hist


class DeviceBackend:
    """Nodal vectors in device memory (torch tensors as plumbing), every operation a
    libhirensi_b200.so kernel; the Solver must hold mesh, history, shots,
    receivers and the measured data (set_data)."""

    def __init__(self, solver, mesh, device=None):
        import torch
        self.torch = torch
        self.s = solver
        self.mesh = mesh
        self.n = mesh.nj
        self.dev = device or torch.device("cuda", torch.cuda.current_device())
        self.map = torch.from_numpy(np.ascontiguousarray(mesh.extend_to, dtype=np.int32)).to(self.dev)
        self.L = solver._L
        self.h = solver.h
        # One stream for the library and for the tensors it reads and writes.  A
        # stream of its own: the library runs a null stream handle on its private
        # non-blocking stream, which would not be ordered with torch's default stream.
        self.stream = torch.cuda.Stream(self.dev)
        solver.set_stream(self.stream.cuda_stream)

    def _on(self):
        return self.torch.cuda.stream(self.stream)

    def _p(self, t):
        return t.data_ptr()

    def _ck(self, rc):
        self.s._check(rc)

    def zeros(self):
        with self._on():
            return self.torch.zeros(self.n, dtype=self.torch.float64, device=self.dev)

    def vec(self, host):
        with self._on():
            return self.torch.from_numpy(np.ascontiguousarray(host, dtype=np.float64)).to(self.dev)

    def host(self, v):
        with self._on():
            return v.cpu().numpy()

    def copy(self, src, dst):
        self.axpby(1.0, src, 0.0, None, dst)

    def axpby(self, a, x, b, y, z):
        import ctypes as C
        self._ck(self.L.hrn_vec_axpby(self.h, self.n, float(a), C.c_void_p(self._p(x)), float(b),
                                      C.c_void_p(self._p(y) if y is not None else 0), C.c_void_p(self._p(z))))

    def mul(self, x, y, z):
        import ctypes as C
        self._ck(self.L.hrn_vec_mul(self.h, self.n, C.c_void_p(self._p(x)), C.c_void_p(self._p(y)), C.c_void_p(self._p(z))))

    def dot(self, x, y):
        import ctypes as C
        out = C.c_double()
        self._ck(self.L.hrn_vec_dot(self.h, self.n, C.c_void_p(self._p(x)), C.c_void_p(self._p(y)), C.byref(out)))
        return out.value

    def norm2(self, x):
        import ctypes as C
        out = C.c_double()
        self._ck(self.L.hrn_vec_norm(self.h, self.n, C.c_void_p(self._p(x)), 2, C.byref(out)))
        return out.value

    def norminf(self, x):
        import ctypes as C
        out = C.c_double()
        self._ck(self.L.hrn_vec_norm(self.h, self.n, C.c_void_p(self._p(x)), 0, C.byref(out)))
        return out.value

    def clip(self, x, lo, hi):
        import ctypes as C
        self._ck(self.L.hrn_vec_clip(self.h, self.n, float(lo), float(hi), C.c_void_p(self._p(x))))

    def extend(self, x):
        import ctypes as C
        # sources of the extension map are fixed points, so the gather can run in place
        self._ck(self.L.hrn_vec_gather(self.h, self.n, C.c_void_p(self._p(self.map)), C.c_void_p(self._p(x)),
                                       C.c_void_p(self._p(x))))

    def gradient_mass_inverse(self):
        import ctypes as C
        mg = self.zeros()
        self._ck(self.L.hrn_gradient_mass(self.h, C.c_void_p(self._p(mg))))
        with self._on():
            keep = mg > 1.0e-10
            img = self.torch.where(keep, 1.0 / self.torch.where(keep, mg, self.torch.ones_like(mg)), self.torch.zeros_like(mg))
            return img.contiguous(), keep.to(self.torch.float64).contiguous()

    def tv(self, lam, mu, reg_l, reg_m):
        import ctypes as C
        cl, cm = C.c_double(), C.c_double()
        self._ck(self.L.hrn_regularization_tv(self.h, C.c_void_p(self._p(lam)), C.c_void_p(self._p(mu)),
                                              C.c_void_p(self._p(reg_l)), C.c_void_p(self._p(reg_m)), C.byref(cl), C.byref(cm)))
        return cl.value, cm.value

    def lbfgs_setup(self, m, restriction):
        import ctypes as C
        self._ck(self.L.hrn_lbfgs_setup(self.h, int(m), C.c_void_p(self._p(restriction))))

    def lbfgs_direction(self, it, it0, g_l, g_m, g_l_pre, g_m_pre, lam, mu, lam_pre, mu_pre, p_l, p_m):
        import ctypes as C
        vp = [C.c_void_p(self._p(v)) for v in (g_l, g_m, g_l_pre, g_m_pre, lam, mu, lam_pre, mu_pre, p_l, p_m)]
        self._ck(self.L.hrn_lbfgs_direction(self.h, int(it), int(it0), *vp, None))

    def forward(self, lam, mu):
        self.s.assemble_device(self._p(lam), self._p(mu))
        self.s.forward()
        return self.s.misfit(None)

    def gradient(self, g_l, g_m):
        self.s.adjoint_gradient(None, to_host=False)
        self.s.gradient_device(self._p(g_l), self._p(g_m))

    def illumination(self):
        """Source illumination of the stored nodes of the last forward (host array)."""
        import ctypes as C
        with self._on():
            out = self.torch.zeros(self.s.nstore // 3, dtype=self.torch.float64, device=self.dev)
            self._ck(self.L.hrn_illumination(self.h, C.c_void_p(self._p(out))))
            return out.cpu().numpy()

    def pseudo_hessian(self):
        """Diagonal pseudo-Hessian (lambda, mu) [nj] of the last forward (host arrays)."""
        import ctypes as C
        nj = self.mesh.nj
        with self._on():
            out = self.torch.zeros(2, nj, dtype=self.torch.float64, device=self.dev)
            self._ck(self.L.hrn_pseudo_hessian(self.h, C.c_void_p(self._p(out[0])), C.c_void_p(self._p(out[1]))))
            h = out.cpu().numpy()
        return h[0], h[1]


class BatchedBackend(DeviceBackend):
    """DeviceBackend over many shots advanced in batches on one context: the misfit of a
    model is the sum over batches (each batch configured in turn, hirensi_b200.batching),
    and the gradient the sum of the batches' adjoint gradients.  The batch left resident by
    the last misfit evaluation takes its adjoint first; the others run their forward again
    before their adjoint (with checkpointing this is the usual recompute).  The reference
    solves one source per call and sums over its sources the same way
    (S4/Program_Main.F90:379-470).  batches: packed batches with their measured data
    (Batch.dis, [nshot][nrec3][nstep+1]); store_position maps receiver equations to
    history positions (Mesh.store_position)."""

    def __init__(self, solver, mesh, batches, dt, store_position, device=None):
        super().__init__(solver, mesh, device)
        self.batches = batches
        self.dt = dt
        self.store_position = store_position
        self.resident = None
        self._g = self.torch.zeros(2, self.n, dtype=self.torch.float64, device=self.dev)

    def _use(self, k):
        from . import batching
        b = self.batches[k]
        batching.configure(self.s, b, self.dt, self.store_position)
        self.s.set_data(b.dis)
        self.resident = k

    def forward(self, lam, mu):
        self.s.assemble_device(self._p(lam), self._p(mu))
        J = 0.0
        for k in range(len(self.batches)):
            self._use(k)
            self.s.forward()
            J += self.s.misfit(None)
        return J

    def gradient(self, g_l, g_m):
        order = list(range(len(self.batches)))
        if self.resident is not None:
            order.remove(self.resident)
            order.insert(0, self.resident)
        self.axpby(0.0, g_l, 0.0, None, g_l)
        self.axpby(0.0, g_m, 0.0, None, g_m)
        first = self.resident
        for i, k in enumerate(order):
            if not (i == 0 and k == first):      # no misfit evaluation left this batch resident
                self._use(k)
                self.s.forward()
            self.s.adjoint_gradient(None, to_host=False)
            self.s.gradient_device(self._p(self._g[0]), self._p(self._g[1]))
            self.axpby(1.0, g_l, 1.0, self._g[0], g_l)
            self.axpby(1.0, g_m, 1.0, self._g[1], g_m)
