"""ctypes wrapper of the CPU FP64 oracle (hrn_oracle.c) plus numpy restatements of
the reference's coupled L-BFGS and model-update step.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py to check (or time, as a baseline) the CUDA path.  The
hirensi_b200 package never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libhrn_oracle.so")
_lib = None

PD = C.POINTER(C.c_double)
PI = C.POINTER(C.c_int)


class _Mesh(C.Structure):
    _fields_ = [("nj", C.c_int), ("nel", C.c_int), ("neq", C.c_int),
                ("xyz", PD), ("inod", PI), ("mtel", PI), ("id", PI), ("rho_el", PD),
                ("pml_param", (C.c_double * 4) * 6)]


def build() -> str:
    """Compile the oracle library with its Makefile (gcc)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(os.path.join(_HERE, "hrn_oracle.c")):
            build()
        L = C.CDLL(_SO)
        L.ora_assemble.restype = C.c_void_p
        L.ora_assemble.argtypes = [C.POINTER(_Mesh), PD, PD, PI, PI]
        L.ora_sys_from_csr.restype = C.c_void_p
        L.ora_sys_from_csr.argtypes = [C.c_int] + [PI, PI, PD] * 3 + [PD]
        L.ora_sys_free.argtypes = [C.c_void_p]
        L.ora_sys_nnz.argtypes = [C.c_void_p, C.c_int]
        L.ora_sys_csr.argtypes = [C.c_void_p, C.c_int, PI, PI, PD]
        L.ora_sys_vectors.argtypes = [C.c_void_p, PD, PD]
        L.ora_forward.argtypes = [C.c_void_p, PD, PD, C.c_int, C.c_double, C.c_int, PI, PD, C.c_int]
        L.ora_adjoint.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int, PI, PD, C.c_int, PI, PI, PD, PD, C.c_int]
        L.ora_control.argtypes = [C.POINTER(_Mesh), C.c_int, C.c_double, C.c_int, PI, PD, PD, PD, PD, C.c_int, C.c_int]
        L.ora_misfit.restype = C.c_double
        L.ora_misfit.argtypes = [C.c_int, C.c_double, C.c_int, PI, PI, C.c_int, PD, PD]
        L.ora_tv_reg.argtypes = [C.POINTER(_Mesh), PD, PD, PD, PD, PD, PD]
        L.ora_rmg.argtypes = [C.POINTER(_Mesh), PD]
        L.ora_time_function.restype = C.c_double
        L.ora_time_function.argtypes = [C.c_double, C.c_int, C.c_double]
        L.ora_shape_3_27.argtypes = [C.c_double] * 3 + [PD, PD]
        L.ora_pml_finder_3d.argtypes = [PD, PD, PD]
        L.ora_element_k.argtypes = [PD, PD, PD, PD]
        L.ora_element_m.argtypes = [PD, C.c_double, PD, C.c_int, PD]
        L.ora_element_en.argtypes = [PD, PD, C.c_int, PD]
        L.ora_element_ea.argtypes = [PD, PD, PD, PD, C.c_int, PD]
        L.ora_element_fs.argtypes = [PD, C.c_int, PD]
        L.ora_element_g.argtypes = [PD, PD, PD, PD, PD, C.c_int]
        L.ora_apply_scaled.argtypes = [C.c_void_p, C.c_int, C.c_int, PD, PD]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(PD)


def _i(a):
    return a.ctypes.data_as(PI)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# --- element level ------------------------------------------------------------

def shape_3_27(x1, x2, x3):
    fn = np.zeros(27)
    d = np.zeros((27, 3))
    lib().ora_shape_3_27(x1, x2, x3, _d(fn), _d(d))
    return fn, d


def pml_finder(xg, pml_param):
    out = np.zeros(19)
    xg = _f64(xg)
    p = _f64(pml_param)
    rc = lib().ora_pml_finder_3d(_d(xg), _d(p), _d(out))
    if rc:
        raise ValueError("point in the top PML zone")
    return out


def element_k(xt, lam_e, mu_e):
    ek = np.zeros((81, 81))
    rc = lib().ora_element_k(_d(_f64(xt)), _d(_f64(lam_e)), _d(_f64(mu_e)), _d(ek))
    assert rc == 0
    return ek


def element_m(xt, rho, pml_param, flag):
    em = np.zeros((81, 81))
    rc = lib().ora_element_m(_d(_f64(xt)), float(rho), _d(_f64(pml_param)), flag, _d(em))
    assert rc == 0, rc
    return em


def element_en(xt, pml_param, flag):
    en = np.zeros((162, 162))
    rc = lib().ora_element_en(_d(_f64(xt)), _d(_f64(pml_param)), flag, _d(en))
    assert rc == 0, rc
    return en


def element_ea(xt, lam_e, mu_e, pml_param, flag):
    ea = np.zeros((81, 162))
    rc = lib().ora_element_ea(_d(_f64(xt)), _d(_f64(lam_e)), _d(_f64(mu_e)), _d(_f64(pml_param)), flag, _d(ea))
    assert rc == 0, rc
    return ea


def element_fs(xt, nface):
    efs = np.zeros(81)
    rc = lib().ora_element_fs(_d(_f64(xt)), nface, _d(efs))
    if rc:
        raise ValueError(f"ELEMENT_FS failed ({rc})")
    return efs


def element_g(xt, eu, ep, lambda_2mu=False):
    gm = np.zeros(27)
    gl = np.zeros(27)
    rc = lib().ora_element_g(_d(_f64(xt)), _d(_f64(eu)), _d(_f64(ep)), _d(gm), _d(gl), int(lambda_2mu))
    assert rc == 0
    return gm, gl


def time_function(t, lcase=2, fr=15.0):
    return lib().ora_time_function(float(t), int(lcase), float(fr))


def time_table(nstep, dt, lcase=2, fr=15.0):
    """TIME_FUNCTION at T, T+dt and T+dt/2 for T = ISTEP*dt, ISTEP = 0..nstep
    (the three calls of S4/Solver_PETSc_Explicit.F90:983-995)."""
    tab = np.zeros((nstep + 1, 3))
    L = lib()
    for i in range(nstep + 1):
        T = float(i) * dt
        tab[i, 0] = L.ora_time_function(T, lcase, fr)
        tab[i, 1] = L.ora_time_function(T + dt, lcase, fr)
        tab[i, 2] = L.ora_time_function(T + 0.5 * dt, lcase, fr)
    return tab


# --- mesh / system level --------------------------------------------------------

class OracleMesh:
    """Holds the C view of a hirensi_b200.mesh.Mesh (arrays are kept alive here)."""

    def __init__(self, mesh, rho=2.0e-3):
        self.mesh = mesh
        self.xyz = _f64(mesh.xyz)
        self.inod = _i32(mesh.inod)
        self.mtel = _i32(mesh.mtel)
        self.id = _i32(mesh.ID)
        self.rho = _f64(np.full(mesh.nel, rho) if np.isscalar(rho) else rho)
        m = _Mesh()
        m.nj, m.nel, m.neq = mesh.nj, mesh.nel, mesh.neq
        m.xyz, m.inod, m.mtel, m.id, m.rho_el = _d(self.xyz), _i(self.inod), _i(self.mtel), _i(self.id), _d(self.rho)
        for r in range(6):
            for c in range(4):
                m.pml_param[r][c] = float(mesh.pml_param[r, c])
        self.c = m


class OracleSystem:
    """Assembled C, K, G (scalar CSR, zeros dropped), DIAG_M and B."""

    def __init__(self, handle, neq):
        self.h = handle
        self.neq = neq

    @classmethod
    def assemble(cls, om: OracleMesh, lam, mu, id_bc=None):
        err = C.c_int(0)
        lam = _f64(lam)
        mu = _f64(mu)
        idb = _i32(id_bc) if id_bc is not None else None
        h = lib().ora_assemble(C.byref(om.c), _d(lam), _d(mu), _i(idb) if idb is not None else None, C.byref(err))
        if not h:
            raise RuntimeError(f"oracle assembly failed ({err.value})")
        return cls(h, om.mesh.neq)

    @classmethod
    def from_csr(cls, neq, mats, diag_m):
        arrs = []
        for ia, ja, a in mats:
            arrs += [_i32(ia), _i32(ja), _f64(a)]
        dm = _f64(diag_m)
        h = lib().ora_sys_from_csr(neq, *[(_i(x) if x.dtype == np.int32 else _d(x)) for x in arrs], _d(dm))
        obj = cls(h, neq)
        obj._keep = (arrs, dm)
        return obj

    def __del__(self):
        if getattr(self, "h", None):
            lib().ora_sys_free(self.h)
            self.h = None

    def csr(self, which):
        nz = lib().ora_sys_nnz(self.h, which)
        ia = np.zeros(self.neq + 1, np.int32)
        ja = np.zeros(nz, np.int32)
        a = np.zeros(nz)
        lib().ora_sys_csr(self.h, which, _i(ia), _i(ja), _d(a))
        return ia, ja, a

    def vectors(self):
        dm = np.zeros(self.neq)
        b = np.zeros(self.neq)
        lib().ora_sys_vectors(self.h, _d(dm), _d(b))
        return dm, b

    def forward(self, b, ftab, nstep, dt, store_eq, nthreads=1):
        store_eq = _i32(store_eq)
        u = np.zeros((nstep + 1, store_eq.size))
        ftab = _f64(ftab)
        assert ftab.shape == (nstep + 1, 3)
        lib().ora_forward(self.h, _d(_f64(b)), _d(ftab), nstep, float(dt), store_eq.size, _i(store_eq), _d(u), int(nthreads))
        return u

    def adjoint(self, nstep, dt, store_eq, u_store, eqdis, eqdis_map, dis_meas, nthreads=1):
        store_eq = _i32(store_eq)
        p = np.zeros((nstep + 1, store_eq.size))
        dis_meas = _f64(dis_meas)
        assert dis_meas.shape == (len(eqdis), nstep + 1)
        lib().ora_adjoint(self.h, nstep, float(dt), store_eq.size, _i(store_eq), _d(_f64(u_store)),
                          len(eqdis), _i(_i32(eqdis)), _i(_i32(eqdis_map)), _d(dis_meas), _d(p), int(nthreads))
        return p

    def apply(self, which, x, transpose_adjoint=False):
        y = np.zeros(self.neq)
        lib().ora_apply_scaled(self.h, which, int(transpose_adjoint), _d(_f64(x)), _d(y))
        return y


def control(om: OracleMesh, nstep, dt, store_eq, u_store, p_store, lambda_2mu=False, nthreads=0):
    """Raw (g_lambda, g_mu) of the control accumulation; nthreads 0 keeps the current
    OpenMP setting, and every thread count gives the same bits."""
    gl = np.zeros(om.mesh.nj)
    gm = np.zeros(om.mesh.nj)
    store_eq = _i32(store_eq)
    rc = lib().ora_control(C.byref(om.c), nstep, float(dt), store_eq.size, _i(store_eq), _d(_f64(u_store)),
                           _d(_f64(p_store)), _d(gl), _d(gm), int(lambda_2mu), int(nthreads))
    assert rc == 0
    return gl, gm


def misfit(nstep, dt, eqdis, eqdis_map, u_store, dis_meas):
    u_store = _f64(u_store)
    return lib().ora_misfit(nstep, float(dt), len(eqdis), _i(_i32(eqdis)), _i(_i32(eqdis_map)),
                            u_store.shape[1], _d(u_store), _d(_f64(dis_meas)))


def tv_reg(om: OracleMesh, lam, mu):
    rl = np.zeros(om.mesh.nj)
    rm = np.zeros(om.mesh.nj)
    cl = C.c_double()
    cm = C.c_double()
    rc = lib().ora_tv_reg(C.byref(om.c), _d(_f64(lam)), _d(_f64(mu)), _d(rl), _d(rm), C.byref(cl), C.byref(cm))
    assert rc == 0
    return rl, rm, cl.value, cm.value


def rmg(om: OracleMesh):
    mg = np.zeros(om.mesh.nj)
    rc = lib().ora_rmg(C.byref(om.c), _d(mg))
    assert rc == 0
    return mg


def inverse_gradient_mass(mg):
    """S4/Control_Problem_Operators.F90:11-22: iMg = 1/Mg where Mg > 1e-10, else 0."""
    img = np.where(mg > 1.0e-10, 1.0 / np.where(mg > 1.0e-10, mg, 1.0), 0.0)
    restriction = (mg > 1.0e-10).astype(np.float64)
    return img, restriction


# --- L-BFGS (S4/LBFGS_Coupled.F90:1-221) --------------------------------------

class LBFGSCoupled:
    """Numpy restatement of the coupled (lambda, mu) L-BFGS include."""

    def __init__(self, nj, m_lbfgs, restriction):
        self.M = m_lbfgs
        self.restriction = restriction
        self.Ys_l = np.zeros((nj, m_lbfgs))
        self.Ys_m = np.zeros((nj, m_lbfgs))
        self.Ss_l = np.zeros((nj, m_lbfgs))
        self.Ss_m = np.zeros((nj, m_lbfgs))
        self.rhos = np.zeros(m_lbfgs)
        self.alphas = np.zeros(m_lbfgs)

    def direction(self, it, it_begin, g_l, g_m, g_l_pre, g_m_pre, lam, mu, lam_pre, mu_pre):
        if it == it_begin:
            return -g_l.copy(), -g_m.copy()
        k = it - it_begin
        M = self.M
        y_l = 0.0 + (1.0 * g_l + -1.0 * g_l_pre)
        s_l = 0.0 + (1.0 * lam + -1.0 * lam_pre)
        y_m = 0.0 + (1.0 * g_m + -1.0 * g_m_pre)
        s_m = 0.0 + (1.0 * mu + -1.0 * mu_pre)
        rho = 1.0 / (float(y_l @ s_l) + float(y_m @ s_m))
        q_l = g_l.copy()
        q_m = g_m.copy()
        if 0 < k <= M:
            n_use = k
            seq = list(range(k, 0, -1))
        else:
            n_use = M
            end = k % M
            seq = list(range(end, 0, -1))
            j = 0
            for _ in range(len(seq), M):
                seq.append(M - j)
                j += 1
        n_store = (k % M) if (k % M) != 0 else M
        self.rhos[n_store - 1] = rho
        self.Ys_l[:, n_store - 1] = y_l
        self.Ys_m[:, n_store - 1] = y_m
        self.Ss_l[:, n_store - 1] = s_l * self.restriction
        self.Ss_m[:, n_store - 1] = s_m * self.restriction
        for iv in range(n_use):
            i = seq[iv] - 1
            a = self.rhos[i] * float(q_l @ self.Ss_l[:, i]) + self.rhos[i] * float(q_m @ self.Ss_m[:, i])
            self.alphas[i] = a
            q_l = q_l - a * self.Ys_l[:, i]
            q_m = q_m - a * self.Ys_m[:, i]
        num = float(y_l @ s_l) + float(y_m @ s_m)
        den = float(y_l @ y_l) + float(y_m @ y_m)
        r_l = (num / den) * q_l
        r_m = (num / den) * q_m
        for iv in range(n_use - 1, -1, -1):
            i = seq[iv] - 1
            beta = self.rhos[i] * float(r_l @ self.Ys_l[:, i]) + self.rhos[i] * float(r_m @ self.Ys_m[:, i])
            r_l = r_l + self.Ss_l[:, i] * (self.alphas[i] - beta)
            r_m = r_m + self.Ss_m[:, i] * (self.alphas[i] - beta)
        return -r_l, -r_m


# --- inversion loop (S4/Program_Main.F90:379-896) ------------------------------

class ArmijoStop(RuntimeError):
    """The reference STOPs after the tenth Armijo trial (S4/Program_Main.F90:883-889)."""


def _extend_and_clip(v, extend_to, lo, hi):
    """VIII (:633-636) then IX (:638-678): the PML nodes take the material of
    their interface node (VecScatter INSERT_VALUES), then every node is clipped
    to the bounds."""
    v = v[extend_to]
    return np.where(v < lo, lo, np.where(v > hi, hi, v))


def inversion_loop(evaluate, gradient, lam0, mu0, n_iter, img, restriction, extend_to, bounds_lambda, bounds_mu,
                   m_lbfgs=15, fac_max_update=(5.0, 5.0), tv=None, reg_factor=0.3, bias_lambda=True,
                   n_iter_bias=50, iter_begin=1):
    """Numpy restatement of the reference's inversion iterations for
    Control_Parameter = 'Lambda_Mu', Lambda_variable = 'Lambda' and
    Search_Direction_Method = 'LBFGS', written from S4/Program_Main.F90:
    * evaluate(lam, mu) -> misfit of the forward solve of that model (Include
      'Solve_Forward.F90' + Compute_Misfit);
    * gradient() -> (g_lambda, g_mu) raw accumulated gradient of the model
      evaluated last (..._Adjoint_OtD + ..._Control_OtD, before the sign flip);
    * tv(lam, mu) -> (reg_lambda, reg_mu, cost_lambda, cost_mu) or None for no
      regularization (Assem_TV_TN_Regularization);
    * img, restriction: the inverse gradient mass and the regular-domain mask
      (S4/Control_Problem_Operators.F90:11-22); extend_to: the PML material
      extension map (vscat_mat_extend).
    Returns a list of per-iteration records (iteration 0 = the initial model):
    misfit, alpha_lambda, alpha_mu, armijo trials, and the model after the
    iteration.  Raises ArmijoStop where the reference STOPs."""
    fac_l, fac_m = float(fac_max_update[0]), float(fac_max_update[1])
    lb = LBFGSCoupled(len(lam0), m_lbfgs, restriction)
    lam = np.array(lam0, dtype=np.float64)
    mu = np.array(mu0, dtype=np.float64)
    lam_pre = np.zeros_like(lam)
    mu_pre = np.zeros_like(mu)
    g_l = np.zeros_like(lam)
    g_m = np.zeros_like(mu)
    J = evaluate(lam, mu)                                         # :327-333
    recs = [dict(iter=0, misfit=J, armijo=0, lam=lam.copy(), mu=mu.copy())]

    def trial(a_l, a_m, it, p_l, p_m):
        """VII (:597-628) + VIII + IX: the model of step sizes a_l, a_m."""
        if bias_lambda and it < n_iter_bias:
            W = 1.0 - float(it // n_iter_bias)                    # DBLE(Iter/NIterBias): integer division
            pm_n = float(np.sqrt(p_m @ p_m))
            pl_n = float(np.sqrt(p_l @ p_l))
            fb_mu = W * pl_n / pm_n * a_l
            fb_lam = (1.0 - W) * pl_n * a_l
            new_l = lam_pre + (fb_mu * p_m + fb_lam * p_l)        # VecCopy + VecMAXPY
        else:
            new_l = a_l * p_l + lam_pre                           # VecWAXPY
        new_m = a_m * p_m + mu_pre
        return (_extend_and_clip(new_l, extend_to, *bounds_lambda),
                _extend_and_clip(new_m, extend_to, *bounds_mu))

    for it in range(iter_begin, iter_begin + n_iter):
        J_pre = J                                                 # II (:384-392)
        g_l_pre, g_m_pre = g_l.copy(), g_m.copy()
        raw_l, raw_m = gradient()                                 # III (:398-409)
        g_l = -np.asarray(raw_l, dtype=np.float64)                # :412-413
        g_m = -np.asarray(raw_m, dtype=np.float64)
        if tv is not None:                                        # IV (:418-450)
            reg_l, reg_m, _, _ = tv(lam, mu)
            f_l = reg_factor * float(np.sqrt(g_l @ g_l)) / float(np.sqrt(reg_l @ reg_l))
            f_m = reg_factor * float(np.sqrt(g_m @ g_m)) / float(np.sqrt(reg_m @ reg_m))
            if it != 1:
                g_l = g_l + f_l * reg_l
                g_m = g_m + f_m * reg_m
        g_l = g_l * img                                           # :454-455
        g_m = g_m * img
        p_l, p_m = lb.direction(it, iter_begin, g_l, g_m, g_l_pre, g_m_pre, lam, mu, lam_pre, mu_pre)   # VI-2
        lam_pre, mu_pre = lam.copy(), mu.copy()                   # VI-3 (:524-526)
        gp_l = float(g_l @ p_l)                                   # VI-4 (:529-556)
        chk_l = gp_l > 0
        if chk_l:
            p_l = -g_l
            gp_l = float(g_l @ p_l)
        gp_m = float(g_m @ p_m)
        chk_m = gp_m > 0
        if chk_m:
            p_m = -g_m
            gp_m = float(g_m @ p_m)
        pl_max = float(np.abs(p_l).max())                         # VI-5 (:558-593)
        pm_max = float(np.abs(p_m).max())
        a_l, a_m = fac_l / pl_max, fac_m / pm_max
        a_l_sd, a_m_sd = a_l, a_m
        if it != iter_begin:
            a_l = a_m = 1.0
            if pl_max > fac_l:
                a_l = fac_l / pl_max
            if pm_max > fac_m:
                a_m = fac_m / pm_max
        if chk_l:
            a_l = a_l_sd
        if chk_m:
            a_m = a_m_sd
        lam, mu = trial(a_l, a_m, it, p_l, p_m)
        J = evaluate(lam, mu)                                     # X-3, X-4
        armijo = 1.0e-4 * abs(a_m) * gp_m + 1.0e-4 * abs(a_l) * gp_l
        count = 0
        while J > J_pre + armijo:                                 # X-5 (:737-896)
            count += 1
            if count == 3:
                fac_l /= 6.0
                fac_m /= 6.0
            a_l *= 0.5
            a_m *= 0.5
            if count == 9:
                a_l, a_m = -a_l, -a_m
            lam, mu = trial(a_l, a_m, it, p_l, p_m)
            J = evaluate(lam, mu)
            armijo = 1.0e-4 * abs(a_m) * gp_m + 1.0e-4 * abs(a_l) * gp_l
            if count == 10:
                raise ArmijoStop(f"Armijo condition failure at iteration {it}")
        recs.append(dict(iter=it, misfit=J, armijo=count, alpha_lambda=a_l, alpha_mu=a_m,
                         lam=lam.copy(), mu=mu.copy()))
    return recs
