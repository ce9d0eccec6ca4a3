"""Host-side mirror of HiReNSI's explicit forward / adjoint / gradient interface.

``Solver`` owns one device context of libhirensi_b200.so.  The module-level
functions keep the names and argument meaning of the reference routines they
replace (S4 = step_4_3D_Forward_and_Inverse):

* ``EXPLICIT_RK4_PETSC_PML_3D``        S4/Solver_PETSc_Explicit.F90:660-1117
* ``EXPLICIT_RK4_PETSC_PML_3D_Adjoint_Control_OtD``
                                         :1125-1405 followed by :1413-1522
* ``Compute_Misfit``                     S4/Solver_PETSc_Inverse.F90:591-657

Errors raise ``HrnError`` with the library's status code, where the reference
would STOP the process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .capi import HrnError, dptr, f64, i32, iptr


class Solver:
    """One device context (stepping precision 'fp64' or 'fp32')."""

    def __init__(self, precision: str = "fp64", device: int = 0):
        self._L = capi.load()
        prec = {"fp64": capi.HRN_FP64, "fp32": capi.HRN_FP32}[precision]
        h = C.c_void_p()
        rc = self._L.hrn_create(device, prec, C.byref(h))
        if rc != capi.HRN_OK:
            raise HrnError(rc, "hrn_create failed (no CUDA device?)")
        self.h = h
        self.precision = precision
        self.nshot = 0
        self.nstep = 0
        self.nstore = 0
        self.nrec3 = 0
        self.nj = 0
        self.nel = 0
        self.neq = 0
        self.ckpt_interval = 0

    # -- plumbing ---------------------------------------------------------------
    def _check(self, rc):
        if rc != capi.HRN_OK:
            msg = self._L.hrn_last_error(self.h)
            raise HrnError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "h", None):
            self._L.hrn_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int | None):
        self._check(self._L.hrn_set_stream(self.h, C.c_void_p(stream_ptr or 0)))

    def set_graphs(self, on: bool):
        """Capture each forward / adjoint call's launches as a CUDA graph and replay
        it on later calls (on by default)."""
        self._check(self._L.hrn_set_graphs(self.h, int(bool(on))))

    def graph_stats(self):
        """(time loops captured, graph launches) so far."""
        a, b = C.c_int64(), C.c_int64()
        self._check(self._L.hrn_graph_stats(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_timing(self, on: bool):
        self._check(self._L.hrn_set_timing(self.h, int(bool(on))))

    def last_timing(self):
        tot, st, n = C.c_double(), C.c_double(), C.c_int64()
        self._check(self._L.hrn_last_timing(self.h, C.byref(tot), C.byref(st), C.byref(n)))
        return tot.value, st.value, n.value

    # -- operator ---------------------------------------------------------------
    def set_operator_csr(self, Cm, Km, Gm, diag_m):
        """Caller-assembled C, K, G as (ia, ja, a) CSR triples and DIAG_M."""
        arrs = []
        for ia, ja, a in (Cm, Km, Gm):
            arrs.append((i32(ia), i32(ja), f64(a)))
        dm = f64(diag_m)
        neq = dm.size
        flat = []
        for ia, ja, a in arrs:
            if ia.size != neq + 1:
                raise ValueError("row pointer length must be neq + 1")
            flat += [iptr(ia), iptr(ja), dptr(a)]
        self._check(self._L.hrn_set_operator_csr(self.h, neq, *flat, dptr(dm)))
        self.neq = neq

    def set_mesh(self, mesh, rho=2.0e-3):
        """Geometry and numbering of a hirensi_b200.mesh.Mesh."""
        rho_el = f64(np.full(mesh.nel, rho) if np.isscalar(rho) else rho)
        self._mesh_keep = (f64(mesh.xyz), i32(mesh.inod), i32(mesh.mtel), i32(mesh.ID), rho_el, f64(mesh.pml_param))
        xyz, inod, mtel, idm, rho_el, pml = self._mesh_keep
        self._check(self._L.hrn_set_mesh(self.h, mesh.nj, mesh.nel, mesh.neq, dptr(xyz), iptr(inod), iptr(mtel),
                                         iptr(idm), dptr(rho_el), dptr(pml)))
        self.nj = mesh.nj
        self.nel = mesh.nel
        self.neq = mesh.neq

    def set_operator_mode(self, matrix_free: bool):
        """True: assemble DIAG_M only and apply C, K, G matrix-free (variants 90-105);
        call after set_mesh, before the first assemble."""
        self._check(self._L.hrn_set_operator_mode(self.h, int(bool(matrix_free))))

    def assemble(self, lam, mu):
        self._check(self._L.hrn_assemble(self.h, dptr(f64(lam)), dptr(f64(mu))))

    def assemble_device(self, lam_ptr: int, mu_ptr: int):
        """Assemble from device-resident nodal lambda, mu (raw device pointers, FP64 [nj])."""
        self._check(self._L.hrn_assemble_device(self.h, C.c_void_p(lam_ptr), C.c_void_p(mu_ptr)))

    def operator_nnz(self, which: int) -> int:
        """Stored entries of C (0), K (1) or G (2)."""
        nnz = C.c_int64()
        self._check(self._L.hrn_get_operator_csr(self.h, which, None, None, None, C.byref(nnz)))
        return nnz.value

    def operator_csr(self, which: int):
        nnz = C.c_int64()
        self._check(self._L.hrn_get_operator_csr(self.h, which, None, None, None, C.byref(nnz)))
        ia = np.zeros(self.neq + 1, np.int32)
        ja = np.zeros(nnz.value, np.int32)
        a = np.zeros(nnz.value)
        self._check(self._L.hrn_get_operator_csr(self.h, which, iptr(ia), iptr(ja), dptr(a), C.byref(nnz)))
        return ia, ja, a

    def apply_operator(self, which: int, x, adjoint: bool = False) -> np.ndarray:
        """One per-step operator on the device: -iM A x (forward) or A'^T x (the
        adjoint-scaled operator, transposed), A = C (0), K (1) or G (2)."""
        xv = f64(x)
        if xv.size != self.neq:
            raise ValueError("x must have neq entries")
        y = np.zeros(self.neq)
        self._check(self._L.hrn_apply_operator(self.h, int(which), int(bool(adjoint)), dptr(xv), dptr(y)))
        return y

    def diag_m(self):
        d = np.zeros(self.neq)
        self._check(self._L.hrn_get_diag_m(self.h, dptr(d)))
        return d

    # -- problem ----------------------------------------------------------------
    def set_history(self, store_eq):
        se = i32(store_eq)
        self._check(self._L.hrn_set_history(self.h, se.size, iptr(se)))
        self.nstore = se.size

    def set_shots(self, nstep: int, dt: float, src_eq, src_b, ftab):
        """src_b [nsrc, nshot] unscaled force entries, ftab [nshot, nstep+1, 3]."""
        se = i32(src_eq)
        sb = f64(src_b)
        ft = f64(ftab)
        if ft.ndim == 2:
            ft = ft[None]
        nshot = ft.shape[0]
        if sb.ndim == 1:
            sb = sb[:, None]
        if sb.shape != (se.size, nshot) or ft.shape != (nshot, nstep + 1, 3):
            raise ValueError("src_b must be [nsrc, nshot] and ftab [nshot, nstep+1, 3]")
        self._check(self._L.hrn_set_shots(self.h, nshot, nstep, float(dt), se.size, iptr(se) if se.size else None,
                                          dptr(np.ascontiguousarray(sb)) if se.size else None, dptr(ft)))
        self.nshot, self.nstep, self.dt = nshot, nstep, dt

    def assemble_face_force(self, nface) -> np.ndarray:
        """ASSEM_FORCE_PETSC_3D on the device: B [neq] of a unit vertical traction on
        the loaded face nface[e] = ID_BC(e, 1) (0 = none) of each regular-domain element."""
        nf = i32(nface)
        if nf.size != self.nel:
            raise ValueError("nface must have one entry per element")
        b = np.zeros(self.neq)
        self._check(self._L.hrn_assemble_face_force(self.h, iptr(nf), dptr(b)))
        return b

    def set_shots_face_force(self, nstep: int, dt: float, ftab):
        """Shots loaded by the device face-force vector, ftab [nshot, nstep+1, 3]."""
        ft = f64(ftab)
        if ft.ndim == 2:
            ft = ft[None]
        if ft.shape[1:] != (nstep + 1, 3):
            raise ValueError("ftab must be [nshot, nstep+1, 3]")
        self._check(self._L.hrn_set_shots_face_force(self.h, ft.shape[0], nstep, float(dt), dptr(ft)))
        self.nshot, self.nstep, self.dt = ft.shape[0], nstep, dt

    def set_receivers(self, eqdis, eqdis_map):
        e, m = i32(eqdis), i32(eqdis_map)
        self._check(self._L.hrn_set_receivers(self.h, e.size, iptr(e), iptr(m)))
        self.nrec3 = e.size

    def set_shot_records(self, nstep_shot=None, rec_mask=None):
        """Uneven shots: record length of each shot (<= nstep of set_shots) and
        rec_mask [nshot, nrec3] of the receivers each shot records (None = all)."""
        ns = None if nstep_shot is None else i32(nstep_shot)
        if ns is not None and ns.size != self.nshot:
            raise ValueError("nstep_shot must have one entry per shot")
        mk = None
        if rec_mask is not None:
            mk = np.ascontiguousarray(np.asarray(rec_mask, dtype=np.uint8))
            if mk.shape != (self.nshot, self.nrec3):
                raise ValueError("rec_mask must be [nshot, nrec3]")
        self._check(self._L.hrn_set_shot_records(self.h, ns.ctypes.data if ns is not None else None,
                                                 mk.ctypes.data if mk is not None else None))
        self._keep_records = (ns, mk)

    def set_data(self, dis_meas=None, device_ptr: int | None = None):
        """Keep the measured data [nshot, nrec3, nstep+1] on the device (host array or device pointer)."""
        if device_ptr is not None:
            self._check(self._L.hrn_set_data(self.h, C.c_void_p(device_ptr), 1))
        else:
            d = self._dis(dis_meas)
            self._check(self._L.hrn_set_data(self.h, d.ctypes.data_as(C.c_void_p), 0))

    def set_checkpointing(self, interval: int):
        """0: keep the whole forward history; K > 0: keep the forward state every
        K steps and recompute each segment's history during the adjoint."""
        self._check(self._L.hrn_set_checkpointing(self.h, int(interval)))
        self.ckpt_interval = int(interval)

    def set_variant(self, forward: int = 0, adjoint: int = 0):
        """Force the stage-kernel variant, 0 = chosen by timing on first use.
        CSR: lanes per row * 10 + stage inputs materialized (1) or rebuilt (0),
        + 2 for the tiled kernel, + 4 for the compact row tiles with staged
        gathers (40-45, 80-85, 160, 161).  Matrix-free (operator
        assembled from the mesh): 90-95 materialized / 100-105 rebuilt inputs,
        even = element slots, odd = atomic row sums, with 1, 2 or 4 shots per thread."""
        self._check(self._L.hrn_set_variant(self.h, int(forward), int(adjoint)))

    def variant(self):
        f, a = C.c_int32(), C.c_int32()
        self._check(self._L.hrn_get_variant(self.h, C.byref(f), C.byref(a)))
        return f.value, a.value

    def time_stage(self, adjoint: bool = False, nsteps: int = 50) -> float:
        """Milliseconds of one stage launch of the tuned variant, from `nsteps` RK4
        steps launched back to back under one pair of CUDA events (no per-launch
        events).  The state buffers are scratch afterwards; the history stays."""
        ms = C.c_double()
        self._check(self._L.hrn_time_stage(self.h, int(bool(adjoint)), int(nsteps), C.byref(ms)))
        return ms.value

    def launch_count(self) -> int:
        n = C.c_int64()
        self._check(self._L.hrn_launch_count(self.h, C.byref(n)))
        return n.value

    # -- time loops ---------------------------------------------------------------
    def forward(self):
        self._check(self._L.hrn_forward(self.h))

    def history(self, shot: int = 0) -> np.ndarray:
        u = np.zeros((self.nstep + 1, self.nstore))
        self._check(self._L.hrn_get_history(self.h, shot, dptr(u)))
        return u

    def state(self, step: int, shot: int = 0):
        """(x1, x2, x3) [neq] of a shot at a checkpointed step (needs set_checkpointing)."""
        x = [np.zeros(self.neq) for _ in range(3)]
        self._check(self._L.hrn_get_state(self.h, int(step), int(shot), *[v.ctypes.data for v in x]))
        return tuple(x)

    def traces(self) -> np.ndarray:
        t = np.zeros((self.nshot, self.nrec3, self.nstep + 1))
        self._check(self._L.hrn_get_traces(self.h, dptr(t)))
        return t

    def _dis(self, dis_meas):
        d = f64(dis_meas)
        if d.ndim == 2:
            d = d[None]
        if d.shape != (self.nshot, self.nrec3, self.nstep + 1):
            raise ValueError("dis_meas must be [nshot, nrec3, nstep+1]")
        return d

    def misfit(self, dis_meas=None) -> float:
        """Misfit against dis_meas, or against the resident data when dis_meas is None."""
        out = C.c_double()
        if dis_meas is None:
            self._check(self._L.hrn_misfit(self.h, None, C.byref(out)))
        else:
            d = self._dis(dis_meas)
            self._check(self._L.hrn_misfit(self.h, dptr(d), C.byref(out)))
        return out.value

    def adjoint_gradient(self, dis_meas=None, lambda_2mu: bool = False, keep_p: bool = False, to_host: bool = True):
        """Raw gradient (g_lambda, g_mu) on the host, or None when to_host is False
        (then fetch it with gradient_device)."""
        d = None if dis_meas is None else self._dis(dis_meas)
        gl = np.zeros(self.nj) if to_host else None
        gm = np.zeros(self.nj) if to_host else None
        self._check(self._L.hrn_adjoint_gradient(self.h, dptr(d) if d is not None else None, int(lambda_2mu), int(keep_p),
                                                 dptr(gl) if to_host else None, dptr(gm) if to_host else None))
        return (gl, gm) if to_host else None

    def gradient_device(self, lam_ptr: int, mu_ptr: int):
        """Copy the accumulated gradient into device buffers (raw pointers, FP64 [nj])."""
        self._check(self._L.hrn_get_gradient_device(self.h, C.c_void_p(lam_ptr), C.c_void_p(mu_ptr)))

    def adjoint_history(self, shot: int = 0) -> np.ndarray:
        p = np.zeros((self.nstep + 1, self.nstore))
        self._check(self._L.hrn_get_adjoint_history(self.h, shot, dptr(p)))
        return p


# -- reference-named entry points ---------------------------------------------

def EXPLICIT_RK4_PETSC_PML_3D(AK, DIAG_M, AC, AG, B, U_Store_Numbers_Global, NSTEP, DT, time_table,
                              precision="fp64", solver: Solver | None = None):
    """Forward RK4 with the assembled (unscaled) operator; returns U_Store_Mapping
    as [NSTEP+1, NStore] (Fortran U_Store_Mapping(NStore, 0:NStep)).

    ``time_table`` [NSTEP+1, 3] holds TIME_FUNCTION at T, T+DT, T+DT/2.  Unlike
    the reference, the caller's matrices are not scaled in place.
    """
    s = solver or Solver(precision)
    s.set_operator_csr(AC, AK, AG, DIAG_M)
    s.set_history(U_Store_Numbers_Global)
    b = f64(B)
    nz = np.nonzero(b)[0]
    s.set_shots(NSTEP, DT, nz, b[nz][:, None], np.asarray(time_table)[None])
    s.forward()
    return s.history(0)


def Compute_Misfit(solver: Solver, Dis_meas) -> float:
    """Sum over shots of 0.5*DT*sum_n ||U_Store(EqDis_MAP, n) - Dis_meas(n, :)||^2."""
    return solver.misfit(Dis_meas)


def EXPLICIT_RK4_PETSC_PML_3D_Adjoint_Control_OtD(solver: Solver, Dis_meas, lambda_2mu=False):
    """Adjoint RK4 (OtD) with the zero-lag control accumulation fused in; returns the
    raw (g_lambda, g_mu) the reference assembles before its sign flip."""
    return solver.adjoint_gradient(Dis_meas, lambda_2mu=lambda_2mu)
