/*
 * hrn_oracle.h -- CPU FP64 restatement of HiReNSI's explicit 3D elastic
 * forward / adjoint / gradient path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path in
 * hirensi_b200: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.  The product path never links or calls it.
 *
 * Conventions (all arrays are plain C, row-major):
 *   xyz   [nj][3]      node coordinates
 *   inod  [nel][27]    0-based node ids, local order of SHAPE_3_27
 *   mtel  [nel]        1 = regular domain (RD), 2 = PML
 *   id    [nj][9]      0-based equation numbers, -1 = constrained
 *                      (columns: ux uy uz sxx syy szz sxy syz szx)
 *   Element matrices are returned as em[row][col] with row/col equal to the
 *   reference's 1-based Fortran indices minus one.
 */
#ifndef HRN_ORACLE_H
#define HRN_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nj, nel, neq;
    const double *xyz;
    const int *inod;
    const int *mtel;
    const int *id;
    const double *rho_el;      /* [nel] density per element (PMAT(MTYPE,3)) */
    double pml_param[6][4];    /* [alpha0, beta0, L, x0] for x+, x-, y+, y-, z+, z- */
} ora_mesh;

typedef struct ora_sys ora_sys;

/* A1 / A2: shape functions and the 3-point rule actually used (GLL). */
void ora_gll3(double x[3], double w[3]);
void ora_shape_3_27(double x1, double x2, double x3, double fn[27], double dfxi[27][3]);
/* A3 */
int  ora_pml_finder_3d(const double xg[3], const double pml_param[6][4], double out[19]);

/* A4 / A5 / A7 element matrices (return 0, or -1 on a non-positive Jacobian). */
int ora_element_k(const double xt[3][27], const double lam_e[27], const double mu_e[27], double ek[81][81]);
int ora_element_m(const double xt[3][27], double rho, const double pml_param[6][4], int flag, double em[81][81]);
int ora_element_en(const double xt[3][27], const double pml_param[6][4], int flag, double en[162][162]);
int ora_element_ea(const double xt[3][27], const double lam_e[27], const double mu_e[27],
                   const double pml_param[6][4], int flag, double ea[81][162]);
int ora_element_fs(const double xt[3][27], int nface, double efs[81]);
/* A12 / A14 element kernels */
int ora_element_g(const double xt[3][27], const double eu[81], const double ep[81],
                  double eg_mu[27], double eg_lam[27], int lambda_2mu);
int ora_element_r_mg(const double xt[3][27], double er[27][27], double emg[27]);
int ora_element_tv(const double xt[3][27], const double e_mu[27], const double e_lam[27],
                   double ereg_mu[27], double ereg_lam[27], double *cost_lam, double *cost_mu);

/* A6 / A5 / A7 assembly (ASSEM_REGULAR_DOMAIN, ASSEM_FORCE, ASSEM_PML). */
ora_sys *ora_assemble(const ora_mesh *m, const double *lam, const double *mu, const int *id_bc, int *err);
void     ora_sys_free(ora_sys *s);
int      ora_sys_nnz(const ora_sys *s, int which);   /* which: 0 = C, 1 = K, 2 = G */
void     ora_sys_csr(const ora_sys *s, int which, int *ia, int *ja, double *a);
void     ora_sys_vectors(const ora_sys *s, double *diag_m, double *b);

/* Operators built from caller CSR arrays (the reference's assembled Mats). */
ora_sys *ora_sys_from_csr(int neq,
                          const int *c_ia, const int *c_ja, const double *c_a,
                          const int *k_ia, const int *k_ja, const double *k_a,
                          const int *g_ia, const int *g_ja, const double *g_a,
                          const double *diag_m);

/* A9: forward RK4.  b[neq] unscaled force vector; ftab[nstep+1][3] holds
 * TIME_FUNCTION at T, T+dt, T+dt/2.  u_store[(nstep+1)][nstore]. */
int ora_forward(const ora_sys *s, const double *b, const double *ftab, int nstep, double dt,
                int nstore, const int *store_eq, double *u_store, int nthreads);
/* A11: adjoint RK4 (OtD).  dis_meas[nrec3][nstep+1] (Fortran Dis_meas(0:NStep,NNDH*3)).
 * p_store[(nstep+1)][nstore]; p_store[0] is left untouched. */
int ora_adjoint(const ora_sys *s, int nstep, double dt, int nstore, const int *store_eq,
                const double *u_store, int nrec3, const int *eqdis, const int *eqdis_map,
                const double *dis_meas, double *p_store, int nthreads);
/* A12: control (gradient) accumulation over steps 1..nstep-1, scale dt.
 * nthreads > 1 computes the element terms in parallel; the result is the same. */
int ora_control(const ora_mesh *m, int nstep, double dt, int nstore, const int *store_eq,
                const double *u_store, const double *p_store, double *g_lam, double *g_mu, int lambda_2mu,
                int nthreads);
/* A13 */
double ora_misfit(int nstep, double dt, int nrec3, const int *eqdis, const int *eqdis_map,
                  int nstore, const double *u_store, const double *dis_meas);
/* A14 helpers: TV regularization vectors and costs; lumped gradient mass. */
int ora_tv_reg(const ora_mesh *m, const double *lam, const double *mu,
               double *reg_lam, double *reg_mu, double *cost_lam, double *cost_mu);
int ora_rmg(const ora_mesh *m, double *mg);

/* A10 */
double ora_time_function(double t, int lcase, double fr);

/* Per-step operator application used by the dot-product tests:
 * y = (scaled forward operator) x  for one matrix (which 0..2), and the
 * transposed adjoint-scaled version. */
int ora_apply_scaled(const ora_sys *s, int which, int transpose_adjoint, const double *x, double *y);

#ifdef __cplusplus
}
#endif
#endif
