/*
 * hrn_oracle.c -- CPU FP64 restatement of HiReNSI's explicit 3D elastic
 * forward / adjoint / gradient arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker the CUDA path in hirensi_b200
 * is compared against.  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py may load it; the product never calls it.
 *
 * Each routine names the reference file:line (paths inside the HiReNSI
 * project, S4 = step_4_3D_Forward_and_Inverse) whose arithmetic it restates.
 * Evaluation order follows the Fortran expressions (left to right) so that
 * element matrices agree with the reference to the last bit wherever the
 * reference's own compiler does not reassociate.
 *
 * The reference cannot be compiled here (Fortran + PETSc 3.4 + MPI are absent)
 * and ships no golden vectors for this path, so parity of this restatement is
 * unpinned against the reference binary; it is pinned by the structural and
 * algebraic tests under tests/ instead.
 */
#include "hrn_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------- */
/* A2: S4/Source1.F90:29-31 -- GAUSS() with NINT = 3 returns the GLL rule.    */
void ora_gll3(double x[3], double w[3])
{
    x[0] = -1.0; x[1] = 0.0; x[2] = 1.0;
    w[0] = 0.33333333333333333333; w[1] = 1.33333333333333333333; w[2] = 0.33333333333333333333;
}

/* A1: S4/Shape_Functions.F90:124-274 (SHAPE_3_27). */
void ora_shape_3_27(double X1, double X2, double X3, double FN[27], double D[27][3])
{
#define F(i) FN[(i) - 1]
#define DF(i, j) D[(i) - 1][(j) - 1]
    F(1) = 0.125 * X1 * -X2 * -X3 * (1.0 + X1) * (1.0 - X2) * (1.0 - X3);
    F(2) = 0.125 * X1 * X2 * -X3 * (1.0 + X1) * (1.0 + X2) * (1.0 - X3);
    F(3) = 0.125 * -X1 * X2 * -X3 * (1.0 - X1) * (1.0 + X2) * (1.0 - X3);
    F(4) = 0.125 * -X1 * -X2 * -X3 * (1.0 - X1) * (1.0 - X2) * (1.0 - X3);
    F(5) = 0.125 * X1 * -X2 * X3 * (1.0 + X1) * (1.0 - X2) * (1.0 + X3);
    F(6) = 0.125 * X1 * X2 * X3 * (1.0 + X1) * (1.0 + X2) * (1.0 + X3);
    F(7) = 0.125 * -X1 * X2 * X3 * (1.0 - X1) * (1.0 + X2) * (1.0 + X3);
    F(8) = 0.125 * -X1 * -X2 * X3 * (1.0 - X1) * (1.0 - X2) * (1.0 + X3);

    F(9) = 0.25 * X1 * -X3 * (1.0 + X1) * (1.0 - X3) * (1.0 - X2 * X2);
    F(11) = 0.25 * -X1 * -X3 * (1.0 - X1) * (1.0 - X3) * (1.0 - X2 * X2);
    F(17) = 0.25 * X1 * X3 * (1.0 + X1) * (1.0 + X3) * (1.0 - X2 * X2);
    F(19) = 0.25 * -X1 * X3 * (1.0 - X1) * (1.0 + X3) * (1.0 - X2 * X2);

    F(10) = 0.25 * X2 * -X3 * (1.0 + X2) * (1.0 - X3) * (1.0 - X1 * X1);
    F(12) = 0.25 * -X2 * -X3 * (1.0 - X2) * (1.0 - X3) * (1.0 - X1 * X1);
    F(18) = 0.25 * X2 * X3 * (1.0 + X2) * (1.0 + X3) * (1.0 - X1 * X1);
    F(20) = 0.25 * -X2 * X3 * (1.0 - X2) * (1.0 + X3) * (1.0 - X1 * X1);

    F(13) = 0.25 * -X2 * X1 * (1.0 - X2) * (1.0 + X1) * (1.0 - X3 * X3);
    F(14) = 0.25 * X2 * X1 * (1.0 + X2) * (1.0 + X1) * (1.0 - X3 * X3);
    F(15) = 0.25 * X2 * -X1 * (1.0 + X2) * (1.0 - X1) * (1.0 - X3 * X3);
    F(16) = 0.25 * -X2 * -X1 * (1.0 - X2) * (1.0 - X1) * (1.0 - X3 * X3);

    F(21) = 0.50 * -X3 * (1.0 - X3) * (1.0 - X1 * X1) * (1.0 - X2 * X2);
    F(26) = 0.50 * X3 * (1.0 + X3) * (1.0 - X1 * X1) * (1.0 - X2 * X2);
    F(22) = 0.50 * X1 * (1.0 + X1) * (1.0 - X2 * X2) * (1.0 - X3 * X3);
    F(24) = 0.50 * -X1 * (1.0 - X1) * (1.0 - X2 * X2) * (1.0 - X3 * X3);
    F(23) = 0.50 * X2 * (1.0 + X2) * (1.0 - X1 * X1) * (1.0 - X3 * X3);
    F(25) = 0.50 * -X2 * (1.0 - X2) * (1.0 - X1 * X1) * (1.0 - X3 * X3);
    F(27) = (1.0 - X1 * X1) * (1.0 - X2 * X2) * (1.0 - X3 * X3);

    DF(1, 1) = 0.125 * -X2 * -X3 * (1.0 - X2) * (1.0 - X3) * (1.0 + 2.0 * X1);
    DF(2, 1) = 0.125 * X2 * -X3 * (1.0 + X2) * (1.0 - X3) * (1.0 + 2.0 * X1);
    DF(3, 1) = 0.125 * X2 * -X3 * (1.0 + X2) * (1.0 - X3) * (-1.0 + 2.0 * X1);
    DF(4, 1) = 0.125 * -X2 * -X3 * (1.0 - X2) * (1.0 - X3) * (-1.0 + 2.0 * X1);
    DF(5, 1) = 0.125 * -X2 * X3 * (1.0 - X2) * (1.0 + X3) * (1.0 + 2.0 * X1);
    DF(6, 1) = 0.125 * X2 * X3 * (1.0 + X2) * (1.0 + X3) * (1.0 + 2.0 * X1);
    DF(7, 1) = 0.125 * X2 * X3 * (1.0 + X2) * (1.0 + X3) * (-1.0 + 2.0 * X1);
    DF(8, 1) = 0.125 * -X2 * X3 * (1.0 - X2) * (1.0 + X3) * (-1.0 + 2.0 * X1);
    DF(9, 1) = 0.25 * -X3 * (1.0 - X3) * (1.0 - X2 * X2) * (1.0 + 2.0 * X1);
    DF(11, 1) = 0.25 * -X3 * (1.0 - X3) * (1.0 - X2 * X2) * (-1.0 + 2.0 * X1);
    DF(17, 1) = 0.25 * X3 * (1.0 + X3) * (1.0 - X2 * X2) * (1.0 + 2.0 * X1);
    DF(19, 1) = 0.25 * X3 * (1.0 + X3) * (1.0 - X2 * X2) * (-1.0 + 2.0 * X1);
    DF(10, 1) = 0.50 * X2 * -X3 * (1.0 + X2) * (1.0 - X3) * (-X1);
    DF(12, 1) = 0.50 * -X2 * -X3 * (1.0 - X2) * (1.0 - X3) * (-X1);
    DF(18, 1) = 0.50 * X2 * X3 * (1.0 + X2) * (1.0 + X3) * (-X1);
    DF(20, 1) = 0.50 * -X2 * X3 * (1.0 - X2) * (1.0 + X3) * (-X1);
    DF(13, 1) = 0.25 * -X2 * (1.0 - X2) * (1.0 - X3 * X3) * (1.0 + 2.0 * X1);
    DF(14, 1) = 0.25 * X2 * (1.0 + X2) * (1.0 - X3 * X3) * (1.0 + 2.0 * X1);
    DF(15, 1) = 0.25 * X2 * (1.0 + X2) * (1.0 - X3 * X3) * (-1.0 + 2.0 * X1);
    DF(16, 1) = 0.25 * -X2 * (1.0 - X2) * (1.0 - X3 * X3) * (-1.0 + 2.0 * X1);
    DF(21, 1) = -X3 * (1.0 - X3) * (-X1) * (1.0 - X2 * X2);
    DF(26, 1) = X3 * (1.0 + X3) * (-X1) * (1.0 - X2 * X2);
    DF(22, 1) = 0.50 * (1.0 - X2 * X2) * (1.0 - X3 * X3) * (1.0 + 2.0 * X1);
    DF(24, 1) = 0.50 * (1.0 - X2 * X2) * (1.0 - X3 * X3) * (-1.0 + 2.0 * X1);
    DF(23, 1) = X2 * (1.0 + X2) * (-X1) * (1.0 - X3 * X3);
    DF(25, 1) = -X2 * (1.0 - X2) * (-X1) * (1.0 - X3 * X3);
    DF(27, 1) = (-2.0 * X1) * (1.0 - X2 * X2) * (1.0 - X3 * X3);

    DF(1, 2) = 0.125 * X1 * -X3 * (1.0 + X1) * (-1.0 + 2.0 * X2) * (1.0 - X3);
    DF(2, 2) = 0.125 * X1 * -X3 * (1.0 + X1) * (+1.0 + 2.0 * X2) * (1.0 - X3);
    DF(3, 2) = 0.125 * -X1 * -X3 * (1.0 - X1) * (+1.0 + 2.0 * X2) * (1.0 - X3);
    DF(4, 2) = 0.125 * -X1 * -X3 * (1.0 - X1) * (-1.0 + 2.0 * X2) * (1.0 - X3);
    DF(5, 2) = 0.125 * X1 * X3 * (1.0 + X1) * (-1.0 + 2.0 * X2) * (1.0 + X3);
    DF(6, 2) = 0.125 * X1 * X3 * (1.0 + X1) * (+1.0 + 2.0 * X2) * (1.0 + X3);
    DF(7, 2) = 0.125 * -X1 * X3 * (1.0 - X1) * (+1.0 + 2.0 * X2) * (1.0 + X3);
    DF(8, 2) = 0.125 * -X1 * X3 * (1.0 - X1) * (-1.0 + 2.0 * X2) * (1.0 + X3);
    DF(9, 2) = 0.50 * X1 * -X3 * (1.0 + X1) * (1.0 - X3) * (-X2);
    DF(11, 2) = 0.50 * -X1 * -X3 * (1.0 - X1) * (1.0 - X3) * (-X2);
    DF(17, 2) = 0.50 * X1 * X3 * (1.0 + X1) * (1.0 + X3) * (-X2);
    DF(19, 2) = 0.50 * -X1 * X3 * (1.0 - X1) * (1.0 + X3) * (-X2);
    DF(10, 2) = 0.25 * -X3 * (+1.0 + 2.0 * X2) * (1.0 - X3) * (1.0 - X1 * X1);
    DF(12, 2) = 0.25 * -X3 * (-1.0 + 2.0 * X2) * (1.0 - X3) * (1.0 - X1 * X1);
    DF(18, 2) = 0.25 * X3 * (+1.0 + 2.0 * X2) * (1.0 + X3) * (1.0 - X1 * X1);
    DF(20, 2) = 0.25 * X3 * (-1.0 + 2.0 * X2) * (1.0 + X3) * (1.0 - X1 * X1);
    DF(13, 2) = 0.25 * X1 * (-1.0 + 2.0 * X2) * (1.0 + X1) * (1.0 - X3 * X3);
    DF(14, 2) = 0.25 * X1 * (+1.0 + 2.0 * X2) * (1.0 + X1) * (1.0 - X3 * X3);
    DF(15, 2) = 0.25 * -X1 * (+1.0 + 2.0 * X2) * (1.0 - X1) * (1.0 - X3 * X3);
    DF(16, 2) = 0.25 * -X1 * (-1.0 + 2.0 * X2) * (1.0 - X1) * (1.0 - X3 * X3);
    DF(21, 2) = -X3 * (1.0 - X3) * (1.0 - X1 * X1) * (-X2);
    DF(26, 2) = X3 * (1.0 + X3) * (1.0 - X1 * X1) * (-X2);
    DF(22, 2) = X1 * (1.0 + X1) * (-X2) * (1.0 - X3 * X3);
    DF(24, 2) = -X1 * (1.0 - X1) * (-X2) * (1.0 - X3 * X3);
    DF(23, 2) = 0.50 * (+1.0 + 2.0 * X2) * (1.0 - X1 * X1) * (1.0 - X3 * X3);
    DF(25, 2) = 0.50 * (-1.0 + 2.0 * X2) * (1.0 - X1 * X1) * (1.0 - X3 * X3);
    DF(27, 2) = (1.0 - X1 * X1) * (-2.0 * X2) * (1.0 - X3 * X3);

    DF(1, 3) = 0.125 * X1 * -X2 * (1.0 + X1) * (1.0 - X2) * (-1.0 + 2.0 * X3);
    DF(2, 3) = 0.125 * X1 * X2 * (1.0 + X1) * (1.0 + X2) * (-1.0 + 2.0 * X3);
    DF(3, 3) = 0.125 * -X1 * X2 * (1.0 - X1) * (1.0 + X2) * (-1.0 + 2.0 * X3);
    DF(4, 3) = 0.125 * -X1 * -X2 * (1.0 - X1) * (1.0 - X2) * (-1.0 + 2.0 * X3);
    DF(5, 3) = 0.125 * X1 * -X2 * (1.0 + X1) * (1.0 - X2) * (+1.0 + 2.0 * X3);
    DF(6, 3) = 0.125 * X1 * X2 * (1.0 + X1) * (1.0 + X2) * (+1.0 + 2.0 * X3);
    DF(7, 3) = 0.125 * -X1 * X2 * (1.0 - X1) * (1.0 + X2) * (+1.0 + 2.0 * X3);
    DF(8, 3) = 0.125 * -X1 * -X2 * (1.0 - X1) * (1.0 - X2) * (+1.0 + 2.0 * X3);
    DF(9, 3) = 0.25 * X1 * (1.0 + X1) * (-1.0 + 2.0 * X3) * (1.0 - X2 * X2);
    DF(11, 3) = 0.25 * -X1 * (1.0 - X1) * (-1.0 + 2.0 * X3) * (1.0 - X2 * X2);
    DF(17, 3) = 0.25 * X1 * (1.0 + X1) * (+1.0 + 2.0 * X3) * (1.0 - X2 * X2);
    DF(19, 3) = 0.25 * -X1 * (1.0 - X1) * (+1.0 + 2.0 * X3) * (1.0 - X2 * X2);
    DF(10, 3) = 0.25 * X2 * (1.0 + X2) * (-1.0 + 2.0 * X3) * (1.0 - X1 * X1);
    DF(12, 3) = 0.25 * -X2 * (1.0 - X2) * (-1.0 + 2.0 * X3) * (1.0 - X1 * X1);
    DF(18, 3) = 0.25 * X2 * (1.0 + X2) * (+1.0 + 2.0 * X3) * (1.0 - X1 * X1);
    DF(20, 3) = 0.25 * -X2 * (1.0 - X2) * (+1.0 + 2.0 * X3) * (1.0 - X1 * X1);
    DF(13, 3) = 0.50 * -X2 * X1 * (1.0 - X2) * (1.0 + X1) * (-X3);
    DF(14, 3) = 0.50 * X2 * X1 * (1.0 + X2) * (1.0 + X1) * (-X3);
    DF(15, 3) = 0.50 * X2 * -X1 * (1.0 + X2) * (1.0 - X1) * (-X3);
    DF(16, 3) = 0.50 * -X2 * -X1 * (1.0 - X2) * (1.0 - X1) * (-X3);
    DF(21, 3) = 0.50 * (-1.0 + 2.0 * X3) * (1.0 - X1 * X1) * (1.0 - X2 * X2);
    DF(26, 3) = 0.50 * (+1.0 + 2.0 * X3) * (1.0 - X1 * X1) * (1.0 - X2 * X2);
    DF(22, 3) = X1 * (1.0 + X1) * (1.0 - X2 * X2) * (-X3);
    DF(24, 3) = -X1 * (1.0 - X1) * (1.0 - X2 * X2) * (-X3);
    DF(23, 3) = X2 * (1.0 + X2) * (1.0 - X1 * X1) * (-X3);
    DF(25, 3) = -X2 * (1.0 - X2) * (1.0 - X1 * X1) * (-X3);
    DF(27, 3) = (1.0 - X1 * X1) * (1.0 - X2 * X2) * (-2.0 * X3);
#undef F
#undef DF
}

/* A3: S4/PML.F90:325-891 (PML_FINDER_3D), polynomial degree 2, ratio 0.
 * pml_param rows: x+, x-, y+, y-, z+, z-; columns: alpha0, beta0, L, x0.
 * Returns -1 when the point lies in the (forbidden) top zone (:615-616). */
int ora_pml_finder_3d(const double XG[3], const double P[6][4], double A[19])
{
    const double deg = 2.0, ratio = 0.0;
    double d_dy_ax = 0, d_dz_ax = 0, d_dx_ay = 0, d_dz_ay = 0, d_dx_az = 0, d_dy_az = 0;
    double d_dy_bx = 0, d_dz_bx = 0, d_dx_by = 0, d_dz_by = 0, d_dx_bz = 0, d_dy_bz = 0;
    for (int i = 0; i < 19; ++i) A[i] = 0.0;
    A[0] = 1.0; A[1] = 1.0; A[2] = 1.0;

    /* x direction (:441-518) */
    int zx = 0;
    if (XG[0] >= P[0][3]) zx = 1; else if (XG[0] <= P[1][3]) zx = 2;
    if (zx) {
        int r = zx - 1;
        double diff = XG[0] - P[r][3], vn = (zx == 1) ? 1.0 : -1.0;
        double a0 = P[r][0], b0 = P[r][1], L = P[r][2];
        double f1 = diff * vn / L, f4 = vn / L;
        double pa = f1 * f1, pd = f1;   /* deg = 2: x**2.0 is evaluated as x*x */
        A[0] = A[0] + a0 * pa;
        A[3] = A[3] + b0 * pa;
        A[1] = A[1] + (a0 * pa) * ratio;
        A[2] = A[2] + (a0 * pa) * ratio;
        A[4] = A[4] + (b0 * pa) * ratio;
        A[5] = A[5] + (b0 * pa) * ratio;
        d_dx_ay = (a0 * deg * f4 * pd) * ratio;
        d_dx_az = (a0 * deg * f4 * pd) * ratio;
        d_dx_by = (b0 * deg * f4 * pd) * ratio;
        d_dx_bz = (b0 * deg * f4 * pd) * ratio;
    }
    /* y direction (:523-601) */
    int zy = 0;
    if (XG[1] >= P[2][3]) zy = 1; else if (XG[1] <= P[3][3]) zy = 2;
    if (zy) {
        int r = 2 + zy - 1;
        double diff = XG[1] - P[r][3], vn = (zy == 1) ? 1.0 : -1.0;
        double a0 = P[r][0], b0 = P[r][1], L = P[r][2];
        double f2 = diff * vn / L, f5 = vn / L;
        double pa = f2 * f2, pd = f2;
        A[1] = A[1] + a0 * pa;
        A[4] = A[4] + b0 * pa;
        A[0] = A[0] + (a0 * pa) * ratio;
        A[2] = A[2] + (a0 * pa) * ratio;
        A[3] = A[3] + (b0 * pa) * ratio;
        A[5] = A[5] + (b0 * pa) * ratio;
        d_dy_ax = (a0 * deg * f5 * pd) * ratio;
        d_dy_az = (a0 * deg * f5 * pd) * ratio;
        d_dy_bx = (b0 * deg * f5 * pd) * ratio;
        d_dy_bz = (b0 * deg * f5 * pd) * ratio;
    }
    /* z direction (:606-655); the top zone stops the reference */
    if (XG[2] > P[4][3]) return -1;
    if (XG[2] <= P[5][3]) {
        double diff = XG[2] - P[5][3], vn = -1.0;
        double a0 = P[5][0], b0 = P[5][1], L = P[5][2];
        double f3 = diff * vn / L, f6 = vn / L;
        double pa = f3 * f3, pd = f3;
        A[2] = A[2] + a0 * pa;
        A[5] = A[5] + b0 * pa;
        A[0] = A[0] + (a0 * pa) * ratio;
        A[1] = A[1] + (a0 * pa) * ratio;
        A[3] = A[3] + (b0 * pa) * ratio;
        A[4] = A[4] + (b0 * pa) * ratio;
        d_dz_ax = (a0 * deg * f6 * pd) * ratio;
        d_dz_ay = (a0 * deg * f6 * pd) * ratio;
        d_dz_bx = (b0 * deg * f6 * pd) * ratio;
        d_dz_by = (b0 * deg * f6 * pd) * ratio;
    }
    /* :827-866 */
    A[6] = A[0] * A[1] * A[2];
    A[7] = A[0] * A[1] * A[5] + A[0] * A[2] * A[4] + A[1] * A[2] * A[3];
    A[8] = A[0] * A[4] * A[5] + A[1] * A[3] * A[5] + A[2] * A[3] * A[4];
    A[9] = A[3] * A[4] * A[5];
    A[10] = d_dz_ax * A[1] + d_dz_ay * A[0];
    A[11] = d_dy_ax * A[2] + d_dy_az * A[0];
    A[12] = d_dx_ay * A[2] + d_dx_az * A[1];
    A[13] = d_dz_ax * A[4] + A[0] * d_dz_by + d_dz_ay * A[3] + A[1] * d_dz_bx;
    A[14] = d_dy_ax * A[5] + A[0] * d_dy_bz + d_dy_az * A[3] + A[2] * d_dy_bx;
    A[15] = d_dx_ay * A[5] + A[1] * d_dx_bz + d_dx_az * A[4] + A[2] * d_dx_by;
    A[16] = d_dz_bx * A[4] + d_dz_by * A[3];
    A[17] = d_dy_bx * A[5] + d_dy_bz * A[3];
    A[18] = d_dx_by * A[5] + d_dx_bz * A[4];
    return 0;
}

/* Jacobian block shared by every element routine, e.g.
 * S4/Element_Matrices_3D.F90:111-139. */
static int geom(const double xt[3][27], double x1, double x2, double x3, double fn[27],
                double dfxi[27][3], double *detj_out, double dfx[27][3], int want_dfx)
{
    double dj[3][3], dji[3][3];
    ora_shape_3_27(x1, x2, x3, fn, dfxi);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 27; ++k) s += xt[i][k] * dfxi[k][j];
            dj[i][j] = s;
        }
    double detj = dj[0][0] * dj[1][1] * dj[2][2] + dj[1][0] * dj[2][1] * dj[0][2] + dj[2][0] * dj[0][1] * dj[1][2]
                - dj[0][2] * dj[1][1] * dj[2][0] - dj[1][2] * dj[2][1] * dj[0][0] - dj[2][2] * dj[0][1] * dj[1][0];
    if (!(detj > 0.0)) return -1;
    *detj_out = detj;
    if (!want_dfx) return 0;
    dji[0][0] = dj[2][2] * dj[1][1] - dj[2][1] * dj[1][2];
    dji[0][1] = -(dj[2][2] * dj[0][1]) + dj[2][1] * dj[0][2];
    dji[0][2] = dj[1][2] * dj[0][1] - dj[1][1] * dj[0][2];
    dji[1][0] = -(dj[2][2] * dj[1][0]) + dj[2][0] * dj[1][2];
    dji[1][1] = dj[2][2] * dj[0][0] - dj[2][0] * dj[0][2];
    dji[1][2] = -(dj[1][2] * dj[0][0]) + dj[1][0] * dj[0][2];
    dji[2][0] = dj[2][1] * dj[1][0] - dj[2][0] * dj[1][1];
    dji[2][1] = -(dj[2][1] * dj[0][0]) + dj[2][0] * dj[0][1];
    dji[2][2] = dj[1][1] * dj[0][0] - dj[1][0] * dj[0][1];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) dji[i][j] = dji[i][j] / detj;
    for (int a = 0; a < 27; ++a)
        for (int k = 0; k < 3; ++k) {
            double s = 0.0;
            for (int m = 0; m < 3; ++m) s += dfxi[a][m] * dji[m][k];
            dfx[a][k] = s;
        }
    return 0;
}

static double dot27(const double *a, const double *b)
{
    double s = 0.0;
    for (int i = 0; i < 27; ++i) s += a[i] * b[i];
    return s;
}

/* A4: S4/Element_Matrices_3D.F90:7-220 (ELEMENT_K_3D). */
int ora_element_k(const double xt[3][27], const double lam_e[27], const double mu_e[27], double ek[81][81])
{
    double xg[3], wg[3], fn[27], dfxi[27][3], dfx[27][3], detj;
    ora_gll3(xg, wg);
    memset(ek, 0, sizeof(double) * 81 * 81);
    for (int lz = 0; lz < 3; ++lz)
        for (int ly = 0; ly < 3; ++ly)
            for (int lx = 0; lx < 3; ++lx) {
                double wstar = wg[lx] * wg[ly] * wg[lz];
                if (geom(xt, xg[lx], xg[ly], xg[lz], fn, dfxi, &detj, dfx, 1)) return -1;
                double fac0 = wstar * detj;
                double zl = dot27(fn, lam_e), zm = dot27(fn, mu_e);
                double f1 = zl + 2.0 * zm, f2 = zl, f3 = zm;
                for (int i = 0; i < 27; ++i)
                    for (int j = 0; j < 27; ++j) {
                        double h1 = dfx[i][0] * dfx[j][0], h2 = dfx[i][1] * dfx[j][1], h3 = dfx[i][2] * dfx[j][2];
                        double h4 = dfx[i][0] * dfx[j][1], h5 = dfx[i][1] * dfx[j][0];
                        double h6 = dfx[i][0] * dfx[j][2], h7 = dfx[i][2] * dfx[j][0];
                        double h8 = dfx[i][1] * dfx[j][2], h9 = dfx[i][2] * dfx[j][1];
                        double g1 = f1 * h1 + f3 * (h2 + h3), g2 = f2 * h4 + f3 * h5, g3 = f2 * h6 + f3 * h7;
                        double g4 = f2 * h5 + f3 * h4, g5 = f1 * h2 + f3 * (h1 + h3), g6 = f2 * h8 + f3 * h9;
                        double g7 = f2 * h7 + f3 * h6, g8 = f2 * h9 + f3 * h8, g9 = f1 * h3 + f3 * (h1 + h2);
                        ek[i][j] += g1 * fac0;           ek[i][j + 27] += g2 * fac0;      ek[i][j + 54] += g3 * fac0;
                        ek[i + 27][j] += g4 * fac0;      ek[i + 27][j + 27] += g5 * fac0; ek[i + 27][j + 54] += g6 * fac0;
                        ek[i + 54][j] += g7 * fac0;      ek[i + 54][j + 27] += g8 * fac0; ek[i + 54][j + 54] += g9 * fac0;
                    }
            }
    return 0;
}

/* A5: S4/Element_Matrices_3D.F90:228-415 (ELEMENT_M_3D), flags 201..205. */
int ora_element_m(const double xt[3][27], double rho, const double P[6][4], int flag, double em[81][81])
{
    double xg[3], wg[3], fn[27], dfxi[27][3], detj, ab[19];
    ora_gll3(xg, wg);
    memset(em, 0, sizeof(double) * 81 * 81);
    if (flag < 201 || flag > 205) return -2;
    for (int lz = 0; lz < 3; ++lz)
        for (int ly = 0; ly < 3; ++ly)
            for (int lx = 0; lx < 3; ++lx) {
                double wstar = wg[lx] * wg[ly] * wg[lz];
                if (geom(xt, xg[lx], xg[ly], xg[lz], fn, dfxi, &detj, NULL, 0)) return -1;
                double fac0 = wstar * detj, fac1 = rho;
                if (flag != 201) {
                    double x[3];
                    for (int d = 0; d < 3; ++d) x[d] = dot27(xt[d], fn);
                    if (ora_pml_finder_3d(x, P, ab)) return -3;
                    fac1 = rho * ab[6 + (flag - 202)];
                }
                for (int i = 0; i < 27; ++i)
                    for (int j = 0; j < 27; ++j) {
                        double g1 = fac1 * (fn[i] * fn[j]);
                        em[i][j] += g1 * fac0;
                        em[i + 27][j + 27] += g1 * fac0;
                        em[i + 54][j + 54] += g1 * fac0;
                    }
            }
    return 0;
}

/* A5: S4/Element_Matrices_3D.F90:423-603 (ELEMENT_EN_3D), flags 301..304. */
int ora_element_en(const double xt[3][27], const double P[6][4], int flag, double en[162][162])
{
    double xg[3], wg[3], fn[27], dfxi[27][3], detj, ab[19];
    ora_gll3(xg, wg);
    memset(en, 0, sizeof(double) * 162 * 162);
    if (flag < 301 || flag > 304) return -2;
    const double fac1 = 2.0;
    for (int lz = 0; lz < 3; ++lz)
        for (int ly = 0; ly < 3; ++ly)
            for (int lx = 0; lx < 3; ++lx) {
                double wstar = wg[lx] * wg[ly] * wg[lz];
                if (geom(xt, xg[lx], xg[ly], xg[lz], fn, dfxi, &detj, NULL, 0)) return -1;
                double fac0 = wstar * detj, x[3];
                for (int d = 0; d < 3; ++d) x[d] = dot27(xt[d], fn);
                if (ora_pml_finder_3d(x, P, ab)) return -3;
                double fac2 = ab[6 + (flag - 301)];
                for (int i = 0; i < 27; ++i)
                    for (int j = 0; j < 27; ++j) {
                        double h1 = fn[i] * fn[j];
                        double g1 = fac2 * h1, g2 = fac1 * fac2 * h1;
                        for (int c = 0; c < 3; ++c) en[i + 27 * c][j + 27 * c] += g1 * fac0;
                        for (int c = 3; c < 6; ++c) en[i + 27 * c][j + 27 * c] += g2 * fac0;
                    }
            }
    return 0;
}

/* A5: S4/Element_Matrices_3D.F90:618-882 (ELEMENT_EA_3D), flags 101..106. */
int ora_element_ea(const double xt[3][27], const double lam_e[27], const double mu_e[27],
                   const double P[6][4], int flag, double ea[81][162])
{
    double xg[3], wg[3], fn[27], dfxi[27][3], dfx[27][3], detj, ab[19];
    ora_gll3(xg, wg);
    memset(ea, 0, sizeof(double) * 81 * 162);
    if (flag < 101 || flag > 106) return -2;
    int upper = flag <= 103;
    int kind = (flag - 101) % 3; /* 0 = e, 1 = p, 2 = w */
    double f7 = 1.0, f8 = 0.0, f9 = 1.0, f10 = 1.0;
    if (!upper) f10 = 0.0;
    for (int lz = 0; lz < 3; ++lz)
        for (int ly = 0; ly < 3; ++ly)
            for (int lx = 0; lx < 3; ++lx) {
                double wstar = wg[lx] * wg[ly] * wg[lz];
                if (geom(xt, xg[lx], xg[ly], xg[lz], fn, dfxi, &detj, dfx, 1)) return -1;
                double fac0 = wstar * detj;
                double zl = dot27(fn, lam_e), zm = dot27(fn, mu_e);
                if (!upper) { f7 = zl + 2.0 * zm; f8 = zl; f9 = 2.0 * zm; }
                double x[3];
                for (int d = 0; d < 3; ++d) x[d] = dot27(xt[d], fn);
                if (ora_pml_finder_3d(x, P, ab)) return -3;
                double f1, f2, f3, f4, f5, f6;
                if (kind == 0) {
                    f1 = ab[0] * ab[1]; f2 = ab[0] * ab[2]; f3 = ab[1] * ab[2];
                    f4 = ab[10]; f5 = ab[11]; f6 = ab[12];
                } else if (kind == 1) {
                    f1 = ab[0] * ab[4] + ab[1] * ab[3]; f2 = ab[0] * ab[5] + ab[2] * ab[3]; f3 = ab[1] * ab[5] + ab[2] * ab[4];
                    f4 = ab[13]; f5 = ab[14]; f6 = ab[15];
                } else {
                    f1 = ab[3] * ab[4]; f2 = ab[3] * ab[5]; f3 = ab[4] * ab[5];
                    f4 = ab[16]; f5 = ab[17]; f6 = ab[18];
                }
                for (int i = 0; i < 27; ++i)
                    for (int j = 0; j < 27; ++j) {
                        double h1 = dfx[i][0] * fn[j], h2 = dfx[i][1] * fn[j], h3 = dfx[i][2] * fn[j], h4 = fn[i] * fn[j];
                        double g1 = f7 * f3 * h1 + f10 * f6 * h4;
                        double g2 = f8 * f3 * h1;
                        double g3 = f9 * f2 * h2 + f10 * f5 * h4;
                        double g4 = f9 * f1 * h3 + f10 * f4 * h4;
                        double g5 = f8 * f2 * h2;
                        double g6 = f7 * f2 * h2 + f10 * f5 * h4;
                        double g7 = f9 * f3 * h1 + f10 * f6 * h4;
                        double g8 = f8 * f1 * h3;
                        double g9 = f7 * f1 * h3 + f10 * f4 * h4;
                        int i1 = i, i2 = i + 27, i3 = i + 54;
                        int j1 = j, j2 = j + 27, j3 = j + 54, j4 = j + 81, j5 = j + 108, j6 = j + 135;
                        ea[i1][j1] += g1 * fac0; ea[i1][j2] += g2 * fac0; ea[i1][j3] += g2 * fac0;
                        ea[i1][j4] += g3 * fac0; ea[i1][j5] += g4 * fac0;
                        ea[i2][j1] += g5 * fac0; ea[i2][j2] += g6 * fac0; ea[i2][j3] += g5 * fac0;
                        ea[i2][j4] += g7 * fac0; ea[i2][j6] += g4 * fac0;
                        ea[i3][j1] += g8 * fac0; ea[i3][j2] += g8 * fac0; ea[i3][j3] += g9 * fac0;
                        ea[i3][j5] += g7 * fac0; ea[i3][j6] += g3 * fac0;
                    }
            }
    return 0;
}

/* A7: S4/Element_Matrices_3D.F90:890-1096 (ELEMENT_FS_3D); unit Tz traction.
 * Returns -4 when the loaded face is not on the surface z = 0 (:1052-1057). */
int ora_element_fs(const double xt[3][27], int nface, double efs[81])
{
    static const int LFACE[6] = {2, 2, 3, 3, 1, 1};
    static const double FVAL[6] = {1.0, -1.0, 1.0, -1.0, 1.0, -1.0};
    static const int IPERM[3] = {2, 3, 1};
    double xg[3], wg[3], fn[27], dfxi[27][3], xi[3] = {0, 0, 0};
    ora_gll3(xg, wg);
    memset(efs, 0, sizeof(double) * 81);
    if (nface == 0) return 0;
    if (nface == 6) nface = 5;
    int L = LFACE[nface - 1], M = IPERM[L - 1], N = IPERM[M - 1];
    xi[N - 1] = FVAL[nface - 1];
    for (int lj = 0; lj < 3; ++lj) {
        xi[M - 1] = xg[lj];
        double wj = wg[lj];
        for (int li = 0; li < 3; ++li) {
            xi[L - 1] = xg[li];
            double wi = wg[li];
            double wstar = wi * wj;
            ora_shape_3_27(xi[0], xi[1], xi[2], fn, dfxi);
            double dj[3][3];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    double s = 0.0;
                    for (int k = 0; k < 27; ++k) s += xt[i][k] * dfxi[k][j];
                    dj[i][j] = s;
                }
            double vr[3], vs[3], vn[3];
            for (int i = 0; i < 3; ++i) { vr[i] = dj[i][L - 1]; vs[i] = dj[i][M - 1]; }
            vn[0] = +vr[1] * vs[2] - vr[2] * vs[1];
            vn[1] = -(vr[0] * vs[2]) + vr[2] * vs[0];
            vn[2] = +vr[0] * vs[1] - vr[1] * vs[0];
            double nrm = 0.0;
            for (int i = 0; i < 3; ++i) nrm = nrm + vn[i] * vn[i];
            nrm = sqrt(nrm);
            double fac0 = wstar * nrm;
            double zc = dot27(xt[2], fn);
            if (fabs(zc) > 1.e-3) return -4;
            for (int i = 0; i < 27; ++i) {
                double h1 = fn[i];
                efs[i] += (0.0 * h1) * fac0;
                efs[i + 27] += (0.0 * h1) * fac0;
                efs[i + 54] += (1.0 * h1) * fac0;
            }
        }
    }
    return 0;
}

/* A12: S4/Element_Matrices_3D.F90:1725-1890 (ELEMENT_g_3D) and :2081-2246 (_v2). */
int ora_element_g(const double xt[3][27], const double eu[81], const double ep[81],
                  double eg_mu[27], double eg_lam[27], int lambda_2mu)
{
    double xg[3], wg[3], fn[27], dfxi[27][3], dfx[27][3], detj;
    double col[3][27];
    ora_gll3(xg, wg);
    for (int i = 0; i < 27; ++i) { eg_mu[i] = 0.0; eg_lam[i] = 0.0; }
    for (int lz = 0; lz < 3; ++lz)
        for (int ly = 0; ly < 3; ++ly)
            for (int lx = 0; lx < 3; ++lx) {
                double wstar = wg[lx] * wg[ly] * wg[lz];
                if (geom(xt, xg[lx], xg[ly], xg[lz], fn, dfxi, &detj, dfx, 1)) return -1;
                double fac0 = wstar * detj;
                for (int k = 0; k < 3; ++k)
                    for (int a = 0; a < 27; ++a) col[k][a] = dfx[a][k];
                double u1x = dot27(eu, col[0]), u2x = dot27(eu + 27, col[0]), u3x = dot27(eu + 54, col[0]);
                double u1y = dot27(eu, col[1]), u2y = dot27(eu + 27, col[1]), u3y = dot27(eu + 54, col[1]);
                double u1z = dot27(eu, col[2]), u2z = dot27(eu + 27, col[2]), u3z = dot27(eu + 54, col[2]);
                double p1x = dot27(ep, col[0]), p2x = dot27(ep + 27, col[0]), p3x = dot27(ep + 54, col[0]);
                double p1y = dot27(ep, col[1]), p2y = dot27(ep + 27, col[1]), p3y = dot27(ep + 54, col[1]);
                double p1z = dot27(ep, col[2]), p2z = dot27(ep + 27, col[2]), p3z = dot27(ep + 54, col[2]);
                double sl = (u1x + u2y + u3z) * (p1x + p2y + p3z);
                double sm;
                if (!lambda_2mu)
                    sm = 2.0 * (u1x * p1x + u2y * p2y + u3z * p3z) + (p1y + p2x) * (u1y + u2x)
                       + (p1z + p3x) * (u1z + u3x) + (p3y + p2z) * (u3y + u2z);
                else
                    sm = -2.0 * (p1x * (u2y + u3z) + p2y * (u1x + u3z) + p3z * (u1x + u2y)) + (p1y + p2x) * (u1y + u2x)
                       + (p1z + p3x) * (u1z + u3x) + (p3y + p2z) * (u3y + u2z);
                for (int i = 0; i < 27; ++i) {
                    eg_mu[i] = eg_mu[i] + fn[i] * sm * fac0;
                    eg_lam[i] = eg_lam[i] + fn[i] * sl * fac0;
                }
            }
    return 0;
}

/* A14: S4/Element_Matrices_3D.F90:1555-1717 (ELEMENT_R_Mg_3D), unweighted. */
int ora_element_r_mg(const double xt[3][27], double er[27][27], double emg[27])
{
    double xg[3], wg[3], fn[27], dfxi[27][3], dfx[27][3], detj;
    double mg[27][27];
    ora_gll3(xg, wg);
    memset(er, 0, sizeof(double) * 27 * 27);
    memset(mg, 0, sizeof(mg));
    for (int lz = 0; lz < 3; ++lz)
        for (int ly = 0; ly < 3; ++ly)
            for (int lx = 0; lx < 3; ++lx) {
                double wstar = wg[lx] * wg[ly] * wg[lz];
                if (geom(xt, xg[lx], xg[ly], xg[lz], fn, dfxi, &detj, dfx, 1)) return -1;
                double fac0 = wstar * detj, fac1 = 1.0;
                for (int i = 0; i < 27; ++i)
                    for (int j = 0; j < 27; ++j) {
                        double h1 = dfx[i][0] * dfx[j][0], h2 = dfx[i][1] * dfx[j][1], h3 = dfx[i][2] * dfx[j][2];
                        er[i][j] = er[i][j] + (h1 + h2 + h3) * fac0 * fac1;
                        mg[i][j] = mg[i][j] + (fn[i] * fn[j]) * fac0;
                    }
            }
    for (int i = 0; i < 27; ++i) emg[i] = mg[i][i];
    return 0;
}

/* A14: S4/Element_Matrices_3D.F90:1899-2074 (ELEMENT_TV_TN_Reg_3D), TV, unweighted. */
int ora_element_tv(const double xt[3][27], const double e_mu[27], const double e_lam[27],
                   double ereg_mu[27], double ereg_lam[27], double *cost_lam, double *cost_mu)
{
    const double eps_tv = 0.01;
    double xg[3], wg[3], fn[27], dfxi[27][3], dfx[27][3], detj, er[27][27], vh[27];
    ora_gll3(xg, wg);
    for (int i = 0; i < 27; ++i) { ereg_mu[i] = 0.0; ereg_lam[i] = 0.0; }
    double cm = 0.0, cl = 0.0;
    for (int lz = 0; lz < 3; ++lz)
        for (int ly = 0; ly < 3; ++ly)
            for (int lx = 0; lx < 3; ++lx) {
                double wstar = wg[lx] * wg[ly] * wg[lz];
                if (geom(xt, xg[lx], xg[ly], xg[lz], fn, dfxi, &detj, dfx, 1)) return -1;
                double fac0 = wstar * detj, fac1 = 1.0;
                for (int i = 0; i < 27; ++i)
                    for (int j = 0; j < 27; ++j)
                        er[i][j] = dfx[i][0] * dfx[j][0] + dfx[i][1] * dfx[j][1] + dfx[i][2] * dfx[j][2];
                for (int pass = 0; pass < 2; ++pass) {
                    const double *e = pass == 0 ? e_mu : e_lam;
                    double *out = pass == 0 ? ereg_mu : ereg_lam;
                    for (int i = 0; i < 27; ++i) {
                        double s = 0.0;
                        for (int j = 0; j < 27; ++j) s += er[i][j] * e[j];
                        vh[i] = s;
                    }
                    double num = dot27(e, vh);
                    double den = sqrt(num + eps_tv);
                    for (int i = 0; i < 27; ++i) out[i] = out[i] + (vh[i] / den) * fac0 * fac1;
                    if (pass == 0) cm = cm + (num / den) * fac0 * fac1;
                    else cl = cl + (num / den) * fac0 * fac1;
                }
            }
    *cost_lam = cl;
    *cost_mu = cm;
    return 0;
}

/* A10: S4/IO.F90:541-728 (TIME_FUNCTION); lcase 2 = Ricker (fr given),
 * 3 = Gaussian (L_Gaussian = 40: mean 0.06, sdev 0.0004). */
double ora_time_function(double T, int lcase, double fr)
{
    const double pi = 3.14159265358979323846264338327950288419716939937510;
    if (lcase == 2) {
        double wr = 2.0 * pi * fr;
        double t_max = 6.0 * sqrt(6.0) / wr;
        double u = wr * T - 3.0 * sqrt(6.0);
        if (T < t_max) {
            double f1 = (0.25 * (u * u) - 0.5) * exp(-0.25 * (u * u)) - 13.0 * exp(-13.5);
            double f2 = 0.50 + 13.0 * exp(-13.5);
            return f1 / f2;
        }
        return 0.0;
    }
    if (lcase == 3) {
        const double gm = 0.06, gs = 0.00040;
        return exp(-(T - gm) * (T - gm) / gs);
    }
    if (lcase == 8) return 1.0;
    return 0.0;
}

/* ------------------------------------------------------------------------- */
/* Assembly (A5/A6/A7): S4/Assemble_PETSc_3D.F90:6-184, :192-436, :444-548.  */

typedef struct { int r, c; double v; } trip;
typedef struct { trip *t; size_t n, cap; } tlist;

static int tl_push(tlist *l, int r, int c, double v)
{
    /* PETSc with MAT_IGNORE_ZERO_ENTRIES drops exact zeros and negative indices. */
    if (r < 0 || c < 0 || v == 0.0) return 0;
    if (l->n == l->cap) {
        size_t nc = l->cap ? 2 * l->cap : 1 << 16;
        trip *nt = (trip *)realloc(l->t, nc * sizeof(trip));
        if (!nt) return -1;
        l->t = nt; l->cap = nc;
    }
    l->t[l->n].r = r; l->t[l->n].c = c; l->t[l->n].v = v; l->n++;
    return 0;
}

struct ora_sys {
    int neq;
    int *ia[3], *ja[3];
    double *a[3];
    int nnz[3];
    double *diag_m, *b;
};

/* Stable CSR build: entries that hit the same (row, col) are summed in call
 * order, like ADD_VALUES into a PETSc AIJ matrix. */
static int tl_to_csr(tlist *l, int neq, int **ia_o, int **ja_o, double **a_o, int *nnz_o)
{
    int *cnt = (int *)calloc((size_t)neq + 1, sizeof(int));
    trip *byrow = (trip *)malloc((l->n ? l->n : 1) * sizeof(trip));
    if (!cnt || !byrow) { free(cnt); free(byrow); return -1; }
    for (size_t k = 0; k < l->n; ++k) cnt[l->t[k].r + 1]++;
    for (int i = 0; i < neq; ++i) cnt[i + 1] += cnt[i];
    int *pos = (int *)malloc(((size_t)neq + 1) * sizeof(int));
    memcpy(pos, cnt, ((size_t)neq + 1) * sizeof(int));
    for (size_t k = 0; k < l->n; ++k) byrow[pos[l->t[k].r]++] = l->t[k];
    free(pos);
    /* within each row: stable insertion sort by column, then merge duplicates */
    int *ia = (int *)malloc(((size_t)neq + 1) * sizeof(int));
    int *ja = (int *)malloc((l->n ? l->n : 1) * sizeof(int));
    double *a = (double *)malloc((l->n ? l->n : 1) * sizeof(double));
    int nz = 0;
    ia[0] = 0;
    for (int i = 0; i < neq; ++i) {
        trip *row = byrow + cnt[i];
        int m = cnt[i + 1] - cnt[i];
        for (int x = 1; x < m; ++x) {
            trip key = row[x];
            int y = x - 1;
            while (y >= 0 && row[y].c > key.c) { row[y + 1] = row[y]; --y; }
            row[y + 1] = key;
        }
        for (int x = 0; x < m;) {
            int c = row[x].c;
            double s = row[x].v;
            int y = x + 1;
            while (y < m && row[y].c == c) { s += row[y].v; ++y; }
            ja[nz] = c; a[nz] = s; ++nz;
            x = y;
        }
        ia[i + 1] = nz;
    }
    free(cnt); free(byrow);
    *ia_o = ia; *ja_o = ja; *a_o = a; *nnz_o = nz;
    return 0;
}

static void gather_xt(const ora_mesh *m, int e, double xt[3][27])
{
    for (int i = 0; i < 27; ++i) {
        int k = m->inod[e * 27 + i];
        for (int d = 0; d < 3; ++d) xt[d][i] = m->xyz[3 * k + d];
    }
}

ora_sys *ora_assemble(const ora_mesh *m, const double *lam, const double *mu, const int *id_bc, int *err)
{
    int n = m->neq;
    tlist L[3] = {{0}};
    ora_sys *s = (ora_sys *)calloc(1, sizeof(ora_sys));
    double (*ek)[81] = malloc(sizeof(double) * 81 * 81);
    double (*em)[81][81] = malloc(sizeof(double) * 4 * 81 * 81);
    double (*en)[162][162] = malloc(sizeof(double) * 4 * 162 * 162);
    double (*ea)[81][162] = malloc(sizeof(double) * 6 * 81 * 162);
    int nd1[81], nd2[162];
    *err = 0;
    s->neq = n;
    s->diag_m = (double *)calloc((size_t)n, sizeof(double));
    s->b = (double *)calloc((size_t)n, sizeof(double));
    #define FAIL(code) do { *err = (code); goto fail; } while (0)

    /* ASSEM_REGULAR_DOMAIN_PETSC_3D: K += EK (row-oriented insertion), DIAG_M += diag(EM). */
    for (int e = 0; e < m->nel; ++e) {
        if (m->mtel[e] != 1) continue;
        double xt[3][27], le[27], me[27];
        gather_xt(m, e, xt);
        for (int i = 0; i < 27; ++i) { le[i] = lam[m->inod[e * 27 + i]]; me[i] = mu[m->inod[e * 27 + i]]; }
        if (ora_element_m(xt, m->rho_el[e], m->pml_param, 201, em[0])) FAIL(1);
        if (ora_element_k(xt, le, me, ek)) FAIL(1);
        for (int c = 0; c < 3; ++c)
            for (int i = 0; i < 27; ++i) nd1[c * 27 + i] = m->id[m->inod[e * 27 + i] * 9 + c];
        for (int i = 0; i < 81; ++i)
            for (int j = 0; j < 81; ++j)
                if (tl_push(&L[1], nd1[i], nd1[j], ek[j][i])) FAIL(9);
        for (int i = 0; i < 81; ++i)
            if (nd1[i] >= 0) s->diag_m[nd1[i]] += em[0][i][i];
    }
    /* ASSEM_FORCE_PETSC_3D: B += EFS on loaded RD faces. */
    if (id_bc) {
        for (int e = 0; e < m->nel; ++e) {
            if (m->mtel[e] != 1 || id_bc[e] == 0) continue;
            double xt[3][27], efs[81];
            gather_xt(m, e, xt);
            int rc = ora_element_fs(xt, id_bc[e], efs);
            if (rc) FAIL(4);
            for (int c = 0; c < 3; ++c)
                for (int i = 0; i < 27; ++i) nd1[c * 27 + i] = m->id[m->inod[e * 27 + i] * 9 + c];
            for (int i = 0; i < 81; ++i)
                if (nd1[i] >= 0) s->b[nd1[i]] += efs[i];
        }
    }
    /* ASSEM_PML_PETSC_3D */
    for (int e = 0; e < m->nel; ++e) {
        if (m->mtel[e] != 2) continue;
        double xt[3][27], le[27], me[27];
        gather_xt(m, e, xt);
        for (int i = 0; i < 27; ++i) { le[i] = lam[m->inod[e * 27 + i]]; me[i] = mu[m->inod[e * 27 + i]]; }
        for (int f = 0; f < 4; ++f)
            if (ora_element_m(xt, m->rho_el[e], m->pml_param, 202 + f, em[f])) FAIL(2);
        for (int f = 0; f < 6; ++f)
            if (ora_element_ea(xt, le, me, m->pml_param, 101 + f, ea[f])) FAIL(2);
        for (int f = 0; f < 4; ++f)
            if (ora_element_en(xt, m->pml_param, 301 + f, en[f])) FAIL(2);
        for (int i = 0; i < 27; ++i) {
            int node = m->inod[e * 27 + i];
            for (int c = 0; c < 3; ++c) nd1[c * 27 + i] = m->id[node * 9 + c];
            for (int c = 0; c < 6; ++c) nd2[c * 27 + i] = m->id[node * 9 + 3 + c];
        }
        /* EM_b -> C, EM_c -> K, EM_d -> G (EM_a goes to the unused AM). */
        for (int f = 1; f < 4; ++f)
            for (int i = 0; i < 81; ++i)
                for (int j = 0; j < 81; ++j)
                    if (tl_push(&L[f - 1], nd1[i], nd1[j], em[f][j][i])) FAIL(9);
        /* EN_b -> C, EN_c -> K, EN_d -> G */
        for (int f = 1; f < 4; ++f)
            for (int i = 0; i < 162; ++i)
                for (int j = 0; j < 162; ++j)
                    if (tl_push(&L[f - 1], nd2[i], nd2[j], en[f][j][i])) FAIL(9);
        /* EA upper (81x162, column-major) inserted with rows = stress dofs:
         * entry(s_i, u_j) = EA_upper(u_j, s_i)   (:414-416) */
        for (int f = 0; f < 3; ++f)
            for (int i = 0; i < 162; ++i)
                for (int j = 0; j < 81; ++j)
                    if (tl_push(&L[f], nd2[i], nd1[j], ea[f][j][i])) FAIL(9);
        /* -transpose(EA_lower) inserted with rows = displacement dofs:
         * entry(u_i, s_j) = -EA_lower(u_i, s_j)   (:418-420) */
        for (int f = 0; f < 3; ++f)
            for (int i = 0; i < 81; ++i)
                for (int j = 0; j < 162; ++j)
                    if (tl_push(&L[f], nd1[i], nd2[j], -ea[3 + f][i][j])) FAIL(9);
        for (int i = 0; i < 81; ++i)
            if (nd1[i] >= 0) s->diag_m[nd1[i]] += em[0][i][i];
        for (int i = 0; i < 162; ++i)
            if (nd2[i] >= 0) s->diag_m[nd2[i]] += en[0][i][i];
    }
    for (int w = 0; w < 3; ++w) {
        if (tl_to_csr(&L[w], n, &s->ia[w], &s->ja[w], &s->a[w], &s->nnz[w])) FAIL(9);
        free(L[w].t); L[w].t = NULL;
    }
    free(ek); free(em); free(en); free(ea);
    return s;
fail:
    for (int w = 0; w < 3; ++w) free(L[w].t);
    free(ek); free(em); free(en); free(ea);
    ora_sys_free(s);
    return NULL;
    #undef FAIL
}

void ora_sys_free(ora_sys *s)
{
    if (!s) return;
    for (int w = 0; w < 3; ++w) { free(s->ia[w]); free(s->ja[w]); free(s->a[w]); }
    free(s->diag_m); free(s->b); free(s);
}

int ora_sys_nnz(const ora_sys *s, int which) { return s->nnz[which]; }

void ora_sys_csr(const ora_sys *s, int which, int *ia, int *ja, double *a)
{
    memcpy(ia, s->ia[which], sizeof(int) * ((size_t)s->neq + 1));
    memcpy(ja, s->ja[which], sizeof(int) * (size_t)s->nnz[which]);
    memcpy(a, s->a[which], sizeof(double) * (size_t)s->nnz[which]);
}

void ora_sys_vectors(const ora_sys *s, double *diag_m, double *b)
{
    if (diag_m) memcpy(diag_m, s->diag_m, sizeof(double) * (size_t)s->neq);
    if (b) memcpy(b, s->b, sizeof(double) * (size_t)s->neq);
}

ora_sys *ora_sys_from_csr(int neq, const int *c_ia, const int *c_ja, const double *c_a,
                          const int *k_ia, const int *k_ja, const double *k_a,
                          const int *g_ia, const int *g_ja, const double *g_a, const double *diag_m)
{
    ora_sys *s = (ora_sys *)calloc(1, sizeof(ora_sys));
    const int *IA[3] = {c_ia, k_ia, g_ia}, *JA[3] = {c_ja, k_ja, g_ja};
    const double *AA[3] = {c_a, k_a, g_a};
    s->neq = neq;
    for (int w = 0; w < 3; ++w) {
        int nz = IA[w][neq];
        s->nnz[w] = nz;
        s->ia[w] = (int *)malloc(sizeof(int) * ((size_t)neq + 1));
        s->ja[w] = (int *)malloc(sizeof(int) * (size_t)(nz ? nz : 1));
        s->a[w] = (double *)malloc(sizeof(double) * (size_t)(nz ? nz : 1));
        memcpy(s->ia[w], IA[w], sizeof(int) * ((size_t)neq + 1));
        memcpy(s->ja[w], JA[w], sizeof(int) * (size_t)nz);
        memcpy(s->a[w], AA[w], sizeof(double) * (size_t)nz);
    }
    s->diag_m = (double *)malloc(sizeof(double) * (size_t)neq);
    s->b = (double *)calloc((size_t)neq, sizeof(double));
    memcpy(s->diag_m, diag_m, sizeof(double) * (size_t)neq);
    return s;
}

/* ------------------------------------------------------------------------- */
/* Time loops (A9, A11): S4/Solver_PETSc_Explicit.F90:660-1117, :1125-1405.  */

typedef struct { int n; const int *ia, *ja; double *a; } csr_t;

static void set_threads(int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

/* MatMultAdd: z = y + A x, per row sum = y_i; sum += a*x[col] in column order. */
static void matmultadd(const csr_t *A, const double *x, double *z)
{
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < A->n; ++i) {
        double s = z[i];
        for (int k = A->ia[i]; k < A->ia[i + 1]; ++k) s += A->a[k] * x[A->ja[k]];
        z[i] = s;
    }
}

/* MatMultTransposeAdd: z = y + A^T x, scattered row by row (PETSc SeqAIJ). */
static void matmulttransposeadd(const csr_t *A, const double *x, double *z)
{
    for (int i = 0; i < A->n; ++i) {
        double al = x[i];
        for (int k = A->ia[i]; k < A->ia[i + 1]; ++k) z[A->ja[k]] += al * A->a[k];
    }
}

/* Parallel transposed product over an explicitly transposed copy (used only
 * when the CPU baseline runs with several threads). */
static void build_transpose(const csr_t *A, int **tia, int **tja, double **ta)
{
    int n = A->n, nz = A->ia[n];
    int *ia = (int *)calloc((size_t)n + 1, sizeof(int));
    int *ja = (int *)malloc(sizeof(int) * (size_t)(nz ? nz : 1));
    double *a = (double *)malloc(sizeof(double) * (size_t)(nz ? nz : 1));
    for (int k = 0; k < nz; ++k) ia[A->ja[k] + 1]++;
    for (int i = 0; i < n; ++i) ia[i + 1] += ia[i];
    int *pos = (int *)malloc(sizeof(int) * ((size_t)n + 1));
    memcpy(pos, ia, sizeof(int) * ((size_t)n + 1));
    for (int i = 0; i < n; ++i)
        for (int k = A->ia[i]; k < A->ia[i + 1]; ++k) {
            int p = pos[A->ja[k]]++;
            ja[p] = i; a[p] = A->a[k];
        }
    free(pos);
    *tia = ia; *tja = ja; *ta = a;
}

#define VLOOP for (int i = 0; i < n; ++i)
#define PVLOOP _Pragma("omp parallel for schedule(static)") for (int i = 0; i < n; ++i)

int ora_forward(const ora_sys *s, const double *b, const double *ftab, int nstep, double dt,
                int nstore, const int *store_eq, double *u_store, int nthreads)
{
    int n = s->neq;
    set_threads(nthreads);
    double *im = (double *)malloc(sizeof(double) * (size_t)n);
    double *bh = (double *)malloc(sizeof(double) * (size_t)n);
    csr_t A[3];
    /* :815-824: MatDiagonalScale(A, iM, NULL), MatScale(A, -1), B <- B * iM */
    VLOOP im[i] = (s->diag_m[i] != 0.0) ? 1.0 / s->diag_m[i] : 0.0;
    for (int w = 0; w < 3; ++w) {
        A[w].n = n; A[w].ia = s->ia[w]; A[w].ja = s->ja[w];
        A[w].a = (double *)malloc(sizeof(double) * (size_t)(s->nnz[w] ? s->nnz[w] : 1));
        for (int i = 0; i < n; ++i)
            for (int k = s->ia[w][i]; k < s->ia[w][i + 1]; ++k) A[w].a[k] = -(s->a[w][k] * im[i]);
    }
    VLOOP bh[i] = b[i] * im[i];
    const csr_t *AC = &A[0], *AK = &A[1], *AG = &A[2];
    size_t vb = sizeof(double) * (size_t)n;
    double *x1 = calloc(n, 8), *x2 = calloc(n, 8), *x3 = calloc(n, 8);
    double *k1t = malloc(vb), *k1m = malloc(vb), *k1b = malloc(vb);
    double *k2t = malloc(vb), *k2m = malloc(vb), *k2b = malloc(vb);
    double *k3t = malloc(vb), *k3m = malloc(vb), *k3b = malloc(vb);
    double *k4t = malloc(vb), *k4m = malloc(vb), *k4b = malloc(vb);
    double *hp = malloc(vb);
    const double h = 0.5 * dt;
    for (int istep = 0; istep <= nstep; ++istep) {
        for (int i = 0; i < nstore; ++i) u_store[(size_t)istep * nstore + i] = x2[store_eq[i]];
        double f7 = ftab[3 * istep + 0], f8 = ftab[3 * istep + 1], f9 = ftab[3 * istep + 2];
        PVLOOP { k1b[i] = 0.0 + f7 * bh[i]; k4b[i] = 0.0 + f8 * bh[i]; k2b[i] = 0.0 + f9 * bh[i]; k3b[i] = 0.0 + f9 * bh[i]; }
        PVLOOP { k1t[i] = x2[i]; k1m[i] = x3[i]; }
        matmultadd(AC, x3, k1b); matmultadd(AK, x2, k1b); matmultadd(AG, x1, k1b);
        PVLOOP { k2t[i] = h * k1m[i] + x2[i]; k2m[i] = h * k1b[i] + x3[i]; hp[i] = h * k1t[i] + x1[i]; }
        matmultadd(AC, k2m, k2b); matmultadd(AK, k2t, k2b); matmultadd(AG, hp, k2b);
        PVLOOP { k3t[i] = h * k2m[i] + x2[i]; k3m[i] = h * k2b[i] + x3[i]; hp[i] = h * k2t[i] + x1[i]; }
        matmultadd(AC, k3m, k3b); matmultadd(AK, k3t, k3b); matmultadd(AG, hp, k3b);
        PVLOOP { k4t[i] = dt * k3m[i] + x2[i]; k4m[i] = dt * k3b[i] + x3[i]; hp[i] = dt * k3t[i] + x1[i]; }
        matmultadd(AC, k4m, k4b); matmultadd(AK, k4t, k4b); matmultadd(AG, hp, k4b);
        /* :1035-1046: help = 0 + (k1 + 2 k2 + 2 k3 + k4) (VecMAXPY, 4 at once); x += dt/6 help */
        const double d6 = dt / 6.0;
        PVLOOP {
            double ht = 0.0 + (((1.0 * k1t[i] + 2.0 * k2t[i]) + 2.0 * k3t[i]) + 1.0 * k4t[i]);
            double hm = 0.0 + (((1.0 * k1m[i] + 2.0 * k2m[i]) + 2.0 * k3m[i]) + 1.0 * k4m[i]);
            double hb = 0.0 + (((1.0 * k1b[i] + 2.0 * k2b[i]) + 2.0 * k3b[i]) + 1.0 * k4b[i]);
            x1[i] = x1[i] + d6 * ht;
            x2[i] = x2[i] + d6 * hm;
            x3[i] = x3[i] + d6 * hb;
        }
    }
    free(x1); free(x2); free(x3); free(k1t); free(k1m); free(k1b); free(k2t); free(k2m); free(k2b);
    free(k3t); free(k3m); free(k3b); free(k4t); free(k4m); free(k4b); free(hp);
    for (int w = 0; w < 3; ++w) free(A[w].a);
    free(im); free(bh);
    return 0;
}

/* Residual vector of the adjoint source at one step (S4/Solver_PETSc_Explicit.F90:1269-1279):
 * B_mis = 0; B_mis(EqDis) += U_Store(map, n) - Dis_meas(n, :).  Only the
 * receiver entries of bm are touched. */
static void misfit_vector(int istep, int nstep, int nrec3, const int *eqdis, const int *emap, int nstore,
                          const double *u_store, const double *dis_meas, double *bm)
{
    for (int q = 0; q < nrec3; ++q) bm[eqdis[q]] = 0.0;
    for (int q = 0; q < nrec3; ++q)
        bm[eqdis[q]] += u_store[(size_t)istep * nstore + emap[q]] - dis_meas[(size_t)q * (nstep + 1) + istep];
}

int ora_adjoint(const ora_sys *s, int nstep, double dt, int nstore, const int *store_eq,
                const double *u_store, int nrec3, const int *eqdis, const int *eqdis_map,
                const double *dis_meas, double *p_store, int nthreads)
{
    int n = s->neq;
    set_threads(nthreads);
    double *im = (double *)malloc(sizeof(double) * (size_t)n);
    VLOOP im[i] = (s->diag_m[i] != 0.0) ? 1.0 / s->diag_m[i] : 0.0;
    /* forward scaling then :1222-1229 (AC,AG *= -1; MatDiagonalScale(A, M, iM)) */
    csr_t A[3];
    int *tia[3] = {0}, *tja[3] = {0};
    double *ta[3] = {0};
    for (int w = 0; w < 3; ++w) {
        A[w].n = n; A[w].ia = s->ia[w]; A[w].ja = s->ja[w];
        A[w].a = (double *)malloc(sizeof(double) * (size_t)(s->nnz[w] ? s->nnz[w] : 1));
        for (int i = 0; i < n; ++i)
            for (int k = s->ia[w][i]; k < s->ia[w][i + 1]; ++k) {
                double v = -(s->a[w][k] * im[i]);
                if (w != 1) v = -v;
                v = v * s->diag_m[i];
                v = v * im[s->ja[w][k]];
                A[w].a[k] = v;
            }
        if (nthreads > 1) build_transpose(&A[w], &tia[w], &tja[w], &ta[w]);
    }
    size_t vb = sizeof(double) * (size_t)n;
    double *x1 = calloc(n, 8), *x2 = calloc(n, 8), *x3 = calloc(n, 8);
    double *k1t = malloc(vb), *k1m = malloc(vb), *k1b = malloc(vb);
    double *k2t = malloc(vb), *k2m = malloc(vb), *k2b = malloc(vb);
    double *k3t = malloc(vb), *k3m = malloc(vb), *k3b = malloc(vb);
    double *k4t = malloc(vb), *k4m = malloc(vb), *k4b = malloc(vb);
    double *hp = malloc(vb), *bm = calloc(n, 8);
    const double h = -0.5 * dt;
    csr_t T[3];
    for (int w = 0; w < 3; ++w) { T[w].n = n; T[w].ia = tia[w]; T[w].ja = tja[w]; T[w].a = ta[w]; }
    #define MTA(w, xx, zz) do { if (nthreads > 1) matmultadd(&T[w], xx, zz); else matmulttransposeadd(&A[w], xx, zz); } while (0)
    for (int istep = nstep; istep >= 1; --istep) {
        for (int i = 0; i < nstore; ++i) p_store[(size_t)istep * nstore + i] = x2[store_eq[i]];
        /* :1269-1306 */
        PVLOOP { k1b[i] = 0.0; k4b[i] = 0.0; }
        misfit_vector(istep, nstep, nrec3, eqdis, eqdis_map, nstore, u_store, dis_meas, bm);
        for (int q = 0; q < nrec3; ++q) { int e = eqdis[q]; k1b[e] = 0.0 + 1.0 * (bm[e] * im[e]); }
        misfit_vector(istep - 1, nstep, nrec3, eqdis, eqdis_map, nstore, u_store, dis_meas, bm);
        for (int q = 0; q < nrec3; ++q) { int e = eqdis[q]; k4b[e] = 0.0 + 1.0 * (bm[e] * im[e]); }
        /* :1309-1312: k2b = k3b = 0 + (0.5 k1b + 0.5 k4b) */
        PVLOOP { double v = 0.0 + (0.5 * k1b[i] + 0.5 * k4b[i]); k2b[i] = v; k3b[i] = v; }
        PVLOOP { k1t[i] = x2[i]; k1m[i] = x3[i]; }
        MTA(0, x3, k1b); MTA(1, x2, k1b); MTA(2, x1, k1b);
        PVLOOP { k2t[i] = h * k1m[i] + x2[i]; k2m[i] = h * k1b[i] + x3[i]; hp[i] = h * k1t[i] + x1[i]; }
        MTA(0, k2m, k2b); MTA(1, k2t, k2b); MTA(2, hp, k2b);
        PVLOOP { k3t[i] = h * k2m[i] + x2[i]; k3m[i] = h * k2b[i] + x3[i]; hp[i] = h * k2t[i] + x1[i]; }
        MTA(0, k3m, k3b); MTA(1, k3t, k3b); MTA(2, hp, k3b);
        PVLOOP { k4t[i] = -dt * k3m[i] + x2[i]; k4m[i] = -dt * k3b[i] + x3[i]; hp[i] = -dt * k3t[i] + x1[i]; }
        MTA(0, k4m, k4b); MTA(1, k4t, k4b); MTA(2, hp, k4b);
        const double d6 = -dt / 6.0;
        PVLOOP {
            double ht = 0.0 + (((1.0 * k1t[i] + 2.0 * k2t[i]) + 2.0 * k3t[i]) + 1.0 * k4t[i]);
            double hm = 0.0 + (((1.0 * k1m[i] + 2.0 * k2m[i]) + 2.0 * k3m[i]) + 1.0 * k4m[i]);
            double hb = 0.0 + (((1.0 * k1b[i] + 2.0 * k2b[i]) + 2.0 * k3b[i]) + 1.0 * k4b[i]);
            x1[i] = x1[i] + d6 * ht;
            x2[i] = x2[i] + d6 * hm;
            x3[i] = x3[i] + d6 * hb;
        }
    }
    #undef MTA
    free(x1); free(x2); free(x3); free(k1t); free(k1m); free(k1b); free(k2t); free(k2m); free(k2b);
    free(k3t); free(k3m); free(k3b); free(k4t); free(k4m); free(k4b); free(hp); free(bm);
    for (int w = 0; w < 3; ++w) { free(A[w].a); free(tia[w]); free(tja[w]); free(ta[w]); }
    free(im);
    return 0;
}

/* A12: S4/Solver_PETSc_Explicit.F90:1413-1522 with Update_g
 * (S4/Assemble_PETSc_3D.F90:556-661).  Node index = material index.
 * The element terms of a step are computed in parallel (nthreads > 1) into one
 * buffer per element and then added to the nodes serially in element order, so
 * every thread count gives the bits of the serial loop.  The reference runs the
 * same element loop on every MPI rank over its own elements. */
int ora_control(const ora_mesh *m, int nstep, double dt, int nstore, const int *store_eq,
                const double *u_store, const double *p_store, double *g_lam, double *g_mu, int lambda_2mu,
                int nthreads)
{
    int n = m->neq;
    set_threads(nthreads);
    int nrd = 0;
    for (int e = 0; e < m->nel; ++e) nrd += m->mtel[e] == 1;
    int *rd = (int *)malloc(sizeof(int) * (size_t)(nrd ? nrd : 1));
    for (int e = 0, k = 0; e < m->nel; ++e) if (m->mtel[e] == 1) rd[k++] = e;
    double *ub = (double *)calloc((size_t)n, sizeof(double));
    double *pb = (double *)calloc((size_t)n, sizeof(double));
    double *egm = (double *)malloc(sizeof(double) * 27 * (size_t)(nrd ? nrd : 1));
    double *egl = (double *)malloc(sizeof(double) * 27 * (size_t)(nrd ? nrd : 1));
    int bad = 0;
    for (int istep = 1; istep <= nstep - 1 && !bad; ++istep) {
        memset(ub, 0, sizeof(double) * (size_t)n);
        memset(pb, 0, sizeof(double) * (size_t)n);
        for (int i = 0; i < nstore; ++i) {
            ub[store_eq[i]] += u_store[(size_t)istep * nstore + i];
            pb[store_eq[i]] += p_store[(size_t)istep * nstore + i];
        }
        #pragma omp parallel for schedule(static) reduction(|:bad)
        for (int k = 0; k < nrd; ++k) {
            int e = rd[k];
            double xt[3][27], eu[81], ep[81];
            gather_xt(m, e, xt);
            for (int c = 0; c < 3; ++c)
                for (int i = 0; i < 27; ++i) {
                    int q = m->id[m->inod[e * 27 + i] * 9 + c];
                    eu[c * 27 + i] = q >= 0 ? ub[q] : 0.0;
                    ep[c * 27 + i] = q >= 0 ? pb[q] : 0.0;
                }
            if (ora_element_g(xt, eu, ep, egm + 27 * (size_t)k, egl + 27 * (size_t)k, lambda_2mu)) bad |= 1;
        }
        if (bad) break;
        for (int k = 0; k < nrd; ++k) {
            int e = rd[k];
            for (int i = 0; i < 27; ++i) {
                int node = m->inod[e * 27 + i];
                g_mu[node] += egm[27 * (size_t)k + i] * dt;
                g_lam[node] += egl[27 * (size_t)k + i] * dt;
            }
        }
    }
    free(ub); free(pb); free(egm); free(egl); free(rd);
    return bad ? -1 : 0;
}

/* A13: S4/Solver_PETSc_Inverse.F90:591-657 (Compute_Misfit). */
double ora_misfit(int nstep, double dt, int nrec3, const int *eqdis, const int *eqdis_map,
                  int nstore, const double *u_store, const double *dis_meas)
{
    /* unique equations in increasing order (VecDot runs over the whole vector) */
    int *uq = (int *)malloc(sizeof(int) * (size_t)(nrec3 ? nrec3 : 1));
    double *acc = (double *)malloc(sizeof(double) * (size_t)(nrec3 ? nrec3 : 1));
    int nu = 0;
    for (int q = 0; q < nrec3; ++q) {
        int e = eqdis[q], found = 0;
        for (int k = 0; k < nu; ++k) if (uq[k] == e) { found = 1; break; }
        if (!found) uq[nu++] = e;
    }
    for (int x = 1; x < nu; ++x) { int k = uq[x], y = x - 1; while (y >= 0 && uq[y] > k) { uq[y + 1] = uq[y]; --y; } uq[y + 1] = k; }
    double cost = 0.0;
    for (int istep = nstep; istep >= 1; --istep) {
        for (int k = 0; k < nu; ++k) acc[k] = 0.0;
        for (int q = 0; q < nrec3; ++q) {
            double r = u_store[(size_t)istep * nstore + eqdis_map[q]] - dis_meas[(size_t)q * (nstep + 1) + istep];
            for (int k = 0; k < nu; ++k) if (uq[k] == eqdis[q]) { acc[k] += r; break; }
        }
        double d = 0.0;
        for (int k = 0; k < nu; ++k) d += acc[k] * acc[k];
        cost = cost + 0.5 * d * dt;
    }
    free(uq); free(acc);
    return cost;
}

/* A14: S4/Assemble_PETSc_3D.F90:755-849 (Assem_TV_TN_Regularization). */
int ora_tv_reg(const ora_mesh *m, const double *lam, const double *mu,
               double *reg_lam, double *reg_mu, double *cost_lam, double *cost_mu)
{
    double cl = 0.0, cm = 0.0;
    for (int e = 0; e < m->nel; ++e) {
        if (m->mtel[e] != 1) continue;
        double xt[3][27], el[27], emu[27], rm[27], rl[27], ecl, ecm;
        gather_xt(m, e, xt);
        for (int i = 0; i < 27; ++i) { el[i] = lam[m->inod[e * 27 + i]]; emu[i] = mu[m->inod[e * 27 + i]]; }
        if (ora_element_tv(xt, emu, el, rm, rl, &ecl, &ecm)) return -1;
        cl = cl + ecl; cm = cm + ecm;
        for (int i = 0; i < 27; ++i) {
            int node = m->inod[e * 27 + i];
            reg_mu[node] += rm[i];
            reg_lam[node] += rl[i];
        }
    }
    *cost_lam = cl; *cost_mu = cm;
    return 0;
}

/* A14: S4/Assemble_PETSc_3D.F90:670-747 (Assem_R_Mg_3D), gradient mass part. */
int ora_rmg(const ora_mesh *m, double *mg)
{
    for (int e = 0; e < m->nel; ++e) {
        if (m->mtel[e] != 1) continue;
        double xt[3][27], er[27][27], emg[27];
        gather_xt(m, e, xt);
        if (ora_element_r_mg(xt, er, emg)) return -1;
        for (int i = 0; i < 27; ++i) mg[m->inod[e * 27 + i]] += emg[i];
    }
    return 0;
}

int ora_apply_scaled(const ora_sys *s, int which, int transpose_adjoint, const double *x, double *y)
{
    int n = s->neq;
    double *im = (double *)malloc(sizeof(double) * (size_t)n);
    VLOOP im[i] = (s->diag_m[i] != 0.0) ? 1.0 / s->diag_m[i] : 0.0;
    csr_t A;
    A.n = n; A.ia = s->ia[which]; A.ja = s->ja[which];
    A.a = (double *)malloc(sizeof(double) * (size_t)(s->nnz[which] ? s->nnz[which] : 1));
    for (int i = 0; i < n; ++i)
        for (int k = s->ia[which][i]; k < s->ia[which][i + 1]; ++k) {
            double v = -(s->a[which][k] * im[i]);
            if (transpose_adjoint) {
                if (which != 1) v = -v;
                v = v * s->diag_m[i];
                v = v * im[s->ja[which][k]];
            }
            A.a[k] = v;
        }
    VLOOP y[i] = 0.0;
    if (transpose_adjoint) matmulttransposeadd(&A, x, y);
    else matmultadd(&A, x, y);
    free(A.a); free(im);
    return 0;
}
