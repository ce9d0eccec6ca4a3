// hrn_elem.cu -- matrix-free application of the assembled operators C, K, G for
// the RK4 stages: the element kernels compute, per 27-node GLL hexahedron, what
// the element matrices of S4/Element_Matrices_3D.F90 do to the stage inputs,
// without forming a matrix.
//
// With the 3-point GLL rule every basis function is a Kronecker delta at the
// quadrature points, so the element operators are local:
//   * regular domain, K (ELEMENT_K_3D :7-220): at each point q the displacement
//     gradient g_ck = sum_m du_c/dxi_m DJI(m,k) (each du/dxi_m a 3-term sum along
//     the xi_m line through q), the isotropic stress
//     sig_cc = lam tr(g) + 2 mu g_cc, sig_ck = mu (g_ck + g_kc), and
//     (K u)_Ic += sum_q w detJ DFX(I,k)(q) sig_ck(q), a line-wise divergence;
//   * PML (ELEMENT_M/EN/EA_3D :228-882 as assembled by
//     S4/Assemble_PETSc_3D.F90:192-436): the mass-type blocks EM_b..d and
//     EN_b..d are diagonal (C, K, G take b, c, d); EA of kind e/p/w (C/K/G)
//     couples the stresses of node J with the displacement gradient at J
//     (upper, rows = stresses) and the displacements with the divergence of the
//     stresses weighted by lam, mu (lower, rows = displacements, negated).  The
//     stretching weight F of a derivative depends only on its direction k:
//     k = x -> F3, y -> F2, z -> F1 of the kind.
// The adjoint applies the transposes (the gradient and divergence swap roles)
// with the signs of the OtD adjoint (C and G negated, S4/Solver_PETSc_Explicit.F90:1222-1229).
//
// A stage is two launches: the element kernel writes each element's
// contribution to its 27 nodes into a slot (or adds it atomically into a row
// accumulator), and the node kernel sums the slots of each row in ascending
// element order, scales by -iM and runs the row epilogue of the stage.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <type_traits>
#include <vector>

#include "hrn_internal.h"
#include "hrn_stage.cuh"

namespace hrn {

__constant__ double e_pml[24];              // PML_PARAM rows x+, x-, y+, y-, z+, z-; cols alpha0, beta0, L, x0

constexpr uint32_t kRdSlot = 0x80000000u;   // slot of a regular-domain element (displacements only)
// Element grids of at least this many blocks per SM (about eight waves of the
// combined kernel) take separate PML and regular-domain launches.
constexpr int kElemSplitBlocksPerSm = 16;

// D[a][b] = l_b'(xi_a) of the 3-point GLL basis: row a (derivative at point a)
// and column b (derivative of basis b at the three points).
__device__ __forceinline__ void gll_row(int a, double &d0, double &d1, double &d2)
{
    d0 = a == 0 ? -1.5 : (a == 1 ? -0.5 : 0.5);
    d1 = a == 0 ? 2.0 : (a == 1 ? 0.0 : -2.0);
    d2 = a == 0 ? -0.5 : (a == 1 ? 0.5 : 1.5);
}
__device__ __forceinline__ void gll_col(int b, double &d0, double &d1, double &d2)
{
    d0 = b == 0 ? -1.5 : (b == 1 ? 2.0 : -0.5);
    d1 = b == 0 ? -0.5 : (b == 1 ? 0.0 : 0.5);
    d2 = b == 0 ? 0.5 : (b == 1 ? -2.0 : 1.5);
}

// PML_FINDER_3D (S4/PML.F90:325-891), degree 2 and ratio 0: alpha (0-2), beta (3-5),
// a, b, c, d (6-9) at a point outside the top zone.
__device__ void pml_coefs(const double *x, double A[10])
{
    A[0] = 1.0; A[1] = 1.0; A[2] = 1.0; A[3] = 0.0; A[4] = 0.0; A[5] = 0.0;
    for (int ax = 0; ax < 2; ++ax) {
        int r = -1;
        if (x[ax] >= e_pml[(2 * ax) * 4 + 3]) r = 2 * ax;
        else if (x[ax] <= e_pml[(2 * ax + 1) * 4 + 3]) r = 2 * ax + 1;
        if (r >= 0) {
            const double vn = (r == 2 * ax) ? 1.0 : -1.0;
            const double f = (x[ax] - e_pml[r * 4 + 3]) * vn / e_pml[r * 4 + 2];
            const double pa = f * f;
            A[ax] += e_pml[r * 4 + 0] * pa;
            A[3 + ax] += e_pml[r * 4 + 1] * pa;
        }
    }
    if (x[2] <= e_pml[5 * 4 + 3]) {
        const double f = -(x[2] - e_pml[5 * 4 + 3]) / e_pml[5 * 4 + 2];
        const double pa = f * f;
        A[2] += e_pml[5 * 4 + 0] * pa;
        A[5] += e_pml[5 * 4 + 1] * pa;
    }
    A[6] = A[0] * A[1] * A[2];
    A[7] = A[0] * A[1] * A[5] + A[0] * A[2] * A[4] + A[1] * A[2] * A[3];
    A[8] = A[0] * A[4] * A[5] + A[1] * A[3] * A[5] + A[2] * A[3] * A[4];
    A[9] = A[3] * A[4] * A[5];
}

template <typename T>
struct ElemArgs {
    int nel_pml, nel_rd, nb_pml;     // elements in processing order: PML first, then the regular domain;
                                     // blocks of PML elements in a combined launch
    const int32_t *el_eq;            // [P][27][9] equation of each point's DOF (-1 fixed)
    const int32_t *el_node;          // [P][27] node of each point
    const double *el_geom;           // [P][27][10] DJI and w*detJ
    const double *el_rho;            // [P]
    const double *lam, *mu, *pmlw;   // nodal lambda, mu; [nj][12] PML weights
    T *slots;                        // [P * 27][9][S]
    T *acc;                          // [neq][S] (atomic variant)
};

// Shot blocking: one thread handles SV consecutive shots of a point (vector
// shared-memory and global accesses), TP = S / SV threads per point, and a block
// takes EPB = 8 / TP elements (216 threads).
template <int S, int SV>
constexpr int elems_per_block() { return (S / SV) >= 8 ? 1 : 8 / (S / SV); }

constexpr int kCoef = 14;   // per point: lam, mu, F3 F2 F1 of kinds e, p, w, then b, c, d

// Per element of a block, PML / regular domain: displacement inputs U
// [3 or 1 inputs][27][3][S], fluxes V [27][9][S], coefficients [27][kCoef or 2]
// (lam, mu only in the regular domain), equation numbers [27][9 or 3] (atomic
// variants).  A regular-domain element needs a third of the PML element's inputs.
template <int S, bool PML>
constexpr int elem_u_stride() { return (PML ? 3 : 1) * 81 * S; }
template <bool PML>
constexpr int elem_ncoef() { return PML ? kCoef : 2; }
template <typename T, int S, int SV, bool PML>
constexpr size_t elem_smem_bytes()
{
    return size_t(elems_per_block<S, SV>()) *
           ((elem_u_stride<S, PML>() + 243 * S + 27 * elem_ncoef<PML>()) * sizeof(T) + 27 * (PML ? 9 : 3) * sizeof(int));
}

// N consecutive values from shared or global memory, vectorized when N values
// fill 8 or 16 bytes (the callers keep such runs aligned to their size).
template <typename T, int N>
__device__ __forceinline__ void ld_n(const T *p, T (&o)[N])
{
    if constexpr (N * sizeof(T) == 16 && sizeof(T) == 4) {
        const float4 v = *reinterpret_cast<const float4 *>(p);
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    } else if constexpr (N * sizeof(T) == 16 && sizeof(T) == 8) {
        const double2 v = *reinterpret_cast<const double2 *>(p);
        o[0] = v.x; o[1] = v.y;
    } else if constexpr (N * sizeof(T) == 8 && sizeof(T) == 4) {
        const float2 v = *reinterpret_cast<const float2 *>(p);
        o[0] = v.x; o[1] = v.y;
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) o[i] = p[i];
    }
}
template <typename T, int N>
__device__ __forceinline__ void ldg_n(const T *p, T (&o)[N])
{
    if constexpr (N * sizeof(T) == 16 && sizeof(T) == 4) {
        const float4 v = __ldg(reinterpret_cast<const float4 *>(p));
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    } else if constexpr (N * sizeof(T) == 16 && sizeof(T) == 8) {
        const double2 v = __ldg(reinterpret_cast<const double2 *>(p));
        o[0] = v.x; o[1] = v.y;
    } else if constexpr (N * sizeof(T) == 8 && sizeof(T) == 4) {
        const float2 v = __ldg(reinterpret_cast<const float2 *>(p));
        o[0] = v.x; o[1] = v.y;
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) o[i] = __ldg(p + i);
    }
}
template <typename T, int N>
__device__ __forceinline__ void st_n(T *p, const T (&o)[N])
{
    if constexpr (N * sizeof(T) == 16 && sizeof(T) == 4) {
        *reinterpret_cast<float4 *>(p) = make_float4(o[0], o[1], o[2], o[3]);
    } else if constexpr (N * sizeof(T) == 16 && sizeof(T) == 8) {
        *reinterpret_cast<double2 *>(p) = make_double2(o[0], o[1]);
    } else if constexpr (N * sizeof(T) == 8 && sizeof(T) == 4) {
        *reinterpret_cast<float2 *>(p) = make_float2(o[0], o[1]);
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) p[i] = o[i];
    }
}
// Atomic add of N consecutive values (vector reductions for FP32).
template <typename T, int N>
__device__ __forceinline__ void red_n(T *p, const T (&o)[N])
{
    if constexpr (sizeof(T) == 4 && N == 4) {
        asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(o[0]), "f"(o[1]), "f"(o[2]), "f"(o[3])
                     : "memory");
    } else if constexpr (sizeof(T) == 4 && N == 2) {
        asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(o[0]), "f"(o[1]) : "memory");
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) atomicAdd(p + i, o[i]);
    }
}

// N shots (from s0) of the stage input of matrix TAG (0 = C, 1 = K, 2 = G) at row
// j: read from the vectors the previous stage materialized (MAT), or rebuilt
// from x1, x2, x3 and the earlier kb with the same fused multiply-adds as the
// row epilogue, e.g. km_3 = c*kb_2 + x3, kt_3 = c*km_2 + x2, h_3 = c*kt_2 + x1.
template <typename T, int S, int N>
__device__ __forceinline__ void stage_input_n(const StageArgs<T> &a, int stage, int mat, int tag, size_t j, int s0, T (&v)[N])
{
    const size_t o = j * S + s0;
    T p1[N], p2[N], p3[N], p4[N];
    if (stage == 1) {
        ldg_n<T, N>((tag == 0 ? a.x3 : (tag == 1 ? a.x2 : a.x1)) + o, v);
        return;
    }
    if (mat) {
        ldg_n<T, N>((tag == 0 ? a.in_m : (tag == 1 ? a.in_t : a.in_h)) + o, v);
        return;
    }
    const T c = a.c, D = a.D;
    if (stage == 2) {
        if (tag == 0) { ldg_n<T, N>(a.kb1 + o, p1); ldg_n<T, N>(a.x3 + o, p2); }
        else if (tag == 1) { ldg_n<T, N>(a.x3 + o, p1); ldg_n<T, N>(a.x2 + o, p2); }
        else { ldg_n<T, N>(a.x2 + o, p1); ldg_n<T, N>(a.x1 + o, p2); }
#pragma unroll
        for (int i = 0; i < N; ++i) v[i] = fmaT(c, p1[i], p2[i]);
    } else if (stage == 3) {
        if (tag == 0) {
            ldg_n<T, N>(a.kb2 + o, p1); ldg_n<T, N>(a.x3 + o, p2);
#pragma unroll
            for (int i = 0; i < N; ++i) v[i] = fmaT(c, p1[i], p2[i]);
        } else if (tag == 1) {
            ldg_n<T, N>(a.kb1 + o, p1); ldg_n<T, N>(a.x3 + o, p2); ldg_n<T, N>(a.x2 + o, p3);
#pragma unroll
            for (int i = 0; i < N; ++i) v[i] = fmaT(c, fmaT(c, p1[i], p2[i]), p3[i]);
        } else {
            ldg_n<T, N>(a.x3 + o, p1); ldg_n<T, N>(a.x2 + o, p2); ldg_n<T, N>(a.x1 + o, p3);
#pragma unroll
            for (int i = 0; i < N; ++i) v[i] = fmaT(c, fmaT(c, p1[i], p2[i]), p3[i]);
        }
    } else {
        if (tag == 0) {
            ldg_n<T, N>(a.kb3 + o, p1); ldg_n<T, N>(a.x3 + o, p2);
#pragma unroll
            for (int i = 0; i < N; ++i) v[i] = fmaT(D, p1[i], p2[i]);
        } else if (tag == 1) {
            ldg_n<T, N>(a.kb2 + o, p1); ldg_n<T, N>(a.x3 + o, p2); ldg_n<T, N>(a.x2 + o, p3);
#pragma unroll
            for (int i = 0; i < N; ++i) v[i] = fmaT(D, fmaT(c, p1[i], p2[i]), p3[i]);
        } else {
            ldg_n<T, N>(a.kb1 + o, p1); ldg_n<T, N>(a.x3 + o, p2); ldg_n<T, N>(a.x2 + o, p3); ldg_n<T, N>(a.x1 + o, p4);
#pragma unroll
            for (int i = 0; i < N; ++i) v[i] = fmaT(D, fmaT(c, fmaT(c, p1[i], p2[i]), p3[i]), p4[i]);
        }
    }
}

template <typename T, int S, int SV, int ADJ, int ACC, bool PML>
__device__ __forceinline__ void elem_body(const ElemArgs<T> &A, const StageArgs<T> &a, int stage, int mat, int pbase, int ngrp,
                                          int e0, T *U, T *V, T *coef, int *eqs)
{
    constexpr int TP = S / SV;
    constexpr int NTAG = PML ? 3 : 1;
    constexpr int NDOF = PML ? 9 : 3;
    const int tid = threadIdx.x;
    const int tp = tid % TP, q = (tid / TP) % 27, el = tid / (27 * TP);
    const int s0 = tp * SV;
    const bool active = e0 + el < ngrp;
    const int p = pbase + e0 + el;
    const size_t pq = size_t(p) * 27 + q;
    constexpr int NC = elem_ncoef<PML>();
    T *Ue = U + el * elem_u_stride<S, PML>();
    T ji[9];
    T f0 = T(0), rho = T(0);
    // all global loads of the block are issued in this one phase; the TP
    // threads of a point share its displacement values and coefficients
    if (active) {
        const double *g = A.el_geom + pq * 10;
#pragma unroll
        for (int k = 0; k < 9; ++k) ji[k] = T(__ldg(g + k));
        f0 = T(__ldg(g + 9));
        if constexpr (PML) rho = T(__ldg(A.el_rho + p));
        const int32_t *eqp = A.el_eq + pq * 9;
        for (int i = tp; i < NTAG * 3; i += TP) {
            const int t = i / 3, c = i % 3;
            const int eq = __ldg(eqp + c);
            T v[S];
            if (eq >= 0) {
                stage_input_n<T, S, S>(a, stage, mat, PML ? t : 1, size_t(eq), 0, v);
            } else {
#pragma unroll
                for (int k = 0; k < S; ++k) v[k] = T(0);
            }
            T *dst = Ue + ((t * 27 + q) * 3 + c) * S;
#pragma unroll
            for (int k = 0; k < S; ++k) dst[k] = v[k];
        }
        if constexpr (ACC == 1)
            for (int d = tp; d < NDOF; d += TP) eqs[(el * 27 + q) * NDOF + d] = __ldg(eqp + d);
        const int node = __ldg(A.el_node + pq);
        T *cf = coef + (el * 27 + q) * NC;
        for (int j = tp; j < NC; j += TP)
            cf[j] = T(j == 0 ? __ldg(A.lam + node) : (j == 1 ? __ldg(A.mu + node) : __ldg(A.pmlw + size_t(node) * 12 + j - 2)));
    }
    __syncthreads();

    const int qm[3] = {q % 3, (q / 3) % 3, q / 9};
    const int base[3] = {q - qm[0], q - 3 * qm[1], q - 9 * qm[2]};
    constexpr int kStride[3] = {1, 3, 9};
    T yu[3][SV], ys[6][SV];
#pragma unroll
    for (int v = 0; v < SV; ++v) {
#pragma unroll
        for (int c = 0; c < 3; ++c) yu[c][v] = T(0);
#pragma unroll
        for (int d = 0; d < 6; ++d) ys[d][v] = T(0);
    }
    // du_c/dxi_m at q along the three lines (component c of input Ut), then
    // gr_k = sum_m du_m DJI(m,k)
    auto grad_c = [&](const T *Ut, int c, T (&gr)[3][SV]) {
        T du[3][SV];
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            double d0, d1, d2;
            gll_row(qm[m], d0, d1, d2);
            const T *pp = Ut + (base[m] * 3 + c) * S + s0;
            const int st = kStride[m] * 3 * S;
            T a0[SV], a1[SV], a2[SV];
            ld_n<T, SV>(pp, a0);
            ld_n<T, SV>(pp + st, a1);
            ld_n<T, SV>(pp + 2 * st, a2);
#pragma unroll
            for (int v = 0; v < SV; ++v) du[m][v] = fmaT(T(d2), a2[v], fmaT(T(d1), a1[v], T(d0) * a0[v]));
        }
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int v = 0; v < SV; ++v) gr[k][v] = fmaT(du[2][v], ji[6 + k], fmaT(du[1][v], ji[3 + k], du[0][v] * ji[k]));
    };
    auto put_flux = [&](const T (&W)[3][3][SV], T sign) {
        T *vb = V + (el * 27 + q) * 9 * S + s0;
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                T o[SV];
#pragma unroll
                for (int v = 0; v < SV; ++v)
                    o[v] = sign * f0 * fmaT(ji[3 * m + 2], W[c][2][v], fmaT(ji[3 * m + 1], W[c][1][v], ji[3 * m] * W[c][0][v]));
                st_n<T, SV>(vb + (c * 3 + m) * S, o);
            }
    };
    if (active) {
        const T *cf = coef + (el * 27 + q) * NC;
        const T lam = cf[0], mu = cf[1];
        const T l2 = lam + T(2) * mu, m2 = T(2) * mu;
        if constexpr (PML) {
            // pass 1: the stresses of the point give the fluxes of the divergence
            // and the diagonal EN terms
            {
                T W[3][3][SV];
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int k = 0; k < 3; ++k)
#pragma unroll
                        for (int v = 0; v < SV; ++v) W[c][k][v] = T(0);
                const int32_t *eqp = A.el_eq + pq * 9;
#pragma unroll
                for (int t = 0; t < 3; ++t) {
                    T sv[6][SV];
#pragma unroll
                    for (int d = 0; d < 6; ++d) {
                        const int eq = __ldg(eqp + 3 + d);
                        if (eq >= 0) {
                            stage_input_n<T, S, SV>(a, stage, mat, t, size_t(eq), s0, sv[d]);
                        } else {
#pragma unroll
                            for (int v = 0; v < SV; ++v) sv[d][v] = T(0);
                        }
                    }
                    const T w0 = cf[2 + 3 * t], w1 = cf[3 + 3 * t], w2 = cf[4 + 3 * t];
                    const T sgn = (ADJ && t != 1) ? T(-1) : T(1);
                    const T dn = sgn * cf[11 + t];
#pragma unroll
                    for (int v = 0; v < SV; ++v) {
                        const T s_0 = sv[0][v], s_1 = sv[1][v], s_2 = sv[2][v], s_3 = sv[3][v], s_4 = sv[4][v], s_5 = sv[5][v];
                        if (!ADJ) {
                            // EA lower: displacement rows take minus the divergence of w_k (C : s)
                            const T sxx = l2 * s_0 + lam * (s_1 + s_2);
                            const T syy = lam * (s_0 + s_2) + l2 * s_1;
                            const T szz = lam * (s_0 + s_1) + l2 * s_2;
                            const T sxy = m2 * s_3, sxz = m2 * s_4, syz = m2 * s_5;
                            W[0][0][v] = fmaT(w0, sxx, W[0][0][v]); W[0][1][v] = fmaT(w1, sxy, W[0][1][v]); W[0][2][v] = fmaT(w2, sxz, W[0][2][v]);
                            W[1][0][v] = fmaT(w0, sxy, W[1][0][v]); W[1][1][v] = fmaT(w1, syy, W[1][1][v]); W[1][2][v] = fmaT(w2, syz, W[1][2][v]);
                            W[2][0][v] = fmaT(w0, sxz, W[2][0][v]); W[2][1][v] = fmaT(w1, syz, W[2][1][v]); W[2][2][v] = fmaT(w2, szz, W[2][2][v]);
                        } else {
                            // transposed EA upper: displacement rows take the divergence of w_k s
                            const T ws0 = sgn * w0, ws1 = sgn * w1, ws2 = sgn * w2;
                            W[0][0][v] = fmaT(ws0, s_0, W[0][0][v]); W[0][1][v] = fmaT(ws1, s_3, W[0][1][v]); W[0][2][v] = fmaT(ws2, s_4, W[0][2][v]);
                            W[1][0][v] = fmaT(ws0, s_3, W[1][0][v]); W[1][1][v] = fmaT(ws1, s_1, W[1][1][v]); W[1][2][v] = fmaT(ws2, s_5, W[1][2][v]);
                            W[2][0][v] = fmaT(ws0, s_4, W[2][0][v]); W[2][1][v] = fmaT(ws1, s_5, W[2][1][v]); W[2][2][v] = fmaT(ws2, s_2, W[2][2][v]);
                        }
                        // diagonal EN (f, 2 f) blocks
                        ys[0][v] = fmaT(dn, s_0, ys[0][v]);
                        ys[1][v] = fmaT(dn, s_1, ys[1][v]);
                        ys[2][v] = fmaT(dn, s_2, ys[2][v]);
                        ys[3][v] = fmaT(T(2) * dn, s_3, ys[3][v]);
                        ys[4][v] = fmaT(T(2) * dn, s_4, ys[4][v]);
                        ys[5][v] = fmaT(T(2) * dn, s_5, ys[5][v]);
                    }
                }
                put_flux(W, ADJ ? T(1) : T(-1));
            }
            // pass 2: displacement gradients give the stress rows, and the
            // diagonal EM terms
#pragma unroll
            for (int t = 0; t < 3; ++t) {
                const T *Ut = Ue + t * 81 * S;
                const T w[3] = {cf[2 + 3 * t], cf[3 + 3 * t], cf[4 + 3 * t]};
                const T sgn = (ADJ && t != 1) ? T(-1) : T(1);
                const T dgu = sgn * rho * cf[11 + t];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    T gr[3][SV];
                    grad_c(Ut, c, gr);
                    T own[SV];
                    ld_n<T, SV>(Ut + (q * 3 + c) * S + s0, own);
#pragma unroll
                    for (int v = 0; v < SV; ++v) {
                        yu[c][v] = fmaT(dgu, own[v], yu[c][v]);
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            const T G = w[k] * gr[k][v];   // weighted strain component (c, k)
                            if (!ADJ) {
                                // EA upper: stress rows take the weighted strain components
                                if (k == c) ys[c][v] += G;
                                else ys[2 + c + k][v] += G;
                            } else {
                                // transposed EA lower: stress rows take minus C : (weighted strain)
                                if (k == c) {
#pragma unroll
                                    for (int d = 0; d < 3; ++d) ys[d][v] -= sgn * (d == c ? l2 : lam) * G;
                                } else {
                                    ys[2 + c + k][v] -= sgn * m2 * G;
                                }
                            }
                        }
                    }
                }
            }
#pragma unroll
            for (int v = 0; v < SV; ++v) {
#pragma unroll
                for (int d = 0; d < 6; ++d) ys[d][v] *= f0;
#pragma unroll
                for (int c = 0; c < 3; ++c) yu[c][v] *= f0;
            }
        } else {
            // regular domain: stress of the K input's gradient gives the fluxes
            T gr[3][3][SV];
#pragma unroll
            for (int c = 0; c < 3; ++c) grad_c(Ue, c, gr[c]);
            T W[3][3][SV];
#pragma unroll
            for (int v = 0; v < SV; ++v) {
                const T tr = gr[0][0][v] + gr[1][1][v] + gr[2][2][v];
                W[0][0][v] = fmaT(m2, gr[0][0][v], lam * tr);
                W[1][1][v] = fmaT(m2, gr[1][1][v], lam * tr);
                W[2][2][v] = fmaT(m2, gr[2][2][v], lam * tr);
                W[0][1][v] = W[1][0][v] = mu * (gr[0][1][v] + gr[1][0][v]);
                W[0][2][v] = W[2][0][v] = mu * (gr[0][2][v] + gr[2][0][v]);
                W[1][2][v] = W[2][1][v] = mu * (gr[1][2][v] + gr[2][1][v]);
            }
            put_flux(W, T(1));
        }
    }
    __syncthreads();
    if (!active) return;
    // divergence at the node of point q: sum over the points of its three lines
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        double d0, d1, d2;
        gll_col(qm[m], d0, d1, d2);
        const T *pp = V + (el * 27 + base[m]) * 9 * S + s0;
        const int st = kStride[m] * 9 * S;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            T a0[SV], a1[SV], a2[SV];
            ld_n<T, SV>(pp + (c * 3 + m) * S, a0);
            ld_n<T, SV>(pp + st + (c * 3 + m) * S, a1);
            ld_n<T, SV>(pp + 2 * st + (c * 3 + m) * S, a2);
#pragma unroll
            for (int v = 0; v < SV; ++v) yu[c][v] += fmaT(T(d2), a2[v], fmaT(T(d1), a1[v], T(d0) * a0[v]));
        }
    }
    if constexpr (ACC == 0) {
        T *o = A.slots + pq * 9 * S + s0;
#pragma unroll
        for (int c = 0; c < 3; ++c) st_n<T, SV>(o + c * S, yu[c]);
        if constexpr (PML) {
#pragma unroll
            for (int d = 0; d < 6; ++d) st_n<T, SV>(o + (3 + d) * S, ys[d]);
        }
    } else {
        const int *eqo = eqs + (el * 27 + q) * NDOF;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int eq = eqo[c];
            if (eq >= 0) red_n<T, SV>(A.acc + size_t(eq) * S + s0, yu[c]);
        }
        if constexpr (PML) {
#pragma unroll
            for (int d = 0; d < 6; ++d) {
                const int eq = eqo[3 + d];
                if (eq >= 0) red_n<T, SV>(A.acc + size_t(eq) * S + s0, ys[d]);
            }
        }
    }
}

// One thread per (element, GLL point, SV shots).  PART 1 takes the PML
// elements and PART 2 the regular-domain elements, one launch each: the
// regular-domain kernel stages a third of the inputs and keeps fewer values
// live, so it runs four blocks per SM to the PML kernel's two.  PART 0 takes
// both in one launch (the first nb_pml blocks PML, shared memory laid out for
// PML elements), which suits grids of a few waves where a second launch would
// add a tail.  Every part computes an element the same way.  ACC = 0: write the
// element's slot; ACC = 1: add into the row accumulator.
template <typename T, int S, int SV, int ADJ, int ACC, int PART>
__global__ void __launch_bounds__(216, PART == 2 ? 4 : 2) k_elem(const ElemArgs<T> A, const StageArgs<T> a, int stage, int mat)
{
    constexpr int EPB = elems_per_block<S, SV>();
    constexpr bool PML_LAYOUT = PART != 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *U = reinterpret_cast<T *>(smem_raw);
    T *V = U + EPB * elem_u_stride<S, PML_LAYOUT>();
    T *coef = V + EPB * 243 * S;
    int *eqs = reinterpret_cast<int *>(coef + EPB * 27 * elem_ncoef<PML_LAYOUT>());
    const int b = int(blockIdx.x);
    if constexpr (PART == 1) {
        elem_body<T, S, SV, ADJ, ACC, true>(A, a, stage, mat, 0, A.nel_pml, b * EPB, U, V, coef, eqs);
    } else if constexpr (PART == 2) {
        elem_body<T, S, SV, ADJ, ACC, false>(A, a, stage, mat, A.nel_pml, A.nel_rd, b * EPB, U, V, coef, eqs);
    } else {
        if (b < A.nb_pml)
            elem_body<T, S, SV, ADJ, ACC, true>(A, a, stage, mat, 0, A.nel_pml, b * EPB, U, V, coef, eqs);
        else
            elem_body<T, S, SV, ADJ, ACC, false>(A, a, stage, mat, A.nel_pml, A.nel_rd, (b - A.nb_pml) * EPB, U, V, coef, eqs);
    }
}

// PML weights of every node: F3, F2, F1 (directions x, y, z) of the kinds
// e, p, w and the diagonal factors b, c, d.
__global__ void k_pml_weights(int nj, const double *__restrict__ xyz, double *__restrict__ out)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nj) return;
    double ab[10];
    pml_coefs(xyz + size_t(j) * 3, ab);
    double *o = out + size_t(j) * 12;
    o[0] = ab[1] * ab[2]; o[1] = ab[0] * ab[2]; o[2] = ab[0] * ab[1];
    o[3] = ab[1] * ab[5] + ab[2] * ab[4]; o[4] = ab[0] * ab[5] + ab[2] * ab[3]; o[5] = ab[0] * ab[4] + ab[1] * ab[3];
    o[6] = ab[4] * ab[5]; o[7] = ab[3] * ab[5]; o[8] = ab[3] * ab[4];
    o[9] = ab[7]; o[10] = ab[8]; o[11] = ab[9];
}

// Element geometry in processing order.
__global__ void k_gather_geom(int np, const int32_t *__restrict__ order, const double *__restrict__ geom, double *__restrict__ out)
{
    const int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (t >= int64_t(np) * 270) return;
    const int p = int(t / 270), k = int(t % 270);
    out[t] = geom[size_t(order[p]) * 270 + k];
}

template <typename T>
struct NodeArgs {
    const int32_t *row_info;   // [neq] node << 4 | dof
    const int32_t *nptr;       // [nj + 1]
    const uint32_t *nslot;     // processing index * 27 + point, | kRdSlot for regular-domain elements
    const T *slots;
    T *acc;
    const double *im;
};

// Row sum of the element contributions, -iM scaling and the stage epilogue.
template <typename T, int S, int STAGE, int ACC, int MAT>
__global__ void __launch_bounds__(256) k_node(const StageArgs<T> a, const NodeArgs<T> na)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= a.n) return;
    T acc[S];
#pragma unroll
    for (int s = 0; s < S; ++s) acc[s] = T(0);
    if constexpr (ACC == 0) {
        const int info = __ldg(na.row_info + row);
        const int node = info >> 4, dof = info & 15;
        const int k1 = __ldg(na.nptr + node + 1);
        for (int k = __ldg(na.nptr + node); k < k1; ++k) {
            const uint32_t sl = __ldg(na.nslot + k);
            if ((sl & kRdSlot) && dof >= 3) continue;
            T v[S];
            ldv<T, S>(na.slots + (size_t(sl & ~kRdSlot) * 9 + dof) * S, v);
#pragma unroll
            for (int s = 0; s < S; ++s) acc[s] += v[s];
        }
    } else {
        T *p = na.acc + size_t(row) * S;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            acc[s] = p[s];
            p[s] = T(0);
        }
    }
    const T im = T(__ldg(na.im + row));
#pragma unroll
    for (int s = 0; s < S; ++s) acc[s] = -im * acc[s];
    finish_row<T, S, STAGE, MAT>(a, row, acc);
}

// ----------------------------------------------------------------------------
// host side

int elem_prepare(hrn_ctx *c)
{
    if (c->have_elem) return 0;
    if (!c->have_mesh) return set_error(c, HRN_ESTATE, "matrix-free operator needs the mesh");
    static const unsigned char ijk[27][3] = {{2, 0, 0}, {2, 2, 0}, {0, 2, 0}, {0, 0, 0}, {2, 0, 2}, {2, 2, 2}, {0, 2, 2},
                                             {0, 0, 2}, {2, 1, 0}, {1, 2, 0}, {0, 1, 0}, {1, 0, 0}, {2, 0, 1}, {2, 2, 1},
                                             {0, 2, 1}, {0, 0, 1}, {2, 1, 2}, {1, 2, 2}, {0, 1, 2}, {1, 0, 2}, {1, 1, 0},
                                             {2, 1, 1}, {1, 2, 1}, {0, 1, 1}, {1, 0, 1}, {1, 1, 2}, {1, 1, 1}};
    unsigned char node_at[27];
    for (int i = 0; i < 27; ++i) node_at[9 * ijk[i][2] + 3 * ijk[i][1] + ijk[i][0]] = (unsigned char)i;
    HRN_CUDA(c, cudaMemcpyToSymbol(e_pml, c->h_pml.data(), 24 * sizeof(double)));
    // processing order: PML elements, then regular-domain elements
    std::vector<int32_t> order;
    for (int e = 0; e < c->nel; ++e)
        if (c->h_mtel[e] == 2) order.push_back(e);
    c->nel_pml_e = int(order.size());
    for (int e = 0; e < c->nel; ++e)
        if (c->h_mtel[e] == 1) order.push_back(e);
    c->nel_rd_e = int(order.size()) - c->nel_pml_e;
    const int np = int(order.size());
    if (int64_t(np) * 27 >= int64_t(kRdSlot)) return set_error(c, HRN_EARG, "too many elements for the slot index");
    std::vector<int32_t> el_eq(size_t(np) * 243), el_node(size_t(np) * 27);
    std::vector<double> el_rho(std::max(np, 1));
    std::vector<int32_t> nptr(size_t(c->nj) + 1, 0);
    for (int p = 0; p < np; ++p) {
        const int e = order[p];
        el_rho[p] = c->h_rho[e];
        for (int q = 0; q < 27; ++q) {
            const int node = c->h_inod[size_t(e) * 27 + node_at[q]];
            el_node[size_t(p) * 27 + q] = node;
            for (int d = 0; d < 9; ++d) el_eq[(size_t(p) * 27 + q) * 9 + d] = c->h_id[size_t(node) * 9 + d];
            nptr[node + 1]++;
        }
    }
    // slots of each node, ascending processing order
    for (int j = 0; j < c->nj; ++j) nptr[j + 1] += nptr[j];
    std::vector<uint32_t> ns(static_cast<size_t>(nptr[c->nj]));
    std::vector<int32_t> pos(nptr.begin(), nptr.end() - 1);
    for (int p = 0; p < np; ++p)
        for (int q = 0; q < 27; ++q)
            ns[pos[el_node[size_t(p) * 27 + q]]++] = uint32_t(p * 27 + q) | (p >= c->nel_pml_e ? kRdSlot : 0u);
    std::vector<int32_t> info(size_t(c->neq), -1);
    for (int j = 0; j < c->nj; ++j)
        for (int d = 0; d < 9; ++d) {
            const int eq = c->h_id[size_t(j) * 9 + d];
            if (eq >= 0 && eq < c->neq) info[eq] = (j << 4) | d;
        }
    for (int32_t v : info)
        if (v < 0) return set_error(c, HRN_EMESH, "an equation has no (node, DOF) in ID");
    const size_t npa = std::max<size_t>(np, 1);
    HRN_CUDA(c, c->d_el_order.alloc(npa * 4));
    HRN_CUDA(c, c->d_el_eq.alloc(npa * 243 * 4));
    HRN_CUDA(c, c->d_el_node.alloc(npa * 27 * 4));
    HRN_CUDA(c, c->d_el_geom.alloc(npa * 270 * 8));
    HRN_CUDA(c, c->d_el_rho.alloc(npa * 8));
    HRN_CUDA(c, c->d_nslot_ptr.alloc(nptr.size() * 4));
    HRN_CUDA(c, c->d_nslot.alloc(std::max<size_t>(ns.size(), 1) * 4));
    HRN_CUDA(c, c->d_row_info.alloc(info.size() * 4));
    HRN_CUDA(c, c->d_pmlw.alloc(size_t(c->nj) * 12 * 8));
    if (np > 0) {
        HRN_CUDA(c, cudaMemcpy(c->d_el_order.p, order.data(), size_t(np) * 4, cudaMemcpyHostToDevice));
        HRN_CUDA(c, cudaMemcpy(c->d_el_eq.p, el_eq.data(), el_eq.size() * 4, cudaMemcpyHostToDevice));
        HRN_CUDA(c, cudaMemcpy(c->d_el_node.p, el_node.data(), el_node.size() * 4, cudaMemcpyHostToDevice));
        HRN_CUDA(c, cudaMemcpy(c->d_el_rho.p, el_rho.data(), size_t(np) * 8, cudaMemcpyHostToDevice));
        k_gather_geom<<<int((int64_t(np) * 270 + 255) / 256), 256, 0, c->stream>>>(np, c->d_el_order.as<int32_t>(),
                                                                                   c->d_asm_geom.as<double>(), c->d_el_geom.as<double>());
        ++c->launches;
    }
    HRN_CUDA(c, cudaMemcpy(c->d_nslot_ptr.p, nptr.data(), nptr.size() * 4, cudaMemcpyHostToDevice));
    if (!ns.empty()) HRN_CUDA(c, cudaMemcpy(c->d_nslot.p, ns.data(), ns.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_row_info.p, info.data(), info.size() * 4, cudaMemcpyHostToDevice));
    k_pml_weights<<<(c->nj + 255) / 256, 256, 0, c->stream>>>(c->nj, c->d_xyz.as<double>(), c->d_pmlw.as<double>());
    ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    c->have_elem = true;
    return 0;
}

// Slot and accumulator buffers for the current precision and shot count.
static int elem_buffers(hrn_ctx *c)
{
    const size_t S = size_t(c->nshot), eb = c->elem_bytes();
    HRN_CUDA(c, c->d_eslots.alloc(std::max<size_t>(size_t(c->nel_pml_e + c->nel_rd_e), 1) * 27 * 9 * S * eb));
    const size_t accb = size_t(c->neq) * S * eb;
    if (c->d_eacc.bytes != accb) {
        HRN_CUDA(c, c->d_eacc.alloc(accb));
        HRN_CUDA(c, cudaMemsetAsync(c->d_eacc.p, 0, accb, c->stream));
    }
    return 0;
}

template <typename T, int S, int SV, int ADJ, int ACC, int PART>
static void launch_elem(const ElemArgs<T> &A, const StageArgs<T> &a, int stage, int mat, int blocks, cudaStream_t st)
{
    static std::atomic<uint64_t> smem_done{0};
    constexpr size_t smem = elem_smem_bytes<T, S, SV, PART != 2>();
    static_assert(smem <= 227 * 1024, "element kernel block exceeds the shared memory of a CTA");
    smem_limit_once(k_elem<T, S, SV, ADJ, ACC, PART>, int(smem), smem_done);
    k_elem<T, S, SV, ADJ, ACC, PART><<<blocks, elems_per_block<S, SV>() * 27 * (S / SV), smem, st>>>(A, a, stage, mat);
}

template <typename T, int S, int SV, int PART>
static void launch_elem_any(const ElemArgs<T> &A, const StageArgs<T> &a, int stage, int mat, int blocks, int adj, int acc,
                            cudaStream_t st)
{
    if (adj) {
        if (acc) launch_elem<T, S, SV, 1, 1, PART>(A, a, stage, mat, blocks, st);
        else launch_elem<T, S, SV, 1, 0, PART>(A, a, stage, mat, blocks, st);
    } else {
        if (acc) launch_elem<T, S, SV, 0, 1, PART>(A, a, stage, mat, blocks, st);
        else launch_elem<T, S, SV, 0, 0, PART>(A, a, stage, mat, blocks, st);
    }
}

template <typename T, int S>
static int elem_stage_t(hrn_ctx *c, const StageArgs<T> &a, int stage, int adj, int acc, int sv, int mat)
{
    ElemArgs<T> A{};
    A.nel_pml = c->nel_pml_e;
    A.nel_rd = c->nel_rd_e;
    A.el_eq = c->d_el_eq.as<int32_t>();
    A.el_node = c->d_el_node.as<int32_t>();
    A.el_geom = c->d_el_geom.as<double>();
    A.el_rho = c->d_el_rho.as<double>();
    A.lam = c->d_lam.as<double>();
    A.mu = c->d_mu.as<double>();
    A.pmlw = c->d_pmlw.as<double>();
    A.slots = c->d_eslots.as<T>();
    A.acc = c->d_eacc.as<T>();
    auto go = [&](auto svc) {
        constexpr int SV = decltype(svc)::value;
        constexpr int EPB = elems_per_block<S, SV>();
        const int nb_pml = (c->nel_pml_e + EPB - 1) / EPB, nb_rd = (c->nel_rd_e + EPB - 1) / EPB;
        if (nb_pml + nb_rd < kElemSplitBlocksPerSm * c->num_sms) {
            // a few waves: one combined launch
            A.nb_pml = nb_pml;
            if (nb_pml + nb_rd > 0) {
                launch_elem_any<T, S, SV, 0>(A, a, stage, mat, nb_pml + nb_rd, adj, acc, c->stream);
                ++c->launches;
            }
            return;
        }
        if (nb_pml > 0) {
            launch_elem_any<T, S, SV, 1>(A, a, stage, mat, nb_pml, adj, acc, c->stream);
            ++c->launches;
        }
        if (nb_rd > 0) {
            launch_elem_any<T, S, SV, 2>(A, a, stage, mat, nb_rd, adj, acc, c->stream);
            ++c->launches;
        }
    };
    bool done = false;
    if constexpr (S % 4 == 0 && sizeof(T) == 4) {
        if (sv == 4) { go(std::integral_constant<int, 4>{}); done = true; }
    }
    if constexpr (S % 2 == 0) {
        if (!done && sv == 2) { go(std::integral_constant<int, 2>{}); done = true; }
    }
    if (!done) go(std::integral_constant<int, 1>{});
    NodeArgs<T> na{c->d_row_info.as<int32_t>(), c->d_nslot_ptr.as<int32_t>(), c->d_nslot.as<uint32_t>(),
                   c->d_eslots.as<T>(), c->d_eacc.as<T>(), c->d_im.as<double>()};
    const int th = 256, nb = (c->neq + th - 1) / th;
    auto node = [&](auto stc, auto accc, auto matc) {
        k_node<T, S, decltype(stc)::value, decltype(accc)::value, decltype(matc)::value><<<nb, th, 0, c->stream>>>(a, na);
    };
    using I0 = std::integral_constant<int, 0>;
    using I1 = std::integral_constant<int, 1>;
    auto node_st = [&](auto accc, auto matc) {
        switch (stage) {
        case 1: node(std::integral_constant<int, 1>{}, accc, matc); break;
        case 2: node(std::integral_constant<int, 2>{}, accc, matc); break;
        case 3: node(std::integral_constant<int, 3>{}, accc, matc); break;
        default: node(std::integral_constant<int, 4>{}, accc, matc); break;
        }
    };
    if (acc) { if (mat) node_st(I1{}, I1{}); else node_st(I1{}, I0{}); }
    else { if (mat) node_st(I0{}, I1{}); else node_st(I0{}, I0{}); }
    return 0;
}

#define HRN_ELEM_DISPATCH(T)                                                       \
    switch (c->nshot) {                                                            \
    case 1: return elem_stage_t<T, 1>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, acc, sv, mat); \
    case 2: return elem_stage_t<T, 2>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, acc, sv, mat); \
    case 3: return elem_stage_t<T, 3>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, acc, sv, mat); \
    case 4: return elem_stage_t<T, 4>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, acc, sv, mat); \
    case 5: return elem_stage_t<T, 5>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, acc, sv, mat); \
    case 6: return elem_stage_t<T, 6>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, acc, sv, mat); \
    case 7: return elem_stage_t<T, 7>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, acc, sv, mat); \
    default: return elem_stage_t<T, 8>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, acc, sv, mat); \
    }

// One matrix-free RK4 stage (element kernel + node kernel) on the stage
// arguments of the CSR kernels; args points to a StageArgs of the context's precision.
int elem_stage(hrn_ctx *c, const void *args, int stage, int adj, int acc, int sv, int mat)
{
    if (c->precision == HRN_FP64) { HRN_ELEM_DISPATCH(double) }
    HRN_ELEM_DISPATCH(float)
}

// Variants 90-95 (stage inputs materialized by the previous stage) and 100-105
// (rebuilt from x and kb): element slots (even) or atomic row sums (odd) with
// 1, 2 or 4 shots per thread; 2 needs an even shot count, 4 a multiple of 4 in FP32.
bool elem_variant_valid(const hrn_ctx *c, int v)
{
    const int b = v >= 100 ? 100 : 90;
    if (v < b || v > b + 5) return false;
    const int sv = 1 << ((v - b) / 2);
    if (c->nshot % sv != 0) return false;
    return sv < 4 || c->precision == HRN_FP32;
}

int elem_ready(hrn_ctx *c)
{
    if (!c->op_from_mesh) return set_error(c, HRN_ESTATE, "the matrix-free variants need an operator assembled from the mesh");
    if (int rc = elem_prepare(c)) return rc;
    return elem_buffers(c);
}

}  // namespace hrn
