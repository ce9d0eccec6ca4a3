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
#include <vector>

#include "hrn_internal.h"
#include "hrn_stage.cuh"

namespace hrn {

__constant__ unsigned char e_node_at[27];   // local node at GLL point q = 9c + 3b + a
__constant__ double e_pml[24];              // PML_PARAM rows x+, x-, y+, y-, z+, z-; cols alpha0, beta0, L, x0

constexpr uint32_t kRdSlot = 0x80000000u;   // slot of a regular-domain element (displacements only)

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
    const int32_t *el_pml, *el_rd;   // element ids by kind
    int nel_pml, nel_rd, nb_pml;     // counts, blocks of PML elements
    const int32_t *inod, *id;
    const double *xyz, *geom, *lam, *mu, *rho;
    const T *in_m, *in_t, *in_h;     // stage inputs of C, K, G
    T *slots;                        // [nel * 27][9][S]
    T *acc;                          // [neq][S] (atomic variant)
};

template <int S>
constexpr int elems_per_block() { return S >= 8 ? 1 : 8 / S; }

template <typename T, int S>
constexpr size_t elem_smem_bytes()
{
    return size_t(elems_per_block<S>()) * (4 * 27 * 9 * S * sizeof(T) + 27 * sizeof(int));
}

// One thread per (element, GLL point, shot).  ACC = 0: write the element's slot;
// ACC = 1: add into the row accumulator.
template <typename T, int S, int ADJ, int ACC>
__global__ void __launch_bounds__(216, 2) k_elem(const ElemArgs<T> A)
{
    constexpr int EPB = elems_per_block<S>();
    constexpr int NT = EPB * 27 * S;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *U = reinterpret_cast<T *>(smem_raw);                 // [EPB][3][27][9][S] stage inputs
    T *V = U + EPB * 3 * 27 * 9 * S;                        // [EPB][27][3 c][3 m][S] divergence fluxes
    int *nodes = reinterpret_cast<int *>(V + EPB * 27 * 9 * S);   // [EPB][27]

    const bool pml = int(blockIdx.x) < A.nb_pml;
    const int e0 = (pml ? int(blockIdx.x) : int(blockIdx.x) - A.nb_pml) * EPB;
    const int ngrp = pml ? A.nel_pml : A.nel_rd;
    const int32_t *list = pml ? A.el_pml : A.el_rd;

    for (int i = threadIdx.x; i < EPB * 27; i += NT) {
        const int el = i / 27;
        nodes[i] = e0 + el < ngrp ? __ldg(A.inod + size_t(__ldg(list + e0 + el)) * 27 + e_node_at[i % 27]) : -1;
    }
    __syncthreads();
    // stage inputs of the element's nodes (PML: C, K, G inputs x 9 DOF; RD: K input x 3 DOF)
    const int ntag = pml ? 3 : 1, ndof = pml ? 9 : 3;
    const int nitem = EPB * ntag * 27 * ndof;
    for (int it = threadIdx.x; it < nitem; it += NT) {
        const int dof = it % ndof;
        int r = it / ndof;
        const int q = r % 27;
        r /= 27;
        const int t = pml ? r % ntag : 1, el = r / ntag;
        const int node = nodes[el * 27 + q];
        const int eq = node >= 0 ? __ldg(A.id + size_t(node) * 9 + dof) : -1;
        T v[S];
        if (eq >= 0) {
            ldv<T, S>((t == 0 ? A.in_m : (t == 1 ? A.in_t : A.in_h)) + size_t(eq) * S, v);
        } else {
#pragma unroll
            for (int s = 0; s < S; ++s) v[s] = T(0);
        }
        T *dst = U + (((el * 3 + t) * 27 + q) * 9 + dof) * S;
#pragma unroll
        for (int s = 0; s < S; ++s) dst[s] = v[s];
    }
    __syncthreads();

    const int tid = threadIdx.x;
    const int s = tid % S, q = (tid / S) % 27, el = tid / (27 * S);
    const bool active = e0 + el < ngrp;
    const int qm[3] = {q % 3, (q / 3) % 3, q / 9};
    const int base[3] = {q - qm[0], q - 3 * qm[1], q - 9 * qm[2]};
    constexpr int kStride[3] = {1, 3, 9};
    T yu[3] = {T(0), T(0), T(0)};
    T ys[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
    T W[3][3] = {{T(0), T(0), T(0)}, {T(0), T(0), T(0)}, {T(0), T(0), T(0)}};
    T ji[9];
    T f0 = T(0);
    if (active) {
        const int e = __ldg(list + e0 + el);
        const double *g = A.geom + (size_t(e) * 27 + q) * 10;
#pragma unroll
        for (int k = 0; k < 9; ++k) ji[k] = T(__ldg(g + k));
        f0 = T(__ldg(g + 9));
        const int node = nodes[el * 27 + q];
        const T lam = T(__ldg(A.lam + node)), mu = T(__ldg(A.mu + node));
        const T *Ue = U + el * 3 * 27 * 9 * S;
        // du_c/dxi_m at q along the three lines, then g_ck = sum_m du_cm DJI(m,k)
        auto grad = [&](const T *Ut, T (&gr)[3][3]) {
            T du[3][3];
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                double d0, d1, d2;
                gll_row(qm[m], d0, d1, d2);
                const T *p = Ut + base[m] * 9 * S + s;
                const int st = kStride[m] * 9 * S;
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    du[c][m] = fmaT(T(d2), p[2 * st + c * S], fmaT(T(d1), p[st + c * S], T(d0) * p[c * S]));
            }
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    gr[c][k] = fmaT(du[c][2], ji[6 + k], fmaT(du[c][1], ji[3 + k], du[c][0] * ji[k]));
        };
        if (pml) {
            double ab[10];
            pml_coefs(A.xyz + size_t(node) * 3, ab);
            const T rho = T(__ldg(A.rho + e));
#pragma unroll
            for (int t = 0; t < 3; ++t) {
                // direction weights (F3, F2, F1) of kind e / p / w and the diagonal factor b / c / d
                T w[3];
                if (t == 0) { w[0] = T(ab[1] * ab[2]); w[1] = T(ab[0] * ab[2]); w[2] = T(ab[0] * ab[1]); }
                else if (t == 1) {
                    w[0] = T(ab[1] * ab[5] + ab[2] * ab[4]);
                    w[1] = T(ab[0] * ab[5] + ab[2] * ab[3]);
                    w[2] = T(ab[0] * ab[4] + ab[1] * ab[3]);
                } else { w[0] = T(ab[4] * ab[5]); w[1] = T(ab[3] * ab[5]); w[2] = T(ab[3] * ab[4]); }
                const T dg = T(ab[7 + t]);
                const T sg = (ADJ && t != 1) ? T(-1) : T(1);
                const T *Ut = Ue + t * 27 * 9 * S;
                T gr[3][3];
                grad(Ut, gr);
                T G[3][3];
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int k = 0; k < 3; ++k) G[c][k] = w[k] * gr[c][k];
                const T *own = Ut + q * 9 * S + s;
                const T s0 = own[3 * S], s1 = own[4 * S], s2 = own[5 * S], s3 = own[6 * S], s4 = own[7 * S], s5 = own[8 * S];
                if (!ADJ) {
                    // EA upper: stress rows take the weighted strain components at q
                    ys[0] += G[0][0];
                    ys[1] += G[1][1];
                    ys[2] += G[2][2];
                    ys[3] += G[0][1] + G[1][0];
                    ys[4] += G[0][2] + G[2][0];
                    ys[5] += G[1][2] + G[2][1];
                    // EA lower: displacement rows take minus the divergence of w_k (C : s)
                    const T l2 = lam + T(2) * mu, m2 = T(2) * mu;
                    const T sxx = l2 * s0 + lam * (s1 + s2), syy = lam * (s0 + s2) + l2 * s1, szz = lam * (s0 + s1) + l2 * s2;
                    const T sxy = m2 * s3, sxz = m2 * s4, syz = m2 * s5;
                    W[0][0] += w[0] * sxx; W[0][1] += w[1] * sxy; W[0][2] += w[2] * sxz;
                    W[1][0] += w[0] * sxy; W[1][1] += w[1] * syy; W[1][2] += w[2] * syz;
                    W[2][0] += w[0] * sxz; W[2][1] += w[1] * syz; W[2][2] += w[2] * szz;
                } else {
                    // transposed EA lower: stress rows take minus C : (weighted strain)
                    const T l2 = lam + T(2) * mu, m2 = T(2) * mu;
                    ys[0] -= sg * (l2 * G[0][0] + lam * (G[1][1] + G[2][2]));
                    ys[1] -= sg * (lam * (G[0][0] + G[2][2]) + l2 * G[1][1]);
                    ys[2] -= sg * (lam * (G[0][0] + G[1][1]) + l2 * G[2][2]);
                    ys[3] -= sg * m2 * (G[0][1] + G[1][0]);
                    ys[4] -= sg * m2 * (G[0][2] + G[2][0]);
                    ys[5] -= sg * m2 * (G[1][2] + G[2][1]);
                    // transposed EA upper: displacement rows take the divergence of w_k s
                    const T ws0 = sg * w[0], ws1 = sg * w[1], ws2 = sg * w[2];
                    W[0][0] += ws0 * s0; W[0][1] += ws1 * s3; W[0][2] += ws2 * s4;
                    W[1][0] += ws0 * s3; W[1][1] += ws1 * s1; W[1][2] += ws2 * s5;
                    W[2][0] += ws0 * s4; W[2][1] += ws1 * s5; W[2][2] += ws2 * s2;
                }
                // diagonal EM (rho * f) and EN (f, 2 f) blocks
                const T du_ = sg * rho * dg, dn = sg * dg;
                yu[0] += du_ * own[0];
                yu[1] += du_ * own[S];
                yu[2] += du_ * own[2 * S];
                ys[0] += dn * s0;
                ys[1] += dn * s1;
                ys[2] += dn * s2;
                ys[3] += T(2) * dn * s3;
                ys[4] += T(2) * dn * s4;
                ys[5] += T(2) * dn * s5;
            }
#pragma unroll
            for (int d = 0; d < 6; ++d) ys[d] *= f0;
#pragma unroll
            for (int c = 0; c < 3; ++c) yu[c] *= f0;
            if (!ADJ) {
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int k = 0; k < 3; ++k) W[c][k] = -W[c][k];
            }
        } else {
            T gr[3][3];
            grad(Ue + 27 * 9 * S, gr);   // K input
            const T tr = gr[0][0] + gr[1][1] + gr[2][2];
            const T m2 = T(2) * mu;
            W[0][0] = fmaT(m2, gr[0][0], lam * tr);
            W[1][1] = fmaT(m2, gr[1][1], lam * tr);
            W[2][2] = fmaT(m2, gr[2][2], lam * tr);
            W[0][1] = W[1][0] = mu * (gr[0][1] + gr[1][0]);
            W[0][2] = W[2][0] = mu * (gr[0][2] + gr[2][0]);
            W[1][2] = W[2][1] = mu * (gr[1][2] + gr[2][1]);
        }
    }
    // fluxes v_cm = w detJ sum_k DJI(m,k) W_ck for the divergence along the xi_m lines
    {
        T *v = V + (el * 27 + q) * 9 * S + s;
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int m = 0; m < 3; ++m)
                v[(c * 3 + m) * S] = active ? f0 * fmaT(ji[3 * m + 2], W[c][2], fmaT(ji[3 * m + 1], W[c][1], ji[3 * m] * W[c][0]))
                                            : T(0);
    }
    __syncthreads();
    if (!active) return;
    // divergence at the node of point q: sum over the points of its three lines
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        double d0, d1, d2;
        gll_col(qm[m], d0, d1, d2);
        const T *p = V + (el * 27 + base[m]) * 9 * S + s;
        const int st = kStride[m] * 9 * S;
#pragma unroll
        for (int c = 0; c < 3; ++c)
            yu[c] += fmaT(T(d2), p[2 * st + (c * 3 + m) * S], fmaT(T(d1), p[st + (c * 3 + m) * S], T(d0) * p[(c * 3 + m) * S]));
    }
    const int e = __ldg(list + e0 + el);
    if constexpr (ACC == 0) {
        T *o = A.slots + (size_t(e) * 27 + q) * 9 * S + s;
#pragma unroll
        for (int c = 0; c < 3; ++c) o[c * S] = yu[c];
        if (pml) {
#pragma unroll
            for (int d = 0; d < 6; ++d) o[(3 + d) * S] = ys[d];
        }
    } else {
        const int node = nodes[el * 27 + q];
        const int32_t *idn = A.id + size_t(node) * 9;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int eq = __ldg(idn + c);
            if (eq >= 0) atomicAdd(A.acc + size_t(eq) * S + s, yu[c]);
        }
        if (pml) {
#pragma unroll
            for (int d = 0; d < 6; ++d) {
                const int eq = __ldg(idn + 3 + d);
                if (eq >= 0) atomicAdd(A.acc + size_t(eq) * S + s, ys[d]);
            }
        }
    }
}

template <typename T>
struct NodeArgs {
    const int32_t *row_info;   // [neq] node << 4 | dof
    const int32_t *nptr;       // [nj + 1]
    const uint32_t *nslot;     // element * 27 + point, | kRdSlot for regular-domain elements
    const T *slots;
    T *acc;
    const double *im;
};

// Row sum of the element contributions, -iM scaling and the stage epilogue.
template <typename T, int S, int STAGE, int ACC>
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
    finish_row<T, S, STAGE, 1>(a, row, acc);
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
    HRN_CUDA(c, cudaMemcpyToSymbol(e_node_at, node_at, sizeof(node_at)));
    HRN_CUDA(c, cudaMemcpyToSymbol(e_pml, c->h_pml.data(), 24 * sizeof(double)));
    std::vector<int32_t> pml, rd;
    for (int e = 0; e < c->nel; ++e) {
        if (c->h_mtel[e] == 2) pml.push_back(e);
        else if (c->h_mtel[e] == 1) rd.push_back(e);
    }
    c->nel_pml_e = int(pml.size());
    c->nel_rd_e = int(rd.size());
    // slots of each node, ascending element order
    std::vector<int32_t> nptr(size_t(c->nj) + 1, 0);
    for (int e = 0; e < c->nel; ++e) {
        if (c->h_mtel[e] != 1 && c->h_mtel[e] != 2) continue;
        for (int q = 0; q < 27; ++q) nptr[c->h_inod[size_t(e) * 27 + node_at[q]] + 1]++;
    }
    for (int j = 0; j < c->nj; ++j) nptr[j + 1] += nptr[j];
    std::vector<uint32_t> ns(static_cast<size_t>(nptr[c->nj]));
    std::vector<int32_t> pos(nptr.begin(), nptr.end() - 1);
    for (int e = 0; e < c->nel; ++e) {
        if (c->h_mtel[e] != 1 && c->h_mtel[e] != 2) continue;
        for (int q = 0; q < 27; ++q) {
            const int node = c->h_inod[size_t(e) * 27 + node_at[q]];
            ns[pos[node]++] = uint32_t(e * 27 + q) | (c->h_mtel[e] == 1 ? kRdSlot : 0u);
        }
    }
    if (int64_t(c->nel) * 27 >= int64_t(kRdSlot)) return set_error(c, HRN_EARG, "too many elements for the slot index");
    std::vector<int32_t> info(size_t(c->neq), -1);
    for (int j = 0; j < c->nj; ++j)
        for (int d = 0; d < 9; ++d) {
            const int eq = c->h_id[size_t(j) * 9 + d];
            if (eq >= 0 && eq < c->neq) info[eq] = (j << 4) | d;
        }
    for (int32_t v : info)
        if (v < 0) return set_error(c, HRN_EMESH, "an equation has no (node, DOF) in ID");
    HRN_CUDA(c, c->d_el_pml.alloc(std::max<size_t>(pml.size(), 1) * 4));
    HRN_CUDA(c, c->d_el_rde.alloc(std::max<size_t>(rd.size(), 1) * 4));
    HRN_CUDA(c, c->d_nslot_ptr.alloc(nptr.size() * 4));
    HRN_CUDA(c, c->d_nslot.alloc(std::max<size_t>(ns.size(), 1) * 4));
    HRN_CUDA(c, c->d_row_info.alloc(info.size() * 4));
    if (!pml.empty()) HRN_CUDA(c, cudaMemcpy(c->d_el_pml.p, pml.data(), pml.size() * 4, cudaMemcpyHostToDevice));
    if (!rd.empty()) HRN_CUDA(c, cudaMemcpy(c->d_el_rde.p, rd.data(), rd.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_nslot_ptr.p, nptr.data(), nptr.size() * 4, cudaMemcpyHostToDevice));
    if (!ns.empty()) HRN_CUDA(c, cudaMemcpy(c->d_nslot.p, ns.data(), ns.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_row_info.p, info.data(), info.size() * 4, cudaMemcpyHostToDevice));
    c->have_elem = true;
    return 0;
}

// Slot and accumulator buffers for the current precision and shot count.
static int elem_buffers(hrn_ctx *c)
{
    const size_t S = size_t(c->nshot), eb = c->elem_bytes();
    HRN_CUDA(c, c->d_eslots.alloc(size_t(c->nel) * 27 * 9 * S * eb));
    const size_t accb = size_t(c->neq) * S * eb;
    if (c->d_eacc.bytes != accb) {
        HRN_CUDA(c, c->d_eacc.alloc(accb));
        HRN_CUDA(c, cudaMemsetAsync(c->d_eacc.p, 0, accb, c->stream));
    }
    return 0;
}

template <typename T, int S, int ADJ, int ACC>
static void launch_elem(const ElemArgs<T> &A, int blocks, cudaStream_t st)
{
    static bool attr_set = false;
    constexpr size_t smem = elem_smem_bytes<T, S>();
    if (!attr_set) {
        cudaFuncSetAttribute(k_elem<T, S, ADJ, ACC>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        attr_set = true;
    }
    k_elem<T, S, ADJ, ACC><<<blocks, elems_per_block<S>() * 27 * S, smem, st>>>(A);
}

template <typename T, int S>
static int elem_stage_t(hrn_ctx *c, const StageArgs<T> &a, int stage, int adj, int acc)
{
    constexpr int EPB = elems_per_block<S>();
    ElemArgs<T> A{};
    A.el_pml = c->d_el_pml.as<int32_t>();
    A.el_rd = c->d_el_rde.as<int32_t>();
    A.nel_pml = c->nel_pml_e;
    A.nel_rd = c->nel_rd_e;
    A.nb_pml = (c->nel_pml_e + EPB - 1) / EPB;
    A.inod = c->d_inod.as<int32_t>();
    A.id = c->d_id.as<int32_t>();
    A.xyz = c->d_xyz.as<double>();
    A.geom = c->d_asm_geom.as<double>();
    A.lam = c->d_lam.as<double>();
    A.mu = c->d_mu.as<double>();
    A.rho = c->d_rho.as<double>();
    if (stage == 1) { A.in_m = a.x3; A.in_t = a.x2; A.in_h = a.x1; }
    else { A.in_m = a.in_m; A.in_t = a.in_t; A.in_h = a.in_h; }
    A.slots = c->d_eslots.as<T>();
    A.acc = c->d_eacc.as<T>();
    const int blocks = A.nb_pml + (c->nel_rd_e + EPB - 1) / EPB;
    if (blocks > 0) {
        if (adj) {
            if (acc) launch_elem<T, S, 1, 1>(A, blocks, c->stream);
            else launch_elem<T, S, 1, 0>(A, blocks, c->stream);
        } else {
            if (acc) launch_elem<T, S, 0, 1>(A, blocks, c->stream);
            else launch_elem<T, S, 0, 0>(A, blocks, c->stream);
        }
        ++c->launches;
    }
    NodeArgs<T> na{c->d_row_info.as<int32_t>(), c->d_nslot_ptr.as<int32_t>(), c->d_nslot.as<uint32_t>(),
                   c->d_eslots.as<T>(), c->d_eacc.as<T>(), c->d_im.as<double>()};
    const int th = 256, nb = (c->neq + th - 1) / th;
    switch (stage * 2 + (acc ? 1 : 0)) {
    case 2: k_node<T, S, 1, 0><<<nb, th, 0, c->stream>>>(a, na); break;
    case 3: k_node<T, S, 1, 1><<<nb, th, 0, c->stream>>>(a, na); break;
    case 4: k_node<T, S, 2, 0><<<nb, th, 0, c->stream>>>(a, na); break;
    case 5: k_node<T, S, 2, 1><<<nb, th, 0, c->stream>>>(a, na); break;
    case 6: k_node<T, S, 3, 0><<<nb, th, 0, c->stream>>>(a, na); break;
    case 7: k_node<T, S, 3, 1><<<nb, th, 0, c->stream>>>(a, na); break;
    case 8: k_node<T, S, 4, 0><<<nb, th, 0, c->stream>>>(a, na); break;
    default: k_node<T, S, 4, 1><<<nb, th, 0, c->stream>>>(a, na); break;
    }
    return 0;
}

#define HRN_ELEM_DISPATCH(T)                                                       \
    switch (c->nshot) {                                                            \
    case 1: return elem_stage_t<T, 1>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, acc); \
    case 2: return elem_stage_t<T, 2>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, acc); \
    case 3: return elem_stage_t<T, 3>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, acc); \
    case 4: return elem_stage_t<T, 4>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, acc); \
    case 5: return elem_stage_t<T, 5>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, acc); \
    case 6: return elem_stage_t<T, 6>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, acc); \
    case 7: return elem_stage_t<T, 7>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, acc); \
    default: return elem_stage_t<T, 8>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, acc); \
    }

// One matrix-free RK4 stage (element kernel + node kernel) on the stage
// arguments of the CSR kernels; args points to a StageArgs of the context's precision.
int elem_stage(hrn_ctx *c, const void *args, int stage, int adj, int acc)
{
    if (c->precision == HRN_FP64) { HRN_ELEM_DISPATCH(double) }
    HRN_ELEM_DISPATCH(float)
}

int elem_ready(hrn_ctx *c)
{
    if (!c->op_from_mesh) return set_error(c, HRN_ESTATE, "the matrix-free variants need an operator assembled from the mesh");
    if (int rc = elem_prepare(c)) return rc;
    return elem_buffers(c);
}

}  // namespace hrn
