// hrn_assemble.cu -- device assembly of C, K, G and DIAG_M for the 27-node GLL
// spectral hexahedra: ASSEM_REGULAR_DOMAIN_PETSC_3D (S4/Assemble_PETSc_3D.F90:6-184)
// with ELEMENT_K_3D / ELEMENT_M_3D (S4/Element_Matrices_3D.F90:7-415) and
// ASSEM_PML_PETSC_3D (:192-436) with ELEMENT_M/EN/EA_3D (:228-882).
//
// With the 3-point GLL rule (GAUSS, S4/Source1.F90:29-31) every shape function
// is a Kronecker delta at the quadrature points and dN_I/dxi_m(q) vanishes
// unless I lies on the xi_m line through q.  Hence
//   * mass-type blocks (M, EM_a..d, EN_a..d) are diagonal: one point q = I;
//   * EA(I c, J d) only receives the point q = J;
//   * EK(I c, J d) only receives the points where both I and J lie on a line
//     through q (at most 7; 513 of the 729 node pairs are reachable).
// Each thread computes one element-matrix entry over its points in the
// reference's point order with the reference's left-to-right arithmetic
// (no fused multiply-add), then adds it to the global CSR entry.  Elements are
// processed colour by colour (no two elements of a colour share a node), so
// the adds need no atomics and the result is reproducible.
//
// The first assembly discovers the sparsity pattern the way MAT_IGNORE_ZERO_ENTRIES
// does (an entry exists when some element contributes a nonzero value): every
// nonzero contribution emits a (row, matrix, column) key, keys are sorted and
// made unique on the device, and the combined C|K|G CSR plus its transpose are
// built from them.
#include <cuda_runtime.h>
#include <thrust/device_ptr.h>
#include <thrust/execution_policy.h>
#include <thrust/merge.h>
#include <thrust/sort.h>
#include <thrust/unique.h>

#include <algorithm>
#include <vector>

#include "hrn_internal.h"

namespace hrn {

__constant__ unsigned char a_ijk[27][3];    // (xi, eta, zeta) index of each local node
__constant__ unsigned char a_node_at[27];   // local node at GLL point q = 9c + 3b + a
__constant__ double a_D[3][3];              // a_D[a][b] = l_b'(xi_a)
__constant__ unsigned char a_kI[513], a_kJ[513], a_kn[513], a_kq[513][7];
__constant__ unsigned char a_eaI[189], a_eaJ[189];

struct AsmArgs {
    const int32_t *elems;      // element ids of this colour
    int nel;
    const int32_t *inod, *id;
    const double *xyz, *geom, *lam, *mu, *rho, *pml;
    // values mode
    const int32_t *rowptr;
    const uint32_t *colx;
    double *raw, *diag_m;
    // discover mode
    int discover;
    int no_csr;                 // matrix-free operator: DIAG_M only, no CSR entries
    unsigned long long *count;
    unsigned long long cap;
    uint64_t *keys;
    int *err;
};

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }

// DFXI(I, m) at GLL point q (exact table values).
__device__ __forceinline__ double dfxi(int I, int m, int q)
{
    const int qa = q % 3, qb = (q / 3) % 3, qc = q / 9;
    const int ia = a_ijk[I][0], ib = a_ijk[I][1], ic = a_ijk[I][2];
    if (m == 0) return (ib == qb && ic == qc) ? a_D[qa][ia] : 0.0;
    if (m == 1) return (ia == qa && ic == qc) ? a_D[qb][ib] : 0.0;
    return (ia == qa && ib == qb) ? a_D[qc][ic] : 0.0;
}

// DFX(I, k) = sum_m DFXI(I, m) DJI(m, k), summed over m = 1..3 like MATMUL.
__device__ __forceinline__ void dfx_row(int I, int q, const double *ji, double out[3])
{
    const double d0 = dfxi(I, 0, q), d1 = dfxi(I, 1, q), d2 = dfxi(I, 2, q);
#pragma unroll
    for (int k = 0; k < 3; ++k) out[k] = add(add(add(0.0, mul(d0, ji[k])), mul(d1, ji[3 + k])), mul(d2, ji[6 + k]));
}

// PML_FINDER_3D (S4/PML.F90:325-891) with polynomial degree 2 and ratio 0:
// returns alpha_x..z (0-2), beta_x..z (3-5) and a, b, c, d (6-9).
__device__ bool pml_ab(const double *x, const double *P, double A[10])
{
    A[0] = 1.0; A[1] = 1.0; A[2] = 1.0; A[3] = 0.0; A[4] = 0.0; A[5] = 0.0;
    // P[r*4 + col]: rows x+, x-, y+, y-, z+, z-; cols alpha0, beta0, L, x0
    for (int ax = 0; ax < 2; ++ax) {
        int r = -1;
        if (x[ax] >= P[(2 * ax) * 4 + 3]) r = 2 * ax;
        else if (x[ax] <= P[(2 * ax + 1) * 4 + 3]) r = 2 * ax + 1;
        if (r >= 0) {
            const double vn = (r == 2 * ax) ? 1.0 : -1.0;
            const double f = (x[ax] - P[r * 4 + 3]) * vn / P[r * 4 + 2];
            const double pa = mul(f, f);
            A[ax] = add(A[ax], mul(P[r * 4 + 0], pa));
            A[3 + ax] = add(A[3 + ax], mul(P[r * 4 + 1], pa));
        }
    }
    if (x[2] > P[4 * 4 + 3]) return false;   // top zone (the reference stops)
    if (x[2] <= P[5 * 4 + 3]) {
        const double f = (x[2] - P[5 * 4 + 3]) * -1.0 / P[5 * 4 + 2];
        const double pa = mul(f, f);
        A[2] = add(A[2], mul(P[5 * 4 + 0], pa));
        A[5] = add(A[5], mul(P[5 * 4 + 1], pa));
    }
    A[6] = mul(mul(A[0], A[1]), A[2]);
    A[7] = add(add(mul(mul(A[0], A[1]), A[5]), mul(mul(A[0], A[2]), A[4])), mul(mul(A[1], A[2]), A[3]));
    A[8] = add(add(mul(mul(A[0], A[4]), A[5]), mul(mul(A[1], A[3]), A[5])), mul(mul(A[2], A[3]), A[4]));
    A[9] = mul(mul(A[3], A[4]), A[5]);
    return true;
}

__device__ __forceinline__ void put(const AsmArgs &A, int row, int col, int tag, double v)
{
    if (row < 0 || col < 0 || v == 0.0 || A.no_csr) return;   // PETSc: negative index ignored, zero not inserted
    if (A.discover) {
        const unsigned long long k = atomicAdd(A.count, 1ull);
        if (k < A.cap) A.keys[k] = (uint64_t(uint32_t(row)) << 32) | (uint64_t(tag) << kTagBits) | uint64_t(col);
        else atomicExch(A.err, 2);
        return;
    }
    const uint32_t key = (uint32_t(tag) << kTagBits) | uint32_t(col);
    int lo = A.rowptr[row], hi = A.rowptr[row + 1] - 1;
    while (lo <= hi) {
        const int mid = lo + ((hi - lo) >> 1);   // no overflow past 2^30 entries
        const uint32_t m = A.colx[mid];
        if (m == key) { A.raw[mid] = add(A.raw[mid], v); return; }
        if (m < key) lo = mid + 1; else hi = mid - 1;
    }
    atomicExch(A.err, 3);   // contribution outside the pattern fixed by the first assembly
}

// One thread per (element, K node pair, c, d): EK of ELEMENT_K_3D (S4/Element_Matrices_3D.F90:160-210).
__global__ void k_asm_rd_k(AsmArgs A)
{
    const int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (t >= int64_t(A.nel) * 513 * 9) return;
    const int cd = int(t % 9), p = int((t / 9) % 513);
    const int e = A.elems[t / (9 * 513)];
    const int c = cd / 3, d = cd % 3;
    const int I = a_kI[p], J = a_kJ[p];
    const int32_t *nd = A.inod + size_t(e) * 27;
    double s = 0.0;
    for (int u = 0; u < a_kn[p]; ++u) {
        const int q = a_kq[p][u];
        const double *g = A.geom + (size_t(e) * 27 + q) * 10;
        double fi[3], fj[3];
        dfx_row(I, q, g, fi);
        dfx_row(J, q, g, fj);
        const int nq = nd[a_node_at[q]];
        const double zl = A.lam[nq], zm = A.mu[nq];
        const double f1 = add(zl, mul(2.0, zm)), f2 = zl, f3 = zm;
        // G(c,d) of ELEMENT_K_3D, H_ab = DFX(I,a) DFX(J,b)
        double G;
        if (c == d) {
            const int o1 = (c + 1) % 3, o2 = (c + 2) % 3;
            // G1 = f1 H11 + f3 (H22 + H33) for c = x; cyclic forms for y, z keep the reference order
            const double hc = mul(fi[c], fj[c]);
            double ha, hb;
            if (c == 0) { ha = mul(fi[1], fj[1]); hb = mul(fi[2], fj[2]); }
            else if (c == 1) { ha = mul(fi[0], fj[0]); hb = mul(fi[2], fj[2]); }
            else { ha = mul(fi[0], fj[0]); hb = mul(fi[1], fj[1]); }
            (void)o1; (void)o2;
            G = add(mul(f1, hc), mul(f3, add(ha, hb)));
        } else {
            // off-diagonal blocks: G = f2 * DFX(I,c) DFX(J,d) + f3 * DFX(I,d) DFX(J,c)
            G = add(mul(f2, mul(fi[c], fj[d])), mul(f3, mul(fi[d], fj[c])));
        }
        s = add(s, mul(G, g[9]));
    }
    put(A, A.id[size_t(nd[I]) * 9 + c], A.id[size_t(nd[J]) * 9 + d], 1, s);
}

// One thread per (element, local node): diagonal mass of the RD (ELEMENT_M_3D, flag 201),
// and for PML elements the diagonal blocks EM_a..d (flags 202-205), EN_a..d (301-304).
__global__ void k_asm_diag(AsmArgs A, int pml)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.nel * 27) return;
    const int I = t % 27;
    const int e = A.elems[t / 27];
    const int node = A.inod[size_t(e) * 27 + I];
    const int q = 9 * a_ijk[I][2] + 3 * a_ijk[I][1] + a_ijk[I][0];
    const double fac0 = A.geom[(size_t(e) * 27 + q) * 10 + 9];
    const double rho = A.rho[e];
    const int32_t *idn = A.id + size_t(node) * 9;
    if (!pml) {
        const double v = mul(mul(rho, 1.0), fac0);   // (RO * FN(I) FN(I)) * FAC0
        if (A.discover) return;
        for (int cc = 0; cc < 3; ++cc)
            if (idn[cc] >= 0) A.diag_m[idn[cc]] = add(A.diag_m[idn[cc]], v);
        return;
    }
    double ab[10];
    const double *x = A.xyz + size_t(node) * 3;
    if (!pml_ab(x, A.pml, ab)) { atomicExch(A.err, 4); return; }
    // EM_f (u) and EN_f (s) diagonal values for f = a, b, c, d
    for (int f = 0; f < 4; ++f) {
        const double fm = mul(rho, ab[6 + f]);
        const double vu = mul(mul(fm, 1.0), fac0);
        const double vs1 = mul(mul(ab[6 + f], 1.0), fac0);
        const double vs2 = mul(mul(mul(2.0, ab[6 + f]), 1.0), fac0);
        if (f == 0) {
            if (A.discover) continue;
            for (int cc = 0; cc < 3; ++cc)
                if (idn[cc] >= 0) A.diag_m[idn[cc]] = add(A.diag_m[idn[cc]], vu);
            for (int cc = 0; cc < 6; ++cc)
                if (idn[3 + cc] >= 0) A.diag_m[idn[3 + cc]] = add(A.diag_m[idn[3 + cc]], cc < 3 ? vs1 : vs2);
            continue;
        }
        for (int cc = 0; cc < 3; ++cc) put(A, idn[cc], idn[cc], f - 1, vu);
        for (int cc = 0; cc < 6; ++cc) put(A, idn[3 + cc], idn[3 + cc], f - 1, cc < 3 ? vs1 : vs2);
    }
}

// One thread per (element, EA pair (I, J), c, d, kind e/p/w): the upper EA value goes
// to (stress J d, displacement I c), minus the lower EA value to (I c, J d)
// (S4/Assemble_PETSc_3D.F90:409-420; ELEMENT_EA_3D, S4/Element_Matrices_3D.F90:618-882).
__global__ void k_asm_ea(AsmArgs A)
{
    const int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (t >= int64_t(A.nel) * 189 * 18 * 3) return;
    const int kind = int(t % 3);
    const int cd = int((t / 3) % 18);
    const int p = int((t / 54) % 189);
    const int e = A.elems[t / (54 * 189)];
    const int c = cd / 6, d = cd % 6;
    // structural zeros EA(I1,J6), EA(I2,J5), EA(I3,J4)
    if ((c == 0 && d == 5) || (c == 1 && d == 4) || (c == 2 && d == 3)) return;
    const int I = a_eaI[p], J = a_eaJ[p];
    const int32_t *nd = A.inod + size_t(e) * 27;
    const int q = 9 * a_ijk[J][2] + 3 * a_ijk[J][1] + a_ijk[J][0];
    const double *g = A.geom + (size_t(e) * 27 + q) * 10;
    const int nq = nd[J];
    double ab[10];
    if (!pml_ab(A.xyz + size_t(nq) * 3, A.pml, ab)) { atomicExch(A.err, 4); return; }
    double F1, F2, F3;
    if (kind == 0) { F1 = mul(ab[0], ab[1]); F2 = mul(ab[0], ab[2]); F3 = mul(ab[1], ab[2]); }
    else if (kind == 1) {
        F1 = add(mul(ab[0], ab[4]), mul(ab[1], ab[3]));
        F2 = add(mul(ab[0], ab[5]), mul(ab[2], ab[3]));
        F3 = add(mul(ab[1], ab[5]), mul(ab[2], ab[4]));
    } else { F1 = mul(ab[3], ab[4]); F2 = mul(ab[3], ab[5]); F3 = mul(ab[4], ab[5]); }
    double fi[3];
    dfx_row(I, q, g, fi);
    const double h1 = mul(fi[0], 1.0), h2 = mul(fi[1], 1.0), h3 = mul(fi[2], 1.0), h4 = (I == J) ? 1.0 : 0.0;
    const double zl = A.lam[nq], zm = A.mu[nq];
    double vals[2];
    for (int lower = 0; lower < 2; ++lower) {
        const double f7 = lower ? add(zl, mul(2.0, zm)) : 1.0;
        const double f8 = lower ? zl : 0.0;
        const double f9 = lower ? mul(2.0, zm) : 1.0;
        const double f10 = lower ? 0.0 : 1.0;
        // FAC4..FAC6 vanish with ratio 0; f10 * 0 * h4 keeps the reference's terms
        const double z = mul(mul(f10, 0.0), h4);
        double G;
        switch (c * 6 + d) {
        case 0: G = add(mul(mul(f7, F3), h1), z); break;       // G1
        case 1: case 2: G = mul(mul(f8, F3), h1); break;      // G2
        case 3: G = add(mul(mul(f9, F2), h2), z); break;       // G3
        case 4: G = add(mul(mul(f9, F1), h3), z); break;       // G4
        case 6: case 8: G = mul(mul(f8, F2), h2); break;      // G5
        case 7: G = add(mul(mul(f7, F2), h2), z); break;       // G6
        case 9: G = add(mul(mul(f9, F3), h1), z); break;       // G7
        case 11: G = add(mul(mul(f9, F1), h3), z); break;      // G4
        case 12: case 13: G = mul(mul(f8, F1), h3); break;    // G8
        case 14: G = add(mul(mul(f7, F1), h3), z); break;      // G9
        case 16: G = add(mul(mul(f9, F3), h1), z); break;      // G7
        default: G = add(mul(mul(f9, F2), h2), z); break;      // 17: G3
        }
        vals[lower] = mul(G, g[9]);
    }
    const int ui = A.id[size_t(nd[I]) * 9 + c];
    const int sj = A.id[size_t(nd[J]) * 9 + 3 + d];
    put(A, sj, ui, kind, vals[0]);
    put(A, ui, sj, kind, -vals[1]);
}

__global__ void k_inv_mass(int n, const double *__restrict__ dm, double *__restrict__ im)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) im[i] = dm[i] != 0.0 ? 1.0 / dm[i] : 0.0;
}

// ----------------------------------------------------------------------------
// host side

static int upload_asm_tables(hrn_ctx *c)
{
    static const unsigned char ijk[27][3] = {{2, 0, 0}, {2, 2, 0}, {0, 2, 0}, {0, 0, 0}, {2, 0, 2}, {2, 2, 2}, {0, 2, 2},
                                             {0, 0, 2}, {2, 1, 0}, {1, 2, 0}, {0, 1, 0}, {1, 0, 0}, {2, 0, 1}, {2, 2, 1},
                                             {0, 2, 1}, {0, 0, 1}, {2, 1, 2}, {1, 2, 2}, {0, 1, 2}, {1, 0, 2}, {1, 1, 0},
                                             {2, 1, 1}, {1, 2, 1}, {0, 1, 1}, {1, 0, 1}, {1, 1, 2}, {1, 1, 1}};
    unsigned char node_at[27];
    for (int i = 0; i < 27; ++i) node_at[9 * ijk[i][2] + 3 * ijk[i][1] + ijk[i][0]] = (unsigned char)i;
    auto on_lines = [&](int I, int q) {
        const int a = q % 3, b = (q / 3) % 3, cc = q / 9;
        return (ijk[I][1] == b && ijk[I][2] == cc) || (ijk[I][0] == a && ijk[I][2] == cc) || (ijk[I][0] == a && ijk[I][1] == b);
    };
    unsigned char kI[513], kJ[513], kn[513], kq[513][7];
    int np = 0;
    for (int I = 0; I < 27; ++I)
        for (int J = 0; J < 27; ++J) {
            int n = 0;
            unsigned char qs[27];
            for (int q = 0; q < 27; ++q)
                if (on_lines(I, q) && on_lines(J, q)) qs[n++] = (unsigned char)q;
            if (!n) continue;
            if (np >= 513 || n > 7) return set_error(c, HRN_ESTATE, "internal: element pair table overflow");
            kI[np] = (unsigned char)I; kJ[np] = (unsigned char)J; kn[np] = (unsigned char)n;
            for (int u = 0; u < 7; ++u) kq[np][u] = u < n ? qs[u] : 0;
            ++np;
        }
    if (np != 513) return set_error(c, HRN_ESTATE, "internal: element pair table size");
    unsigned char eI[189], eJ[189];
    int ne = 0;
    for (int J = 0; J < 27; ++J) {
        const int q = 9 * ijk[J][2] + 3 * ijk[J][1] + ijk[J][0];
        for (int I = 0; I < 27; ++I)
            if (on_lines(I, q)) { eI[ne] = (unsigned char)I; eJ[ne] = (unsigned char)J; ++ne; }
    }
    if (ne != 189) return set_error(c, HRN_ESTATE, "internal: EA pair table size");
    const double D[3][3] = {{-1.5, 2.0, -0.5}, {-0.5, 0.0, 0.5}, {0.5, -2.0, 1.5}};
    HRN_CUDA(c, cudaMemcpyToSymbol(a_ijk, ijk, sizeof(ijk)));
    HRN_CUDA(c, cudaMemcpyToSymbol(a_node_at, node_at, sizeof(node_at)));
    HRN_CUDA(c, cudaMemcpyToSymbol(a_D, D, sizeof(D)));
    HRN_CUDA(c, cudaMemcpyToSymbol(a_kI, kI, sizeof(kI)));
    HRN_CUDA(c, cudaMemcpyToSymbol(a_kJ, kJ, sizeof(kJ)));
    HRN_CUDA(c, cudaMemcpyToSymbol(a_kn, kn, sizeof(kn)));
    HRN_CUDA(c, cudaMemcpyToSymbol(a_kq, kq, sizeof(kq)));
    HRN_CUDA(c, cudaMemcpyToSymbol(a_eaI, eI, sizeof(eI)));
    HRN_CUDA(c, cudaMemcpyToSymbol(a_eaJ, eJ, sizeof(eJ)));
    return 0;
}

// Greedy element colouring: elements of one colour share no node.
static int build_colors(hrn_ctx *c)
{
    const int nel = c->nel, nj = c->nj;
    std::vector<int> cnt(size_t(nj) + 1, 0);
    for (int e = 0; e < nel; ++e)
        for (int i = 0; i < 27; ++i) cnt[c->h_inod[size_t(e) * 27 + i] + 1]++;
    for (int j = 0; j < nj; ++j) cnt[j + 1] += cnt[j];
    std::vector<int> adj(static_cast<size_t>(cnt[nj])), pos(cnt.begin(), cnt.end() - 1);
    for (int e = 0; e < nel; ++e)
        for (int i = 0; i < 27; ++i) adj[pos[c->h_inod[size_t(e) * 27 + i]]++] = e;
    std::vector<int> color(size_t(nel), -1);
    int ncol = 0;
    std::vector<int> mark;
    for (int e = 0; e < nel; ++e) {
        mark.assign(size_t(ncol) + 1, 0);
        for (int i = 0; i < 27; ++i) {
            const int j = c->h_inod[size_t(e) * 27 + i];
            for (int k = cnt[j]; k < cnt[j + 1]; ++k) {
                const int o = adj[k];
                if (color[o] >= 0) mark[color[o]] = 1;
            }
        }
        int col = 0;
        while (col < ncol && mark[col]) ++col;
        color[e] = col;
        if (col == ncol) ++ncol;
    }
    // per colour: RD elements, then PML elements
    std::vector<int32_t> list;
    c->color_off.assign(1, 0);
    for (int col = 0; col < ncol; ++col)
        for (int kind = 1; kind <= 2; ++kind) {
            for (int e = 0; e < nel; ++e)
                if (color[e] == col && c->h_mtel[e] == kind) list.push_back(e);
            c->color_off.push_back(int(list.size()));
        }
    HRN_CUDA(c, c->d_el_color_list.alloc(list.size() * 4));
    HRN_CUDA(c, cudaMemcpy(c->d_el_color_list.p, list.data(), list.size() * 4, cudaMemcpyHostToDevice));
    return 0;
}

// The kernels of elements [off, off + n) of one (colour, kind) group.
static int run_group(hrn_ctx *c, AsmArgs A, int g, int off, int n)
{
    const int th = 256;
    if (n <= 0) return 0;
    A.elems = c->d_el_color_list.as<int32_t>() + c->color_off[g] + off;
    A.nel = n;
    const bool pml = (g % 2) == 1;
    k_asm_diag<<<(n * 27 + th - 1) / th, th, 0, c->stream>>>(A, pml ? 1 : 0); ++c->launches;
    if (!pml) {
        const int64_t tot = int64_t(n) * 513 * 9;
        k_asm_rd_k<<<unsigned((tot + th - 1) / th), th, 0, c->stream>>>(A); ++c->launches;
    } else {
        const int64_t tot = int64_t(n) * 189 * 54;
        k_asm_ea<<<unsigned((tot + th - 1) / th), th, 0, c->stream>>>(A); ++c->launches;
    }
    HRN_CUDA(c, cudaGetLastError());
    return 0;
}

static int run_kernels(hrn_ctx *c, AsmArgs A)
{
    const int ngroups = int(c->color_off.size()) - 1;   // (colour, kind) groups
    for (int g = 0; g < ngroups; ++g)
        if (int rc = run_group(c, A, g, 0, c->color_off[g + 1] - c->color_off[g])) return rc;
    return 0;
}

// Most candidate keys one element of a kind can emit (diagonal, stiffness, PML blocks).
constexpr unsigned long long kKeysRd = 513ull * 9, kKeysPml = 27ull * 9 + 189ull * 15 * 2 * 3;
constexpr unsigned long long kKeysPerSlice = 1ull << 29;   // 4 GiB of candidate keys per slice

// Matrix-free operator: only DIAG_M and its inverse (the element kernels apply C, K
// and G from the mesh and the nodal material).
static int assemble_mass_only(hrn_ctx *c, AsmArgs A)
{
    const int th = 256;
    HRN_CUDA(c, c->d_diag_m.alloc(size_t(c->neq) * 8));
    HRN_CUDA(c, c->d_im.alloc(size_t(c->neq) * 8));
    HRN_CUDA(c, cudaMemsetAsync(c->d_diag_m.p, 0, size_t(c->neq) * 8, c->stream));
    A.discover = 0;
    A.no_csr = 1;
    A.diag_m = c->d_diag_m.as<double>();
    const int ngroups = int(c->color_off.size()) - 1;
    for (int g = 0; g < ngroups; ++g) {
        const int n = c->color_off[g + 1] - c->color_off[g];
        if (n == 0) continue;
        A.elems = c->d_el_color_list.as<int32_t>() + c->color_off[g];
        A.nel = n;
        k_asm_diag<<<(n * 27 + th - 1) / th, th, 0, c->stream>>>(A, (g % 2) == 1 ? 1 : 0); ++c->launches;
        HRN_CUDA(c, cudaGetLastError());
    }
    k_inv_mass<<<(c->neq + 255) / 256, 256, 0, c->stream>>>(c->neq, c->d_diag_m.as<double>(), c->d_im.as<double>()); ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    int err = 0;
    HRN_CUDA(c, cudaMemcpyAsync(&err, c->d_asm_err.p, 4, cudaMemcpyDeviceToHost, c->stream));
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    if (err == 4) return set_error(c, HRN_EMESH, "a PML point lies in the top PML zone");
    if (err) return set_error(c, HRN_ESTATE, "internal: assembly error flag");
    return 0;
}

int assemble_device(hrn_ctx *c, bool discover_pattern)
{
    if (int rc = upload_asm_tables(c)) return rc;
    if (c->color_off.empty())
        if (int rc = build_colors(c)) return rc;
    AsmArgs A{};
    A.inod = c->d_inod.as<int32_t>();
    A.id = c->d_id.as<int32_t>();
    A.xyz = c->d_xyz.as<double>();
    A.geom = c->d_asm_geom.as<double>();
    A.lam = c->d_lam.as<double>();
    A.mu = c->d_mu.as<double>();
    A.rho = c->d_rho.as<double>();
    A.pml = c->d_pml.as<double>();
    A.err = c->d_asm_err.as<int>();
    HRN_CUDA(c, cudaMemsetAsync(c->d_asm_err.p, 0, 16, c->stream));
    if (c->mf_only) return assemble_mass_only(c, A);
    if (discover_pattern) {
        // Candidate keys slice by slice of each (colour, kind) group: each slice's keys
        // are sorted and made unique, then merged into the sorted set of all keys so
        // far, so device memory stays bounded by one slice plus the final pattern.
        DevBuf keys, count, acc, tmp;
        HRN_CUDA(c, keys.alloc(size_t(kKeysPerSlice) * 8));
        HRN_CUDA(c, count.alloc(8));
        size_t na = 0;
        A.discover = 1;
        A.keys = keys.as<uint64_t>();
        A.count = count.as<unsigned long long>();
        const int ngroups = int(c->color_off.size()) - 1;
        for (int g = 0; g < ngroups; ++g) {
            const int ng = c->color_off[g + 1] - c->color_off[g];
            const unsigned long long per = (g % 2) == 1 ? kKeysPml : kKeysRd;
            const int slice = int(std::max<unsigned long long>(1, kKeysPerSlice / per));
            for (int off = 0; off < ng; off += slice) {
                const int n = std::min(slice, ng - off);
                A.cap = (unsigned long long)n * per;
                HRN_CUDA(c, cudaMemsetAsync(count.p, 0, 8, c->stream));
                if (int rc = run_group(c, A, g, off, n)) return rc;
                unsigned long long nk = 0;
                int err = 0;
                HRN_CUDA(c, cudaMemcpyAsync(&nk, count.p, 8, cudaMemcpyDeviceToHost, c->stream));
                HRN_CUDA(c, cudaMemcpyAsync(&err, c->d_asm_err.p, 4, cudaMemcpyDeviceToHost, c->stream));
                HRN_CUDA(c, cudaStreamSynchronize(c->stream));
                if (err == 4) return set_error(c, HRN_EMESH, "a PML point lies in the top PML zone");
                if (err || nk > A.cap) return set_error(c, HRN_ESTATE, "internal: pattern discovery overflow");
                thrust::device_ptr<uint64_t> kp(keys.as<uint64_t>());
                thrust::sort(thrust::cuda::par.on(c->stream), kp, kp + nk);
                const size_t nu = size_t(thrust::unique(thrust::cuda::par.on(c->stream), kp, kp + nk) - kp);
                // merge with the keys found so far
                HRN_CUDA(c, tmp.alloc(std::max<size_t>(na + nu, 1) * 8));
                thrust::device_ptr<uint64_t> ap(acc.as<uint64_t>()), tp(tmp.as<uint64_t>());
                const size_t nm = size_t(thrust::merge(thrust::cuda::par.on(c->stream), ap, ap + na, kp, kp + nu, tp) - tp);
                na = size_t(thrust::unique(thrust::cuda::par.on(c->stream), tp, tp + nm) - tp);
                std::swap(acc.p, tmp.p);
                std::swap(acc.bytes, tmp.bytes);
            }
        }
        keys.release();
        tmp.release();
        std::vector<uint64_t> hk(na);
        if (na) HRN_CUDA(c, cudaMemcpyAsync(hk.data(), acc.p, na * 8, cudaMemcpyDeviceToHost, c->stream));
        HRN_CUDA(c, cudaStreamSynchronize(c->stream));
        acc.release();
        if (int rc = finalize_pattern_from_keys(c, hk)) return rc;
    }
    // values
    HRN_CUDA(c, c->d_diag_m.alloc(size_t(c->neq) * 8));
    HRN_CUDA(c, c->d_im.alloc(size_t(c->neq) * 8));
    HRN_CUDA(c, cudaMemsetAsync(c->d_raw.p, 0, size_t(std::max<int64_t>(c->nnz, 1)) * 8, c->stream));
    HRN_CUDA(c, cudaMemsetAsync(c->d_diag_m.p, 0, size_t(c->neq) * 8, c->stream));
    HRN_CUDA(c, cudaMemsetAsync(c->d_asm_err.p, 0, 16, c->stream));
    A.discover = 0;
    A.rowptr = c->d_rowptr.as<int32_t>();
    A.colx = c->d_colx.as<uint32_t>();
    A.raw = c->d_raw.as<double>();
    A.diag_m = c->d_diag_m.as<double>();
    if (int rc = run_kernels(c, A)) return rc;
    k_inv_mass<<<(c->neq + 255) / 256, 256, 0, c->stream>>>(c->neq, c->d_diag_m.as<double>(), c->d_im.as<double>()); ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    int err = 0;
    HRN_CUDA(c, cudaMemcpyAsync(&err, c->d_asm_err.p, 4, cudaMemcpyDeviceToHost, c->stream));
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    if (err == 4) return set_error(c, HRN_EMESH, "a PML point lies in the top PML zone");
    if (err == 3) return set_error(c, HRN_EARG, "a nonzero contribution fell outside the sparsity pattern of the first assembly");
    if (err) return set_error(c, HRN_ESTATE, "internal: assembly error flag");
    return launch_scale_operator(c);
}

// ----------------------------------------------------------------------------
// Face traction: ASSEM_FORCE_PETSC_3D (S4/Assemble_PETSc_3D.F90:444-548) with
// ELEMENT_FS_3D (S4/Element_Matrices_3D.F90:890-1096).  A unit vertical
// traction (Tx = Ty = 0, Tz = 1) is integrated over the loaded face of every
// regular-domain element with the 3-point GLL rule.  Every face point is a GLL
// node, so the shape functions there are Kronecker deltas: node I at point q
// receives w_i w_j |dx/dxi_L x dx/dxi_M| of that point alone, in its z entry.
// DJ(:, L) and DJ(:, M) are summed over the 27 nodes in local order without
// fused multiply-adds, as MATMUL(XT, DFXI); the normal is the reference's CROSS.

__constant__ double a_gll_w[3];

// One thread per loaded element: efs[k][27] (z entries) and an error flag when a
// face point is off the surface (|z| > 1e-3), where the reference STOPs.
__global__ void k_face_force(int nload, const int32_t *__restrict__ elem, const int32_t *__restrict__ face,
                             const int32_t *__restrict__ inod, const double *__restrict__ xyz, double *__restrict__ efs,
                             int *__restrict__ err)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nload) return;
    const int e = elem[k];
    int nface = face[k];
    if (nface == 6) nface = 5;                  // the reference's temporary adjustment (:945-948)
    const int lface[6] = {2, 2, 3, 3, 1, 1};
    const int fsign[6] = {1, -1, 1, -1, 1, -1};
    const int iperm[3] = {2, 3, 1};
    const int L = lface[nface - 1], M = iperm[L - 1], N = iperm[M - 1];
    double xt[3][27];
    for (int i = 0; i < 27; ++i) {
        const int n = inod[size_t(e) * 27 + i];
        xt[0][i] = xyz[3 * size_t(n) + 0];
        xt[1][i] = xyz[3 * size_t(n) + 1];
        xt[2][i] = xyz[3 * size_t(n) + 2];
    }
    double *out = efs + size_t(k) * 27;
    for (int i = 0; i < 27; ++i) out[i] = 0.0;
    int idx[3];
    idx[N - 1] = fsign[nface - 1] > 0 ? 2 : 0;
    for (int lj = 0; lj < 3; ++lj) {
        idx[M - 1] = lj;
        for (int li = 0; li < 3; ++li) {
            idx[L - 1] = li;
            const int q = 9 * idx[2] + 3 * idx[1] + idx[0];
            const double wstar = mul(a_gll_w[li], a_gll_w[lj]);
            double vr[3], vs[3];
            for (int d = 0; d < 3; ++d) {
                double sr = 0.0, ss = 0.0;
                for (int I = 0; I < 27; ++I) {
                    sr = add(sr, mul(xt[d][I], dfxi(I, L - 1, q)));
                    ss = add(ss, mul(xt[d][I], dfxi(I, M - 1, q)));
                }
                vr[d] = sr;
                vs[d] = ss;
            }
            const double vn0 = __dsub_rn(mul(vr[1], vs[2]), mul(vr[2], vs[1]));
            const double vn1 = add(-mul(vr[0], vs[2]), mul(vr[2], vs[0]));
            const double vn2 = __dsub_rn(mul(vr[0], vs[1]), mul(vr[1], vs[0]));
            const double nrm = __dsqrt_rn(add(add(add(0.0, mul(vn0, vn0)), mul(vn1, vn1)), mul(vn2, vn2)));
            const int I = a_node_at[q];
            if (fabs(xt[2][I]) > 1.e-3) atomicExch(err, 5);
            out[I] = add(out[I], mul(wstar, nrm));
        }
    }
}

// B of the loaded elements, added per equation in element order (VecSetValues
// with ADD_VALUES, element by element): b[eq] = sum over its (slot, node) list.
__global__ void k_face_force_add(int nrow, const int32_t *__restrict__ row_eq, const int32_t *__restrict__ ptr,
                                 const int32_t *__restrict__ src, const double *__restrict__ efs, double *__restrict__ b)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrow) return;
    double v = 0.0;
    for (int t = ptr[r]; t < ptr[r + 1]; ++t) v = add(v, efs[src[t]]);
    b[row_eq[r]] = v;
}

int face_force(hrn_ctx *c, const int32_t *nface)
{
    if (int rc = upload_asm_tables(c)) return rc;
    const double w[3] = {0.33333333333333333333, 1.33333333333333333333, 0.33333333333333333333};
    HRN_CUDA(c, cudaMemcpyToSymbol(a_gll_w, w, sizeof(w)));
    // loaded regular-domain elements in element order, and per z equation of their
    // nodes the (slot, local node) contributions in that order
    std::vector<int32_t> elem, face;
    for (int e = 0; e < c->nel; ++e) {
        if (c->h_mtel[e] != 1 || nface[e] == 0) continue;
        if (nface[e] < 1 || nface[e] > 6) return set_error(c, HRN_EARG, "nface must be 0 (no load) or 1..6");
        elem.push_back(e);
        face.push_back(nface[e]);
    }
    const int nload = int(elem.size());
    std::vector<std::vector<int32_t>> per_eq;
    std::vector<int32_t> eq_of, slot_of_eq(size_t(c->neq), -1);
    for (int k = 0; k < nload; ++k)
        for (int i = 0; i < 27; ++i) {
            const int eq = c->h_id[size_t(c->h_inod[size_t(elem[k]) * 27 + i]) * 9 + 2];
            if (eq < 0) continue;
            if (slot_of_eq[eq] < 0) {
                slot_of_eq[eq] = int(eq_of.size());
                eq_of.push_back(eq);
                per_eq.emplace_back();
            }
            per_eq[slot_of_eq[eq]].push_back(k * 27 + i);
        }
    std::vector<int32_t> ptr(1, 0), src;
    for (auto &v : per_eq) {
        src.insert(src.end(), v.begin(), v.end());
        ptr.push_back(int32_t(src.size()));
    }
    HRN_CUDA(c, c->d_face_b.alloc(size_t(c->neq) * 8));
    HRN_CUDA(c, cudaMemsetAsync(c->d_face_b.p, 0, size_t(c->neq) * 8, c->stream));
    c->have_face_b = true;
    if (nload == 0) return 0;
    DevBuf d_elem, d_face, d_efs, d_eq, d_ptr, d_src, d_err;
    HRN_CUDA(c, d_elem.alloc(size_t(nload) * 4));
    HRN_CUDA(c, d_face.alloc(size_t(nload) * 4));
    HRN_CUDA(c, d_efs.alloc(size_t(nload) * 27 * 8));
    HRN_CUDA(c, d_eq.alloc(eq_of.size() * 4));
    HRN_CUDA(c, d_ptr.alloc(ptr.size() * 4));
    HRN_CUDA(c, d_src.alloc(src.size() * 4));
    HRN_CUDA(c, d_err.alloc(4));
    HRN_CUDA(c, cudaMemcpyAsync(d_elem.p, elem.data(), elem.size() * 4, cudaMemcpyHostToDevice, c->stream));
    HRN_CUDA(c, cudaMemcpyAsync(d_face.p, face.data(), face.size() * 4, cudaMemcpyHostToDevice, c->stream));
    HRN_CUDA(c, cudaMemcpyAsync(d_eq.p, eq_of.data(), eq_of.size() * 4, cudaMemcpyHostToDevice, c->stream));
    HRN_CUDA(c, cudaMemcpyAsync(d_ptr.p, ptr.data(), ptr.size() * 4, cudaMemcpyHostToDevice, c->stream));
    HRN_CUDA(c, cudaMemcpyAsync(d_src.p, src.data(), src.size() * 4, cudaMemcpyHostToDevice, c->stream));
    HRN_CUDA(c, cudaMemsetAsync(d_err.p, 0, 4, c->stream));
    k_face_force<<<(nload + 63) / 64, 64, 0, c->stream>>>(nload, d_elem.as<int32_t>(), d_face.as<int32_t>(),
                                                          c->d_inod.as<int32_t>(), c->d_xyz.as<double>(),
                                                          d_efs.as<double>(), d_err.as<int>()); ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    const int nrow = int(eq_of.size());
    k_face_force_add<<<(nrow + 127) / 128, 128, 0, c->stream>>>(nrow, d_eq.as<int32_t>(), d_ptr.as<int32_t>(),
                                                               d_src.as<int32_t>(), d_efs.as<double>(),
                                                               c->d_face_b.as<double>()); ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    int err = 0;
    HRN_CUDA(c, cudaMemcpyAsync(&err, d_err.p, 4, cudaMemcpyDeviceToHost, c->stream));
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    if (err) {
        c->have_face_b = false;
        return set_error(c, HRN_EMESH, "loaded face not on the surface (|z| > 1e-3 at a face point)");
    }
    return 0;
}

}  // namespace hrn
