// hrn_step.cu -- fused RK4 stage kernels of the explicit forward and adjoint
// time loops, the adjoint source, the fused zero-lag gradient and the misfit.
//
// One RK4 step of S4/Solver_PETSc_Explicit.F90:983-1046 (forward) or
// :1269-1364 (adjoint) is four launches of rk4_stage<STAGE>.  Stage s computes
//     kb_s = src_s + C^ km_s + K^ kt_s + G^ h_s
// over one combined CSR (C, K and G entries of a row back to back, matrix id in
// the top bits of the column index).  The stage inputs km_s, kt_s, h_s are not
// stored: every gathered column value is rebuilt from x1, x2, x3 and the earlier
// kb vectors with the same fused multiply-adds the row owner uses, e.g.
//     km_3 = c*kb_2 + x3,   kt_3 = c*km_2 + x2,   h_3 = c*kt_2 + x1   (c = dt/2).
// The fourth stage applies x <- x + dt/6 (k1 + 2 k2 + 2 k3 + k4) for its own
// rows and writes the new state into the other half of a ping-pong buffer.
// All S shots of a batch share each matrix entry (vectors are [row][shot]).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "hrn_internal.h"
#include "hrn_misfit.cuh"
#include "hrn_stage.cuh"

namespace hrn {


// Stage input of the entry's matrix at column j: rebuilt from x and earlier kb
// (MAT = 0), or read from the vectors the previous stage materialized (MAT = 1).
template <typename T, int S, int STAGE, int MAT>
__device__ __forceinline__ void gather_any(const StageArgs<T> &a, int tag, size_t j, T (&v)[S])
{
    if constexpr (MAT == 1 && STAGE > 1) {
        const T *src = tag == 0 ? a.in_m : (tag == 1 ? a.in_t : a.in_h);
        ldv<T, S>(src + j * S, v);
    } else {
        if (tag == 0) gather<T, S, STAGE, 0>(a, j, v);
        else if (tag == 1) gather<T, S, STAGE, 1>(a, j, v);
        else gather<T, S, STAGE, 2>(a, j, v);
    }
}


// G lanes per row; rows of a warp are independent sub-groups.  A row holds its
// C, K and G entries back to back; seg[row] = (first K entry, first G entry).
// Each lane takes four entries per trip so that their loads are in flight together.
template <typename T, int S, int STAGE, int G, int MAT>
__global__ void __launch_bounds__(256) rk4_stage(const StageArgs<T> a)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = tid / G;
    const int lane = threadIdx.x & (G - 1);
    if (row >= a.n) return;   // uniform over the G lanes of a row
    const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));

    T acc[S];
#pragma unroll
    for (int s = 0; s < S; ++s) acc[s] = T(0);
    const int k0 = __ldg(a.rowptr + row), k3 = __ldg(a.rowptr + row + 1);
    const int2 sg = __ldg(a.seg + row);
    // four entries per lane per trip: all column/value loads (streamed, evict-first)
    // issue before the gathers that depend on them
    for (int k = k0 + lane; k < k3; k += 4 * G) {
        uint32_t cx[4];
        T vv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int kk = k + u * G;
            const bool in = kk < k3;
            cx[u] = in ? __ldcs(a.colx + kk) : __ldcs(a.colx + k);
            vv[u] = in ? __ldcs(a.val + kk) : T(0);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int kk = k + u * G;
            T x[S];
            gather_any<T, S, STAGE, MAT>(a, kk >= sg.y ? 2 : (kk >= sg.x ? 1 : 0), size_t(cx[u] & kColMask), x);
#pragma unroll
            for (int s = 0; s < S; ++s) acc[s] = fmaT(vv[u], x[s], acc[s]);
        }
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1)
#pragma unroll
        for (int s = 0; s < S; ++s) acc[s] += __shfl_xor_sync(gmask, acc[s], off, G);
    if (lane != 0) return;

    finish_row<T, S, STAGE, MAT>(a, row, acc);
}

// ----------------------------------------------------------------------------
// tiled stage kernel: each CTA walks tiles of consecutive rows (at most
// kTileE entries); the column and value slab of the next tile is streamed into
// shared memory by 1-D bulk copies (cp.async.bulk, completion on an mbarrier)
// while the current tile is processed, so the gathers only wait on
// shared-memory reads.  Waits are bounded; a timeout sets *err and stops the CTA.

constexpr int kTileE = kTileEntries;  // entries per tile
constexpr int kTileThreads = 512;
constexpr int kTileSlack = 8;         // alignment slack of a buffer, entries

template <typename T>
constexpr size_t tile_smem_bytes()
{
    return 128 + 2 * (size_t(kTileE + kTileSlack) * 4 + size_t(kTileE + kTileSlack) * sizeof(T));
}

template <typename T>
__device__ __forceinline__ void tile_issue(const StageArgs<T> &a, const int32_t *tiles, int t, uint32_t *cb, T *vb,
                                           uint64_t *bar)
{
    const int e0 = __ldg(a.rowptr + __ldg(tiles + t)), e1 = __ldg(a.rowptr + __ldg(tiles + t + 1));
    constexpr int va_mask = int(16 / sizeof(T)) - 1;
    const int ca = e0 & ~3, va = e0 & ~va_mask;
    const uint32_t cn = uint32_t(((e1 - ca) * 4 + 15) & ~15);
    const uint32_t vn = uint32_t(((e1 - va) * int(sizeof(T)) + 15) & ~15);
    if (e1 == e0) {
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
        return;
    }
    mbar_expect_tx(bar, cn + vn);
    bulk_g2s(cb, a.colx + ca, cn, bar);
    bulk_g2s(vb, a.val + va, vn, bar);
}

template <typename T, int S, int STAGE, int G, int MAT>
__global__ void __launch_bounds__(kTileThreads) rk4_stage_tile(const StageArgs<T> a, const int32_t *__restrict__ tiles,
                                                               int ntiles, int *__restrict__ err)
{
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem);
    uint32_t *cbuf[2];
    T *vbuf[2];
    {
        size_t off = 128;
        for (int b = 0; b < 2; ++b) {
            cbuf[b] = reinterpret_cast<uint32_t *>(smem + off);
            off += size_t(kTileE + kTileSlack) * 4;
            vbuf[b] = reinterpret_cast<T *>(smem + off);
            off += size_t(kTileE + kTileSlack) * sizeof(T);
        }
    }
    __shared__ int abort_flag;
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_flag = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0 && int(blockIdx.x) < ntiles) tile_issue<T>(a, tiles, blockIdx.x, cbuf[0], vbuf[0], bar);
    const int lane = threadIdx.x & (G - 1);
    const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
    int it = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
        const int b = it & 1;
        const int tn = t + gridDim.x;
        if (threadIdx.x == 0 && tn < ntiles) tile_issue<T>(a, tiles, tn, cbuf[b ^ 1], vbuf[b ^ 1], bar + (b ^ 1));
        const bool ok = mbar_wait(bar + b, uint32_t((it >> 1) & 1));
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) {
                atomicExch(err, 1);
                abort_flag = 1;
            }
            break;
        }
        const int r0 = __ldg(tiles + t), r1 = __ldg(tiles + t + 1);
        const int e0 = __ldg(a.rowptr + r0);
        const int ca = e0 & ~3, va = e0 & ~(int(16 / sizeof(T)) - 1);
        const uint32_t *cb = cbuf[b];
        const T *vb = vbuf[b];
        for (int row = r0 + int(threadIdx.x) / G; row < r1; row += kTileThreads / G) {
            T acc[S];
#pragma unroll
            for (int s = 0; s < S; ++s) acc[s] = T(0);
            const int k0 = __ldg(a.rowptr + row), k3 = __ldg(a.rowptr + row + 1);
            const int2 sg = __ldg(a.seg + row);
            for (int k = k0 + lane; k < k3; k += 4 * G) {
                uint32_t cx[4];
                T vv[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int kk = k + u * G;
                    const bool in = kk < k3;
                    cx[u] = cb[(in ? kk : k) - ca];
                    vv[u] = in ? vb[kk - va] : T(0);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int kk = k + u * G;
                    T x[S];
                    gather_any<T, S, STAGE, MAT>(a, kk >= sg.y ? 2 : (kk >= sg.x ? 1 : 0), size_t(cx[u] & kColMask), x);
#pragma unroll
                    for (int s = 0; s < S; ++s) acc[s] = fmaT(vv[u], x[s], acc[s]);
                }
            }
#pragma unroll
            for (int off = G / 2; off > 0; off >>= 1)
#pragma unroll
                for (int s = 0; s < S; ++s) acc[s] += __shfl_xor_sync(gmask, acc[s], off, G);
            if (lane == 0) finish_row<T, S, STAGE, MAT>(a, row, acc);
        }
        __syncthreads();   // buffer b is refilled only after every thread is done with it
    }
    // on abort, let the copy still in flight into the other buffer land (bounded)
    if (abort_flag && threadIdx.x == 0) mbar_wait(bar + ((it & 1) ^ 1), uint32_t(((it + 1) >> 1) & 1));
}

// ----------------------------------------------------------------------------
// operator scaling

// forward: -(a_ij * iM_i)            (S4/Solver_PETSc_Explicit.F90:815-824)
template <typename T>
__global__ void k_scale_fwd(int64_t nnz, const int32_t *__restrict__ rowidx, const double *__restrict__ raw,
                            const double *__restrict__ im, T *__restrict__ out)
{
    for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < nnz; k += int64_t(gridDim.x) * blockDim.x)
        out[k] = T(-__dmul_rn(raw[k], im[rowidx[k]]));
}

// adjoint, stored transposed: ((+-(a_ij iM_i)) M_i) iM_j  (:1222-1229)
template <typename T>
__global__ void k_scale_adj(int64_t nnz, const int64_t *__restrict__ permT, const int32_t *__restrict__ rowidx,
                            const uint32_t *__restrict__ colx, const double *__restrict__ raw,
                            const double *__restrict__ dm, const double *__restrict__ im, T *__restrict__ out)
{
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < nnz; t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t k = permT[t];
        const int i = rowidx[k];
        const uint32_t cx = colx[k];
        double v = -__dmul_rn(raw[k], im[i]);
        if ((cx >> kTagBits) != 1u) v = -v;
        v = __dmul_rn(v, dm[i]);
        v = __dmul_rn(v, im[cx & kColMask]);
        out[t] = T(v);
    }
}

// One per-step operator applied to an FP64 vector: y_i = sum over the row's
// entries of matrix `which` of val * x[col], from the values the stage kernels
// stream (forward: -iM A, row order; adjoint: the transposed adjoint-scaled
// values, so y = A'^T x).  Used by the dot-product tests of the device operator.
template <typename T>
__global__ void k_apply_operator(int n, const int32_t *__restrict__ rowptr, const uint32_t *__restrict__ colx,
                                 const T *__restrict__ val, uint32_t which, const double *__restrict__ x,
                                 double *__restrict__ y)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int32_t k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            const uint32_t cw = colx[k];
            if ((cw >> kTagBits) != which) continue;
            s = fma(double(val[k]), x[cw & kColMask], s);
        }
        y[i] = s;
    }
}

// ----------------------------------------------------------------------------
// sources

// Forward stage sources for every step: f(T) b^, f(T+dt/2) b^ (twice), f(T+dt) b^,
// b^ = B * iM.  src_b [nslot][S], ftab [S][nstep+1][3] (T, T+dt, T+dt/2).
template <typename T, int S>
__global__ void k_src_fwd(int nstep, int nslot, const int32_t *__restrict__ slot_eq, const double *__restrict__ src_b,
                          const double *__restrict__ ftab, const double *__restrict__ im, T *__restrict__ srcv)
{
    const int64_t total = int64_t(nstep + 1) * nslot * S;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
        const int s = int(t % S);
        const int sl = int((t / S) % nslot);
        const int n = int(t / (int64_t(S) * nslot));
        const double bh = src_b[sl * S + s] * im[slot_eq[sl]];
        const double *f = ftab + (size_t(s) * (nstep + 1) + n) * 3;
        T *o = srcv + (size_t(n) * 4 * nslot) * S;
        o[(0 * size_t(nslot) + sl) * S + s] = T(0.0 + f[0] * bh);
        o[(1 * size_t(nslot) + sl) * S + s] = T(0.0 + f[2] * bh);
        o[(2 * size_t(nslot) + sl) * S + s] = T(0.0 + f[2] * bh);
        o[(3 * size_t(nslot) + sl) * S + s] = T(0.0 + f[1] * bh);
    }
}

// Adjoint stage sources of step n (S4/Solver_PETSc_Explicit.F90:1269-1312):
// k1 = iM r_n, k4 = iM r_{n-1}, k2 = k3 = (k1 + k4)/2 with
// r_m = U_Store(EqDis_MAP, m) - Dis_meas(m, :) summed over duplicate equations.
// Receiver displacements of one step (checkpointed forward): out[q][s] = x2[eqdis[q]][s].
template <typename T, int S>
__global__ void k_traces(int nrec3, const int32_t *__restrict__ eq, const T *__restrict__ x2, T *__restrict__ out)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nrec3 * S) return;
    const int q = t / S, s = t % S;
    out[t] = x2[size_t(eq[q]) * S + s];
}

// Uneven shots (shot_nstep / mask not null): shot s records steps 0..shot_nstep[s]
// at the receivers q with mask[s][q] != 0.  Its adjoint starts at its own last
// step: for n > shot_nstep[s] every source of the shot is zero, so its state stays
// exactly zero until then and the batch reproduces the shot run alone.
template <typename T, int S>
__global__ void k_src_adj(int n, int nstep, int nstore, int nrec3, int nslot, const int32_t *__restrict__ ptr,
                          const int32_t *__restrict__ qlist, const int32_t *__restrict__ slot_eq,
                          const int32_t *__restrict__ emap, const T *__restrict__ hist,
                          const double *__restrict__ dis, const double *__restrict__ im, T *__restrict__ srcv,
                          const int32_t *__restrict__ shot_nstep, const uint8_t *__restrict__ mask)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nslot * S) return;
    const int s = t % S, sl = t / S;
    if (shot_nstep && n > shot_nstep[s]) {
#pragma unroll
        for (int k = 0; k < 4; ++k) srcv[(k * size_t(nslot) + sl) * S + s] = T(0);
        return;
    }
    double r1 = 0.0, r4 = 0.0;
    for (int k = ptr[sl]; k < ptr[sl + 1]; ++k) {
        const int q = qlist[k];
        if (mask && !mask[size_t(s) * nrec3 + q]) continue;
        const size_t pos = size_t(emap[q]) * S + s;
        const double *d = dis + (size_t(s) * nrec3 + q) * (nstep + 1);
        r1 += double(hist[size_t(n) * nstore * S + pos]) - d[n];
        r4 += double(hist[size_t(n - 1) * nstore * S + pos]) - d[n - 1];
    }
    const double m = im[slot_eq[sl]];
    const double v1 = 0.0 + 1.0 * (r1 * m), v4 = 0.0 + 1.0 * (r4 * m);
    const double v2 = 0.0 + (0.5 * v1 + 0.5 * v4);
    srcv[(0 * size_t(nslot) + sl) * S + s] = T(v1);
    srcv[(1 * size_t(nslot) + sl) * S + s] = T(v2);
    srcv[(2 * size_t(nslot) + sl) * S + s] = T(v2);
    srcv[(3 * size_t(nslot) + sl) * S + s] = T(v4);
}

// ----------------------------------------------------------------------------
// zero-lag gradient (ELEMENT_g_3D, S4/Element_Matrices_3D.F90:1725-1890, and
// Update_g, S4/Assemble_PETSc_3D.F90:556-661), one thread per GLL point.
// With the GLL rule FN(I) at point q is the Kronecker delta, so the element
// contribution to node I is the point scalar at q = I times w*detJ.

__constant__ int c_node_at[27];   // local node at GLL point q = 9c + 3b + a
__constant__ double c_D[3][3];    // c_D[a][b] = l_b'(xi_a)

constexpr int kGradElems = 4;

template <typename T, int S>
__global__ void __launch_bounds__(128) k_gradient(int nel_rd, const int32_t *__restrict__ rd_store,
                                                  const int32_t *__restrict__ rd_elems, const int32_t *__restrict__ inod,
                                                  const double *__restrict__ geom, const T *__restrict__ hist_n,
                                                  const T *__restrict__ x2, const int32_t *__restrict__ store_eq,
                                                  double *__restrict__ g_lam, double *__restrict__ g_mu, double dt,
                                                  int lambda_2mu)   // g_lam, g_mu: [nel_rd][27] point slots
{
    __shared__ T su[kGradElems][27][3][S];
    __shared__ T sp[kGradElems][27][3][S];
    const int le = threadIdx.x / 27, q = threadIdx.x % 27;
    const int e = blockIdx.x * kGradElems + le;
    const bool active = threadIdx.x < 27 * kGradElems && e < nel_rd;
    if (active) {
        const int sn = rd_store[size_t(e) * 27 + q];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int pos = 3 * sn + c;
            const int eq = store_eq[pos];
#pragma unroll
            for (int s = 0; s < S; ++s) {
                su[le][q][c][s] = hist_n[size_t(pos) * S + s];
                sp[le][q][c][s] = x2[size_t(eq) * S + s];
            }
        }
    }
    __syncthreads();
    if (!active) return;
    const int aq = q % 3, bq = (q / 3) % 3, cq = q / 9;
    const double *gm = geom + (size_t(e) * 27 + q) * 10;
    double J[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) J[k] = gm[k];
    const double fac0 = gm[9];
    double tl = 0.0, tm = 0.0;
    for (int s = 0; s < S; ++s) {
        double du[3][3], dp[3][3];   // d(comp)/d(xi_m)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double ux = 0, uy = 0, uz = 0, px = 0, py = 0, pz = 0;
#pragma unroll
            for (int t = 0; t < 3; ++t) {
                const int nx = c_node_at[9 * cq + 3 * bq + t];
                const int ny = c_node_at[9 * cq + 3 * t + aq];
                const int nz = c_node_at[9 * t + 3 * bq + aq];
                ux += c_D[aq][t] * double(su[le][nx][c][s]);
                uy += c_D[bq][t] * double(su[le][ny][c][s]);
                uz += c_D[cq][t] * double(su[le][nz][c][s]);
                px += c_D[aq][t] * double(sp[le][nx][c][s]);
                py += c_D[bq][t] * double(sp[le][ny][c][s]);
                pz += c_D[cq][t] * double(sp[le][nz][c][s]);
            }
            du[c][0] = ux; du[c][1] = uy; du[c][2] = uz;
            dp[c][0] = px; dp[c][1] = py; dp[c][2] = pz;
        }
        // physical gradients: d/dx_k = sum_m DJI(m,k) d/dxi_m
        double gu[3][3], gp[3][3];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                gu[c][k] = du[c][0] * J[0 * 3 + k] + du[c][1] * J[1 * 3 + k] + du[c][2] * J[2 * 3 + k];
                gp[c][k] = dp[c][0] * J[0 * 3 + k] + dp[c][1] * J[1 * 3 + k] + dp[c][2] * J[2 * 3 + k];
            }
        const double u1x = gu[0][0], u2x = gu[1][0], u3x = gu[2][0];
        const double u1y = gu[0][1], u2y = gu[1][1], u3y = gu[2][1];
        const double u1z = gu[0][2], u2z = gu[1][2], u3z = gu[2][2];
        const double p1x = gp[0][0], p2x = gp[1][0], p3x = gp[2][0];
        const double p1y = gp[0][1], p2y = gp[1][1], p3y = gp[2][1];
        const double p1z = gp[0][2], p2z = gp[1][2], p3z = gp[2][2];
        const double sl = (u1x + u2y + u3z) * (p1x + p2y + p3z);
        const double cross = (p1y + p2x) * (u1y + u2x) + (p1z + p3x) * (u1z + u3x) + (p3y + p2z) * (u3y + u2z);
        double sm;
        if (!lambda_2mu) sm = 2.0 * (u1x * p1x + u2y * p2y + u3z * p3z) + cross;
        else sm = -2.0 * (p1x * (u2y + u3z) + p2y * (u1x + u3z) + p3z * (u1x + u2y)) + cross;
        tl += (sl * fac0) * dt;
        tm += (sm * fac0) * dt;
    }
    // one thread owns each (element, point) slot: the sum over steps needs no atomics
    g_lam[size_t(e) * 27 + q] += tl;
    g_mu[size_t(e) * 27 + q] += tm;
}

// Node sums of the gradient slots in a fixed order (ascending element, then point),
// so the gradient is the same bit for bit from run to run.  Nodes without a slot
// (PML-only nodes) get 0.
__global__ void k_gradient_nodes(int nj, const int32_t *__restrict__ ptr, const int32_t *__restrict__ slots,
                                 const double *__restrict__ slot_l, const double *__restrict__ slot_m,
                                 double *__restrict__ g_lam, double *__restrict__ g_mu)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nj) return;
    double sl = 0.0, sm = 0.0;
    for (int k = ptr[j]; k < ptr[j + 1]; ++k) {
        sl += slot_l[slots[k]];
        sm += slot_m[slots[k]];
    }
    g_lam[j] = sl;
    g_mu[j] = sm;
}

// ----------------------------------------------------------------------------
// misfit (Compute_Misfit, S4/Solver_PETSc_Inverse.F90:591-657)

// Uneven shots: the terms of a shot past its record length are zero, and masked
// receivers do not enter it (see k_src_adj).
template <typename T, int S>
__global__ void k_misfit_terms(int nstep, int nstore, int nrec3, int nslot, const int32_t *__restrict__ ptr,
                               const int32_t *__restrict__ qlist, const int32_t *__restrict__ emap,
                               const T *__restrict__ hist, const double *__restrict__ dis, double *__restrict__ terms,
                               const int32_t *__restrict__ shot_nstep, const uint8_t *__restrict__ mask)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (nstep + 1) * S) return;
    const int s = t % S, n = t / S;
    terms[size_t(s) * (nstep + 1) + n] =
        misfit_term<T>(S, s, n, nstep, nstore, nrec3, nslot, ptr, qlist, emap, hist, dis, shot_nstep, mask);
}

__global__ void k_misfit_sum(int nshot, int nstep, double dt, const double *__restrict__ terms, double *__restrict__ cost)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    misfit_sum(nshot, nstep, dt, terms, cost);
}

// ----------------------------------------------------------------------------
// host side

static int blocks_for(int64_t work, int threads, int64_t cap = 148LL * 32)
{
    int64_t b = (work + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return int(b);
}

template <typename T>
static int scale_operator_t(hrn_ctx *c)
{
    const int th = 256;
    const size_t vb = size_t(c->nnz) * sizeof(T) + kBulkPad;
    if (c->d_fwd.bytes != vb) HRN_CUDA(c, c->d_fwd.alloc(vb));
    if (c->d_adj.bytes != vb) HRN_CUDA(c, c->d_adj.alloc(vb));
    if (c->nnz == 0) return 0;
    k_scale_fwd<T><<<blocks_for(c->nnz, th), th, 0, c->stream>>>(c->nnz, c->d_rowidx.as<int32_t>(), c->d_raw.as<double>(),
                                                                  c->d_im.as<double>(), c->d_fwd.as<T>()); ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    k_scale_adj<T><<<blocks_for(c->nnz, th), th, 0, c->stream>>>(c->nnz, c->d_permT.as<int64_t>(), c->d_rowidx.as<int32_t>(),
                                                                  c->d_colx.as<uint32_t>(), c->d_raw.as<double>(),
                                                                  c->d_diag_m.as<double>(), c->d_im.as<double>(), c->d_adj.as<T>()); ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    return 0;
}

int run_apply_operator(hrn_ctx *c, int which, int adj, const double *d_x, double *d_y)
{
    const int th = 256;
    const int32_t *rp = adj ? c->d_rowptrT.as<int32_t>() : c->d_rowptr.as<int32_t>();
    const uint32_t *cx = adj ? c->d_colxT.as<uint32_t>() : c->d_colx.as<uint32_t>();
    const int grid = blocks_for(c->neq, th);
    if (c->precision == HRN_FP64)
        k_apply_operator<double><<<grid, th, 0, c->stream>>>(c->neq, rp, cx, adj ? c->d_adj.as<double>() : c->d_fwd.as<double>(),
                                                              uint32_t(which), d_x, d_y);
    else
        k_apply_operator<float><<<grid, th, 0, c->stream>>>(c->neq, rp, cx, adj ? c->d_adj.as<float>() : c->d_fwd.as<float>(),
                                                             uint32_t(which), d_x, d_y);
    ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    return 0;
}

int launch_scale_operator(hrn_ctx *c)
{
    ++c->val_version;
    return c->precision == HRN_FP64 ? scale_operator_t<double>(c) : scale_operator_t<float>(c);
}

struct TileArgs {
    const int32_t *tiles;
    int ntiles, grid;
    int *err;
};

// Stage-kernel variant: lanes per row (4, 8, 16) x stage inputs rebuilt at the
// gather (0) or materialized by the previous stage (1) x row-parallel (0) or
// tiled with bulk-copied matrix slabs (2); encoded lanes * 10 + mat + tiled,
// chosen per operator by timing.
constexpr int kVariants[10] = {40, 80, 160, 41, 81, 161, 42, 43, 82, 83};
// 90-95 / 100-105: matrix-free element kernels with the stage inputs
// materialized / rebuilt from x and kb; element slots (even) or atomic row sums
// (odd), with 1 (+0, +1), 2 (+2, +3) or 4 (+4, +5) shots per thread
inline bool is_elem_variant(int v) { return (v >= 90 && v <= 95) || (v >= 100 && v <= 105); }

template <typename T, int S, int STAGE, int G, int MAT>
static void launch_tile(const StageArgs<T> &a, const TileArgs &ta, cudaStream_t st)
{
    static std::atomic<uint64_t> smem_done{0};
    constexpr size_t smem = tile_smem_bytes<T>();
    smem_limit_once(rk4_stage_tile<T, S, STAGE, G, MAT>, int(smem), smem_done);
    rk4_stage_tile<T, S, STAGE, G, MAT><<<ta.grid, kTileThreads, smem, st>>>(a, ta.tiles, ta.ntiles, ta.err);
}

template <typename T, int S, int STAGE>
static void launch_stage(const StageArgs<T> &a, int variant, cudaStream_t st, const TileArgs &ta)
{
    switch (variant) {
    case 42: launch_tile<T, S, STAGE, 4, 0>(a, ta, st); return;
    case 43: launch_tile<T, S, STAGE, 4, 1>(a, ta, st); return;
    case 82: launch_tile<T, S, STAGE, 8, 0>(a, ta, st); return;
    case 83: launch_tile<T, S, STAGE, 8, 1>(a, ta, st); return;
    default: break;
    }
    const int th = 256;
    const int lanes = variant / 10;
    const int64_t threads = int64_t(a.n) * lanes;
    const int blocks = int((threads + th - 1) / th);
    switch (variant) {
    case 40: rk4_stage<T, S, STAGE, 4, 0><<<blocks, th, 0, st>>>(a); break;
    case 160: rk4_stage<T, S, STAGE, 16, 0><<<blocks, th, 0, st>>>(a); break;
    case 41: rk4_stage<T, S, STAGE, 4, 1><<<blocks, th, 0, st>>>(a); break;
    case 81: rk4_stage<T, S, STAGE, 8, 1><<<blocks, th, 0, st>>>(a); break;
    case 161: rk4_stage<T, S, STAGE, 16, 1><<<blocks, th, 0, st>>>(a); break;
    default: rk4_stage<T, S, STAGE, 8, 0><<<blocks, th, 0, st>>>(a); break;
    }
}

struct StageTimer {
    hrn_ctx *c;
    size_t used = 0;
    explicit StageTimer(hrn_ctx *cc) : c(cc) {}
    cudaEvent_t get()
    {
        if (used == c->ev_pool.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            c->ev_pool.push_back(e);
        }
        return c->ev_pool[used++];
    }
};


// ----------------------------------------------------------------------------
// element geometry at the 27 GLL points: DJI (row m = xi direction, column k =
// x direction) and w*detJ, from the Jacobian of S4/Element_Matrices_3D.F90:111-139.
// With the GLL rule only the 3 nodes on the xi_m line through a point carry a
// nonzero dN/dxi_m there, so DJ(i,m) is a 3-term sum; the terms are added in
// ascending local node order (the order of MATMUL(XT, DFXI)) without fused
// multiply-adds, so DJ, detJ and DJI equal the reference's left-to-right values.
__constant__ double c_w[3];
__constant__ unsigned char c_gnode[27][3][3];   // [q][m][t] local nodes on the xi_m line, ascending
__constant__ double c_gd[27][3][3];             // matching dN/dxi_m values at q

__global__ void k_geometry(int nel, const int32_t *__restrict__ elems, const int32_t *__restrict__ inod,
                           const double *__restrict__ xyz, double *__restrict__ out, int *__restrict__ bad)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nel * 27) return;
    const int le = t / 27, q = t % 27;
    const int e = elems ? elems[le] : le;
    const int aq = q % 3, bq = (q / 3) % 3, cq = q / 9;
    const int32_t *nd = inod + size_t(e) * 27;
    double dj[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            double s = 0.0;
#pragma unroll
            for (int tt = 0; tt < 3; ++tt)
                s = __dadd_rn(s, __dmul_rn(xyz[size_t(nd[c_gnode[q][m][tt]]) * 3 + i], c_gd[q][m][tt]));
            dj[i][m] = s;
        }
#define M_(a, b) __dmul_rn(a, b)
#define A_(a, b) __dadd_rn(a, b)
#define S_(a, b) __dsub_rn(a, b)
    const double detj = S_(S_(S_(A_(A_(M_(M_(dj[0][0], dj[1][1]), dj[2][2]), M_(M_(dj[1][0], dj[2][1]), dj[0][2])),
                                     M_(M_(dj[2][0], dj[0][1]), dj[1][2])),
                                  M_(M_(dj[0][2], dj[1][1]), dj[2][0])),
                               M_(M_(dj[1][2], dj[2][1]), dj[0][0])),
                            M_(M_(dj[2][2], dj[0][1]), dj[1][0]));
    double *o = out + size_t(t) * 10;
    if (!(detj > 0.0)) {
        atomicExch(bad, 1);
        for (int k = 0; k < 10; ++k) o[k] = 0.0;
        return;
    }
    double ji[9];
    ji[0] = S_(M_(dj[2][2], dj[1][1]), M_(dj[2][1], dj[1][2]));
    ji[1] = A_(-M_(dj[2][2], dj[0][1]), M_(dj[2][1], dj[0][2]));
    ji[2] = S_(M_(dj[1][2], dj[0][1]), M_(dj[1][1], dj[0][2]));
    ji[3] = A_(-M_(dj[2][2], dj[1][0]), M_(dj[2][0], dj[1][2]));
    ji[4] = S_(M_(dj[2][2], dj[0][0]), M_(dj[2][0], dj[0][2]));
    ji[5] = A_(-M_(dj[1][2], dj[0][0]), M_(dj[1][0], dj[0][2]));
    ji[6] = S_(M_(dj[2][1], dj[1][0]), M_(dj[2][0], dj[1][1]));
    ji[7] = A_(-M_(dj[2][1], dj[0][0]), M_(dj[2][0], dj[0][1]));
    ji[8] = S_(M_(dj[1][1], dj[0][0]), M_(dj[1][0], dj[0][1]));
#pragma unroll
    for (int k = 0; k < 9; ++k) o[k] = __ddiv_rn(ji[k], detj);
    o[9] = M_(M_(M_(c_w[aq], c_w[bq]), c_w[cq]), detj);
#undef M_
#undef A_
#undef S_
}

static const int kLocalIjk[27][3] = {{2, 0, 0}, {2, 2, 0}, {0, 2, 0}, {0, 0, 0}, {2, 0, 2}, {2, 2, 2}, {0, 2, 2}, {0, 0, 2},
                                     {2, 1, 0}, {1, 2, 0}, {0, 1, 0}, {1, 0, 0}, {2, 0, 1}, {2, 2, 1}, {0, 2, 1}, {0, 0, 1},
                                     {2, 1, 2}, {1, 2, 2}, {0, 1, 2}, {1, 0, 2}, {1, 1, 0}, {2, 1, 1}, {1, 2, 1}, {0, 1, 1},
                                     {1, 0, 1}, {1, 1, 2}, {1, 1, 1}};

// local node at GLL point q = 9c + 3b + a
static void gll_node_at(int (&node_at)[27])
{
    for (int i = 0; i < 27; ++i) node_at[9 * kLocalIjk[i][2] + 3 * kLocalIjk[i][1] + kLocalIjk[i][0]] = i;
}

static int upload_tables(hrn_ctx *c)
{
    static const int ijk[27][3] = {{2, 0, 0}, {2, 2, 0}, {0, 2, 0}, {0, 0, 0}, {2, 0, 2}, {2, 2, 2}, {0, 2, 2}, {0, 0, 2},
                                   {2, 1, 0}, {1, 2, 0}, {0, 1, 0}, {1, 0, 0}, {2, 0, 1}, {2, 2, 1}, {0, 2, 1}, {0, 0, 1},
                                   {2, 1, 2}, {1, 2, 2}, {0, 1, 2}, {1, 0, 2}, {1, 1, 0}, {2, 1, 1}, {1, 2, 1}, {0, 1, 1},
                                   {1, 0, 1}, {1, 1, 2}, {1, 1, 1}};
    int node_at[27];
    for (int i = 0; i < 27; ++i) node_at[9 * ijk[i][2] + 3 * ijk[i][1] + ijk[i][0]] = i;
    // derivative of the 1D quadratic Lagrange basis l_b at GLL point xi_a
    const double D[3][3] = {{-1.5, 2.0, -0.5}, {-0.5, 0.0, 0.5}, {0.5, -2.0, 1.5}};
    const double w[3] = {0.33333333333333333333, 1.33333333333333333333, 0.33333333333333333333};
    HRN_CUDA(c, cudaMemcpyToSymbol(c_node_at, node_at, sizeof(node_at)));
    HRN_CUDA(c, cudaMemcpyToSymbol(c_D, D, sizeof(D)));
    HRN_CUDA(c, cudaMemcpyToSymbol(c_w, w, sizeof(w)));
    unsigned char gnode[27][3][3];
    double gd[27][3][3];
    for (int q = 0; q < 27; ++q) {
        const int qi[3] = {q % 3, (q / 3) % 3, q / 9};
        for (int m = 0; m < 3; ++m) {
            int t = 0;
            for (int I = 0; I < 27; ++I) {   // ascending local node order
                bool on = true;
                for (int k = 0; k < 3; ++k)
                    if (k != m && ijk[I][k] != qi[k]) on = false;
                if (!on) continue;
                gnode[q][m][t] = (unsigned char)I;
                gd[q][m][t] = D[qi[m]][ijk[I][m]];
                ++t;
            }
        }
    }
    HRN_CUDA(c, cudaMemcpyToSymbol(c_gnode, gnode, sizeof(gnode)));
    HRN_CUDA(c, cudaMemcpyToSymbol(c_gd, gd, sizeof(gd)));
    return 0;
}

int build_rd_geometry(hrn_ctx *c)
{
    if (int rc = upload_tables(c)) return rc;
    std::vector<int32_t> rd;
    for (int e = 0; e < c->nel; ++e)
        if (c->h_mtel[e] == 1) rd.push_back(e);
    c->nel_rd = int(rd.size());
    HRN_CUDA(c, c->d_rd_elems.alloc(rd.size() * 4));
    if (!rd.empty()) HRN_CUDA(c, cudaMemcpy(c->d_rd_elems.p, rd.data(), rd.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, c->d_rd_geom.alloc(size_t(c->nel_rd) * 27 * 10 * 8));
    HRN_CUDA(c, c->d_asm_geom.alloc(size_t(c->nel) * 27 * 10 * 8));
    HRN_CUDA(c, c->d_asm_err.alloc(16));
    HRN_CUDA(c, cudaMemsetAsync(c->d_asm_err.p, 0, 16, c->stream));
    const int th = 256;
    if (c->nel_rd > 0)
        k_geometry<<<(c->nel_rd * 27 + th - 1) / th, th, 0, c->stream>>>(c->nel_rd, c->d_rd_elems.as<int32_t>(), c->d_inod.as<int32_t>(),
                                                                           c->d_xyz.as<double>(), c->d_rd_geom.as<double>(), c->d_asm_err.as<int>()); ++c->launches;
    k_geometry<<<(c->nel * 27 + th - 1) / th, th, 0, c->stream>>>(c->nel, nullptr, c->d_inod.as<int32_t>(), c->d_xyz.as<double>(),
                                                                   c->d_asm_geom.as<double>(), c->d_asm_err.as<int>()); ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    int bad = 0;
    HRN_CUDA(c, cudaMemcpyAsync(&bad, c->d_asm_err.p, 4, cudaMemcpyDeviceToHost, c->stream));
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    if (bad) return set_error(c, HRN_EMESH, "non-positive Jacobian determinant in an element");
    c->have_rd_store = false;
    return 0;
}

// History node index of every RD element node (nodes of RD elements are all stored).
static int build_rd_store(hrn_ctx *c)
{
    if (c->have_rd_store) return 0;
    std::vector<int32_t> inv(size_t(c->neq), -1);
    for (int p = 0; p < c->nstore; ++p) inv[c->h_store_eq[p]] = p;
    std::vector<int32_t> rs(size_t(c->nel_rd) * 27);
    int k = 0;
    for (int e = 0; e < c->nel; ++e) {
        if (c->h_mtel[e] != 1) continue;
        for (int i = 0; i < 27; ++i) {
            const int node = c->h_inod[size_t(e) * 27 + i];
            int pos[3];
            for (int d = 0; d < 3; ++d) {
                const int eq = c->h_id[size_t(node) * 9 + d];
                pos[d] = eq >= 0 ? inv[eq] : -1;
            }
            if (pos[0] < 0 || pos[0] % 3 != 0 || pos[1] != pos[0] + 1 || pos[2] != pos[0] + 2)
                return set_error(c, HRN_EARG, "history equations must hold the x, y, z displacement of every regular-domain node, in that order");
            rs[size_t(k) * 27 + i] = pos[0] / 3;
        }
        ++k;
    }
    HRN_CUDA(c, c->d_rd_store.alloc(rs.size() * 4));
    if (!rs.empty()) HRN_CUDA(c, cudaMemcpy(c->d_rd_store.p, rs.data(), rs.size() * 4, cudaMemcpyHostToDevice));
    // gradient slots of every node, in ascending (element, point) order
    int node_at[27];
    gll_node_at(node_at);
    std::vector<int32_t> ptr(size_t(c->nj) + 1, 0), slots(size_t(c->nel_rd) * 27);
    std::vector<int32_t> slot_node(slots.size());
    k = 0;
    for (int e = 0; e < c->nel; ++e) {
        if (c->h_mtel[e] != 1) continue;
        for (int q = 0; q < 27; ++q) {
            const int node = c->h_inod[size_t(e) * 27 + node_at[q]];
            slot_node[size_t(k) * 27 + q] = node;
            ptr[size_t(node) + 1]++;
        }
        ++k;
    }
    for (int j = 0; j < c->nj; ++j) ptr[j + 1] += ptr[j];
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (size_t sidx = 0; sidx < slot_node.size(); ++sidx) slots[fill[slot_node[sidx]]++] = int32_t(sidx);
    HRN_CUDA(c, c->d_gnode_ptr.alloc(ptr.size() * 4));
    HRN_CUDA(c, c->d_gnode_slot.alloc(std::max<size_t>(slots.size(), 1) * 4));
    HRN_CUDA(c, c->d_gslot.alloc(std::max<size_t>(slots.size(), 1) * 2 * 8));
    HRN_CUDA(c, cudaMemcpy(c->d_gnode_ptr.p, ptr.data(), ptr.size() * 4, cudaMemcpyHostToDevice));
    if (!slots.empty()) HRN_CUDA(c, cudaMemcpy(c->d_gnode_slot.p, slots.data(), slots.size() * 4, cudaMemcpyHostToDevice));
    // identity map of the history rows (the pseudo-Hessian reads u through it), allocated
    // here with the other gradient tables so that later calls allocate nothing
    std::vector<int32_t> iota(static_cast<size_t>(std::max(c->nstore, 1)));
    for (int i = 0; i < c->nstore; ++i) iota[i] = i;
    HRN_CUDA(c, c->d_store_iota.alloc(iota.size() * 4));
    HRN_CUDA(c, cudaMemcpy(c->d_store_iota.p, iota.data(), iota.size() * 4, cudaMemcpyHostToDevice));
    c->have_rd_store = true;
    return 0;
}

// Zero the gradient slots (on the stream) / sum them into node vectors g_l, g_m [nj].
static int gradient_slots_clear(hrn_ctx *c)
{
    HRN_CUDA(c, cudaMemsetAsync(c->d_gslot.p, 0, c->d_gslot.bytes, c->stream));
    return 0;
}

static int gradient_slots_to_nodes(hrn_ctx *c, double *g_l, double *g_m)
{
    const size_t ns = size_t(c->nel_rd) * 27;
    k_gradient_nodes<<<(c->nj + 255) / 256, 256, 0, c->stream>>>(c->nj, c->d_gnode_ptr.as<int32_t>(),
                                                                 c->d_gnode_slot.as<int32_t>(), c->d_gslot.as<double>(),
                                                                 c->d_gslot.as<double>() + ns, g_l, g_m);
    ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    return 0;
}

// ----------------------------------------------------------------------------
// time loops

template <typename T, int S>
static void launch_step(hrn_ctx *c, StageArgs<T> a, T *X, T *Y, StageTimer *tm, int lanes, const TileArgs &ta, int adj)
{
    const size_t vn = size_t(c->neq) * S;
    T *kb = c->d_KB.as<T>();
    a.x1 = X; a.x2 = X + vn; a.x3 = X + 2 * vn;
    a.kb1 = kb; a.kb2 = kb + vn; a.kb3 = kb + 2 * vn;
    a.y1 = Y; a.y2 = Y + vn; a.y3 = Y + 2 * vn;
    T *mA = c->d_MB.as<T>(), *mB = mA + 3 * vn;   // two sets of materialized stage inputs
    for (int st = 1; st <= 4; ++st) {
        if (tm) cudaEventRecord(tm->get(), c->stream);
        a.kb_out = st < 4 ? kb + size_t(st - 1) * vn : nullptr;
        T *in = (st == 3) ? mB : mA, *out = (st == 2) ? mB : mA;   // stage s reads set (s%2), writes the other
        a.in_t = in; a.in_m = in + vn; a.in_h = in + 2 * vn;
        a.out_t = out; a.out_m = out + vn; a.out_h = out + 2 * vn;
        if (is_elem_variant(lanes)) {
            const int b = lanes >= 100 ? 100 : 90;
            elem_stage(c, &a, st, adj, (lanes - b) % 2, 1 << ((lanes - b) / 2), b == 90 ? 1 : 0);
        } else if (is_gt_variant(lanes)) {
            gt_stage(c, &a, st, adj, lanes);
        } else {
            switch (st) {
            case 1: launch_stage<T, S, 1>(a, lanes, c->stream, ta); break;
            case 2: launch_stage<T, S, 2>(a, lanes, c->stream, ta); break;
            case 3: launch_stage<T, S, 3>(a, lanes, c->stream, ta); break;
            default: launch_stage<T, S, 4>(a, lanes, c->stream, ta); break;
            }
        }
        ++c->launches;
        if (tm) cudaEventRecord(tm->get(), c->stream);
        a.hist = nullptr;   // history only in stage 1
    }
}

static double sum_timer(hrn_ctx *c, const StageTimer &tm)
{
    double tot = 0.0;
    for (size_t i = 0; i + 1 < tm.used; i += 2) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev_pool[i], c->ev_pool[i + 1]);
        tot += ms;
    }
    return tot;
}

// Lanes per row for one operator: the fastest of 4, 8 and 16 over a few full
// RK4 steps on the zero state (the traffic does not depend on the values).
template <typename T, int S>
static int autotune_lanes(hrn_ctx *c, StageArgs<T> a, T *X, T *Y, const TileArgs &ta, int adj)
{
    a.hist = nullptr;
    float best = 1e30f;
    int pick = 80;
    std::vector<int> cand;
    if (c->have_pattern) cand.assign(kVariants, kVariants + 10);   // none with a matrix-free operator
    if (c->have_pattern && gt_ready(c, adj) == 0)
        // 47 / 87 (pipelined tiles) stay selectable but are not timed here: their many
        // small bulk copies are limited by the copy engine's rate (about 2x slower)
        for (int v : {44, 45, 84, 85, 46, 86})
            if (gt_runs_valid(v, c->nshot, c->elem_bytes())) cand.push_back(v);
    if (c->op_from_mesh) {
        if (int rc = elem_ready(c)) return rc;
        for (int v : {90, 91, 92, 93, 94, 95, 100, 101, 102, 103, 104, 105})
            if (elem_variant_valid(c, v)) cand.push_back(v);
    }
    if (cand.empty())
        return set_error(c, HRN_EARG, "no stage variant serves this operator, shot count and precision");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int lanes : cand) {
        launch_step<T, S>(c, a, X, Y, nullptr, lanes, ta, adj);   // warm-up
        cudaEventRecord(e0, c->stream);
        for (int r = 0; r < 3; ++r) launch_step<T, S>(c, a, X, Y, nullptr, lanes, ta, adj);
        cudaEventRecord(e1, c->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) { best = ms; pick = lanes; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    HRN_CUDA(c, cudaGetLastError());
    return pick;
}

static int check_step_error(hrn_ctx *c)
{
    int err = 0;
    HRN_CUDA(c, cudaMemcpy(&err, c->d_step_err.p, 4, cudaMemcpyDeviceToHost));
    if (err) {
        cudaMemset(c->d_step_err.p, 0, 4);
        if (err == 2) return set_error(c, HRN_ESTATE, "a stage ran without the tables of its kernel variant");
        return set_error(c, HRN_ECUDA, "a bounded wait of a stage kernel (bulk copies into shared memory) timed out");
    }
    return 0;
}

// Stage arguments of the forward operator (CSR, forward sources, history rows).
template <typename T, int S>
static StageArgs<T> forward_args(hrn_ctx *c)
{
    StageArgs<T> a{};
    a.n = c->neq;
    a.rowptr = c->d_rowptr.as<int32_t>();
    a.seg = c->d_seg.as<int2>();
    a.colx = c->d_colx.as<uint32_t>();
    a.val = c->d_fwd.as<T>();
    a.slot = c->d_slot_f.as<int32_t>();
    a.nslot = c->nslot_f;
    a.store_pos = c->d_store_pos.as<int32_t>();
    a.c = T(0.5 * c->dt);
    a.D = T(c->dt);
    a.d6 = T(c->dt / 6.0);
    return a;
}

template <typename T, int S>
static const T *forward_src(hrn_ctx *c, int n)
{
    return c->nslot_f ? c->d_srcv_f.as<T>() + size_t(n) * 4 * c->nslot_f * S : nullptr;
}

// ----------------------------------------------------------------------------
// CUDA graphs of the time loops.  A call's stream work (memsets, source tables,
// every stage, history, trace and gradient launch of all steps) is captured once
// and replayed while nothing it names can have changed: the allocation
// generation (every DevBuf allocation or release), the settings epoch (every
// setter), the variant and the call's flags.  Values in the buffers -- the
// scaled operator after a reassembly, the data, the time functions -- may
// change between replays.  Host work (autotuning, table builds, allocations)
// stays outside the capture.

static bool graph_usable(const hrn_ctx *c)
{
    return c->graphs && !c->timing && c->stream != nullptr && c->stream != cudaStreamLegacy;
}

// Capture body(c) on the context's stream into g (replacing an older graph).
// Returns false, with the stream usable and no error pending, if capture or
// instantiation fails; the caller then runs the body directly.
template <typename F>
static bool graph_capture(hrn_ctx *c, LoopGraph &g, const uint64_t (&sig)[6], F body)
{
    g.reset();
    const int64_t l0 = c->launches;
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const int rc = body();
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(c->stream, &graph);
    const int64_t captured = c->launches - l0;
    c->launches = l0;
    bool ok = rc == 0 && ec == cudaSuccess && graph != nullptr;
    if (ok) ok = cudaGraphInstantiate(&g.exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    if (!ok) {
        cudaGetLastError();
        g.reset();
        return false;
    }
    for (int k = 0; k < 6; ++k) g.sig[k] = sig[k];
    g.launches = captured;
    return true;
}

// Run body(c) through the graph g when possible, directly otherwise.
template <typename F>
static int run_loop(hrn_ctx *c, LoopGraph &g, const uint64_t (&sig)[6], F body)
{
    if (graph_usable(c)) {
        bool same = g.exec != nullptr;
        for (int k = 0; k < 6 && same; ++k) same = g.sig[k] == sig[k];
        if (!same && graph_capture(c, g, sig, body)) {
            same = true;
            ++c->graph_captures;
        }
        if (same) {
            HRN_CUDA(c, cudaGraphLaunch(g.exec, c->stream));
            c->launches += g.launches;
            ++c->graph_replays;
            return 0;
        }
    }
    return body();
}

template <typename T, int S>
static int forward_t(hrn_ctx *c)
{
    const size_t vn = size_t(c->neq) * S;
    T *X0 = c->d_X.as<T>(), *X1 = X0 + 3 * vn;
    StageArgs<T> a = forward_args<T, S>(c);
    TileArgs ta{c->d_tiles.as<int32_t>(), c->ntiles, std::min(c->ntiles, 2 * c->num_sms), c->d_step_err.as<int>()};
    // variant choice and its tables: host work, before any capture
    if (c->lanes_f <= 0) {
        // first use: the source table, then time the variants on the zero state
        HRN_CUDA(c, cudaMemsetAsync(X0, 0, 3 * vn * sizeof(T), c->stream));
        if (c->nslot_f > 0) {
            const int64_t tot = int64_t(c->nstep + 1) * c->nslot_f * S;
            k_src_fwd<T, S><<<blocks_for(tot, 256), 256, 0, c->stream>>>(c->nstep, c->nslot_f, c->d_fslot_eq.as<int32_t>(),
                                                                         c->d_fsrc_b.as<double>(), c->d_ftab.as<double>(),
                                                                         c->d_im.as<double>(), c->d_srcv_f.as<T>()); ++c->launches;
            HRN_CUDA(c, cudaGetLastError());
        }
        a.srcv = c->d_srcv_f.as<T>();
        const int r = autotune_lanes<T, S>(c, a, X0, X1, ta, 0);
        if (r < 40) return r;
        c->lanes_f = r;
    }
    if (c->mf_only && !is_elem_variant(c->lanes_f))
        return set_error(c, HRN_EARG, "the operator is matrix-free: use variants 90-95 / 100-105");
    if (is_elem_variant(c->lanes_f)) {
        if (!elem_variant_valid(c, c->lanes_f)) return set_error(c, HRN_EARG, "matrix-free variant not available for this shot count and precision");
        if (int rc = elem_ready(c)) return rc;
    } else if (is_gt_variant(c->lanes_f)) {
        if (!gt_runs_valid(c->lanes_f, c->nshot, c->elem_bytes()))
            return set_error(c, HRN_EARG, "variants 46, 47, 86, 87 need records (shots x value size) of a multiple of 16 bytes");
        if (int rc = gt_ready(c, 0)) return rc;
        if (is_gtp_variant(c->lanes_f))
            if (int rc = gtp_prepare(c, 0)) return rc;
    }
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, c->stream);
    StageTimer tm(c);
    // stream work only: memsets, source table, every step
    auto body = [&]() -> int {
        HRN_CUDA(c, cudaMemsetAsync(X0, 0, 3 * vn * sizeof(T), c->stream));
        if (c->nslot_f > 0) {
            const int64_t tot = int64_t(c->nstep + 1) * c->nslot_f * S;
            k_src_fwd<T, S><<<blocks_for(tot, 256), 256, 0, c->stream>>>(c->nstep, c->nslot_f, c->d_fslot_eq.as<int32_t>(),
                                                                         c->d_fsrc_b.as<double>(), c->d_ftab.as<double>(),
                                                                         c->d_im.as<double>(), c->d_srcv_f.as<T>()); ++c->launches;
            HRN_CUDA(c, cudaGetLastError());
        }
        const int K = c->ckpt;
        for (int n = 0; n <= c->nstep; ++n) {
            a.srcv = forward_src<T, S>(c, n);
            T *X = (n & 1) ? X1 : X0, *Y = (n & 1) ? X0 : X1;
            if (K > 0) {
                // checkpointed: the state every K steps and the receiver rows of every step
                if (n % K == 0)
                    HRN_CUDA(c, cudaMemcpyAsync(c->d_ckpt.as<T>() + size_t(n / K) * 3 * vn, X, 3 * vn * sizeof(T),
                                                cudaMemcpyDeviceToDevice, c->stream));
                if (c->nrec3 > 0) {
                    k_traces<T, S><<<(c->nrec3 * S + 127) / 128, 128, 0, c->stream>>>(
                        c->nrec3, c->d_eqdis.as<int32_t>(), X + vn, c->d_traces.as<T>() + size_t(n) * c->nrec3 * S);
                    ++c->launches;
                }
                a.hist = nullptr;
            } else {
                a.hist = c->d_hist.as<T>() + size_t(n) * c->nstore * S;
            }
            launch_step<T, S>(c, a, X, Y, c->timing ? &tm : nullptr, c->lanes_f, ta, 0);
        }
        HRN_CUDA(c, cudaGetLastError());
        return 0;
    };
    const uint64_t sig[6] = {alloc_generation().load(), c->epoch, uint64_t(c->lanes_f), 0, 0, uintptr_t(c->stream)};
    const int rc = run_loop(c, c->gfwd, sig, body);
    cudaEventRecord(t1, c->stream);
    if (rc) {
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        return rc;
    }
    HRN_CUDA(c, cudaEventSynchronize(t1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    c->last_total_ms = ms;
    c->last_stage_ms = c->timing ? sum_timer(c, tm) : 0.0;
    c->last_stage_launches = c->timing ? int64_t(tm.used / 2) : 0;
    c->acc_stage_ms += c->last_stage_ms;
    c->acc_stage_launches += c->last_stage_launches;
    if (int rc2 = check_step_error(c)) return rc2;
    c->have_forward = true;
    c->have_phist = false;
    return 0;
}

template <typename T, int S>
static int adjoint_t(hrn_ctx *c, int lambda_2mu, int keep_p)
{
    if (int rc = build_rd_store(c)) return rc;
    if (!c->side_stream) {
        HRN_CUDA(c, cudaStreamCreateWithFlags(&c->side_stream, cudaStreamNonBlocking));
        HRN_CUDA(c, cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
        HRN_CUDA(c, cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
    }
    const size_t vn = size_t(c->neq) * S;
    T *X0 = c->d_X.as<T>(), *X1 = X0 + 3 * vn;
    if (keep_p) HRN_CUDA(c, c->d_phist.alloc(size_t(c->nstep + 1) * c->nstore * S * sizeof(T)));
    StageArgs<T> a{};
    a.n = c->neq;
    a.rowptr = c->d_rowptrT.as<int32_t>();
    a.seg = c->d_segT.as<int2>();
    a.colx = c->d_colxT.as<uint32_t>();
    a.val = c->d_adj.as<T>();
    a.slot = c->d_slot_a.as<int32_t>();
    a.nslot = c->nslot_a;
    a.srcv = c->d_srcv_a.as<T>();
    a.store_pos = c->d_store_pos.as<int32_t>();
    a.c = T(-0.5 * c->dt);
    a.D = T(-c->dt);
    a.d6 = T(-c->dt / 6.0);
    TileArgs ta{c->d_tilesT.as<int32_t>(), c->ntilesT, std::min(c->ntilesT, 2 * c->num_sms), c->d_step_err.as<int>()};
    // variant choice and its tables: host work, before any capture
    if (c->lanes_a <= 0) {
        HRN_CUDA(c, cudaMemsetAsync(X0, 0, 3 * vn * sizeof(T), c->stream));
        const int r = autotune_lanes<T, S>(c, a, X0, X1, ta, 1);
        if (r < 40) return r;
        c->lanes_a = r;
    }
    if (c->mf_only && !is_elem_variant(c->lanes_a))
        return set_error(c, HRN_EARG, "the operator is matrix-free: use variants 90-95 / 100-105");
    if (is_elem_variant(c->lanes_a)) {
        if (!elem_variant_valid(c, c->lanes_a)) return set_error(c, HRN_EARG, "matrix-free variant not available for this shot count and precision");
        if (int rc = elem_ready(c)) return rc;
    } else if (is_gt_variant(c->lanes_a)) {
        if (!gt_runs_valid(c->lanes_a, c->nshot, c->elem_bytes()))
            return set_error(c, HRN_EARG, "variants 46, 47, 86, 87 need records (shots x value size) of a multiple of 16 bytes");
        if (int rc = gt_ready(c, 1)) return rc;
        if (is_gtp_variant(c->lanes_a))
            if (int rc = gtp_prepare(c, 1)) return rc;
    }
    if (c->ckpt > 0 && is_gt_variant(c->lanes_f)) {   // the recomputed forward segments
        if (int rc = gt_ready(c, 0)) return rc;
        if (is_gtp_variant(c->lanes_f))
            if (int rc = gtp_prepare(c, 0)) return rc;
    }
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, c->stream);
    StageTimer tm(c);
    double *gl = c->d_g.as<double>(), *gmu = gl + c->nj;
    double *gsl = c->d_gslot.as<double>(), *gsm = gsl + size_t(c->nel_rd) * 27;   // point slots
    const int gblocks = (c->nel_rd + kGradElems - 1) / kGradElems;
    const RecView rv = rec_view(c);
    const int K = c->ckpt;
    StageArgs<T> af = forward_args<T, S>(c);
    TileArgs taf{c->d_tiles.as<int32_t>(), c->ntiles, std::min(c->ntiles, 2 * c->num_sms), c->d_step_err.as<int>()};
    // stream work only: memsets, every adjoint step with its sources, the recomputed
    // forward segments and the gradient
    auto body = [&]() -> int {
        HRN_CUDA(c, cudaMemsetAsync(X0, 0, 3 * vn * sizeof(T), c->stream));
        if (int rc = gradient_slots_clear(c)) return rc;
        if (keep_p) HRN_CUDA(c, cudaMemsetAsync(c->d_phist.p, 0, c->d_phist.bytes, c->stream));
        int it = 0;
        bool forked = false;   // a gradient launch is pending on the side stream
        for (int n = c->nstep; n >= 1; --n, ++it) {
            // the previous step's gradient read the state this step overwrites and the
            // history segment a recompute overwrites: it must be done first
            if (forked) HRN_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_join, 0));
            const int k0 = K > 0 ? (n / K) * K : 0;   // first step of n's checkpoint segment
            if (K > 0 && (n == c->nstep || n % K == K - 1)) {
                // recompute the forward history of steps k0 .. min(k0 + K - 1, nstep - 1) from the checkpoint
                T *R0 = c->d_Xr.as<T>(), *R1 = R0 + 3 * vn;
                HRN_CUDA(c, cudaMemcpyAsync(R0, c->d_ckpt.as<T>() + size_t(n / K) * 3 * vn, 3 * vn * sizeof(T),
                                            cudaMemcpyDeviceToDevice, c->stream));
                const int m1 = std::min(k0 + K - 1, c->nstep - 1);
                for (int m = k0; m <= m1; ++m) {
                    af.srcv = forward_src<T, S>(c, m);
                    af.hist = c->d_ckseg.as<T>() + size_t(m - k0) * c->nstore * S;
                    T *Xm = ((m - k0) & 1) ? R1 : R0, *Ym = ((m - k0) & 1) ? R0 : R1;
                    launch_step<T, S>(c, af, Xm, Ym, c->timing ? &tm : nullptr, c->lanes_f, taf, 0);
                }
            }
            const T *u_n = K > 0 ? c->d_ckseg.as<T>() + size_t(n - k0) * c->nstore * S
                                 : c->d_hist.as<T>() + size_t(n) * c->nstore * S;
            if (c->nslot_a > 0)
                k_src_adj<T, S><<<(c->nslot_a * S + 127) / 128, 128, 0, c->stream>>>(
                    n, c->nstep, rv.stride, c->nrec3, c->nslot_a, c->d_aslot_ptr.as<int32_t>(), c->d_aslot_q.as<int32_t>(),
                    c->d_aslot_eq.as<int32_t>(), rv.map, static_cast<const T *>(rv.hist), c->d_dis.as<double>(),
                    c->d_im.as<double>(), c->d_srcv_a.as<T>(), shot_nstep_ptr(c), rec_mask_ptr(c)); ++c->launches;
            a.hist = keep_p ? c->d_phist.as<T>() + size_t(n) * c->nstore * S : nullptr;
            T *X = (it & 1) ? X1 : X0, *Y = (it & 1) ? X0 : X1;
            if (n <= c->nstep - 1 && c->nel_rd > 0) {
                // the zero-lag correlation of this step's state runs on the side stream,
                // next to the step's stages (they read X and write Y, KB, MB)
                HRN_CUDA(c, cudaEventRecord(c->ev_fork, c->stream));
                HRN_CUDA(c, cudaStreamWaitEvent(c->side_stream, c->ev_fork, 0));
                k_gradient<T, S><<<gblocks, 128, 0, c->side_stream>>>(c->nel_rd, c->d_rd_store.as<int32_t>(), c->d_rd_elems.as<int32_t>(),
                                                                      c->d_inod.as<int32_t>(), c->d_rd_geom.as<double>(),
                                                                      u_n, X + vn,
                                                                      c->d_store_eq.as<int32_t>(), gsl, gsm, c->dt, lambda_2mu); ++c->launches;
                HRN_CUDA(c, cudaEventRecord(c->ev_join, c->side_stream));
                forked = true;
            }
            launch_step<T, S>(c, a, X, Y, c->timing ? &tm : nullptr, c->lanes_a, ta, 1);
        }
        if (forked) HRN_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_join, 0));
        if (int rc = gradient_slots_to_nodes(c, gl, gmu)) return rc;
        HRN_CUDA(c, cudaGetLastError());
        return 0;
    };
    const uint64_t sig[6] = {alloc_generation().load(), c->epoch, uint64_t(c->lanes_a) | (uint64_t(c->lanes_f) << 32),
                             uint64_t(keep_p != 0), uint64_t(lambda_2mu != 0), uintptr_t(c->stream)};
    const int rc = run_loop(c, c->gadj, sig, body);
    cudaEventRecord(t1, c->stream);
    if (rc) {
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        return rc;
    }
    HRN_CUDA(c, cudaEventSynchronize(t1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    c->last_total_ms = ms;
    c->last_stage_ms = c->timing ? sum_timer(c, tm) : 0.0;
    c->last_stage_launches = c->timing ? int64_t(tm.used / 2) : 0;
    c->acc_stage_ms += c->last_stage_ms;
    c->acc_stage_launches += c->last_stage_launches;
    if (int rc2 = check_step_error(c)) return rc2;
    c->have_phist = keep_p != 0;
    return 0;
}

template <typename T, int S>
static int misfit_t(hrn_ctx *c, double *cost)
{
    const int tot = (c->nstep + 1) * S;
    const RecView rv = rec_view(c);
    k_misfit_terms<T, S><<<(tot + 127) / 128, 128, 0, c->stream>>>(c->nstep, rv.stride, c->nrec3, c->nslot_a,
                                                                   c->d_aslot_ptr.as<int32_t>(), c->d_aslot_q.as<int32_t>(),
                                                                   rv.map, static_cast<const T *>(rv.hist),
                                                                   c->d_dis.as<double>(), c->d_mis_terms.as<double>(),
                                                                   shot_nstep_ptr(c), rec_mask_ptr(c)); ++c->launches;
    k_misfit_sum<<<1, 1, 0, c->stream>>>(S, c->nstep, c->dt, c->d_mis_terms.as<double>(), c->d_cost.as<double>()); ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    std::vector<double> h(size_t(1 + S));
    HRN_CUDA(c, cudaMemcpyAsync(h.data(), c->d_cost.p, h.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int s = 0; s < 1 + S; ++s) cost[s] = h[s];
    return 0;
}

// Diagonal pseudo-Hessian of the lambda / mu model: the gradient's zero-lag
// correlation (k_gradient) with the forward wavefield in place of the adjoint one,
// sum over n = 1 .. nstep-1 and shots of dt * [ (div u)^2 ] and of the strain-energy
// term, at the regular-domain nodes.  hl, hm: device arrays [nj].
template <typename T, int S>
static int pseudo_hessian_t(hrn_ctx *c, double *hl, double *hm)
{
    if (int rc = build_rd_store(c)) return rc;   // also the identity map of the history rows
    if (int rc = gradient_slots_clear(c)) return rc;
    double *gsl = c->d_gslot.as<double>(), *gsm = gsl + size_t(c->nel_rd) * 27;
    const int gblocks = (c->nel_rd + kGradElems - 1) / kGradElems;
    if (c->nel_rd > 0)
        for (int n = 1; n <= c->nstep - 1; ++n) {
            const T *u_n = c->d_hist.as<T>() + size_t(n) * c->nstore * S;
            // p := u: the history row read again through the identity position map
            k_gradient<T, S><<<gblocks, 128, 0, c->stream>>>(c->nel_rd, c->d_rd_store.as<int32_t>(), c->d_rd_elems.as<int32_t>(),
                                                             c->d_inod.as<int32_t>(), c->d_rd_geom.as<double>(), u_n, u_n,
                                                             c->d_store_iota.as<int32_t>(), gsl, gsm, c->dt, 0);
            ++c->launches;
        }
    if (int rc = gradient_slots_to_nodes(c, hl, hm)) return rc;
    HRN_CUDA(c, cudaGetLastError());
    return 0;
}

#define HRN_DISPATCH_S(FN, T, ...)                        \
    switch (c->nshot) {                                   \
    case 1: return FN<T, 1>(c, ##__VA_ARGS__);            \
    case 2: return FN<T, 2>(c, ##__VA_ARGS__);            \
    case 3: return FN<T, 3>(c, ##__VA_ARGS__);            \
    case 4: return FN<T, 4>(c, ##__VA_ARGS__);            \
    case 5: return FN<T, 5>(c, ##__VA_ARGS__);            \
    case 6: return FN<T, 6>(c, ##__VA_ARGS__);            \
    case 7: return FN<T, 7>(c, ##__VA_ARGS__);            \
    case 8: return FN<T, 8>(c, ##__VA_ARGS__);            \
    default: return set_error(c, HRN_EARG, "nshot out of range"); \
    }

// Device time of the stage kernel alone: nsteps RK4 steps (4 stage launches
// each) of the tuned variant, back to back from the zero state with the first
// step's sources and no history, bracketed by one pair of CUDA events on the
// context's stream.  The traffic of a stage does not depend on the values.  The forward history and
// the checkpoints are untouched; the state and stage buffers are scratch.
template <typename T, int S>
static int time_stage_t(hrn_ctx *c, int adj, int nsteps, double *avg_ms)
{
    const int lanes = adj ? c->lanes_a : c->lanes_f;
    if (lanes <= 0) return set_error(c, HRN_ESTATE, "no tuned stage variant: run hrn_forward (and hrn_adjoint_gradient) first");
    const size_t vn = size_t(c->neq) * S;
    T *X0 = c->d_X.as<T>(), *X1 = X0 + 3 * vn;
    StageArgs<T> a = forward_args<T, S>(c);
    TileArgs ta{c->d_tiles.as<int32_t>(), c->ntiles, std::min(c->ntiles, 2 * c->num_sms), c->d_step_err.as<int>()};
    if (adj) {
        a.rowptr = c->d_rowptrT.as<int32_t>();
        a.seg = c->d_segT.as<int2>();
        a.colx = c->d_colxT.as<uint32_t>();
        a.val = c->d_adj.as<T>();
        a.slot = c->d_slot_a.as<int32_t>();
        a.nslot = c->nslot_a;
        a.c = T(-0.5 * c->dt);
        a.D = T(-c->dt);
        a.d6 = T(-c->dt / 6.0);
        ta = TileArgs{c->d_tilesT.as<int32_t>(), c->ntilesT, std::min(c->ntilesT, 2 * c->num_sms), c->d_step_err.as<int>()};
    }
    // the sources of the first step (the tables exist once the variant is tuned)
    a.srcv = adj ? c->d_srcv_a.as<T>() : forward_src<T, S>(c, 0);
    a.hist = nullptr;
    if (a.nslot > 0 && !a.srcv) return set_error(c, HRN_ESTATE, "no source table: run the time loop first");
    if (is_elem_variant(lanes)) {
        if (int rc = elem_ready(c)) return rc;
    } else if (is_gt_variant(lanes)) {
        if (!gt_runs_valid(lanes, c->nshot, c->elem_bytes())) return set_error(c, HRN_EARG, "variant needs 16-byte records");
        if (int rc = gt_ready(c, adj)) return rc;
        if (is_gtp_variant(lanes))
            if (int rc = gtp_prepare(c, adj)) return rc;
    }
    HRN_CUDA(c, cudaMemsetAsync(X0, 0, 6 * vn * sizeof(T), c->stream));
    launch_step<T, S>(c, a, X0, X1, nullptr, lanes, ta, adj);   // warm-up
    cudaEvent_t e0, e1;
    HRN_CUDA(c, cudaEventCreate(&e0));
    HRN_CUDA(c, cudaEventCreate(&e1));
    cudaEventRecord(e0, c->stream);
    for (int n = 0; n < nsteps; ++n) {
        T *X = (n & 1) ? X1 : X0, *Y = (n & 1) ? X0 : X1;
        launch_step<T, S>(c, a, X, Y, nullptr, lanes, ta, adj);
    }
    cudaEventRecord(e1, c->stream);
    const cudaError_t es = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (es == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    HRN_CUDA(c, es);
    HRN_CUDA(c, cudaGetLastError());
    if (int rc = check_step_error(c)) return rc;
    *avg_ms = double(ms) / (4.0 * nsteps);
    return 0;
}

int run_time_stage(hrn_ctx *c, int adj, int nsteps, double *avg_ms)
{
    if (c->precision == HRN_FP64) { HRN_DISPATCH_S(time_stage_t, double, adj, nsteps, avg_ms) }
    HRN_DISPATCH_S(time_stage_t, float, adj, nsteps, avg_ms)
}

int run_forward(hrn_ctx *c)
{
    if (c->precision == HRN_FP64) { HRN_DISPATCH_S(forward_t, double) }
    HRN_DISPATCH_S(forward_t, float)
}

int run_adjoint_gradient(hrn_ctx *c, int lambda_2mu, int keep_p)
{
    if (c->precision == HRN_FP64) { HRN_DISPATCH_S(adjoint_t, double, lambda_2mu, keep_p) }
    HRN_DISPATCH_S(adjoint_t, float, lambda_2mu, keep_p)
}

int run_pseudo_hessian(hrn_ctx *c, double *hl, double *hm)
{
    if (c->precision == HRN_FP64) { HRN_DISPATCH_S(pseudo_hessian_t, double, hl, hm) }
    HRN_DISPATCH_S(pseudo_hessian_t, float, hl, hm)
}

int run_misfit(hrn_ctx *c, double *cost)
{
    if (c->precision == HRN_FP64) { HRN_DISPATCH_S(misfit_t, double, cost) }
    HRN_DISPATCH_S(misfit_t, float, cost)
}

}  // namespace hrn
