// hrn_inv.cu -- device side of the model update of the inversion loop
// (S4/Program_Main.F90:411-896, S4/LBFGS_Coupled.F90, S4/Control_Problem_Operators.F90):
// FP64 vector algebra with deterministic reductions, the TV regularization and
// lumped gradient mass element kernels, and the coupled L-BFGS two-loop
// recursion.  All vectors are nodal (length nj) FP64 device arrays; the driver
// keeps its control flow on the host and reads back scalars only.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "hrn_internal.h"

namespace hrn {

constexpr int kRedBlocks = 296;   // 2 x 148 SMs
constexpr int kRedThreads = 256;

// partial[b] = sum over the grid-stride slice of block b, in a fixed order
template <int KIND>
__global__ void k_reduce_partial(int n, const double *__restrict__ x, const double *__restrict__ y, double *__restrict__ part)
{
    __shared__ double sh[kRedThreads];
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if constexpr (KIND == 0) acc += x[i] * y[i];          // dot
        else if constexpr (KIND == 1) acc += x[i] * x[i];     // squared 2-norm
        else acc = fmax(acc, fabs(x[i]));                      // inf-norm
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            if constexpr (KIND == 2) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + s]);
            else sh[threadIdx.x] += sh[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

template <int KIND>
__global__ void k_reduce_final(int np, const double *__restrict__ part, double *__restrict__ out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double acc = 0.0;
    for (int i = 0; i < np; ++i) {
        if constexpr (KIND == 2) acc = fmax(acc, part[i]);
        else acc += part[i];
    }
    out[0] = KIND == 1 ? sqrt(acc) : acc;
}

// z = a x + b y  (y may be null: z = a x)
__global__ void k_axpby(int n, double a, const double *__restrict__ x, double b, const double *__restrict__ y, double *__restrict__ z)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        z[i] = y ? a * x[i] + b * y[i] : a * x[i];
}

__global__ void k_mul(int n, const double *__restrict__ x, const double *__restrict__ y, double *__restrict__ z)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) z[i] = x[i] * y[i];
}

__global__ void k_clip(int n, double lo, double hi, double *__restrict__ x)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double v = x[i];
        x[i] = v < lo ? lo : (v > hi ? hi : v);
    }
}

__global__ void k_gather(int n, const int32_t *__restrict__ map, const double *__restrict__ x, double *__restrict__ y)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = x[map[i]];
}

// ----------------------------------------------------------------------------
// element kernels over the regular domain (GLL points, one thread per point)

__constant__ int v_node_at[27];
__constant__ double v_D[3][3];

// TV regularization (ELEMENT_TV_TN_Reg_3D, S4/Element_Matrices_3D.F90:1899-2074, unweighted):
// per point, ER = sum_k dN_I/dx_k dN_J/dx_k, vh = ER e, den = sqrt(e.vh + 0.01),
// E_Reg += vh / den * w detJ, cost += (e.vh) / den * w detJ.  With the GLL rule
// vh_I = sum_k dN_I/dx_k g_k and e.vh = |g|^2 where g = grad e at the point, and
// only the 7 nodes on the lines through the point receive a contribution.
__global__ void k_tv(int nel_rd, const int32_t *__restrict__ rd_elems, const int32_t *__restrict__ inod,
                     const double *__restrict__ geom, const double *__restrict__ lam, const double *__restrict__ mu,
                     double *__restrict__ reg_l, double *__restrict__ reg_m, double *__restrict__ cost_part)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double cl = 0.0, cm = 0.0;
    if (t < nel_rd * 27) {
        const int e = t / 27, q = t % 27;
        const int aq = q % 3, bq = (q / 3) % 3, cq = q / 9;
        const int32_t *nd = inod + size_t(rd_elems[e]) * 27;
        const double *g = geom + size_t(t) * 10;
        int ln[3][3];   // [direction][t] local node on the line through q
        for (int u = 0; u < 3; ++u) {
            ln[0][u] = v_node_at[9 * cq + 3 * bq + u];
            ln[1][u] = v_node_at[9 * cq + 3 * u + aq];
            ln[2][u] = v_node_at[9 * u + 3 * bq + aq];
        }
        const int qi[3] = {aq, bq, cq};
        for (int f = 0; f < 2; ++f) {
            const double *val = f == 0 ? mu : lam;
            double *reg = f == 0 ? reg_m : reg_l;
            double dxi[3];
            for (int m = 0; m < 3; ++m) {
                double s = 0.0;
                for (int u = 0; u < 3; ++u) s += v_D[qi[m]][u] * val[nd[ln[m][u]]];
                dxi[m] = s;
            }
            double gr[3];
            for (int k = 0; k < 3; ++k) gr[k] = dxi[0] * g[0 * 3 + k] + dxi[1] * g[1 * 3 + k] + dxi[2] * g[2 * 3 + k];
            const double num = gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2];
            const double den = sqrt(num + 0.01);
            const double w = g[9] / den;
            // vh_I = sum_k DFX(I,k) gr_k with DFX(I,k) = sum_m DFXI(I,m) DJI(m,k)
            for (int m = 0; m < 3; ++m) {
                const double proj = g[m * 3 + 0] * gr[0] + g[m * 3 + 1] * gr[1] + g[m * 3 + 2] * gr[2];
                for (int u = 0; u < 3; ++u) atomicAdd(reg + nd[ln[m][u]], v_D[qi[m]][u] * proj * w);
            }
            if (f == 0) cm = num / den * g[9];
            else cl = num / den * g[9];
        }
    }
    // deterministic per-block cost partials
    __shared__ double shl[256], shm[256];
    shl[threadIdx.x] = cl;
    shm[threadIdx.x] = cm;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            shl[threadIdx.x] += shl[threadIdx.x + s];
            shm[threadIdx.x] += shm[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        cost_part[2 * blockIdx.x] = shl[0];
        cost_part[2 * blockIdx.x + 1] = shm[0];
    }
}

// Lumped gradient mass (ELEMENT_R_Mg_3D diagonal): Mg(node) += w detJ at the node's point.
__global__ void k_gradient_mass(int nel_rd, const int32_t *__restrict__ rd_elems, const int32_t *__restrict__ inod,
                                const double *__restrict__ geom, double *__restrict__ mg)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nel_rd * 27) return;
    const int e = t / 27, q = t % 27;
    atomicAdd(mg + inod[size_t(rd_elems[e]) * 27 + v_node_at[q]], geom[size_t(t) * 10 + 9]);
}

// ----------------------------------------------------------------------------
// host helpers

static int grid_for(int n) { return std::min(std::max((n + 255) / 256, 1), 148 * 8); }

int vec_reduce(hrn_ctx *c, int kind, int n, const double *x, const double *y, double *out)
{
    if (!c->d_red.p) HRN_CUDA(c, c->d_red.alloc((kRedBlocks + 1) * 8));
    double *part = c->d_red.as<double>();
    if (kind == 0) k_reduce_partial<0><<<kRedBlocks, kRedThreads, 0, c->stream>>>(n, x, y, part);
    else if (kind == 1) k_reduce_partial<1><<<kRedBlocks, kRedThreads, 0, c->stream>>>(n, x, y, part);
    else k_reduce_partial<2><<<kRedBlocks, kRedThreads, 0, c->stream>>>(n, x, y, part);
    ++c->launches;
    if (kind == 0) k_reduce_final<0><<<1, 32, 0, c->stream>>>(kRedBlocks, part, part + kRedBlocks);
    else if (kind == 1) k_reduce_final<1><<<1, 32, 0, c->stream>>>(kRedBlocks, part, part + kRedBlocks);
    else k_reduce_final<2><<<1, 32, 0, c->stream>>>(kRedBlocks, part, part + kRedBlocks);
    ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    HRN_CUDA(c, cudaMemcpyAsync(out, part + kRedBlocks, 8, cudaMemcpyDeviceToHost, c->stream));
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    return 0;
}

int vec_axpby(hrn_ctx *c, int n, double a, const double *x, double b, const double *y, double *z)
{
    k_axpby<<<grid_for(n), 256, 0, c->stream>>>(n, a, x, b, y, z);
    ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    return 0;
}

static int upload_inv_tables(hrn_ctx *c)
{
    static const int ijk[27][3] = {{2, 0, 0}, {2, 2, 0}, {0, 2, 0}, {0, 0, 0}, {2, 0, 2}, {2, 2, 2}, {0, 2, 2}, {0, 0, 2},
                                   {2, 1, 0}, {1, 2, 0}, {0, 1, 0}, {1, 0, 0}, {2, 0, 1}, {2, 2, 1}, {0, 2, 1}, {0, 0, 1},
                                   {2, 1, 2}, {1, 2, 2}, {0, 1, 2}, {1, 0, 2}, {1, 1, 0}, {2, 1, 1}, {1, 2, 1}, {0, 1, 1},
                                   {1, 0, 1}, {1, 1, 2}, {1, 1, 1}};
    int node_at[27];
    for (int i = 0; i < 27; ++i) node_at[9 * ijk[i][2] + 3 * ijk[i][1] + ijk[i][0]] = i;
    const double D[3][3] = {{-1.5, 2.0, -0.5}, {-0.5, 0.0, 0.5}, {0.5, -2.0, 1.5}};
    HRN_CUDA(c, cudaMemcpyToSymbol(v_node_at, node_at, sizeof(node_at)));
    HRN_CUDA(c, cudaMemcpyToSymbol(v_D, D, sizeof(D)));
    return 0;
}

int regularization_tv(hrn_ctx *c, const double *lam, const double *mu, double *reg_l, double *reg_m, double *cost_l, double *cost_m)
{
    if (int rc = upload_inv_tables(c)) return rc;
    HRN_CUDA(c, cudaMemsetAsync(reg_l, 0, size_t(c->nj) * 8, c->stream));
    HRN_CUDA(c, cudaMemsetAsync(reg_m, 0, size_t(c->nj) * 8, c->stream));
    const int th = 256, nb = std::max((c->nel_rd * 27 + th - 1) / th, 1);
    DevBuf &part = c->d_tv_part;   // kept, so that repeated calls allocate nothing
    HRN_CUDA(c, part.alloc(size_t(2) * nb * 8));
    k_tv<<<nb, th, 0, c->stream>>>(c->nel_rd, c->d_rd_elems.as<int32_t>(), c->d_inod.as<int32_t>(), c->d_rd_geom.as<double>(),
                                   lam, mu, reg_l, reg_m, part.as<double>());
    ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    std::vector<double> h(size_t(2) * nb);
    HRN_CUDA(c, cudaMemcpyAsync(h.data(), part.p, h.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    double sl = 0.0, sm = 0.0;
    for (int b = 0; b < nb; ++b) { sl += h[2 * b]; sm += h[2 * b + 1]; }
    *cost_l = sl;
    *cost_m = sm;
    return 0;
}

int gradient_mass(hrn_ctx *c, double *mg)
{
    if (int rc = upload_inv_tables(c)) return rc;
    HRN_CUDA(c, cudaMemsetAsync(mg, 0, size_t(c->nj) * 8, c->stream));
    const int th = 256;
    if (c->nel_rd > 0)
        k_gradient_mass<<<(c->nel_rd * 27 + th - 1) / th, th, 0, c->stream>>>(c->nel_rd, c->d_rd_elems.as<int32_t>(),
                                                                               c->d_inod.as<int32_t>(), c->d_rd_geom.as<double>(), mg);
    ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    return 0;
}

}  // namespace hrn

using namespace hrn;

namespace hrn {
// Source illumination of every stored node: the sum over steps, shots and the three
// displacement components of u^2 in the forward history [nstep+1][nstore][S].
template <typename T>
__global__ void k_illumination(int nnode, int nstore, int nstep, int S, const T *__restrict__ hist, double *__restrict__ out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nnode) return;
    double acc = 0.0;
    for (int n = 0; n <= nstep; ++n) {
        const T *h = hist + (size_t(n) * nstore + 3 * size_t(k)) * S;
        for (int i = 0; i < 3 * S; ++i) {
            const double v = double(h[i]);
            acc = fma(v, v, acc);
        }
    }
    out[k] = acc;
}

}  // namespace hrn

extern "C" {

int hrn_vec_dot(hrn_ctx *c, int32_t n, const double *x, const double *y, double *out)
{
    if (!c || !x || !y || !out || n < 0) return HRN_EARG;
    return vec_reduce(c, 0, n, x, y, out);
}

int hrn_vec_norm(hrn_ctx *c, int32_t n, const double *x, int32_t kind, double *out)
{
    if (!c || !x || !out || n < 0 || (kind != 2 && kind != 0)) return c ? set_error(c, HRN_EARG, "norm kind must be 2 or 0 (infinity)") : HRN_EARG;
    return vec_reduce(c, kind == 2 ? 1 : 2, n, x, nullptr, out);
}

int hrn_vec_axpby(hrn_ctx *c, int32_t n, double a, const double *x, double b, const double *y, double *z)
{
    if (!c || !x || !z || n < 0) return HRN_EARG;
    return vec_axpby(c, n, a, x, b, y, z);
}

int hrn_vec_mul(hrn_ctx *c, int32_t n, const double *x, const double *y, double *z)
{
    if (!c || !x || !y || !z || n < 0) return HRN_EARG;
    k_mul<<<grid_for(n), 256, 0, c->stream>>>(n, x, y, z);
    ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    return HRN_OK;
}

int hrn_vec_clip(hrn_ctx *c, int32_t n, double lo, double hi, double *x)
{
    if (!c || !x || n < 0) return HRN_EARG;
    k_clip<<<grid_for(n), 256, 0, c->stream>>>(n, lo, hi, x);
    ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    return HRN_OK;
}

int hrn_vec_gather(hrn_ctx *c, int32_t n, const int32_t *map, const double *x, double *y)
{
    if (!c || !map || !x || !y || n < 0) return HRN_EARG;
    k_gather<<<grid_for(n), 256, 0, c->stream>>>(n, map, x, y);
    ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    return HRN_OK;
}

int hrn_regularization_tv(hrn_ctx *c, const double *d_lambda, const double *d_mu, double *d_reg_lambda, double *d_reg_mu,
                          double *cost_lambda, double *cost_mu)
{
    if (!c || !d_lambda || !d_mu || !d_reg_lambda || !d_reg_mu || !cost_lambda || !cost_mu) return HRN_EARG;
    if (!c->have_mesh) return set_error(c, HRN_ESTATE, "no mesh: call hrn_set_mesh first");
    return regularization_tv(c, d_lambda, d_mu, d_reg_lambda, d_reg_mu, cost_lambda, cost_mu);
}

int hrn_illumination(hrn_ctx *c, double *d_out)
{
    if (!c || !d_out) return HRN_EARG;
    if (!c->have_forward) return set_error(c, HRN_ESTATE, "no forward history: call hrn_forward first");
    if (c->ckpt > 0) return set_error(c, HRN_ESTATE, "illumination needs the whole forward history (checkpointing is on)");
    if (c->nstore % 3 != 0) return set_error(c, HRN_EARG, "history rows must come in x, y, z triples");
    cudaSetDevice(c->device);
    const int nnode = c->nstore / 3, th = 128;
    if (c->precision == HRN_FP64)
        k_illumination<double><<<(nnode + th - 1) / th, th, 0, c->stream>>>(nnode, c->nstore, c->nstep, c->nshot,
                                                                          c->d_hist.as<double>(), d_out);
    else
        k_illumination<float><<<(nnode + th - 1) / th, th, 0, c->stream>>>(nnode, c->nstore, c->nstep, c->nshot,
                                                                         c->d_hist.as<float>(), d_out);
    ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    return HRN_OK;
}

int hrn_pseudo_hessian(hrn_ctx *c, double *d_h_lambda, double *d_h_mu)
{
    if (!c || !d_h_lambda || !d_h_mu) return HRN_EARG;
    if (!c->have_forward) return set_error(c, HRN_ESTATE, "no forward history: call hrn_forward first");
    if (c->ckpt > 0) return set_error(c, HRN_ESTATE, "the pseudo-Hessian needs the whole forward history (checkpointing is on)");
    if (!c->have_mesh) return set_error(c, HRN_ESTATE, "no mesh: call hrn_set_mesh first");
    cudaSetDevice(c->device);
    return run_pseudo_hessian(c, d_h_lambda, d_h_mu);
}

int hrn_gradient_mass(hrn_ctx *c, double *d_mg)
{
    if (!c || !d_mg) return HRN_EARG;
    if (!c->have_mesh) return set_error(c, HRN_ESTATE, "no mesh: call hrn_set_mesh first");
    return gradient_mass(c, d_mg);
}

// Coupled L-BFGS memory (S4/LBFGS_Coupled.F90; M_LBFGS in S4/Adjustments.F90:180).
int hrn_lbfgs_setup(hrn_ctx *c, int32_t m, const double *d_restriction)
{
    if (!c || m < 1 || !d_restriction) return HRN_EARG;
    if (!c->have_mesh) return set_error(c, HRN_ESTATE, "no mesh: call hrn_set_mesh first");
    const size_t nj = size_t(c->nj);
    HRN_CUDA(c, c->d_lbfgs.alloc((4 * size_t(m) + 6) * nj * 8));
    HRN_CUDA(c, cudaMemsetAsync(c->d_lbfgs.p, 0, (4 * size_t(m) + 6) * nj * 8, c->stream));
    HRN_CUDA(c, c->d_restrict.alloc(nj * 8));
    HRN_CUDA(c, cudaMemcpyAsync(c->d_restrict.p, d_restriction, nj * 8, cudaMemcpyDeviceToDevice, c->stream));
    c->lbfgs_m = m;
    c->lbfgs_rho.assign(size_t(m), 0.0);
    c->lbfgs_alpha.assign(size_t(m), 0.0);
    return HRN_OK;
}

// Search direction p = -H g of the coupled L-BFGS two-loop recursion
// (S4/LBFGS_Coupled.F90:4-218); every vector is a device array [nj].
int hrn_lbfgs_direction(hrn_ctx *c, int32_t iter, int32_t iter_begin, const double *g_l, const double *g_m,
                        const double *g_l_pre, const double *g_m_pre, const double *lam, const double *mu,
                        const double *lam_pre, const double *mu_pre, double *p_l, double *p_m, double *rho_out)
{
    if (!c || !g_l || !g_m || !p_l || !p_m) return HRN_EARG;
    if (c->lbfgs_m < 1) return set_error(c, HRN_ESTATE, "call hrn_lbfgs_setup first");
    const int n = c->nj, M = c->lbfgs_m;
    if (iter == iter_begin) {   // p = -g
        if (int rc = vec_axpby(c, n, -1.0, g_l, 0.0, nullptr, p_l)) return rc;
        if (int rc = vec_axpby(c, n, -1.0, g_m, 0.0, nullptr, p_m)) return rc;
        if (rho_out) *rho_out = 0.0;
        return HRN_OK;
    }
    if (!g_l_pre || !g_m_pre || !lam || !mu || !lam_pre || !mu_pre) return HRN_EARG;
    const int k = iter - iter_begin;
    double *base = c->d_lbfgs.as<double>();
    auto Ys_l = [&](int i) { return base + (size_t(0) * M + i) * n; };
    auto Ys_m = [&](int i) { return base + (size_t(1) * M + i) * n; };
    auto Ss_l = [&](int i) { return base + (size_t(2) * M + i) * n; };
    auto Ss_m = [&](int i) { return base + (size_t(3) * M + i) * n; };
    double *y_l = base + 4 * size_t(M) * n, *y_m = y_l + n, *s_l = y_m + n, *s_m = s_l + n, *q_l = s_m + n, *q_m = q_l + n;
#define CK(call) do { if (int _rc = (call)) return _rc; } while (0)
    CK(vec_axpby(c, n, 1.0, g_l, -1.0, g_l_pre, y_l));
    CK(vec_axpby(c, n, 1.0, lam, -1.0, lam_pre, s_l));
    CK(vec_axpby(c, n, 1.0, g_m, -1.0, g_m_pre, y_m));
    CK(vec_axpby(c, n, 1.0, mu, -1.0, mu_pre, s_m));
    double rl, rm;
    CK(vec_reduce(c, 0, n, y_l, s_l, &rl));
    CK(vec_reduce(c, 0, n, y_m, s_m, &rm));
    const double rho = 1.0 / (rl + rm);
    if (rho_out) *rho_out = rho;
    CK(vec_axpby(c, n, 1.0, g_l, 0.0, nullptr, q_l));
    CK(vec_axpby(c, n, 1.0, g_m, 0.0, nullptr, q_m));
    std::vector<int> seq;
    int n_use;
    if (k > 0 && k <= M) {
        n_use = k;
        for (int i = k; i >= 1; --i) seq.push_back(i);
    } else {
        n_use = M;
        const int end = k % M;
        for (int i = end; i >= 1; --i) seq.push_back(i);
        int j = 0;
        while (int(seq.size()) < M) seq.push_back(M - j++);
    }
    const int n_store = (k % M) != 0 ? (k % M) : M;
    c->lbfgs_rho[n_store - 1] = rho;
    const double *rs = c->d_restrict.as<double>();
    HRN_CUDA(c, cudaMemcpyAsync(Ys_l(n_store - 1), y_l, size_t(n) * 8, cudaMemcpyDeviceToDevice, c->stream));
    HRN_CUDA(c, cudaMemcpyAsync(Ys_m(n_store - 1), y_m, size_t(n) * 8, cudaMemcpyDeviceToDevice, c->stream));
    CK(hrn_vec_mul(c, n, s_l, rs, Ss_l(n_store - 1)));
    CK(hrn_vec_mul(c, n, s_m, rs, Ss_m(n_store - 1)));
    for (int iv = 0; iv < n_use; ++iv) {   // loop 1
        const int i = seq[iv] - 1;
        double a1, a2;
        CK(vec_reduce(c, 0, n, q_l, Ss_l(i), &a1));
        CK(vec_reduce(c, 0, n, q_m, Ss_m(i), &a2));
        const double a = c->lbfgs_rho[i] * a1 + c->lbfgs_rho[i] * a2;
        c->lbfgs_alpha[i] = a;
        CK(vec_axpby(c, n, 1.0, q_l, -a, Ys_l(i), q_l));
        CK(vec_axpby(c, n, 1.0, q_m, -a, Ys_m(i), q_m));
    }
    double hn1, hn2, hd1, hd2;   // H0 = (y.s) / (y.y)
    CK(vec_reduce(c, 0, n, y_l, s_l, &hn1));
    CK(vec_reduce(c, 0, n, y_l, y_l, &hd1));
    CK(vec_reduce(c, 0, n, y_m, s_m, &hn2));
    CK(vec_reduce(c, 0, n, y_m, y_m, &hd2));
    const double h0 = (hn1 + hn2) / (hd1 + hd2);
    CK(vec_axpby(c, n, h0, q_l, 0.0, nullptr, p_l));   // r, kept in p
    CK(vec_axpby(c, n, h0, q_m, 0.0, nullptr, p_m));
    for (int iv = n_use - 1; iv >= 0; --iv) {   // loop 2
        const int i = seq[iv] - 1;
        double b1, b2;
        CK(vec_reduce(c, 0, n, p_l, Ys_l(i), &b1));
        CK(vec_reduce(c, 0, n, p_m, Ys_m(i), &b2));
        const double beta = c->lbfgs_rho[i] * b1 + c->lbfgs_rho[i] * b2;
        const double w = c->lbfgs_alpha[i] - beta;
        CK(vec_axpby(c, n, 1.0, p_l, w, Ss_l(i), p_l));
        CK(vec_axpby(c, n, 1.0, p_m, w, Ss_m(i), p_m));
    }
    CK(vec_axpby(c, n, -1.0, p_l, 0.0, nullptr, p_l));
    CK(vec_axpby(c, n, -1.0, p_m, 0.0, nullptr, p_m));
#undef CK
    return HRN_OK;
}

}  // extern "C"
