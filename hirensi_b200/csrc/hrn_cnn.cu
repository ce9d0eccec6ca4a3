// hrn_cnn.cu -- 3-D convolution layers of the learned gradient preconditioner:
// 3x3x3 kernels with zero padding on a [channel][z][y][x] grid, BF16 weights
// and activations, FP32 accumulation; forward, data gradient and weight / bias
// gradient (deterministic reductions).  At most 16 input and 16 output channels.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/hirensi_b200.h"

namespace {

constexpr int kMaxC = 16;

struct Grid {
    int nz, ny, nx;
    __device__ __forceinline__ int size() const { return nz * ny * nx; }
};

// offset of kernel tap k = 9 dz + 3 dy + dx (each in 0..2) from voxel (z, y, x); -1 if outside
__device__ __forceinline__ int tap(const Grid &g, int z, int y, int x, int k, int sign)
{
    const int zz = z + sign * (k / 9 - 1), yy = y + sign * ((k / 3) % 3 - 1), xx = x + sign * (k % 3 - 1);
    if (zz < 0 || zz >= g.nz || yy < 0 || yy >= g.ny || xx < 0 || xx >= g.nx) return -1;
    return (zz * g.ny + yy) * g.nx + xx;
}

// y[co][v] = act(b[co] + sum_ci sum_k w[co][ci][k] x[ci][v + off(k)])
__global__ void k_conv_fwd(int cin, int cout, Grid g, const __nv_bfloat16 *__restrict__ x,
                           const __nv_bfloat16 *__restrict__ w, const float *__restrict__ b, int relu,
                           __nv_bfloat16 *__restrict__ y)
{
    __shared__ float ws[kMaxC * kMaxC * 27];
    for (int i = threadIdx.x; i < cout * cin * 27; i += blockDim.x) ws[i] = __bfloat162float(w[i]);
    __syncthreads();
    const int V = g.size();
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const int xx = v % g.nx, yy = (v / g.nx) % g.ny, zz = v / (g.nx * g.ny);
    float acc[kMaxC];
#pragma unroll
    for (int co = 0; co < kMaxC; ++co) acc[co] = co < cout ? b[co] : 0.f;
    for (int k = 0; k < 27; ++k) {
        const int u = tap(g, zz, yy, xx, k, 1);
        if (u < 0) continue;
        for (int ci = 0; ci < cin; ++ci) {
            const float xv = __bfloat162float(x[size_t(ci) * V + u]);
#pragma unroll
            for (int co = 0; co < kMaxC; ++co)
                if (co < cout) acc[co] = fmaf(ws[(co * cin + ci) * 27 + k], xv, acc[co]);
        }
    }
    for (int co = 0; co < cout; ++co) {
        const float a = relu ? fmaxf(acc[co], 0.f) : acc[co];
        y[size_t(co) * V + v] = __float2bfloat16_rn(a);
    }
}

// gradient at the pre-activation: gy masked by the activation's derivative
__device__ __forceinline__ float gz_at(const float *__restrict__ gy, const __nv_bfloat16 *__restrict__ y, int relu, size_t i)
{
    const float g = gy[i];
    if (!relu) return g;
    return __bfloat162float(y[i]) > 0.f ? g : 0.f;
}

// gx[ci][v] = sum_co sum_k w[co][ci][k] gz[co][v - off(k)]
__global__ void k_conv_bwd_data(int cin, int cout, Grid g, const __nv_bfloat16 *__restrict__ w,
                                const __nv_bfloat16 *__restrict__ y, int relu, const float *__restrict__ gy,
                                float *__restrict__ gx)
{
    __shared__ float ws[kMaxC * kMaxC * 27];
    for (int i = threadIdx.x; i < cout * cin * 27; i += blockDim.x) ws[i] = __bfloat162float(w[i]);
    __syncthreads();
    const int V = g.size();
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const int xx = v % g.nx, yy = (v / g.nx) % g.ny, zz = v / (g.nx * g.ny);
    float acc[kMaxC];
#pragma unroll
    for (int ci = 0; ci < kMaxC; ++ci) acc[ci] = 0.f;
    for (int k = 0; k < 27; ++k) {
        const int u = tap(g, zz, yy, xx, k, -1);
        if (u < 0) continue;
        for (int co = 0; co < cout; ++co) {
            const float gz = gz_at(gy, y, relu, size_t(co) * V + u);
#pragma unroll
            for (int ci = 0; ci < kMaxC; ++ci)
                if (ci < cin) acc[ci] = fmaf(ws[(co * cin + ci) * 27 + k], gz, acc[ci]);
        }
    }
    for (int ci = 0; ci < cin; ++ci) gx[size_t(ci) * V + v] = acc[ci];
}

// one block per (co, ci): gw[co][ci][k] = sum_v gz[co][v] x[ci][v + off(k)];
// the ci = 0 block also writes gb[co] = sum_v gz[co][v]
constexpr int kWThreads = 256;

__global__ void __launch_bounds__(kWThreads) k_conv_bwd_weight(int cin, int cout, Grid g, const __nv_bfloat16 *__restrict__ x,
                                                               const __nv_bfloat16 *__restrict__ y, int relu,
                                                               const float *__restrict__ gy, float *__restrict__ gw,
                                                               float *__restrict__ gb)
{
    const int co = blockIdx.x / cin, ci = blockIdx.x % cin;
    const int V = g.size();
    float acc[28];
#pragma unroll
    for (int k = 0; k < 28; ++k) acc[k] = 0.f;
    for (int v = threadIdx.x; v < V; v += kWThreads) {
        const float gz = gz_at(gy, y, relu, size_t(co) * V + v);
        if (gz == 0.f) continue;
        const int xx = v % g.nx, yy = (v / g.nx) % g.ny, zz = v / (g.nx * g.ny);
#pragma unroll
        for (int k = 0; k < 27; ++k) {
            const int u = tap(g, zz, yy, xx, k, 1);
            if (u >= 0) acc[k] = fmaf(gz, __bfloat162float(x[size_t(ci) * V + u]), acc[k]);
        }
        acc[27] += gz;
    }
    // fixed-order reduction: warp shuffles, then the warps' partials in order
    __shared__ float part[kWThreads / 32][28];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 28; ++k) {
        float s = acc[k];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (lane == 0) part[wid][k] = s;
    }
    __syncthreads();
    if (threadIdx.x < 28) {
        float s = 0.f;
        for (int i = 0; i < kWThreads / 32; ++i) s += part[i][threadIdx.x];
        if (threadIdx.x < 27) gw[(size_t(co) * cin + ci) * 27 + threadIdx.x] = s;
        else if (ci == 0) gb[co] = s;
    }
}

int check(int cin, int cout, int nz, int ny, int nx)
{
    if (cin < 1 || cin > kMaxC || cout < 1 || cout > kMaxC || nz < 1 || ny < 1 || nx < 1) return HRN_EARG;
    if (int64_t(nz) * ny * nx > (int64_t(1) << 30)) return HRN_EARG;
    return HRN_OK;
}

}  // namespace

extern "C" int hrn_cnn_conv3d_forward(int32_t cin, int32_t cout, int32_t nz, int32_t ny, int32_t nx, const void *x,
                                      const void *w, const float *bias, int32_t relu, void *y, void *stream)
{
    if (int rc = check(cin, cout, nz, ny, nx)) return rc;
    if (!x || !w || !bias || !y) return HRN_EARG;
    const Grid g{nz, ny, nx};
    const int V = nz * ny * nx, th = 128;
    k_conv_fwd<<<(V + th - 1) / th, th, 0, static_cast<cudaStream_t>(stream)>>>(
        cin, cout, g, static_cast<const __nv_bfloat16 *>(x), static_cast<const __nv_bfloat16 *>(w), bias, relu,
        static_cast<__nv_bfloat16 *>(y));
    return cudaGetLastError() == cudaSuccess ? HRN_OK : HRN_ECUDA;
}

extern "C" int hrn_cnn_conv3d_backward(int32_t cin, int32_t cout, int32_t nz, int32_t ny, int32_t nx, const void *x,
                                       const void *w, const void *y, int32_t relu, const float *gy, float *gx, float *gw,
                                       float *gb, void *stream)
{
    if (int rc = check(cin, cout, nz, ny, nx)) return rc;
    if (!x || !w || !y || !gy || !gw || !gb) return HRN_EARG;
    const Grid g{nz, ny, nx};
    const int V = nz * ny * nx, th = 128;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (gx)
        k_conv_bwd_data<<<(V + th - 1) / th, th, 0, st>>>(cin, cout, g, static_cast<const __nv_bfloat16 *>(w),
                                                          static_cast<const __nv_bfloat16 *>(y), relu, gy, gx);
    k_conv_bwd_weight<<<cin * cout, kWThreads, 0, st>>>(cin, cout, g, static_cast<const __nv_bfloat16 *>(x),
                                                        static_cast<const __nv_bfloat16 *>(y), relu, gy, gw, gb);
    return cudaGetLastError() == cudaSuccess ? HRN_OK : HRN_ECUDA;
}
