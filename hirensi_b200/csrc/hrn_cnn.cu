// hrn_cnn.cu -- 3-D convolution layers of the learned gradient preconditioner on
// the 5th-generation tensor cores: 3x3x3 kernels with zero padding, BF16 operands,
// FP32 accumulation in tensor memory (TMEM), at most 16 input and 16 output
// channels.  Activations are channels-last with a channel stride of 16: voxel v
// holds channels 0..15 in 32 contiguous bytes.
//
// Each layer is an implicit GEMM over the 27 kernel taps:
//   forward      y[v][co]  = b[co] + sum_tap sum_ci x[v + off(tap)][ci] w[co][ci][tap]
//                D (128 voxels x 16 co) += A_tap (128 x 16 ci) B_tap (16 ci x 16 co)
//   data grad.   gx[v][ci] = sum_tap sum_co gz[v - off(tap)][co] w[co][ci][tap]
//                the same kernel with the neighbour offset negated and B_tap transposed
//   weight grad. gw[co][ci][tap] = sum_v x[v + off(tap)][ci] gz[v][co]
//                D ((8 taps x 16 ci) x 16 co) += A (128 x 16 voxels) B (16 voxels x 16 co),
//                voxel chunks in parallel, partial sums added in a fixed order.
// gz = gy masked by the ReLU of y and rounded to BF16 (the tensor-core operand).
// The forward and data-gradient kernels read a copy of their A source with a
// one-voxel zero border, where every tap is a shift of the voxel index: a tile
// copies each of the nine (dz, dy) row bands once and takes the three dx taps as
// 16-byte shifts of the same band.
//
// One elected thread issues tcgen05.mma (kind::f16, M = 128, N = 16, K = 16) on
// operands staged in shared memory in the canonical no-swizzle core-matrix layout
// (8 rows x 16 bytes per core matrix), commits to an mbarrier, and the CTA reads
// the accumulator back with tcgen05.ld.  Every wait is bounded: on a timeout the
// kernel flags an error, waits (bounded) once more and frees its TMEM.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "../../include/hirensi_b200.h"

namespace {

constexpr int kC = 16;            // channel stride of the activations (and the padded GEMM K and N)
constexpr int kM = 128;           // voxels per tile (MMA M)
constexpr int kThreads = 128;     // one warpgroup: warp w reads TMEM lanes 32w..32w+31
constexpr int kTmemCols = 32;     // smallest TMEM allocation; the accumulator uses 16 columns
constexpr int kWgSteps = 8;       // K steps (16 voxels each) staged per round of the weight-gradient kernel
constexpr int kWgChunk = 1024;    // voxels of one weight-gradient CTA

struct Grid {
    int nz, ny, nx;
    __host__ __device__ int size() const { return nz * ny * nx; }
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return uint32_t(__cvta_generic_to_shared(p)); }

// Shared-memory matrix descriptor, no swizzle: start address, leading-dimension
// byte offset (between core matrices along K for K-major operands, along K groups
// for MN-major ones), stride byte offset (between 8-row groups), version 1.
__device__ __forceinline__ uint64_t smem_desc(const void *p, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = uint64_t((smem_u32(p) >> 4) & 0x3FFFu);
    d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
    d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
    d |= uint64_t(1) << 46;
    return d;
}

// Instruction descriptor of kind::f16: BF16 A and B, FP32 D, M x N, operand majors.
constexpr uint32_t instr_desc(int M, int N, int a_mn_major, int b_mn_major)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(a_mn_major) << 15) | (uint32_t(b_mn_major) << 16) |
           (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// bounded wait for the phase with the given parity; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    const uint32_t addr = smem_u32(bar);
    for (int i = 0; i < (1 << 20); ++i) {
        uint32_t done;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                     : "=r"(done) : "r"(addr), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tmem_alloc(uint32_t *dst)   // whole warp
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr)   // whole warp
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(kTmemCols) : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mma_bf16(uint32_t taddr, uint64_t adesc, uint64_t bdesc, uint32_t idesc, int accumulate)
{
    asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                 " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}"
                 ::"r"(taddr), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate) : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 16 FP32 accumulator columns of this thread's TMEM lane (warp w: lanes 32w..32w+31)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&o)[16])
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) o[i] = __uint_as_float(r[i]);
}

// 16-byte asynchronous copy global -> shared; valid = false writes 16 zero bytes and
// reads nothing (source size 0)
__device__ __forceinline__ void cp_async16_zfill(void *dst, const void *src, bool valid)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ uint32_t pack2(float a, float b)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&h);
}

// Eight channels (one 16-byte core-matrix row) of the A operand at voxel u:
// the activations (forward) or gz = gy masked by ReLU(y), rounded to BF16 (data gradient).
template <bool GRAD>
__device__ __forceinline__ uint4 channels8(const void *src, const __nv_bfloat16 *y, int relu, int u, int half)
{
    if (u < 0) return make_uint4(0, 0, 0, 0);
    if constexpr (!GRAD) {
        return __ldg(reinterpret_cast<const uint4 *>(static_cast<const __nv_bfloat16 *>(src) + size_t(u) * kC) + half);
    } else {
        const float4 *g = reinterpret_cast<const float4 *>(static_cast<const float *>(src) + size_t(u) * kC + 8 * half);
        const float4 a = __ldg(g), b = __ldg(g + 1);
        float f[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        if (relu) {
            const uint4 yy = __ldg(reinterpret_cast<const uint4 *>(y + size_t(u) * kC) + half);
            const __nv_bfloat16 *yh = reinterpret_cast<const __nv_bfloat16 *>(&yy);
#pragma unroll
            for (int i = 0; i < 8; ++i)
                if (!(__bfloat162float(yh[i]) > 0.f)) f[i] = 0.f;
        }
        return make_uint4(pack2(f[0], f[1]), pack2(f[2], f[3]), pack2(f[4], f[5]), pack2(f[6], f[7]));
    }
}

// B operand of every tap in the canonical layout, written once per call into
// global memory (27 x 512 bytes) for the tiles to copy: core matrix (n / 8, k / 8)
// at ((n / 8) * 2 + k / 8) * 128, row n % 8.  Forward: B_tap[n = co][k = ci];
// data gradient: B_tap[n = ci][k = co].
template <bool GRAD>
__global__ void k_conv_pack_b(int cin, int cout, const __nv_bfloat16 *__restrict__ w, unsigned char *__restrict__ bpack)
{
    const int nrow = GRAD ? cin : cout, ncol = GRAD ? cout : cin;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 27 * kC * kC; i += gridDim.x * blockDim.x) {
        const int tap = i / (kC * kC), n = (i / kC) % kC, k = i % kC;
        __nv_bfloat16 val = __float2bfloat16_rn(0.f);
        if (n < nrow && k < ncol) {
            const int co = GRAD ? k : n, ci = GRAD ? n : k;
            val = w[(size_t(co) * cin + ci) * 27 + tap];
        }
        *reinterpret_cast<__nv_bfloat16 *>(bpack + tap * 512 + ((n >> 3) * 2 + (k >> 3)) * 128 + (n & 7) * 16 + (k & 7) * 2) = val;
    }
}

// Forward (GRAD = false) and data gradient (GRAD = true) on the padded grid: the A
// operand comes from a copy of the input with a one-voxel zero border (k_conv_pad),
// so that every tap is a pure shift of the padded voxel index
//   off(tap) = dz Sz + dy Sy + dx,  Sz = (ny + 2)(nx + 2), Sy = nx + 2,
// negated for the data gradient.  A tile is 128 consecutive padded voxels p0..p0+127.
// For each (dz, dy) the tile needs the rows p0 + sgn (dz Sz + dy Sy) - 1 .. +128
// (130 rows, covering the three dx); the CTA copies each such band once into shared
// memory as two half-planes of 16-byte rows ([h][row][8 channels]), and the A operand
// of tap (dz, dy, dx) is the band seen from row 1 + sgn dx: in the no-swizzle
// K-major layout a core matrix is 8 consecutive 16-byte rows, so the shift is only
// the descriptor's start address (16 bytes per row), with the half-planes one
// leading-byte offset apart.  The 27 MMAs run in the tap order of the unpadded
// formulation on the same operand values, so the result is the same.
//   forward: src = x padded (BF16), B_tap[n = co][k = ci], out = y (BF16 [V][16]);
//   data gradient: src = gz padded (BF16, k_conv_pad<true>), B_tap[n = ci][k = co],
//   out = gx (FP32 [V][16]).
// Output rows of border voxels are not written.
constexpr int kBandRows = kM + 2;
constexpr int kBandBytes = 2 * kBandRows * 16;     // two half-planes
constexpr int kBandLbo = kBandRows * 16;           // between the half-planes (K direction)

template <bool GRAD>
__global__ void __launch_bounds__(kThreads) k_conv_band(int cin, int cout, Grid g, const __nv_bfloat16 *__restrict__ srcp,
                                                        const unsigned char *__restrict__ bpack,
                                                        const float *__restrict__ bias, int relu, void *__restrict__ out,
                                                        int *__restrict__ err)
{
    static_assert(kThreads == kM, "one thread per voxel of the tile in the epilogue");
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *Bs = smem;                         // 27 x 512
    unsigned char *As = smem + 27 * 512;              // 9 bands
    uint64_t *bar = reinterpret_cast<uint64_t *>(As + 9 * kBandBytes);
    uint32_t *s_taddr = reinterpret_cast<uint32_t *>(bar + 1);
    const int Sy = g.nx + 2, Sz = (g.ny + 2) * Sy;
    const int Vp = (g.nz + 2) * Sz;
    const int p0 = blockIdx.x * kM;
    const int warp = threadIdx.x >> 5;
    constexpr int sgn = GRAD ? -1 : 1;

    for (int i = threadIdx.x; i < 27 * 512 / 16; i += kThreads)
        reinterpret_cast<uint4 *>(Bs)[i] = __ldg(reinterpret_cast<const uint4 *>(bpack) + i);
    // bands: a thread copies one 32-byte row into the two half-planes; consecutive
    // threads take consecutive rows (contiguous 16-byte stores in each plane); rows
    // outside the padded grid are zero-filled
    for (int i = threadIdx.x; i < 9 * kBandRows; i += kThreads) {
        const int b = i / kBandRows, j = i % kBandRows;
        const int dz = b / 3 - 1, dy = b % 3 - 1;
        const int row = p0 + sgn * (dz * Sz + dy * Sy) - 1 + j;
        const bool in = row >= 0 && row < Vp;
        const uint4 *q = reinterpret_cast<const uint4 *>(srcp + (in ? size_t(row) * kC : 0));
        cp_async16_zfill(As + b * kBandBytes + j * 16, q, in);
        cp_async16_zfill(As + b * kBandBytes + kBandLbo + j * 16, q + 1, in);
    }
    cp_async_wait_all();
    if (threadIdx.x == 0) mbar_init(bar);
    if (warp == 0) tmem_alloc(s_taddr);
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t taddr = *s_taddr;
    constexpr uint32_t idesc = instr_desc(kM, kC, 0, 0);
    if (threadIdx.x == 0) {
        for (int tap = 0; tap < 27; ++tap) {
            const int b = tap / 3, dx = tap % 3 - 1;     // band (dz, dy) = (tap / 9, tap / 3 % 3)
            mma_bf16(taddr, smem_desc(As + b * kBandBytes + (1 + sgn * dx) * 16, kBandLbo, 128),
                     smem_desc(Bs + tap * 512, 128, 256), idesc, tap != 0);
        }
        mma_commit(bar);
    }
    bool ok = mbar_wait(bar, 0);
    ok = __syncthreads_and(ok);
    if (!ok) {
        if (threadIdx.x == 0) {
            atomicExch(err, 1);
            mbar_wait(bar, 0);
        }
    } else {
        fence_after();
        float acc[16];
        tmem_ld16(taddr + (uint32_t(32 * warp) << 16), acc);   // this thread's TMEM lane is its voxel
        const int p = p0 + threadIdx.x;
        const int px = p % Sy, py = (p / Sy) % (g.ny + 2), pz = p / Sz;
        if (p < Vp && px >= 1 && px <= g.nx && py >= 1 && py <= g.ny && pz >= 1 && pz <= g.nz) {
            const int v = ((pz - 1) * g.ny + (py - 1)) * g.nx + (px - 1);
            if constexpr (!GRAD) {
                uint32_t o[8];
#pragma unroll
                for (int c = 0; c < 16; c += 2) {
                    float a = c < cout ? acc[c] + bias[c] : 0.f, b = c + 1 < cout ? acc[c + 1] + bias[c + 1] : 0.f;
                    if (relu) { a = fmaxf(a, 0.f); b = fmaxf(b, 0.f); }
                    o[c / 2] = pack2(a, b);
                }
                uint4 *dst = reinterpret_cast<uint4 *>(static_cast<__nv_bfloat16 *>(out) + size_t(v) * kC);
                dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
                dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
            } else {
                float4 *dst = reinterpret_cast<float4 *>(static_cast<float *>(out) + size_t(v) * kC);
#pragma unroll
                for (int c = 0; c < 16; c += 4)
                    dst[c / 4] = make_float4(c < cin ? acc[c] : 0.f, c + 1 < cin ? acc[c + 1] : 0.f,
                                             c + 2 < cin ? acc[c + 2] : 0.f, c + 3 < cin ? acc[c + 3] : 0.f);
            }
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(taddr);
}

// Copy of the A source with a one-voxel zero border, BF16 [Vp][16]: the activations
// (forward) or gz = gy masked by ReLU(y) and rounded to BF16 (data gradient).  One
// thread per (padded voxel, channel half).
template <bool GRAD>
__global__ void k_conv_pad(Grid g, const void *__restrict__ src, const __nv_bfloat16 *__restrict__ y_act, int relu,
                           __nv_bfloat16 *__restrict__ dstp)
{
    const int Sy = g.nx + 2, Sz = (g.ny + 2) * Sy;
    const int n = 2 * (g.nz + 2) * Sz;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int p = i >> 1, h = i & 1;
        const int px = p % Sy, py = (p / Sy) % (g.ny + 2), pz = p / Sz;
        const bool interior = px >= 1 && px <= g.nx && py >= 1 && py <= g.ny && pz >= 1 && pz <= g.nz;
        const int u = interior ? ((pz - 1) * g.ny + (py - 1)) * g.nx + (px - 1) : -1;
        reinterpret_cast<uint4 *>(dstp + size_t(p) * kC)[h] = channels8<GRAD>(src, y_act, relu, u, h);
    }
}

// Weight gradient, partial sums of one chunk of voxels for one M tile of 8 taps:
//   part[chunk][mt * 128 + (tap - 8 mt) * 16 + ci][co] = sum_v x[v + off(tap)][ci] gz[v][co]
// Both operands are MN-major (the GEMM's K runs over voxels): core matrix
// (8 M or N elements) x (8 voxels), row = voxel, at (group * 2 + voxel / 8) * 128.
__global__ void __launch_bounds__(kThreads) k_conv_wgrad_tc(Grid g, const __nv_bfloat16 *__restrict__ x,
                                                            const float *__restrict__ gy,
                                                            const __nv_bfloat16 *__restrict__ y_act, int relu,
                                                            float *__restrict__ part, int *__restrict__ err)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *As = smem;                         // kWgSteps x 4096
    unsigned char *Bs = smem + kWgSteps * 4096;       // kWgSteps x 512
    uint64_t *bar = reinterpret_cast<uint64_t *>(Bs + kWgSteps * 512);
    uint32_t *s_taddr = reinterpret_cast<uint32_t *>(bar + 1);
    const int V = g.size();
    const int mt = blockIdx.x, chunk = blockIdx.y;
    const int c0 = chunk * kWgChunk;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) mbar_init(bar);
    if (warp == 0) tmem_alloc(s_taddr);
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t taddr = *s_taddr;
    constexpr uint32_t idesc = instr_desc(kM, kC, 1, 1);
    constexpr int kRoundVox = kWgSteps * 16;
    const int nround = kWgChunk / kRoundVox;
    bool ok = true;
    int issued = 0;
    for (int r = 0; r < nround && ok; ++r) {
        const int vr = c0 + r * kRoundVox;
        if (vr >= V) break;
        // Thread m stages voxel vr + m (step s = m / 16, voxel kv = m % 16 of the step).
        // A: 16 M groups (tap, channel half) x 16 voxels per step; B: 2 N groups x 16 voxels.
        // A quarter-warp's 16-byte stores fill one contiguous 128-byte core matrix.
        const int m = threadIdx.x, s = m >> 4, kv = m & 15, v = vr + m;
        const bool inside = v < V;
        int vx = 0, vy = 0, vz = 0;
        if (inside) {
            vx = v % g.nx;
            const int q = v / g.nx;
            vy = q % g.ny;
            vz = q / g.ny;
        }
        unsigned char *arow = As + s * 4096 + (kv >> 3) * 128 + (kv & 7) * 16;
#pragma unroll
        for (int tl = 0; tl < 8; ++tl) {
            const int tap = mt * 8 + tl;
            const int zz = vz + tap / 9 - 1, yy = vy + (tap / 3) % 3 - 1, xx = vx + tap % 3 - 1;
            const bool nb = inside && tap < 27 && zz >= 0 && zz < g.nz && yy >= 0 && yy < g.ny && xx >= 0 && xx < g.nx;
            const uint4 *p = reinterpret_cast<const uint4 *>(x + (nb ? size_t((zz * g.ny + yy) * g.nx + xx) * kC : 0));
            cp_async16_zfill(arow + (tl * 2 + 0) * 256, p, nb);
            cp_async16_zfill(arow + (tl * 2 + 1) * 256, p + 1, nb);
        }
        unsigned char *brow = Bs + s * 512 + (kv >> 3) * 128 + (kv & 7) * 16;
        const uint4 b0 = channels8<true>(gy, y_act, relu, inside ? v : -1, 0);
        const uint4 b1 = channels8<true>(gy, y_act, relu, inside ? v : -1, 1);
        *reinterpret_cast<uint4 *>(brow) = b0;
        *reinterpret_cast<uint4 *>(brow + 256) = b1;
        cp_async_wait_all();
        fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            fence_after();
            for (int s = 0; s < kWgSteps; ++s)
                mma_bf16(taddr, smem_desc(As + s * 4096, 128, 256), smem_desc(Bs + s * 512, 128, 256), idesc,
                         (r | s) != 0);
            mma_commit(bar);
        }
        ++issued;
        ok = mbar_wait(bar, uint32_t(r & 1));
        ok = __syncthreads_and(ok);
    }
    float *dst = part + (size_t(chunk) * 4 * kM + size_t(mt) * kM + 32 * warp + lane) * kC;
    if (!ok) {
        if (threadIdx.x == 0) {
            atomicExch(err, 1);
            mbar_wait(bar, uint32_t((issued - 1) & 1));
        }
    } else if (issued == 0) {
#pragma unroll
        for (int c = 0; c < 16; ++c) dst[c] = 0.f;
    } else {
        fence_after();
        float acc[16];
        tmem_ld16(taddr + (uint32_t(32 * warp) << 16), acc);
#pragma unroll
        for (int c = 0; c < 16; c += 4) reinterpret_cast<float4 *>(dst)[c / 4] = make_float4(acc[c], acc[c + 1], acc[c + 2], acc[c + 3]);
    }
    fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(taddr);
}

// gw[co][ci][tap] = sum over chunks, in chunk order, of the partial sums
__global__ void k_conv_wgrad_sum(int cin, int cout, int nchunk, const float *__restrict__ part, float *__restrict__ gw)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cout * cin * 27) return;
    const int co = i / (cin * 27), ci = (i / 27) % cin, tap = i % 27;
    const size_t row = size_t(tap) * kC + ci;        // = mt * 128 + (tap - 8 mt) * 16 + ci
    float s = 0.f;
    for (int c = 0; c < nchunk; ++c) s += part[(size_t(c) * 4 * kM + row) * kC + co];
    gw[i] = s;
}

// gb[co] = sum_v gz[v][co] (FP32 gz), one block per output channel, fixed-order reduction
constexpr int kBThreads = 256;
__global__ void __launch_bounds__(kBThreads) k_conv_bias_grad(Grid g, const float *__restrict__ gy,
                                                              const __nv_bfloat16 *__restrict__ y_act, int relu,
                                                              float *__restrict__ gb)
{
    const int co = blockIdx.x;
    const int V = g.size();
    float s = 0.f;
    for (int v = threadIdx.x; v < V; v += kBThreads) {
        const float gz = gy[size_t(v) * kC + co];
        if (!relu || __bfloat162float(y_act[size_t(v) * kC + co]) > 0.f) s += gz;
    }
    __shared__ float part[kBThreads / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int i = 0; i < kBThreads / 32; ++i) t += part[i];
        gb[co] = t;
    }
}

constexpr size_t kConvSmem = 27 * 512 + 9 * kBandBytes + 16;
constexpr size_t kWgSmem = kWgSteps * (4096 + 512) + 16;

int check(int cin, int cout, int nz, int ny, int nx)
{
    if (cin < 1 || cin > kC || cout < 1 || cout > kC || nz < 1 || ny < 1 || nx < 1) return HRN_EARG;
    if (int64_t(nz + 2) * (ny + 2) * (nx + 2) > (int64_t(1) << 30)) return HRN_EARG;   // padded grid
    return HRN_OK;
}

// Per-device scratch of the layers (the error flag, the packed B operand, the padded
// copy of the A source and the weight-gradient partial sums), grown on demand and
// kept until the process exits.  Calls that overlap on one device share it, as they
// share the error flag: the calls synchronize their stream before returning.
struct Scratch {
    int *err = nullptr;
    unsigned char *bpack = nullptr;   // 27 x 512 bytes
    __nv_bfloat16 *pad = nullptr;     // [(nz + 2)(ny + 2)(nx + 2)][16]
    size_t pad_bytes = 0;
    float *part = nullptr;
    size_t part_bytes = 0;
};

size_t pad_bytes(const Grid &g) { return size_t(g.nz + 2) * (g.ny + 2) * (g.nx + 2) * kC * sizeof(__nv_bfloat16); }

int scratch(int dev, size_t part_bytes, size_t padded_bytes, Scratch &out)
{
    static std::mutex mu;
    static Scratch per[64];
    if (dev < 0 || dev >= 64) return HRN_EARG;
    std::lock_guard<std::mutex> lock(mu);
    Scratch &s = per[dev];
    if (!s.err) {
        if (cudaMalloc(&s.err, sizeof(int)) != cudaSuccess) return HRN_EOOM;
        if (cudaMemset(s.err, 0, sizeof(int)) != cudaSuccess) return HRN_ECUDA;
    }
    if (!s.bpack && cudaMalloc(&s.bpack, 27 * 512) != cudaSuccess) return HRN_EOOM;
    if (padded_bytes > s.pad_bytes) {
        if (s.pad) cudaFree(s.pad);
        s.pad = nullptr;
        s.pad_bytes = 0;
        if (cudaMalloc(&s.pad, padded_bytes) != cudaSuccess) return HRN_EOOM;
        s.pad_bytes = padded_bytes;
    }
    if (part_bytes > s.part_bytes) {
        if (s.part) cudaFree(s.part);
        s.part = nullptr;
        s.part_bytes = 0;
        if (cudaMalloc(&s.part, part_bytes) != cudaSuccess) return HRN_EOOM;
        s.part_bytes = part_bytes;
    }
    out = s;
    return HRN_OK;
}

int check_err(const Scratch &s, cudaStream_t st)
{
    int e = 0;
    if (cudaMemcpyAsync(&e, s.err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return HRN_ECUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return HRN_ECUDA;
    if (e) {
        cudaMemsetAsync(s.err, 0, sizeof(int), st);
        return HRN_ECUDA;
    }
    return HRN_OK;
}

template <bool GRAD>
void set_smem_once()
{
    static std::atomic<uint64_t> done{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t bit = dev >= 0 && dev < 64 ? (uint64_t(1) << dev) : 0;
    if (bit && (done.load() & bit)) return;
    cudaFuncSetAttribute(k_conv_band<GRAD>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kConvSmem));
    done.fetch_or(bit);
}

}  // namespace

extern "C" int hrn_cnn_conv3d_forward(int32_t cin, int32_t cout, int32_t nz, int32_t ny, int32_t nx, const void *x,
                                      const void *w, const float *bias, int32_t relu, void *y, void *stream)
{
    if (int rc = check(cin, cout, nz, ny, nx)) return rc;
    if (!x || !w || !bias || !y) return HRN_EARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return HRN_ECUDA;
    const Grid g{nz, ny, nx};
    Scratch s;
    if (int rc = scratch(dev, 0, pad_bytes(g), s)) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int np = (nz + 2) * (ny + 2) * (nx + 2);
    set_smem_once<false>();
    k_conv_pack_b<false><<<27, 256, 0, st>>>(cin, cout, static_cast<const __nv_bfloat16 *>(w), s.bpack);
    k_conv_pad<false><<<std::min((2 * np + 255) / 256, 148 * 16), 256, 0, st>>>(g, x, nullptr, 0, s.pad);
    k_conv_band<false><<<(np + kM - 1) / kM, kThreads, kConvSmem, st>>>(cin, cout, g, s.pad, s.bpack, bias, relu, y,
                                                                        s.err);
    if (cudaGetLastError() != cudaSuccess) return HRN_ECUDA;
    return check_err(s, st);
}

extern "C" int hrn_cnn_conv3d_backward(int32_t cin, int32_t cout, int32_t nz, int32_t ny, int32_t nx, const void *x,
                                       const void *w, const void *y, int32_t relu, const float *gy, float *gx, float *gw,
                                       float *gb, void *stream)
{
    if (int rc = check(cin, cout, nz, ny, nx)) return rc;
    if (!x || !w || !y || !gy || !gw || !gb) return HRN_EARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return HRN_ECUDA;
    const Grid g{nz, ny, nx};
    const int V = g.size();
    const int nchunk = (V + kWgChunk - 1) / kWgChunk;
    Scratch s;
    if (int rc = scratch(dev, size_t(nchunk) * 4 * kM * kC * sizeof(float), gx ? pad_bytes(g) : 0, s)) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const __nv_bfloat16 *yb = static_cast<const __nv_bfloat16 *>(y);
    if (gx) {
        const int np = (nz + 2) * (ny + 2) * (nx + 2);
        set_smem_once<true>();
        k_conv_pack_b<true><<<27, 256, 0, st>>>(cin, cout, static_cast<const __nv_bfloat16 *>(w), s.bpack);
        k_conv_pad<true><<<std::min((2 * np + 255) / 256, 148 * 16), 256, 0, st>>>(g, gy, yb, relu, s.pad);
        k_conv_band<true><<<(np + kM - 1) / kM, kThreads, kConvSmem, st>>>(cin, cout, g, s.pad, s.bpack, nullptr, relu,
                                                                           gx, s.err);
    }
    k_conv_wgrad_tc<<<dim3(4, nchunk), kThreads, kWgSmem, st>>>(g, static_cast<const __nv_bfloat16 *>(x), gy, yb, relu,
                                                                 s.part, s.err);
    k_conv_wgrad_sum<<<(cout * cin * 27 + 127) / 128, 128, 0, st>>>(cin, cout, nchunk, s.part, gw);
    k_conv_bias_grad<<<cout, kBThreads, 0, st>>>(g, gy, yb, relu, gb);
    if (cudaGetLastError() != cudaSuccess) return HRN_ECUDA;
    return check_err(s, st);
}
