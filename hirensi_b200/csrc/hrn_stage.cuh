// hrn_stage.cuh -- device helpers shared by the stage kernels: shot-vector
// loads and stores, the stage argument block and the row epilogue of one RK4
// stage (source, history, next-stage inputs or the state update).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hrn {

// ----------------------------------------------------------------------------
// small vector helpers

// Read-only vector loads of the S shots of one row: one 256-bit load for 32
// bytes (sm_100 ld.global.nc.v4.f64 / v8.f32), 128-bit or narrower otherwise, so
// each gathered row record costs one request per 32-byte sector.
__device__ __forceinline__ void ld256(const double *p, double &a, double &b, double &c, double &d)
{
    asm volatile("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p));
}
__device__ __forceinline__ void ld256(const float *p, float (&o)[8])
{
    asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(o[0]), "=f"(o[1]), "=f"(o[2]), "=f"(o[3]), "=f"(o[4]), "=f"(o[5]), "=f"(o[6]), "=f"(o[7])
                 : "l"(p));
}

template <typename T, int S>
__device__ __forceinline__ void ldv(const T *__restrict__ p, T (&o)[S])
{
    if constexpr (sizeof(T) == 8 && S % 4 == 0) {
#pragma unroll
        for (int s = 0; s < S; s += 4) ld256(p + s, o[s], o[s + 1], o[s + 2], o[s + 3]);
    } else if constexpr (sizeof(T) == 8 && S % 2 == 0) {
#pragma unroll
        for (int s = 0; s < S; s += 2) {
            double2 v = __ldg(reinterpret_cast<const double2 *>(p) + s / 2);
            o[s] = v.x;
            o[s + 1] = v.y;
        }
    } else if constexpr (sizeof(T) == 4 && S % 8 == 0) {
        ld256(p, o);
    } else if constexpr (sizeof(T) == 4 && S % 4 == 0) {
#pragma unroll
        for (int s = 0; s < S; s += 4) {
            float4 v = __ldg(reinterpret_cast<const float4 *>(p) + s / 4);
            o[s] = v.x; o[s + 1] = v.y; o[s + 2] = v.z; o[s + 3] = v.w;
        }
    } else if constexpr (sizeof(T) == 4 && S % 2 == 0) {
#pragma unroll
        for (int s = 0; s < S; s += 2) {
            float2 v = __ldg(reinterpret_cast<const float2 *>(p) + s / 2);
            o[s] = v.x; o[s + 1] = v.y;
        }
    } else {
#pragma unroll
        for (int s = 0; s < S; ++s) o[s] = __ldg(p + s);
    }
}

template <typename T, int S>
__device__ __forceinline__ void stv(T *__restrict__ p, const T (&o)[S])
{
    if constexpr (sizeof(T) == 8 && S % 2 == 0) {
#pragma unroll
        for (int s = 0; s < S; s += 2) reinterpret_cast<double2 *>(p)[s / 2] = make_double2(o[s], o[s + 1]);
    } else if constexpr (sizeof(T) == 4 && S % 4 == 0) {
#pragma unroll
        for (int s = 0; s < S; s += 4)
            reinterpret_cast<float4 *>(p)[s / 4] = make_float4(o[s], o[s + 1], o[s + 2], o[s + 3]);
    } else {
#pragma unroll
        for (int s = 0; s < S; ++s) p[s] = o[s];
    }
}

// ----------------------------------------------------------------------------
// mbarrier and 1-D bulk copies (global -> shared), with bounded waits

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
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

__device__ __forceinline__ double fmaT(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float fmaT(float a, float b, float c) { return fmaf(a, b, c); }

// ----------------------------------------------------------------------------
// stage kernel

template <typename T>
struct StageArgs {
    int n;
    const int32_t *__restrict__ rowptr;
    const int2 *__restrict__ seg;           // [n] first K entry, first G entry of each row
    const uint32_t *__restrict__ colx;
    const T *__restrict__ val;
    const T *__restrict__ x1, *__restrict__ x2, *__restrict__ x3;
    const T *__restrict__ kb1, *__restrict__ kb2, *__restrict__ kb3;
    T *__restrict__ kb_out;                 // stages 1-3
    T *__restrict__ y1, *__restrict__ y2, *__restrict__ y3;   // stage 4
    const T *__restrict__ in_t, *__restrict__ in_m, *__restrict__ in_h;   // materialized stage inputs
    T *__restrict__ out_t, *__restrict__ out_m, *__restrict__ out_h;      // next-stage inputs
    const int32_t *__restrict__ slot;       // [n] source slot or -1
    const T *__restrict__ srcv;             // [4][nslot][S] this step
    int nslot;
    const int32_t *__restrict__ store_pos;  // [n] history position or -1 (stage 1)
    T *__restrict__ hist;                   // [nstore][S] of this step, or null
    T c, D, d6;                             // dt/2, dt, dt/6 (negated for the adjoint)
};

// Stage-input value of matrix TAG (0 = C, 1 = K, 2 = G) at row j, rebuilt from
// x1, x2, x3 and the earlier kb with the fused multiply-adds the row owner uses,
// e.g. km_3 = c*kb_2 + x3, kt_3 = c*km_2 + x2, h_3 = c*kt_2 + x1 (c = dt/2).
template <typename T, int S, int STAGE, int TAG>
__device__ __forceinline__ void gather(const StageArgs<T> &a, size_t j, T (&v)[S])
{
    const size_t o = j * S;
    if constexpr (STAGE == 1) {
        ldv<T, S>((TAG == 0 ? a.x3 : (TAG == 1 ? a.x2 : a.x1)) + o, v);
    } else if constexpr (STAGE == 2) {
        T p[S], q[S];
        if constexpr (TAG == 0) { ldv<T, S>(a.kb1 + o, p); ldv<T, S>(a.x3 + o, q); }
        else if constexpr (TAG == 1) { ldv<T, S>(a.x3 + o, p); ldv<T, S>(a.x2 + o, q); }
        else { ldv<T, S>(a.x2 + o, p); ldv<T, S>(a.x1 + o, q); }
#pragma unroll
        for (int s = 0; s < S; ++s) v[s] = fmaT(a.c, p[s], q[s]);
    } else if constexpr (STAGE == 3) {
        if constexpr (TAG == 0) {
            T p[S], q[S];
            ldv<T, S>(a.kb2 + o, p); ldv<T, S>(a.x3 + o, q);
#pragma unroll
            for (int s = 0; s < S; ++s) v[s] = fmaT(a.c, p[s], q[s]);
        } else if constexpr (TAG == 1) {
            T k1[S], x3[S], x2[S];
            ldv<T, S>(a.kb1 + o, k1); ldv<T, S>(a.x3 + o, x3); ldv<T, S>(a.x2 + o, x2);
#pragma unroll
            for (int s = 0; s < S; ++s) v[s] = fmaT(a.c, fmaT(a.c, k1[s], x3[s]), x2[s]);
        } else {
            T x3[S], x2[S], x1[S];
            ldv<T, S>(a.x3 + o, x3); ldv<T, S>(a.x2 + o, x2); ldv<T, S>(a.x1 + o, x1);
#pragma unroll
            for (int s = 0; s < S; ++s) v[s] = fmaT(a.c, fmaT(a.c, x3[s], x2[s]), x1[s]);
        }
    } else {
        if constexpr (TAG == 0) {
            T p[S], q[S];
            ldv<T, S>(a.kb3 + o, p); ldv<T, S>(a.x3 + o, q);
#pragma unroll
            for (int s = 0; s < S; ++s) v[s] = fmaT(a.D, p[s], q[s]);
        } else if constexpr (TAG == 1) {
            T k2[S], x3[S], x2[S];
            ldv<T, S>(a.kb2 + o, k2); ldv<T, S>(a.x3 + o, x3); ldv<T, S>(a.x2 + o, x2);
#pragma unroll
            for (int s = 0; s < S; ++s) v[s] = fmaT(a.D, fmaT(a.c, k2[s], x3[s]), x2[s]);
        } else {
            T k1[S], x3[S], x2[S], x1[S];
            ldv<T, S>(a.kb1 + o, k1); ldv<T, S>(a.x3 + o, x3); ldv<T, S>(a.x2 + o, x2); ldv<T, S>(a.x1 + o, x1);
#pragma unroll
            for (int s = 0; s < S; ++s) v[s] = fmaT(a.D, fmaT(a.c, fmaT(a.c, k1[s], x3[s]), x2[s]), x1[s]);
        }
    }
}

// Row epilogue: stage source, history (stage 1), kb or the next-stage inputs
// (stages 1-3) or the RK4 update into the other state buffer (stage 4).
// sl = the row's source slot (-1 none); pos = its history position (-1 none),
// read only in stage 1 with a history to write.
template <typename T, int S, int STAGE, int MAT>
__device__ __forceinline__ void finish_row_sp(const StageArgs<T> &a, int row, int sl, int pos, const T (&acc)[S])
{
    const size_t o = size_t(row) * S;
    T kb[S];
    if (sl >= 0) {
        T sv[S];
        ldv<T, S>(a.srcv + (size_t(STAGE - 1) * a.nslot + sl) * S, sv);
#pragma unroll
        for (int s = 0; s < S; ++s) kb[s] = sv[s] + acc[s];
    } else {
#pragma unroll
        for (int s = 0; s < S; ++s) kb[s] = acc[s];
    }
    if constexpr (STAGE == 1) {
        if (a.hist && pos >= 0) {
            T x2[S];
            ldv<T, S>(a.x2 + o, x2);
            stv<T, S>(a.hist + size_t(pos) * S, x2);
        }
    }
    if constexpr (STAGE < 4) {
        stv<T, S>(a.kb_out + o, kb);
        if constexpr (MAT == 1) {
            // next-stage inputs of this row: kt' = c km + x2, km' = c kb + x3, h' = c kt + x1
            T x1[S], x2[S], x3[S], kt[S], km[S], nt[S], nm[S], nh[S];
            ldv<T, S>(a.x1 + o, x1); ldv<T, S>(a.x2 + o, x2); ldv<T, S>(a.x3 + o, x3);
            if constexpr (STAGE == 1) {
#pragma unroll
                for (int s = 0; s < S; ++s) { kt[s] = x2[s]; km[s] = x3[s]; }
            } else {
                ldv<T, S>(a.in_t + o, kt);
                ldv<T, S>(a.in_m + o, km);
            }
            const T cc = STAGE == 3 ? a.D : a.c;
#pragma unroll
            for (int s = 0; s < S; ++s) {
                nt[s] = fmaT(cc, km[s], x2[s]);
                nm[s] = fmaT(cc, kb[s], x3[s]);
                nh[s] = fmaT(cc, kt[s], x1[s]);
            }
            stv<T, S>(a.out_t + o, nt);
            stv<T, S>(a.out_m + o, nm);
            stv<T, S>(a.out_h + o, nh);
        }
    } else {
        T x1[S], x2[S], x3[S], k1[S], k2[S], k3[S], n1[S], n2[S], n3[S];
        ldv<T, S>(a.x1 + o, x1); ldv<T, S>(a.x2 + o, x2); ldv<T, S>(a.x3 + o, x3);
        ldv<T, S>(a.kb1 + o, k1); ldv<T, S>(a.kb2 + o, k2); ldv<T, S>(a.kb3 + o, k3);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            // stage inputs of this row, built exactly as gather() builds them
            const T km2 = fmaT(a.c, k1[s], x3[s]);
            const T km3 = fmaT(a.c, k2[s], x3[s]);
            const T km4 = fmaT(a.D, k3[s], x3[s]);
            const T kt2 = fmaT(a.c, x3[s], x2[s]);
            const T kt3 = fmaT(a.c, km2, x2[s]);
            const T kt4 = fmaT(a.D, km3, x2[s]);
            const T ht = ((x2[s] + T(2) * kt2) + T(2) * kt3) + kt4;
            const T hm = ((x3[s] + T(2) * km2) + T(2) * km3) + km4;
            const T hb = ((k1[s] + T(2) * k2[s]) + T(2) * k3[s]) + kb[s];
            n1[s] = fmaT(a.d6, ht, x1[s]);
            n2[s] = fmaT(a.d6, hm, x2[s]);
            n3[s] = fmaT(a.d6, hb, x3[s]);
        }
        stv<T, S>(a.y1 + o, n1);
        stv<T, S>(a.y2 + o, n2);
        stv<T, S>(a.y3 + o, n3);
    }
}

template <typename T, int S, int STAGE, int MAT>
__device__ __forceinline__ void finish_row(const StageArgs<T> &a, int row, const T (&acc)[S])
{
    const int sl = __ldg(a.slot + row);
    const int pos = (STAGE == 1 && a.hist) ? __ldg(a.store_pos + row) : -1;
    finish_row_sp<T, S, STAGE, MAT>(a, row, sl, pos, acc);
}

}  // namespace hrn
