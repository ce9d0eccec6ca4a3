// hrn_gtile.cu -- RK4 stage kernel over spatially compact row tiles whose
// gathered stage inputs are staged in shared memory (variants 44, 45, 84, 85,
// and 46, 86 with the staged records moved by bulk copies).
//
// The row-parallel stage kernel gathers one row record ([S] shots of the stage
// input of the entry's matrix) per stored entry: about 18 gathers per row on the
// 27-node meshes.  Here the rows are cut into tiles of nodes that lie close
// together (nodes along a Morton curve of their coordinates when the mesh is
// known, consecutive rows otherwise), and a tile needs only about 8 distinct
// (matrix, column) records per row.  One CTA per tile:
//   1. one thread starts 1-D bulk copies of the tile's entry slab (values and
//      16-bit positions in the staged set) into shared memory;
//   2. meanwhile the threads load the tile's rows with their source slots and
//      history positions, and the tile's distinct records, ascending, into shared
//      memory (asynchronous 16-byte copies when the stage inputs are materialized);
//   3. after a bounded wait for the bulk copies, G lanes per row sum the row's
//      entries from shared memory;
//   4. one thread per row finishes it as the other stage kernels do (source,
//      history, kb or the next-stage inputs, or the RK4 update).
// Entries keep their order within a row and the lane split of the row-parallel
// kernel, so the row sums equal that kernel's bit for bit.
//
// A tile's distinct keys, sorted, fall into runs of consecutive columns of one
// matrix (about 1.5 runs per row and 6 records per run on the 27-node meshes), and
// a run is contiguous both in the stage-input array and in the staged set.  With
// materialized stage inputs and records of a multiple of 16 bytes, variants 46
// and 86 move each run with one 1-D bulk copy (the tensor memory accelerator)
// into shared memory, completing on the tile's mbarrier together with the entry
// slab, so the gathered records take no load/store-unit instructions at all.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "hrn_internal.h"
#include "hrn_stage.cuh"

namespace hrn {

#ifndef HRN_GT_BUDGET_KB
#define HRN_GT_BUDGET_KB 36    // shared memory per tile: up to six CTAs per SM
#endif
#ifndef HRN_GT_ROWS
#define HRN_GT_ROWS 64         // rows per tile before halving to fit the budget
#endif

#ifndef HRN_GT_THREADS
#define HRN_GT_THREADS 128
#endif

constexpr int kGtThreads = HRN_GT_THREADS;
constexpr size_t kGtBudget = size_t(HRN_GT_BUDGET_KB) * 1024;
constexpr int kGtRows = HRN_GT_ROWS;

template <typename T>
struct GtArgs {
    const int4 *__restrict__ tinfo;     // [ntiles][2]
    const int32_t *__restrict__ row;
    const int32_t *__restrict__ ent;
    const uint32_t *__restrict__ ukey;
    const uint16_t *__restrict__ lidx;
    const T *__restrict__ val;
    const int4 *__restrict__ runs;      // [nruns] staged index, matrix, first column, records (variants 46, 86)
    int *__restrict__ err;
};

__host__ __device__ constexpr size_t a16(size_t x) { return (x + 15) & ~size_t(15); }

// shared-memory footprint of a tile: barrier, four row arrays, row sums, entry slab, records
__host__ __device__ constexpr size_t gt_footprint(int nrows, int nent_pad, int nu, size_t elem, size_t rec)
{
    return 16 + 4 * a16(size_t(nrows) * 4) + a16(size_t(nrows) * rec) + a16(size_t(nent_pad) * 2) +
           a16(size_t(nent_pad) * elem) + size_t(nu) * rec;
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

template <typename T, int S>
__device__ __forceinline__ void sts_rec(T *d, const T (&v)[S])
{
    if constexpr (sizeof(T) == 8 && S % 2 == 0) {
#pragma unroll
        for (int s = 0; s < S; s += 2) reinterpret_cast<double2 *>(d)[s / 2] = make_double2(v[s], v[s + 1]);
    } else if constexpr (sizeof(T) == 4 && S % 4 == 0) {
#pragma unroll
        for (int s = 0; s < S; s += 4) reinterpret_cast<float4 *>(d)[s / 4] = make_float4(v[s], v[s + 1], v[s + 2], v[s + 3]);
    } else if constexpr (sizeof(T) == 4 && S % 2 == 0) {
#pragma unroll
        for (int s = 0; s < S; s += 2) reinterpret_cast<float2 *>(d)[s / 2] = make_float2(v[s], v[s + 1]);
    } else {
#pragma unroll
        for (int s = 0; s < S; ++s) d[s] = v[s];
    }
}

template <typename T, int S>
__device__ __forceinline__ void lds_rec(const T *p, T (&o)[S])
{
    if constexpr (sizeof(T) == 8 && S % 2 == 0) {
#pragma unroll
        for (int s = 0; s < S; s += 2) {
            const double2 v = reinterpret_cast<const double2 *>(p)[s / 2];
            o[s] = v.x;
            o[s + 1] = v.y;
        }
    } else if constexpr (sizeof(T) == 4 && S % 4 == 0) {
#pragma unroll
        for (int s = 0; s < S; s += 4) {
            const float4 v = reinterpret_cast<const float4 *>(p)[s / 4];
            o[s] = v.x; o[s + 1] = v.y; o[s + 2] = v.z; o[s + 3] = v.w;
        }
    } else if constexpr (sizeof(T) == 4 && S % 2 == 0) {
#pragma unroll
        for (int s = 0; s < S; s += 2) {
            const float2 v = reinterpret_cast<const float2 *>(p)[s / 2];
            o[s] = v.x; o[s + 1] = v.y;
        }
    } else {
#pragma unroll
        for (int s = 0; s < S; ++s) o[s] = p[s];
    }
}

// 32-byte staged records placed with their two 16-byte halves swapped when bit 2 of
// the record's index is set.  Eight lanes reading eight random records then spread over
// all eight 16-byte bank groups instead of the four even (or odd) ones, which cuts the
// shared-memory bank conflicts of the row sums; the values and the order of the sums
// are unchanged.
template <typename T, int S>
constexpr bool kSwizzleRec = (S * sizeof(T)) == 32;

__device__ __forceinline__ uint32_t rec_swz(uint32_t idx) { return ((idx >> 2) & 1u) * 16u; }

template <typename T, int S>
__device__ __forceinline__ void sts_rec_swz(T *base, uint32_t idx, const T (&v)[S])
{
    if constexpr (kSwizzleRec<T, S>) {
        char *rec = reinterpret_cast<char *>(base) + size_t(idx) * 32;
        const uint32_t sw = rec_swz(idx);
        const T *lo = v, *hi = v + S / 2;
        if constexpr (sizeof(T) == 8) {
            *reinterpret_cast<double2 *>(rec + sw) = make_double2(lo[0], lo[1]);
            *reinterpret_cast<double2 *>(rec + (16u ^ sw)) = make_double2(hi[0], hi[1]);
        } else {
            *reinterpret_cast<float4 *>(rec + sw) = make_float4(lo[0], lo[1], lo[2], lo[3]);
            *reinterpret_cast<float4 *>(rec + (16u ^ sw)) = make_float4(hi[0], hi[1], hi[2], hi[3]);
        }
    } else {
        sts_rec<T, S>(base + size_t(idx) * S, v);
    }
}

template <typename T, int S>
__device__ __forceinline__ void lds_rec_swz(const T *base, uint32_t idx, T (&o)[S])
{
    if constexpr (kSwizzleRec<T, S>) {
        const char *rec = reinterpret_cast<const char *>(base) + size_t(idx) * 32;
        const uint32_t sw = rec_swz(idx);
        if constexpr (sizeof(T) == 8) {
            const double2 a = *reinterpret_cast<const double2 *>(rec + sw);
            const double2 b = *reinterpret_cast<const double2 *>(rec + (16u ^ sw));
            o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
        } else {
            const float4 a = *reinterpret_cast<const float4 *>(rec + sw);
            const float4 b = *reinterpret_cast<const float4 *>(rec + (16u ^ sw));
            o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
            o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
        }
    } else {
        lds_rec<T, S>(base + size_t(idx) * S, o);
    }
}

// Stage input of matrix TAG at row j (same values as the gathers of rk4_stage).
template <typename T, int S, int STAGE, int MAT>
__device__ __forceinline__ void staged_input(const StageArgs<T> &a, uint32_t key, T (&v)[S])
{
    const int tag = int(key >> kTagBits);
    const size_t j = size_t(key & kColMask);
    if constexpr (MAT == 1 && STAGE > 1) {
        const T *src = tag == 0 ? a.in_m : (tag == 1 ? a.in_t : a.in_h);
        ldv<T, S>(src + j * S, v);
    } else {
        if (tag == 0) gather<T, S, STAGE, 0>(a, j, v);
        else if (tag == 1) gather<T, S, STAGE, 1>(a, j, v);
        else gather<T, S, STAGE, 2>(a, j, v);
    }
}

template <typename T, int S, int STAGE, int G, int MAT, bool RUNS = false>
__global__ void __launch_bounds__(kGtThreads) rk4_stage_gt(const StageArgs<T> a, const GtArgs<T> g)
{
    static_assert(!RUNS || (MAT == 1 && (S * sizeof(T)) % 16 == 0), "bulk-copied runs need materialized inputs and 16-byte records");
    extern __shared__ __align__(128) unsigned char gt_smem[];
    const int4 ti0 = __ldg(g.tinfo + 2 * blockIdx.x), ti1 = __ldg(g.tinfo + 2 * blockIdx.x + 1);
    const int row_off = ti0.x, nrows = ti0.y, ent_off = ti0.z, nent = ti0.w, u_off = ti1.x, nu = ti1.y;
    const int run_off = ti1.z, nruns = ti1.w;
    uint64_t *bar = reinterpret_cast<uint64_t *>(gt_smem);
    size_t off = 16;
    int32_t *s_row = reinterpret_cast<int32_t *>(gt_smem + off); off += a16(size_t(nrows) * 4);
    int32_t *s_ent = reinterpret_cast<int32_t *>(gt_smem + off); off += a16(size_t(nrows) * 4);
    int32_t *s_slot = reinterpret_cast<int32_t *>(gt_smem + off); off += a16(size_t(nrows) * 4);
    int32_t *s_pos = reinterpret_cast<int32_t *>(gt_smem + off); off += a16(size_t(nrows) * 4);
    T *s_acc = reinterpret_cast<T *>(gt_smem + off); off += a16(size_t(nrows) * S * sizeof(T));
    uint16_t *s_lidx = reinterpret_cast<uint16_t *>(gt_smem + off); off += a16(size_t(nent) * 2);
    T *s_val = reinterpret_cast<T *>(gt_smem + off); off += a16(size_t(nent) * sizeof(T));
    T *sx = reinterpret_cast<T *>(gt_smem + off);

    constexpr size_t kRec = S * sizeof(T);
    // 1. entry slab by bulk copies (sizes and addresses are multiples of 16 bytes); with
    //    RUNS the staged records too, one bulk copy per run of consecutive columns, all
    //    completing on the same barrier, whose byte count is set before any copy starts
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        const uint32_t bytes = uint32_t(nent) * uint32_t(2 + sizeof(T)) + (RUNS ? uint32_t(nu) * uint32_t(kRec) : 0u);
        if (bytes > 0) mbar_expect_tx(bar, bytes);
        else asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0 && nent > 0) {
        bulk_g2s(s_lidx, g.lidx + ent_off, uint32_t(nent) * 2u, bar);
        bulk_g2s(s_val, g.val + ent_off, uint32_t(nent) * uint32_t(sizeof(T)), bar);
    }
    if constexpr (RUNS) {
        for (int q = threadIdx.x; q < nruns; q += kGtThreads) {
            const int4 rn = __ldg(g.runs + run_off + q);   // staged index, matrix, first column, records
            const T *src = STAGE == 1 ? (rn.y == 0 ? a.x3 : (rn.y == 1 ? a.x2 : a.x1))
                                      : (rn.y == 0 ? a.in_m : (rn.y == 1 ? a.in_t : a.in_h));
            bulk_g2s(sx + size_t(rn.x) * S, src + size_t(rn.z) * S, uint32_t(rn.w) * uint32_t(kRec), bar);
        }
    }
    // 2. rows of the tile with their source slot and history position
    for (int r = threadIdx.x; r < nrows; r += kGtThreads) {
        const int row = __ldg(g.row + row_off + r);
        s_row[r] = row;
        s_ent[r] = __ldg(g.ent + row_off + r);
        s_slot[r] = __ldg(a.slot + row);
        s_pos[r] = (STAGE == 1 && a.hist) ? __ldg(a.store_pos + row) : -1;
    }
    //    staged set, ascending keys, adjacent threads on adjacent keys
    if constexpr (RUNS) {
        // the records arrive by the bulk copies above
    } else if constexpr (MAT == 1 && STAGE > 1 && kRec % 16 == 0) {
        // materialized inputs: asynchronous 16-byte copies straight into shared memory,
        // eight keys per thread in flight before their copies are issued
        for (int u = threadIdx.x; u < nu; u += 8 * kGtThreads) {
            uint32_t key[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int uu = u + q * kGtThreads;
                key[q] = uu < nu ? __ldg(g.ukey + u_off + uu) : 0u;
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int uu = u + q * kGtThreads;
                if (uu < nu) {
                    const int tag = int(key[q] >> kTagBits);
                    const T *src = (tag == 0 ? a.in_m : (tag == 1 ? a.in_t : a.in_h)) + size_t(key[q] & kColMask) * S;
                    T *d = sx + size_t(uu) * S;
                    if constexpr (kSwizzleRec<T, S>) {
                        const uint32_t sw = rec_swz(uint32_t(uu));
                        cp_async16(reinterpret_cast<char *>(d) + sw, reinterpret_cast<const char *>(src));
                        cp_async16(reinterpret_cast<char *>(d) + (16u ^ sw), reinterpret_cast<const char *>(src) + 16);
                    } else {
#pragma unroll
                        for (size_t b = 0; b < kRec; b += 16)
                            cp_async16(reinterpret_cast<char *>(d) + b, reinterpret_cast<const char *>(src) + b);
                    }
                }
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 0;" ::: "memory");
    } else {
        // Q records per thread per trip, all loads issued before the stores
        constexpr int Q = (kRec >= 64) ? 2 : 4;
        for (int u = threadIdx.x; u < nu; u += Q * kGtThreads) {
            T v[Q][S];
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const int uu = u + q * kGtThreads;
                if (uu < nu) staged_input<T, S, STAGE, MAT>(a, __ldg(g.ukey + u_off + uu), v[q]);
            }
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const int uu = u + q * kGtThreads;
                if (uu < nu) sts_rec_swz<T, S>(sx, uint32_t(uu), v[q]);
            }
        }
    }
    // bounded wait for the slab; on a timeout flag the error, let the copy land (bounded) and stop
    const bool ok = mbar_wait(bar, 0);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) {
            atomicExch(g.err, 1);
            mbar_wait(bar, 0);
        }
        return;
    }

    // 3. row sums, G lanes per row, everything read from shared memory
    const int lane = threadIdx.x & (G - 1);
    const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
    for (int i = int(threadIdx.x) / G; i < nrows; i += kGtThreads / G) {
        const uint32_t pe = uint32_t(s_ent[i]);
        const int k0 = int(pe & 0xffffu), k3 = k0 + int(pe >> 16);
        T acc[S];
#pragma unroll
        for (int s = 0; s < S; ++s) acc[s] = T(0);
        for (int k = k0 + lane; k < k3; k += 4 * G) {
#pragma unroll
            for (int uu = 0; uu < 4; ++uu) {
                const int kk = k + uu * G;
                if (kk < k3) {
                    T x[S];
                    if constexpr (RUNS) lds_rec<T, S>(sx + size_t(s_lidx[kk]) * S, x);   // bulk copies keep the plain layout
                    else lds_rec_swz<T, S>(sx, s_lidx[kk], x);
                    const T w = s_val[kk];
#pragma unroll
                    for (int s = 0; s < S; ++s) acc[s] = fmaT(w, x[s], acc[s]);
                }
            }
        }
#pragma unroll
        for (int off2 = G / 2; off2 > 0; off2 >>= 1)
#pragma unroll
            for (int s = 0; s < S; ++s) acc[s] += __shfl_xor_sync(gmask, acc[s], off2, G);
        if (lane == 0) sts_rec<T, S>(s_acc + size_t(i) * S, acc);
    }
    __syncthreads();
    // 4. one thread per row: source, history, kb / next-stage inputs or the RK4 update
    for (int r = threadIdx.x; r < nrows; r += kGtThreads) {
        T acc[S];
        lds_rec<T, S>(s_acc + size_t(r) * S, acc);
        finish_row_sp<T, S, STAGE, MAT>(a, s_row[r], s_slot[r], s_pos[r], acc);
    }
}

// ----------------------------------------------------------------------------
// Pipelined staged tiles (variants 47, 87): persistent CTAs of four consumer warps
// and one producer warp with two shared-memory buffers.  For its next tile the
// producer waits until the consumers have released that buffer, sets the byte count
// on the buffer's mbarrier and starts 1-D bulk copies of everything the tile needs:
// its header, the row metadata (entry range, source slot, history position, row),
// the entry slab, the staged records (one copy per run of consecutive columns) and
// the epilogue's row operands (x1, x2, x3 and the stage's inputs or kb, one copy per
// run of consecutive rows and operand).  Meanwhile the consumers sum and finish the
// previous tile from shared memory alone, so no phase of a tile waits on a global
// load.  The row sums and the epilogue use the arithmetic of the other stage kernels
// (equal to variants 41 / 81 bit for bit).

constexpr int kGtpConsumers = 128;
constexpr int kGtpThreads = kGtpConsumers + 32;
constexpr int kGtpHdr = 64;               // tile header: tinfo (32 B) and tinfo2 (16 B)
constexpr int kGtpRows = kGtRows;         // rows of a tile, at most

// buffer: header | meta [kGtpRows][4] int32 | operands [6][kGtpRows][S] | lidx | values | records
__host__ __device__ constexpr size_t gtp_fixed(size_t rec) { return kGtpHdr + size_t(kGtpRows) * 16 + 6 * size_t(kGtpRows) * rec; }
__host__ __device__ constexpr size_t gtp_buffer(size_t rec) { return gtp_fixed(rec) + kGtBudget; }
__host__ __device__ constexpr size_t gtp_smem(size_t rec) { return 64 + 2 * gtp_buffer(rec) + size_t(kGtpRows) * rec; }

template <typename T>
struct GtpArgs {
    const int32_t *__restrict__ tinfo;    // [ntiles][8]
    const int32_t *__restrict__ tinfo2;   // [ntiles][4] first operand run, runs
    const int4 *__restrict__ meta;        // [rows in tile order] entry range, slot, history position, row
    const int4 *__restrict__ eruns;       // [n] first tile row, first row (equation), rows
    const int4 *__restrict__ runs;        // record runs (as variants 46, 86)
    const uint16_t *__restrict__ lidx;
    const T *__restrict__ val;
    int ntiles;
    int *__restrict__ err;
};

__device__ __forceinline__ void bar_named_consumers() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// the stage's epilogue operands: x1, x2, x3, then (stages 2, 3) in_t, in_m or (stage 4) kb1, kb2, kb3
template <typename T, int STAGE>
__device__ __forceinline__ const T *gtp_operand(const StageArgs<T> &a, int v)
{
    if (v == 0) return a.x1;
    if (v == 1) return a.x2;
    if (v == 2) return a.x3;
    if constexpr (STAGE == 4) return v == 3 ? a.kb1 : (v == 4 ? a.kb2 : a.kb3);
    else return v == 3 ? a.in_t : a.in_m;
}

template <typename T, int STAGE>
constexpr int gtp_noperands() { return STAGE == 1 ? 3 : (STAGE == 4 ? 6 : 5); }

// Row epilogue of finish_row_sp with the row's operands read from shared memory
// (op(v) = operand v of this row); the same arithmetic, so the same bits.
template <typename T, int S, int STAGE>
__device__ __forceinline__ void gtp_finish(const StageArgs<T> &a, int row, int sl, int pos, const T (&acc)[S],
                                           const T *ops, int r)
{
    auto op = [&](int v, T (&o)[S]) { lds_rec<T, S>(ops + (size_t(v) * kGtpRows + r) * S, o); };
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
    T x1[S], x2[S], x3[S];
    op(0, x1);
    op(1, x2);
    op(2, x3);
    if constexpr (STAGE == 1) {
        if (a.hist && pos >= 0) stv<T, S>(a.hist + size_t(pos) * S, x2);
    }
    if constexpr (STAGE < 4) {
        stv<T, S>(a.kb_out + o, kb);
        T kt[S], km[S], nt[S], nm[S], nh[S];
        if constexpr (STAGE == 1) {
#pragma unroll
            for (int s = 0; s < S; ++s) { kt[s] = x2[s]; km[s] = x3[s]; }
        } else {
            op(3, kt);
            op(4, km);
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
    } else {
        T k1[S], k2[S], k3[S], n1[S], n2[S], n3[S];
        op(3, k1);
        op(4, k2);
        op(5, k3);
#pragma unroll
        for (int s = 0; s < S; ++s) {
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

template <typename T, int S, int STAGE, int G>
__global__ void __launch_bounds__(kGtpThreads) rk4_stage_gtp(const StageArgs<T> a, const GtpArgs<T> g)
{
    constexpr size_t kRec = S * sizeof(T);
    static_assert(kRec % 16 == 0, "pipelined tiles need 16-byte records");
    constexpr int NV = gtp_noperands<T, STAGE>();
    extern __shared__ __align__(128) unsigned char gtp_shm[];
    uint64_t *full = reinterpret_cast<uint64_t *>(gtp_shm);
    uint64_t *empty = full + 2;
    int *s_fail = reinterpret_cast<int *>(full + 4);
    unsigned char *buf0 = gtp_shm + 64;
    T *s_acc = reinterpret_cast<T *>(buf0 + 2 * gtp_buffer(kRec));
    const int tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        mbar_init(&empty[0], 1);
        mbar_init(&empty[1], 1);
        *s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int ntiles = g.ntiles;
    if (tid >= kGtpConsumers) {
        // ---- producer warp
        const int lane = tid - kGtpConsumers;
        int i = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
            const int b = i & 1, k = i >> 1;
            if (k >= 1 && !mbar_wait(&empty[b], uint32_t((k - 1) & 1))) {
                if (lane == 0) atomicExch(g.err, 1);
                break;
            }
            unsigned char *buf = buf0 + size_t(b) * gtp_buffer(kRec);
            const int4 ti0 = __ldg(reinterpret_cast<const int4 *>(g.tinfo) + 2 * t);
            const int4 ti1 = __ldg(reinterpret_cast<const int4 *>(g.tinfo) + 2 * t + 1);
            const int4 ti2 = __ldg(reinterpret_cast<const int4 *>(g.tinfo2) + t);
            const int row_off = ti0.x, nrows = ti0.y, ent_off = ti0.z, nent = ti0.w, nu = ti1.y;
            const int run_off = ti1.z, nruns = ti1.w, erun_off = ti2.x, neruns = ti2.y;
            uint16_t *s_lidx = reinterpret_cast<uint16_t *>(buf + gtp_fixed(kRec));
            T *s_val = reinterpret_cast<T *>(buf + gtp_fixed(kRec) + a16(size_t(nent) * 2));
            T *sx = reinterpret_cast<T *>(reinterpret_cast<unsigned char *>(s_val) + a16(size_t(nent) * sizeof(T)));
            T *ops = reinterpret_cast<T *>(buf + kGtpHdr + size_t(kGtpRows) * 16);
            if (lane == 0) {
                const uint32_t bytes = 48u + uint32_t(nrows) * 16u + uint32_t(nent) * uint32_t(2 + sizeof(T)) +
                                       uint32_t(nu) * uint32_t(kRec) + uint32_t(NV) * uint32_t(nrows) * uint32_t(kRec);
                mbar_expect_tx(&full[b], bytes);
            }
            __syncwarp();
            if (lane == 0) {
                bulk_g2s(buf, g.tinfo + 8 * size_t(t), 32u, &full[b]);
                bulk_g2s(buf + 32, g.tinfo2 + 4 * size_t(t), 16u, &full[b]);
                bulk_g2s(buf + kGtpHdr, g.meta + row_off, uint32_t(nrows) * 16u, &full[b]);
            } else if (lane == 1 && nent > 0) {
                bulk_g2s(s_lidx, g.lidx + ent_off, uint32_t(nent) * 2u, &full[b]);
            } else if (lane == 2 && nent > 0) {
                bulk_g2s(s_val, g.val + ent_off, uint32_t(nent) * uint32_t(sizeof(T)), &full[b]);
            }
            for (int q = lane; q < nruns; q += 32) {
                const int4 rn = __ldg(g.runs + run_off + q);
                const T *src = STAGE == 1 ? (rn.y == 0 ? a.x3 : (rn.y == 1 ? a.x2 : a.x1))
                                          : (rn.y == 0 ? a.in_m : (rn.y == 1 ? a.in_t : a.in_h));
                bulk_g2s(sx + size_t(rn.x) * S, src + size_t(rn.z) * S, uint32_t(rn.w) * uint32_t(kRec), &full[b]);
            }
            for (int q = lane; q < neruns * NV; q += 32) {
                const int v = q / neruns;
                const int4 er = __ldg(g.eruns + erun_off + (q - v * neruns));   // first tile row, first row, rows
                bulk_g2s(ops + (size_t(v) * kGtpRows + er.x) * S, gtp_operand<T, STAGE>(a, v) + size_t(er.y) * S,
                         uint32_t(er.z) * uint32_t(kRec), &full[b]);
            }
        }
        return;
    }
    // ---- consumer warps
    int i = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
        const int b = i & 1, k = i >> 1;
        const bool ok = mbar_wait(&full[b], uint32_t(k & 1));
        if (!ok) *s_fail = 1;
        bar_named_consumers();
        if (*s_fail) {
            if (tid == 0) {
                atomicExch(g.err, 1);
                mbar_wait(&full[b], uint32_t(k & 1));   // the copies in flight into this buffer
            }
            break;
        }
        const unsigned char *buf = buf0 + size_t(b) * gtp_buffer(kRec);
        const int4 ti0 = *reinterpret_cast<const int4 *>(buf);
        const int nrows = ti0.y, nent = ti0.w;
        const int4 *meta = reinterpret_cast<const int4 *>(buf + kGtpHdr);
        const uint16_t *s_lidx = reinterpret_cast<const uint16_t *>(buf + gtp_fixed(kRec));
        const T *s_val = reinterpret_cast<const T *>(buf + gtp_fixed(kRec) + a16(size_t(nent) * 2));
        const T *sx = reinterpret_cast<const T *>(reinterpret_cast<const unsigned char *>(s_val) + a16(size_t(nent) * sizeof(T)));
        const T *ops = reinterpret_cast<const T *>(buf + kGtpHdr + size_t(kGtpRows) * 16);
        // row sums, G lanes per row, from shared memory
        const int lane = tid & (G - 1);
        const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << ((tid & 31) & ~(G - 1)));
        for (int r = tid / G; r < nrows; r += kGtpConsumers / G) {
            const uint32_t pe = uint32_t(meta[r].x);
            const int k0 = int(pe & 0xffffu), k3 = k0 + int(pe >> 16);
            T acc[S];
#pragma unroll
            for (int s = 0; s < S; ++s) acc[s] = T(0);
            for (int kk0 = k0 + lane; kk0 < k3; kk0 += 4 * G) {
#pragma unroll
                for (int uu = 0; uu < 4; ++uu) {
                    const int kk = kk0 + uu * G;
                    if (kk < k3) {
                        T x[S];
                        lds_rec<T, S>(sx + size_t(s_lidx[kk]) * S, x);
                        const T w = s_val[kk];
#pragma unroll
                        for (int s = 0; s < S; ++s) acc[s] = fmaT(w, x[s], acc[s]);
                    }
                }
            }
#pragma unroll
            for (int off2 = G / 2; off2 > 0; off2 >>= 1)
#pragma unroll
                for (int s = 0; s < S; ++s) acc[s] += __shfl_xor_sync(gmask, acc[s], off2, G);
            if (lane == 0) sts_rec<T, S>(s_acc + size_t(r) * S, acc);
        }
        bar_named_consumers();
        // epilogue, one thread per row, operands from shared memory
        for (int r = tid; r < nrows; r += kGtpConsumers) {
            const int4 mt = meta[r];   // entry range, source slot, history position, row
            T acc[S];
            lds_rec<T, S>(s_acc + size_t(r) * S, acc);
            gtp_finish<T, S, STAGE>(a, mt.w, mt.y, mt.z, acc, ops, r);
        }
        bar_named_consumers();
        if (tid == 0) mbar_arrive(&empty[b]);
    }
}

// Row metadata of the pipelined tiles in tile order: entry range, source slot,
// history position, row (the slots and positions of the direction's current set-up).
__global__ void k_gtp_meta(int n, const int32_t *__restrict__ row, const int32_t *__restrict__ ent,
                           const int32_t *__restrict__ slot, const int32_t *__restrict__ store_pos, int4 *__restrict__ meta)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int q = row[r];
    meta[r] = make_int4(ent[r], slot[q], store_pos[q], q);
}

template <typename T>
__global__ void k_gt_values(int64_t nnz, const int32_t *__restrict__ perm, const T *__restrict__ src, T *__restrict__ dst)
{
    for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < nnz; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int32_t p = perm[k];
        dst[k] = p >= 0 ? src[p] : T(0);
    }
}

// ----------------------------------------------------------------------------
// tile construction (host)

static uint64_t spread3(uint32_t v)
{
    uint64_t r = 0;
    for (int b = 0; b < 10; ++b) r |= uint64_t((v >> b) & 1u) << (3 * b);
    return r;
}

// Rows in tile order, grouped by node (a group never straddles two tiles).
// With the mesh: the equations of each node (ID order), nodes along a Morton
// curve of their coordinates; without it, or if the mesh's ID does not number
// the operator's rows exactly once: consecutive rows, one row per group.
static void row_order(const hrn_ctx *c, std::vector<int32_t> &order, std::vector<int32_t> &gstart)
{
    const int n = c->neq;
    order.clear();
    gstart.clear();
    if (c->have_mesh && c->nj > 0 && c->h_id.size() == size_t(c->nj) * 9 && c->h_xyz.size() == size_t(c->nj) * 3) {
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int j = 0; j < c->nj; ++j)
            for (int d = 0; d < 3; ++d) {
                lo[d] = std::min(lo[d], c->h_xyz[size_t(j) * 3 + d]);
                hi[d] = std::max(hi[d], c->h_xyz[size_t(j) * 3 + d]);
            }
        const double ext = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-300});
        std::vector<std::pair<uint64_t, int32_t>> key(size_t(c->nj));
        for (int j = 0; j < c->nj; ++j) {
            uint64_t code = 0;
            for (int d = 0; d < 3; ++d) {
                const double f = (c->h_xyz[size_t(j) * 3 + d] - lo[d]) / ext;
                const uint32_t q = uint32_t(std::min(1023.0, std::max(0.0, f * 1023.999)));
                code |= spread3(q) << d;
            }
            key[j] = {code, j};
        }
        std::sort(key.begin(), key.end());
        std::vector<char> seen(size_t(n), 0);
        bool ok = true;
        for (const auto &kj : key) {
            const int j = kj.second;
            const size_t g0 = order.size();
            for (int d = 0; d < 9 && ok; ++d) {
                const int eq = c->h_id[size_t(j) * 9 + d];
                if (eq < 0) continue;
                if (eq >= n || seen[eq]) { ok = false; break; }
                seen[eq] = 1;
                order.push_back(eq);
            }
            if (!ok) break;
            if (order.size() > g0) gstart.push_back(int32_t(g0));
        }
        if (ok && order.size() == size_t(n)) {
            gstart.push_back(n);
            return;
        }
        order.clear();
        gstart.clear();
    }
    order.resize(size_t(n));
    std::iota(order.begin(), order.end(), 0);
    gstart.resize(size_t(n) + 1);
    std::iota(gstart.begin(), gstart.end(), 0);
}

static int gt_build(hrn_ctx *c, int adj, size_t rec_bytes)
{
    GtSet &gs = c->gt[adj];
    gs.built = false;
    const int n = c->neq;
    const int64_t nnz = c->nnz;
    const size_t elem = c->elem_bytes();
    std::vector<int32_t> rowptr;
    std::vector<uint32_t> colx;
    if (adj == 0) {
        rowptr = c->h_rowptr;
        colx = c->h_colx;
    } else {
        rowptr.resize(size_t(n) + 1);
        colx.resize(size_t(nnz));
        HRN_CUDA(c, cudaMemcpy(rowptr.data(), c->d_rowptrT.p, rowptr.size() * 4, cudaMemcpyDeviceToHost));
        if (nnz) HRN_CUDA(c, cudaMemcpy(colx.data(), c->d_colxT.p, colx.size() * 4, cudaMemcpyDeviceToHost));
    }
    std::vector<int32_t> order, gstart;
    row_order(c, order, gstart);
    const int ngroups = int(gstart.size()) - 1;

    // Distinct keys of a range of groups, counted with a per-key mark of the last
    // range that saw it (no clearing between ranges).  Key index = matrix * n + column.
    auto kidx = [n](uint32_t key) { return size_t(key >> kTagBits) * size_t(n) + size_t(key & kColMask); };
    std::vector<int32_t> mark(size_t(3) * n, -1), pos(size_t(3) * n, 0);
    int range_id = 0;
    auto count = [&](int g0, int g1, int64_t &nent, int &nu) {
        ++range_id;
        nent = 0;
        nu = 0;
        for (int r = gstart[g0]; r < gstart[g1]; ++r) {
            const int row = order[r];
            for (int32_t p = rowptr[row]; p < rowptr[row + 1]; ++p) {
                const size_t k = kidx(colx[p]);
                if (mark[k] != range_id) {
                    mark[k] = range_id;
                    ++nu;
                }
            }
            nent += rowptr[row + 1] - rowptr[row];
        }
    };
    auto pad8 = [](int64_t x) { return (x + 7) & ~int64_t(7); };
    std::vector<int32_t> h_tinfo, h_ent(size_t(std::max(n, 1)), 0);
    std::vector<uint32_t> h_ukey;
    std::vector<uint16_t> h_lidx;
    std::vector<int32_t> h_perm;
    std::vector<int32_t> h_runs;   // [nruns][4] staged index, matrix, first column, records
    std::vector<int32_t> h_eruns;  // [n][4] first tile row, first row, rows: runs of consecutive rows of a tile
    std::vector<int32_t> h_tinfo2; // [ntiles][4] first operand run, operand runs
    int max_rows = 0;
    std::vector<uint32_t> keys;
    size_t smem = 0;
    bool fit = true;
    // accept groups [g0, g1) as a tile: its ascending keys, rows, entries and slab padding
    auto emit = [&](int g0, int g1) {
        ++range_id;
        keys.clear();
        for (int r = gstart[g0]; r < gstart[g1]; ++r)
            for (int32_t p = rowptr[order[r]]; p < rowptr[order[r] + 1]; ++p) {
                const size_t k = kidx(colx[p]);
                if (mark[k] != range_id) {
                    mark[k] = range_id;
                    keys.push_back(colx[p]);
                }
            }
        std::sort(keys.begin(), keys.end());
        for (size_t q = 0; q < keys.size(); ++q) pos[kidx(keys[q])] = int32_t(q);
        const int64_t e0 = int64_t(h_lidx.size());
        for (int r = gstart[g0]; r < gstart[g1]; ++r) {
            const int row = order[r];
            const int cnt = rowptr[row + 1] - rowptr[row];
            h_ent[r] = int32_t(uint32_t(int64_t(h_lidx.size()) - e0) | (uint32_t(cnt) << 16));
            for (int32_t p = rowptr[row]; p < rowptr[row + 1]; ++p) {
                h_lidx.push_back(uint16_t(pos[kidx(colx[p])]));
                h_perm.push_back(p);
            }
        }
        const int64_t ne = int64_t(h_lidx.size()) - e0;
        h_lidx.resize(size_t(e0 + pad8(ne)), 0);
        h_perm.resize(size_t(e0 + pad8(ne)), -1);
        // runs of consecutive keys: consecutive columns of one matrix, contiguous in the
        // stage-input array and in the staged set
        const int32_t r0 = int32_t(h_runs.size() / 4);
        for (size_t q = 0; q < keys.size();) {
            size_t q1 = q + 1;
            while (q1 < keys.size() && keys[q1] == keys[q1 - 1] + 1u) ++q1;
            const int32_t rn[4] = {int32_t(q), int32_t(keys[q] >> kTagBits), int32_t(keys[q] & kColMask), int32_t(q1 - q)};
            h_runs.insert(h_runs.end(), rn, rn + 4);
            q = q1;
        }
        const int32_t ti[8] = {gstart[g0], gstart[g1] - gstart[g0], int32_t(e0), int32_t(pad8(ne)),
                               int32_t(h_ukey.size()), int32_t(keys.size()), r0, int32_t(h_runs.size() / 4) - r0};
        // runs of consecutive rows (equations) among the tile's rows, for the epilogue's operand copies
        const int32_t er0 = int32_t(h_eruns.size() / 4);
        for (int r = gstart[g0]; r < gstart[g1];) {
            int r1 = r + 1;
            while (r1 < gstart[g1] && order[r1] == order[r1 - 1] + 1) ++r1;
            const int32_t er[4] = {r - gstart[g0], order[r], r1 - r, 0};
            h_eruns.insert(h_eruns.end(), er, er + 4);
            r = r1;
        }
        const int32_t ti2[4] = {er0, int32_t(h_eruns.size() / 4) - er0, 0, 0};
        h_tinfo2.insert(h_tinfo2.end(), ti2, ti2 + 4);
        max_rows = std::max(max_rows, gstart[g1] - gstart[g0]);
        h_tinfo.insert(h_tinfo.end(), ti, ti + 8);
        h_ukey.insert(h_ukey.end(), keys.begin(), keys.end());
    };
    // cut a range of groups into tiles: halve until the tile's footprint fits
    std::vector<std::pair<int, int>> stack;
    auto cut = [&](int g0, int g1) {
        stack.assign(1, {g0, g1});
        while (!stack.empty() && fit) {
            const auto [a0, a1] = stack.back();
            stack.pop_back();
            int64_t nent = 0;
            int nu = 0;
            count(a0, a1, nent, nu);
            const int nrows = gstart[a1] - gstart[a0];
            const int64_t ne = pad8(nent);
            const bool small = ne <= 65535 && nu <= 65535;
            const size_t f = small ? gt_footprint(nrows, int(ne), nu, elem, rec_bytes) : ~size_t(0);
            if (f > kGtBudget) {
                if (a1 - a0 == 1) { fit = false; break; }
                const int mid = (a0 + a1) / 2;
                stack.push_back({mid, a1});
                stack.push_back({a0, mid});
                continue;
            }
            emit(a0, a1);
            smem = std::max(smem, f);
        }
    };
    int g = 0;
    while (g < ngroups && fit) {
        int g1 = g;
        while (g1 < ngroups && (g1 == g || gstart[g1 + 1] - gstart[g] <= kGtRows)) ++g1;
        cut(g, g1);
        g = g1;
    }
    if (!fit) return set_error(c, HRN_EARG, "a node's rows need more shared memory than a staged tile holds");
    if (int64_t(h_ukey.size()) >= (int64_t(1) << 31) || int64_t(h_lidx.size()) >= (int64_t(1) << 31))
        return set_error(c, HRN_EARG, "staged-gather tiles need fewer than 2^31 entries and keys");
    const int ntiles = int(h_tinfo.size() / 8);
    const int64_t total = int64_t(h_lidx.size());
    if (h_lidx.size() < 8) {
        h_lidx.resize(8, 0);
        h_perm.resize(8, -1);
    }

    HRN_CUDA(c, gs.d_tinfo.alloc(std::max<size_t>(h_tinfo.size(), 8) * 4));
    HRN_CUDA(c, gs.d_row.alloc(std::max<size_t>(order.size(), 1) * 4));
    HRN_CUDA(c, gs.d_ent.alloc(h_ent.size() * 4));
    HRN_CUDA(c, gs.d_ukey.alloc(std::max<size_t>(h_ukey.size(), 1) * 4));
    HRN_CUDA(c, gs.d_lidx.alloc(h_lidx.size() * 2));
    HRN_CUDA(c, gs.d_perm.alloc(h_perm.size() * 4));
    HRN_CUDA(c, gs.d_runs.alloc(std::max<size_t>(h_runs.size(), 4) * 4));
    HRN_CUDA(c, gs.d_eruns.alloc(std::max<size_t>(h_eruns.size(), 4) * 4));
    HRN_CUDA(c, gs.d_tinfo2.alloc(std::max<size_t>(h_tinfo2.size(), 4) * 4));
    HRN_CUDA(c, gs.d_meta.alloc(std::max<size_t>(order.size(), 1) * 16));
    if (!h_eruns.empty()) HRN_CUDA(c, cudaMemcpy(gs.d_eruns.p, h_eruns.data(), h_eruns.size() * 4, cudaMemcpyHostToDevice));
    if (!h_tinfo2.empty()) HRN_CUDA(c, cudaMemcpy(gs.d_tinfo2.p, h_tinfo2.data(), h_tinfo2.size() * 4, cudaMemcpyHostToDevice));
    if (!h_runs.empty()) HRN_CUDA(c, cudaMemcpy(gs.d_runs.p, h_runs.data(), h_runs.size() * 4, cudaMemcpyHostToDevice));
    if (!h_tinfo.empty()) HRN_CUDA(c, cudaMemcpy(gs.d_tinfo.p, h_tinfo.data(), h_tinfo.size() * 4, cudaMemcpyHostToDevice));
    if (!order.empty()) HRN_CUDA(c, cudaMemcpy(gs.d_row.p, order.data(), order.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(gs.d_ent.p, h_ent.data(), h_ent.size() * 4, cudaMemcpyHostToDevice));
    if (!h_ukey.empty()) HRN_CUDA(c, cudaMemcpy(gs.d_ukey.p, h_ukey.data(), h_ukey.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(gs.d_lidx.p, h_lidx.data(), h_lidx.size() * 2, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(gs.d_perm.p, h_perm.data(), h_perm.size() * 4, cudaMemcpyHostToDevice));
    gs.ntiles = ntiles;
    gs.smem = smem;
    gs.nu = int64_t(h_ukey.size());
    gs.nent = total;
    gs.nruns = int64_t(h_runs.size() / 4);
    gs.max_rows = max_rows;
    gs.rec_bytes = rec_bytes;
    gs.val_version = -1;
    gs.built = true;
    return 0;
}

template <typename T>
static int gt_values(hrn_ctx *c, int adj)
{
    GtSet &gs = c->gt[adj];
    if (gs.val_version == c->val_version && gs.val_elem == sizeof(T)) return 0;
    const int64_t ne = std::max<int64_t>(gs.nent, 8);
    const size_t vb = size_t(ne) * sizeof(T);
    if (gs.d_val.bytes != vb) HRN_CUDA(c, gs.d_val.alloc(vb));
    const T *src = adj ? c->d_adj.as<T>() : c->d_fwd.as<T>();
    const int th = 256;
    const int blocks = int(std::min<int64_t>((ne + th - 1) / th, int64_t(c->num_sms) * 16));
    k_gt_values<T><<<blocks, th, 0, c->stream>>>(ne, gs.d_perm.as<int32_t>(), src, gs.d_val.as<T>());
    ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    gs.val_version = c->val_version;
    gs.val_elem = sizeof(T);
    return 0;
}

int gtp_prepare(hrn_ctx *c, int adj)
{
    GtSet &gs = c->gt[adj];
    if (!gs.built) return set_error(c, HRN_ESTATE, "staged-gather tables not built");
    if (gs.max_rows > kGtpRows) return set_error(c, HRN_EARG, "a tile has more rows than the pipelined tiles hold");
    const int n = c->neq;
    if (n == 0) return 0;
    k_gtp_meta<<<(n + 255) / 256, 256, 0, c->stream>>>(n, gs.d_row.as<int32_t>(), gs.d_ent.as<int32_t>(),
                                                       (adj ? c->d_slot_a : c->d_slot_f).as<int32_t>(),
                                                       c->d_store_pos.as<int32_t>(), gs.d_meta.as<int4>());
    ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    return 0;
}

int gt_ready(hrn_ctx *c, int adj)
{
    if (!c->have_pattern || !c->have_operator) return set_error(c, HRN_ESTATE, "no operator");
    if (c->nshot < 1) return set_error(c, HRN_ESTATE, "no shots");
    const size_t rec = size_t(c->nshot) * c->elem_bytes();
    GtSet &gs = c->gt[adj];
    if (!gs.built || gs.rec_bytes != rec)
        if (int rc = gt_build(c, adj, rec)) return rc;
    return c->precision == HRN_FP64 ? gt_values<double>(c, adj) : gt_values<float>(c, adj);
}

// ----------------------------------------------------------------------------
// launch

template <typename T, int S, int STAGE, int G, int MAT, bool RUNS = false>
static void launch_gt(const StageArgs<T> &a, const GtArgs<T> &g, int ntiles, size_t smem, cudaStream_t st)
{
    static std::atomic<uint64_t> smem_done{0};
    smem_limit_once(rk4_stage_gt<T, S, STAGE, G, MAT, RUNS>, int(kGtBudget), smem_done);
    rk4_stage_gt<T, S, STAGE, G, MAT, RUNS><<<ntiles, kGtThreads, smem, st>>>(a, g);
}

template <typename T, int S, int STAGE, int G>
static void launch_gtp(const StageArgs<T> &a, const GtpArgs<T> &g, int num_sms, cudaStream_t st)
{
    if constexpr ((S * sizeof(T)) % 16 == 0) {
        static std::atomic<uint64_t> smem_done{0};
        constexpr size_t smem = gtp_smem(S * sizeof(T));
        smem_limit_once(rk4_stage_gtp<T, S, STAGE, G>, int(smem), smem_done);
        const int per_sm = std::max(1, int((227 * 1024) / smem));
        const int grid = std::min(g.ntiles, num_sms * per_sm);
        rk4_stage_gtp<T, S, STAGE, G><<<grid, kGtpThreads, smem, st>>>(a, g);
    }
}

template <typename T, int S, int STAGE>
static void launch_gt_variant(const StageArgs<T> &a, const GtArgs<T> &g, int ntiles, size_t smem, int variant,
                              cudaStream_t st)
{
    switch (variant) {
    case 44: launch_gt<T, S, STAGE, 4, 0>(a, g, ntiles, smem, st); break;
    case 45: launch_gt<T, S, STAGE, 4, 1>(a, g, ntiles, smem, st); break;
    case 84: launch_gt<T, S, STAGE, 8, 0>(a, g, ntiles, smem, st); break;
    case 46:
    case 86:
        if constexpr ((S * sizeof(T)) % 16 == 0) {
            if (variant == 46) launch_gt<T, S, STAGE, 4, 1, true>(a, g, ntiles, smem, st);
            else launch_gt<T, S, STAGE, 8, 1, true>(a, g, ntiles, smem, st);
        }
        break;
    default: launch_gt<T, S, STAGE, 8, 1>(a, g, ntiles, smem, st); break;
    }
}

template <typename T, int S>
static int gt_stage_t(hrn_ctx *c, const StageArgs<T> &a, int stage, int adj, int variant)
{
    const GtSet &gs = c->gt[adj];
    if (!gs.built) {
        // the tables are built before every time loop; reaching here without them is an
        // internal error, flagged so that the call fails instead of skipping the stage
        static const int two = 2;
        cudaMemcpyAsync(c->d_step_err.p, &two, sizeof(int), cudaMemcpyHostToDevice, c->stream);
        return set_error(c, HRN_ESTATE, "staged-gather tables not built");
    }
    if (gs.ntiles == 0) return 0;   // no rows
    if ((variant == 46 || variant == 86 || variant == 47 || variant == 87) && (S * sizeof(T)) % 16 != 0) {
        static const int two = 2;
        cudaMemcpyAsync(c->d_step_err.p, &two, sizeof(int), cudaMemcpyHostToDevice, c->stream);
        return set_error(c, HRN_EARG, "variants 46, 47, 86, 87 need records of a multiple of 16 bytes");
    }
    if (variant == 47 || variant == 87) {
        const GtpArgs<T> gp{gs.d_tinfo.as<int32_t>(), gs.d_tinfo2.as<int32_t>(), gs.d_meta.as<int4>(), gs.d_eruns.as<int4>(),
                            gs.d_runs.as<int4>(), gs.d_lidx.as<uint16_t>(), gs.d_val.as<T>(), gs.ntiles, c->d_step_err.as<int>()};
        switch (stage * 100 + variant) {
        case 147: launch_gtp<T, S, 1, 4>(a, gp, c->num_sms, c->stream); break;
        case 247: launch_gtp<T, S, 2, 4>(a, gp, c->num_sms, c->stream); break;
        case 347: launch_gtp<T, S, 3, 4>(a, gp, c->num_sms, c->stream); break;
        case 447: launch_gtp<T, S, 4, 4>(a, gp, c->num_sms, c->stream); break;
        case 187: launch_gtp<T, S, 1, 8>(a, gp, c->num_sms, c->stream); break;
        case 287: launch_gtp<T, S, 2, 8>(a, gp, c->num_sms, c->stream); break;
        case 387: launch_gtp<T, S, 3, 8>(a, gp, c->num_sms, c->stream); break;
        default: launch_gtp<T, S, 4, 8>(a, gp, c->num_sms, c->stream); break;
        }
        return 0;
    }
    const GtArgs<T> g{gs.d_tinfo.as<int4>(), gs.d_row.as<int32_t>(), gs.d_ent.as<int32_t>(), gs.d_ukey.as<uint32_t>(),
                      gs.d_lidx.as<uint16_t>(), gs.d_val.as<T>(), gs.d_runs.as<int4>(), c->d_step_err.as<int>()};
    switch (stage) {
    case 1: launch_gt_variant<T, S, 1>(a, g, gs.ntiles, gs.smem, variant, c->stream); break;
    case 2: launch_gt_variant<T, S, 2>(a, g, gs.ntiles, gs.smem, variant, c->stream); break;
    case 3: launch_gt_variant<T, S, 3>(a, g, gs.ntiles, gs.smem, variant, c->stream); break;
    default: launch_gt_variant<T, S, 4>(a, g, gs.ntiles, gs.smem, variant, c->stream); break;
    }
    return 0;
}

#define HRN_GT_DISPATCH(T)                                                              \
    switch (c->nshot) {                                                                 \
    case 1: return gt_stage_t<T, 1>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, variant); \
    case 2: return gt_stage_t<T, 2>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, variant); \
    case 3: return gt_stage_t<T, 3>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, variant); \
    case 4: return gt_stage_t<T, 4>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, variant); \
    case 5: return gt_stage_t<T, 5>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, variant); \
    case 6: return gt_stage_t<T, 6>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, variant); \
    case 7: return gt_stage_t<T, 7>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, variant); \
    case 8: return gt_stage_t<T, 8>(c, *static_cast<const StageArgs<T> *>(args), stage, adj, variant); \
    default: return set_error(c, HRN_EARG, "nshot out of range");                      \
    }

int gt_stage(hrn_ctx *c, const void *args, int stage, int adj, int variant)
{
    if (c->precision == HRN_FP64) { HRN_GT_DISPATCH(double) }
    HRN_GT_DISPATCH(float)
}

}  // namespace hrn
