// hrn_internal.h -- context layout and helpers shared by the CUDA sources of
// libhirensi_b200.so.  Not part of the public C ABI (include/hirensi_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <vector>

#include "../../include/hirensi_b200.h"

namespace hrn {

// Incremented by every device allocation or release of a DevBuf, so that a
// captured graph can tell whether any buffer it names may have moved.
inline std::atomic<uint64_t> &alloc_generation()
{
    static std::atomic<uint64_t> g{0};
    return g;
}

// Raise a kernel's dynamic shared-memory limit once per device: the attribute
// belongs to the device that is current, and contexts on several devices or
// threads may launch the same kernel.  `done` holds one bit per device.
template <typename K>
inline void smem_limit_once(K kernel, int bytes, std::atomic<uint64_t> &done)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t bit = dev >= 0 && dev < 64 ? (uint64_t(1) << dev) : 0;
    if (bit && (done.load() & bit)) return;
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    done.fetch_or(bit);
}

// Owning device buffer (cudaMalloc / cudaFree).
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) {
            cudaFree(p);
            alloc_generation()++;
        }
        p = nullptr;
        bytes = 0;
    }
    cudaError_t alloc(size_t n) {
        if (n == bytes && p) return cudaSuccess;
        release();
        if (n == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(&p, n);
        alloc_generation()++;
        if (e == cudaSuccess) bytes = n;
        else p = nullptr;
        return e;
    }
    template <typename T> T *as() const { return static_cast<T *>(p); }
};

constexpr int kTagBits = 30;
constexpr int kTileEntries = 4096;     // entries per tile of the tiled stage kernel
constexpr size_t kBulkPad = 64;        // bytes past the end of bulk-copied arrays
constexpr uint32_t kColMask = (1u << kTagBits) - 1u;

// One time loop (every launch of a forward or adjoint call) captured as a CUDA
// graph and replayed while its signature -- allocation generation, settings
// epoch, variant and flags -- is unchanged.
struct LoopGraph {
    cudaGraphExec_t exec = nullptr;
    uint64_t sig[6] = {0, 0, 0, 0, 0, 0};
    int64_t launches = 0;      // kernels launched by one replay
    void reset() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        for (auto &v : sig) v = 0;
        launches = 0;
    }
    ~LoopGraph() { reset(); }
};

// Row tiles of the staged-gather stage kernel (variants 44-46, 84-86) for one
// operator direction: spatially compact sets of rows whose gathered (matrix,
// column) pairs, entries and row data fit in one CTA's shared memory.
struct GtSet {
    bool built = false;
    size_t rec_bytes = 0;       // bytes of one staged record (S values) the tiles were cut for
    int ntiles = 0;
    size_t smem = 0;            // largest shared-memory footprint of a tile (bytes)
    int64_t nu = 0;             // staged records over all tiles
    int64_t nent = 0;           // entries over all tiles, each tile padded to a multiple of 8
    DevBuf d_tinfo;             // [ntiles][8] first tile row, rows, first entry, padded entries, first key, keys
    DevBuf d_row;               // [neq] row of each tile row
    DevBuf d_ent;               // [neq] first entry (relative to the tile) | entry count << 16
    DevBuf d_ukey;              // [nu] matrix id << 30 | column, ascending within a tile
    DevBuf d_lidx;              // [nent] uint16 position of the entry's key in its tile's set
    DevBuf d_perm;              // [nent] int32 entry of the scaled value array (-1: padding)
    DevBuf d_val;               // [nent] scaled values in tile order (T)
    DevBuf d_runs;              // [nruns][4] staged index, matrix, first column, records of each run of consecutive keys
    int64_t nruns = 0;
    DevBuf d_eruns;             // [n][4] first tile row, first row, rows: runs of consecutive rows inside a tile
    DevBuf d_tinfo2;            // [ntiles][4] first operand run, operand runs
    DevBuf d_meta;              // [neq] int4 per tile row: entry range, source slot, history position, row (pipelined tiles)
    int max_rows = 0;           // rows of the largest tile
    int64_t val_version = -1;   // value version d_val was built from
    size_t val_elem = 0;
};

}  // namespace hrn

struct hrn_ctx {
    int device = 0;
    int precision = HRN_FP64;
    std::string err;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t side_stream = nullptr;       // the adjoint's gradient launches, beside the stages
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;

    // ---- operator: one CSR per row holding the C, K and G entries in that order;
    // the top 2 bits of each column index name the matrix (0 = C, 1 = K, 2 = G).
    int neq = 0;
    int64_t nnz = 0;
    int64_t nnz_w[3] = {0, 0, 0};
    bool have_operator = false;    // values present
    bool have_pattern = false;
    std::vector<int32_t> h_rowptr;            // host copy of the combined pattern
    std::vector<uint32_t> h_colx;
    hrn::DevBuf d_rowptr, d_colx, d_rowidx;   // forward pattern (+ row of each entry)
    hrn::DevBuf d_rowptrT, d_colxT, d_permT;  // transposed pattern, perm into forward entries
    hrn::DevBuf d_seg, d_segT;                // [neq] int2: first K and first G entry of each row
    int lanes_f = 0, lanes_a = 0;             // stage-kernel variant, lanes*10+mat (0 = tune on first use)
    hrn::DevBuf d_tiles, d_tilesT;            // row boundaries of the tiles of the tiled stage kernel
    int ntiles = 0, ntilesT = 0;
    int num_sms = 148;
    hrn::DevBuf d_step_err;                   // device flag: a bounded wait of a stage kernel timed out
    hrn::DevBuf d_raw;                        // unscaled values (FP64)
    hrn::DevBuf d_fwd, d_adj;                 // scaled forward values, transposed adjoint values (T)
    int64_t val_version = 0;                  // incremented whenever d_fwd / d_adj are rewritten
    hrn::GtSet gt[2];                         // staged-gather row tiles: forward, adjoint
    hrn::DevBuf d_diag_m, d_im;               // FP64 mass diagonal and its reciprocal

    // ---- mesh (device assembly and gradient)
    bool have_mesh = false;
    int nj = 0, nel = 0, nel_rd = 0;
    std::vector<double> h_xyz, h_rho, h_pml;
    std::vector<int32_t> h_inod, h_mtel, h_id;
    hrn::DevBuf d_xyz, d_inod, d_id, d_rho, d_pml;
    hrn::DevBuf d_rd_elems;       // [nel_rd] element ids of the regular domain
    hrn::DevBuf d_rd_geom;        // [nel_rd][27][10] DJI (9) and w*detJ per GLL point (FP64)
    hrn::DevBuf d_rd_store;       // [nel_rd][27] history node index (store index / 3)
    bool have_rd_store = false;
    hrn::DevBuf d_gslot;          // [2][nel_rd][27] gradient of each element point, summed over steps (FP64)
    hrn::DevBuf d_gnode_ptr, d_gnode_slot;   // [nj + 1], [nel_rd * 27]: the slots of every node, ascending
    // device assembly
    hrn::DevBuf d_asm_geom;       // [nel][27][10] for all elements
    hrn::DevBuf d_el_color_list;  // elements sorted by colour
    std::vector<int> color_off;   // [ncolor + 1]
    hrn::DevBuf d_lam, d_mu;      // nodal material (FP64)
    hrn::DevBuf d_touched;        // pattern discovery flags
    hrn::DevBuf d_asm_err;        // device error flag of the assembly kernels
    hrn::DevBuf d_face_b;         // [neq] face-traction force vector B (FP64)
    bool have_face_b = false;
    // matrix-free element operator (variants 90 and 91 of the stage kernels)
    bool op_from_mesh = false;    // the operator was assembled from the current mesh and material
    bool mf_only = false;         // assemble DIAG_M only: the operator is applied matrix-free (no CSR)
    bool have_elem = false;       // element lists, node slot lists and the row map are built
    int nel_pml_e = 0, nel_rd_e = 0;
    hrn::DevBuf d_el_order;       // element ids in processing order: PML, then regular domain
    hrn::DevBuf d_el_eq;          // [P][27][9] equations of each point's DOF (-1 fixed)
    hrn::DevBuf d_el_node;        // [P][27] node of each point
    hrn::DevBuf d_el_geom;        // [P][27][10] DJI and w*detJ (FP64)
    hrn::DevBuf d_el_rho;         // [P] density
    hrn::DevBuf d_nslot_ptr, d_nslot; // [nj + 1], per node: processing index * 27 + point (top bit: RD element)
    hrn::DevBuf d_row_info;       // [neq] node << 4 | DOF
    hrn::DevBuf d_pmlw;           // [nj][12] PML direction weights of kinds e, p, w and b, c, d (FP64)
    hrn::DevBuf d_eslots;         // [P * 27][9][S] element contributions (T)
    hrn::DevBuf d_eacc;           // [neq][S] row accumulator of the atomic variant (T), kept zero between stages

    // ---- history
    int nstore = 0;
    std::vector<int32_t> h_store_eq;
    hrn::DevBuf d_store_eq, d_store_pos;      // [nstore], [neq] (-1 = not stored)
    hrn::DevBuf d_store_iota;                 // [nstore] 0 .. nstore-1 (pseudo-Hessian)

    // ---- shots
    int nshot = 0, nstep = 0;
    double dt = 0.0;
    int nslot_f = 0;
    hrn::DevBuf d_slot_f;         // [neq] forward source slot of each row (-1 none)
    hrn::DevBuf d_fslot_eq;       // [nslot_f] equation of each source slot
    hrn::DevBuf d_fsrc_b;         // [nslot_f][S] unscaled B values (FP64)
    hrn::DevBuf d_ftab;           // [S][nstep+1][3] TIME_FUNCTION samples (FP64)
    hrn::DevBuf d_srcv_f;         // [nstep+1][4][nslot_f][S] stage source values (T)
    std::vector<int32_t> h_src_eq;
    std::vector<double> h_src_b, h_ftab;

    // ---- receivers
    int nrec3 = 0, nslot_a = 0;
    std::vector<int32_t> h_eqdis, h_eqdis_map;
    hrn::DevBuf d_slot_a;         // [neq] receiver slot of each row (-1 none)
    hrn::DevBuf d_aslot_ptr, d_aslot_q, d_aslot_eq;   // receiver lists per slot (CSR) and slot equation
    hrn::DevBuf d_eqdis_map;
    hrn::DevBuf d_srcv_a;         // [4][nslot_a][S]
    hrn::DevBuf d_dis;            // [nshot][nrec3][nstep+1] FP64
    // uneven shots: per-shot record length and receiver selection (empty = all shots
    // nstep long with every receiver)
    std::vector<int32_t> h_shot_nstep;
    std::vector<uint8_t> h_rec_mask;
    hrn::DevBuf d_shot_nstep;     // [nshot] int32, or unset
    hrn::DevBuf d_rec_mask;       // [nshot][nrec3] uint8, or unset
    hrn::DevBuf d_mis_terms;      // [nshot][nstep+1] FP64
    hrn::DevBuf d_cost;           // [1 + nshot] FP64

    // ---- checkpointing of the forward wavefield (0: keep the whole history)
    int ckpt = 0;                 // steps between stored forward states
    hrn::DevBuf d_ckpt;           // [nstep / ckpt + 1][3][neq][S] forward state at steps 0, ckpt, 2 ckpt, ...
    hrn::DevBuf d_ckseg;          // [ckpt][nstore][S] history of the segment being recomputed
    hrn::DevBuf d_traces;         // [nstep+1][nrec3][S] receiver displacements of every step
    hrn::DevBuf d_Xr;             // [2][3][neq][S] state of the recomputed forward
    hrn::DevBuf d_eqdis, d_iota;  // [nrec3] receiver equations; 0 .. nrec3-1

    // ---- state and histories
    hrn::DevBuf d_X;              // [2][3][neq][S]
    hrn::DevBuf d_KB;             // [3][neq][S]
    hrn::DevBuf d_MB;             // [2][3][neq][S] materialized stage inputs
    hrn::DevBuf d_hist;           // [nstep+1][nstore][S]
    hrn::DevBuf d_phist;          // adjoint history (optional)
    bool have_forward = false;
    bool have_phist = false;
    hrn::DevBuf d_g;              // [2][nj] FP64 gradient accumulators (lambda, mu)
    bool have_data = false;       // measured data resident on the device

    // ---- inversion (model update)
    hrn::DevBuf d_red;            // reduction partials
    hrn::DevBuf d_tv_part;        // per-block partial sums of the TV regularization
    int lbfgs_m = 0;
    hrn::DevBuf d_lbfgs;          // [4][M][nj] Ys_l, Ys_m, Ss_l, Ss_m, then 6 scratch vectors [nj]
    hrn::DevBuf d_restrict;       // [nj] restriction to the regular domain (1 / 0)
    std::vector<double> lbfgs_rho, lbfgs_alpha;

    // ---- CUDA graphs of the time loops (on unless disabled or timing per launch)
    bool graphs = true;
    uint64_t epoch = 1;            // incremented by every setting change
    hrn::LoopGraph gfwd, gadj;
    int64_t graph_captures = 0, graph_replays = 0;

    // ---- timing
    int64_t launches = 0;          // kernels launched by this context (cumulative)
    bool timing = false;
    double last_total_ms = 0.0, last_stage_ms = 0.0;
    int64_t last_stage_launches = 0;
    double acc_stage_ms = 0.0;      // summed since timing was last enabled
    int64_t acc_stage_launches = 0;
    std::vector<cudaEvent_t> ev_pool;

    size_t elem_bytes() const { return precision == HRN_FP64 ? 8 : 4; }
};

// Kernel launchers implemented in the .cu files.
namespace hrn {
// Where the receiver displacements of every step live: the forward history
// (rows = history positions) or, with checkpointing, the trace buffer (rows =
// receivers).  Row q of step n: hist + (n * stride + map[q]) * S.
struct RecView {
    const void *hist;
    int stride;
    const int32_t *map;
};
inline RecView rec_view(const hrn_ctx *c)
{
    if (c->ckpt > 0) return RecView{c->d_traces.p, c->nrec3, c->d_iota.as<int32_t>()};
    return RecView{c->d_hist.p, c->nstore, c->d_eqdis_map.as<int32_t>()};
}
// Per-shot record lengths and receiver masks on the device, or null when the
// batch is even.
inline const int32_t *shot_nstep_ptr(const hrn_ctx *c)
{
    return c->h_shot_nstep.empty() ? nullptr : c->d_shot_nstep.as<int32_t>();
}
inline const uint8_t *rec_mask_ptr(const hrn_ctx *c)
{
    return c->h_rec_mask.empty() ? nullptr : c->d_rec_mask.as<uint8_t>();
}
int launch_scale_operator(hrn_ctx *c);
int run_apply_operator(hrn_ctx *c, int which, int adj, const double *d_x, double *d_y);
int run_forward(hrn_ctx *c);
int run_adjoint_gradient(hrn_ctx *c, int lambda_2mu, int keep_p);
int run_misfit(hrn_ctx *c, double *cost);
int run_time_stage(hrn_ctx *c, int adj, int nsteps, double *avg_ms);
int run_pseudo_hessian(hrn_ctx *c, double *hl, double *hm);
int build_rd_geometry(hrn_ctx *c);
int assemble_device(hrn_ctx *c, bool discover_pattern);
int face_force(hrn_ctx *c, const int32_t *nface);
int finalize_pattern_from_keys(hrn_ctx *c, const std::vector<uint64_t> &keys);
int vec_reduce(hrn_ctx *c, int kind, int n, const double *x, const double *y, double *out);
int gt_ready(hrn_ctx *c, int adj);
int gtp_prepare(hrn_ctx *c, int adj);
int gt_stage(hrn_ctx *c, const void *stage_args, int stage, int adj, int variant);
inline bool is_gt_variant(int v) { return v == 44 || v == 45 || v == 84 || v == 85 || v == 46 || v == 86 || v == 47 || v == 87; }
// pipelined staged tiles: persistent CTAs, producer warp, per-call row metadata
inline bool is_gtp_variant(int v) { return v == 47 || v == 87; }
// staged-gather variants whose records move by bulk copies: records of a multiple of 16 bytes
inline bool gt_runs_valid(int v, int nshot, size_t elem) { return (v != 46 && v != 86 && v != 47 && v != 87) || (size_t(nshot) * elem) % 16 == 0; }
int elem_prepare(hrn_ctx *c);
int elem_ready(hrn_ctx *c);
int elem_stage(hrn_ctx *c, const void *stage_args, int stage, int adj, int acc, int shots_per_thread, int mat);
bool elem_variant_valid(const hrn_ctx *c, int variant);
int vec_axpby(hrn_ctx *c, int n, double a, const double *x, double b, const double *y, double *z);
int set_error(hrn_ctx *c, int code, const std::string &msg);
int cuda_error(hrn_ctx *c, cudaError_t e, const char *what);
}  // namespace hrn

#define HRN_CUDA(ctx, call)                                           \
    do {                                                              \
        cudaError_t _e = (call);                                      \
        if (_e != cudaSuccess) return hrn::cuda_error((ctx), _e, #call); \
    } while (0)
