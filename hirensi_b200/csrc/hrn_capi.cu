// hrn_capi.cu -- extern "C" entry points of libhirensi_b200.so (see
// include/hirensi_b200.h): argument checking, pattern set-up and buffer
// management around the kernels of hrn_step.cu and hrn_assemble.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "hrn_internal.h"

namespace hrn {

int set_error(hrn_ctx *c, int code, const std::string &msg)
{
    if (c) c->err = msg;
    return code;
}

int cuda_error(hrn_ctx *c, cudaError_t e, const char *what)
{
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) return set_error(c, HRN_EOOM, m);
    return set_error(c, HRN_ECUDA, m);
}

// Install a combined forward pattern (row i: C, then K, then G entries, each
// sorted by column; matrix id in the top bits of the column) and its transpose
// (row j: per matrix in the same order, the rows i with a_ij stored).
static int install_pattern(hrn_ctx *c, int32_t neq, std::vector<int32_t> &rowptr, std::vector<uint32_t> &colx)
{
    const int64_t nnz = rowptr[neq];
    std::vector<int32_t> rowidx(static_cast<size_t>(nnz));
    c->nnz_w[0] = c->nnz_w[1] = c->nnz_w[2] = 0;
    for (int32_t i = 0; i < neq; ++i)
        for (int32_t p = rowptr[i]; p < rowptr[i + 1]; ++p) {
            rowidx[p] = i;
            c->nnz_w[colx[p] >> kTagBits]++;
        }
    std::vector<int32_t> rowptrT(static_cast<size_t>(neq) + 1, 0);
    for (int64_t p = 0; p < nnz; ++p) rowptrT[(colx[p] & kColMask) + 1]++;
    for (int32_t j = 0; j < neq; ++j) rowptrT[j + 1] += rowptrT[j];
    std::vector<int32_t> pos(rowptrT.begin(), rowptrT.end() - 1);
    std::vector<uint32_t> colxT(static_cast<size_t>(nnz));
    std::vector<int64_t> permT(static_cast<size_t>(nnz));
    for (uint32_t w = 0; w < 3; ++w)
        for (int32_t i = 0; i < neq; ++i)
            for (int32_t p = rowptr[i]; p < rowptr[i + 1]; ++p) {
                if ((colx[p] >> kTagBits) != w) continue;
                const int32_t j = int32_t(colx[p] & kColMask);
                const int32_t t = pos[j]++;
                colxT[t] = uint32_t(i) | (w << kTagBits);
                permT[t] = p;
            }
    // segment starts (first K entry, first G entry) of every forward and transposed row
    std::vector<int32_t> seg(2 * static_cast<size_t>(neq)), segT(2 * static_cast<size_t>(neq));
    for (int32_t i = 0; i < neq; ++i) {
        int32_t p = rowptr[i];
        while (p < rowptr[i + 1] && (colx[p] >> kTagBits) < 1u) ++p;
        seg[2 * i] = p;
        while (p < rowptr[i + 1] && (colx[p] >> kTagBits) < 2u) ++p;
        seg[2 * i + 1] = p;
        p = rowptrT[i];
        while (p < rowptrT[i + 1] && (colxT[p] >> kTagBits) < 1u) ++p;
        segT[2 * i] = p;
        while (p < rowptrT[i + 1] && (colxT[p] >> kTagBits) < 2u) ++p;
        segT[2 * i + 1] = p;
    }
    // tiles of consecutive rows with at most kTileEntries entries (tiled stage kernel)
    auto make_tiles = [&](const std::vector<int32_t> &rp, std::vector<int32_t> &tl) -> bool {
        tl.assign(1, 0);
        for (int32_t i = 0; i < neq; ++i) {
            if (rp[i + 1] - rp[i] > kTileEntries) return false;
            if (rp[i + 1] - rp[tl.back()] > kTileEntries) tl.push_back(i);
        }
        tl.push_back(neq);
        return true;
    };
    std::vector<int32_t> tiles, tilesT;
    if (!make_tiles(rowptr, tiles) || !make_tiles(rowptrT, tilesT))
        return set_error(c, HRN_EARG, "a row has more stored entries than a tile holds");
    HRN_CUDA(c, c->d_tiles.alloc(tiles.size() * 4));
    HRN_CUDA(c, c->d_tilesT.alloc(tilesT.size() * 4));
    HRN_CUDA(c, cudaMemcpy(c->d_tiles.p, tiles.data(), tiles.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_tilesT.p, tilesT.data(), tilesT.size() * 4, cudaMemcpyHostToDevice));
    c->ntiles = int(tiles.size()) - 1;
    c->ntilesT = int(tilesT.size()) - 1;
    c->neq = neq;
    c->nnz = nnz;
    c->lanes_f = c->lanes_a = 0;
    HRN_CUDA(c, c->d_seg.alloc(seg.size() * 4));
    HRN_CUDA(c, c->d_segT.alloc(segT.size() * 4));
    HRN_CUDA(c, cudaMemcpy(c->d_seg.p, seg.data(), seg.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_segT.p, segT.data(), segT.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, c->d_rowptr.alloc(rowptr.size() * 4));
    HRN_CUDA(c, c->d_colx.alloc(colx.size() * 4 + kBulkPad));
    HRN_CUDA(c, c->d_rowidx.alloc(std::max<size_t>(rowidx.size(), 1) * 4));
    HRN_CUDA(c, c->d_rowptrT.alloc(rowptrT.size() * 4));
    HRN_CUDA(c, c->d_colxT.alloc(colxT.size() * 4 + kBulkPad));
    HRN_CUDA(c, c->d_permT.alloc(std::max<size_t>(permT.size(), 1) * 8));
    HRN_CUDA(c, c->d_raw.alloc(std::max<size_t>(size_t(nnz), 1) * 8));
    HRN_CUDA(c, cudaMemcpy(c->d_rowptr.p, rowptr.data(), rowptr.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_colx.p, colx.data(), colx.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_rowidx.p, rowidx.data(), rowidx.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_rowptrT.p, rowptrT.data(), rowptrT.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_colxT.p, colxT.data(), colxT.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_permT.p, permT.data(), permT.size() * 8, cudaMemcpyHostToDevice));
    c->h_rowptr.swap(rowptr);
    c->h_colx.swap(colx);
    c->have_pattern = true;
    c->gt[0].built = c->gt[1].built = false;
    return 0;
}

// Pattern from three caller CSRs.
static int build_pattern(hrn_ctx *c, int32_t neq, const int32_t *ia[3], const int32_t *ja[3])
{
    int64_t nnz = 0;
    for (int w = 0; w < 3; ++w) {
        if (ia[w][0] != 0) return set_error(c, HRN_EARG, "CSR row pointer must start at 0");
        for (int32_t i = 0; i < neq; ++i)
            if (ia[w][i + 1] < ia[w][i]) return set_error(c, HRN_EARG, "CSR row pointer must be non-decreasing");
        nnz += ia[w][neq];
        for (int64_t k = 0; k < ia[w][neq]; ++k)
            if (ja[w][k] < 0 || ja[w][k] >= neq) return set_error(c, HRN_EARG, "CSR column index out of range");
        for (int32_t i = 0; i < neq; ++i)
            for (int32_t p = ia[w][i] + 1; p < ia[w][i + 1]; ++p)
                if (ja[w][p] <= ja[w][p - 1]) return set_error(c, HRN_EARG, "CSR columns must be sorted and unique within a row");
    }
    if (nnz >= (int64_t(1) << 31)) return set_error(c, HRN_EARG, "more than 2^31 stored entries");
    std::vector<int32_t> rowptr(static_cast<size_t>(neq) + 1);
    std::vector<uint32_t> colx(static_cast<size_t>(nnz));
    int64_t k = 0;
    rowptr[0] = 0;
    for (int32_t i = 0; i < neq; ++i) {
        for (int w = 0; w < 3; ++w)
            for (int32_t p = ia[w][i]; p < ia[w][i + 1]; ++p) colx[k++] = uint32_t(ja[w][p]) | (uint32_t(w) << kTagBits);
        rowptr[i + 1] = int32_t(k);
    }
    return install_pattern(c, neq, rowptr, colx);
}

}  // namespace hrn

// Pattern from sorted unique keys (row << 32 | matrix << 30 | column), device assembly.
int hrn::finalize_pattern_from_keys(hrn_ctx *c, const std::vector<uint64_t> &keys)
{
    if (keys.size() >= (size_t(1) << 31)) return set_error(c, HRN_EARG, "more than 2^31 stored entries");
    std::vector<int32_t> rowptr(static_cast<size_t>(c->neq) + 1, 0);
    std::vector<uint32_t> colx(keys.size());
    for (size_t k = 0; k < keys.size(); ++k) {
        rowptr[(keys[k] >> 32) + 1]++;
        colx[k] = uint32_t(keys[k] & 0xffffffffu);
    }
    for (int32_t i = 0; i < c->neq; ++i) rowptr[i + 1] += rowptr[i];
    return install_pattern(c, c->neq, rowptr, colx);
}

namespace hrn {

static int set_mass(hrn_ctx *c, const double *diag_m, bool device_src)
{
    HRN_CUDA(c, c->d_diag_m.alloc(size_t(c->neq) * 8));
    HRN_CUDA(c, c->d_im.alloc(size_t(c->neq) * 8));
    std::vector<double> im(size_t(c->neq));
    std::vector<double> dm(size_t(c->neq));
    if (device_src) HRN_CUDA(c, cudaMemcpy(dm.data(), diag_m, dm.size() * 8, cudaMemcpyDeviceToHost));
    else std::memcpy(dm.data(), diag_m, dm.size() * 8);
    for (int i = 0; i < c->neq; ++i) {
        if (!std::isfinite(dm[i])) return set_error(c, HRN_ENAN, "non-finite mass diagonal");
        im[i] = dm[i] != 0.0 ? 1.0 / dm[i] : 0.0;   // VecReciprocal leaves zeros alone
    }
    HRN_CUDA(c, cudaMemcpy(c->d_diag_m.p, dm.data(), dm.size() * 8, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_im.p, im.data(), im.size() * 8, cudaMemcpyHostToDevice));
    return 0;
}

// Per-row slot map for the history.
static int upload_store_pos(hrn_ctx *c)
{
    if (c->neq == 0 || c->nstore == 0) return 0;
    std::vector<int32_t> sp(size_t(c->neq), -1);
    for (int p = 0; p < c->nstore; ++p) {
        const int32_t e = c->h_store_eq[p];
        if (e < 0 || e >= c->neq) return set_error(c, HRN_EARG, "history equation out of range");
        if (sp[e] >= 0) return set_error(c, HRN_EARG, "history equation listed twice");
        sp[e] = p;
    }
    HRN_CUDA(c, c->d_store_pos.alloc(sp.size() * 4));
    HRN_CUDA(c, cudaMemcpy(c->d_store_pos.p, sp.data(), sp.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, c->d_store_eq.alloc(size_t(c->nstore) * 4));
    HRN_CUDA(c, cudaMemcpy(c->d_store_eq.p, c->h_store_eq.data(), size_t(c->nstore) * 4, cudaMemcpyHostToDevice));
    return 0;
}

static int upload_sources(hrn_ctx *c)
{
    if (c->neq == 0 || c->nshot == 0) return 0;
    const int S = c->nshot;
    std::map<int32_t, int> slot_of;
    for (int32_t e : c->h_src_eq) {
        if (e < 0 || e >= c->neq) return set_error(c, HRN_EARG, "source equation out of range");
        slot_of.emplace(e, 0);
    }
    int k = 0;
    std::vector<int32_t> slot_eq;
    for (auto &kv : slot_of) { kv.second = k++; slot_eq.push_back(kv.first); }
    c->nslot_f = k;
    std::vector<double> b(size_t(k) * S, 0.0);
    for (size_t r = 0; r < c->h_src_eq.size(); ++r)
        for (int s = 0; s < S; ++s) b[size_t(slot_of[c->h_src_eq[r]]) * S + s] += c->h_src_b[r * S + s];
    std::vector<int32_t> slot(size_t(c->neq), -1);
    for (int i = 0; i < k; ++i) slot[slot_eq[i]] = i;
    HRN_CUDA(c, c->d_slot_f.alloc(slot.size() * 4));
    HRN_CUDA(c, cudaMemcpy(c->d_slot_f.p, slot.data(), slot.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, c->d_fslot_eq.alloc(std::max(k, 1) * 4));
    HRN_CUDA(c, c->d_fsrc_b.alloc(std::max<size_t>(b.size(), 1) * 8));
    HRN_CUDA(c, c->d_ftab.alloc(c->h_ftab.size() * 8));
    HRN_CUDA(c, c->d_srcv_f.alloc(std::max<size_t>(size_t(c->nstep + 1) * 4 * k * S, 1) * c->elem_bytes()));
    if (k) {
        HRN_CUDA(c, cudaMemcpy(c->d_fslot_eq.p, slot_eq.data(), size_t(k) * 4, cudaMemcpyHostToDevice));
        HRN_CUDA(c, cudaMemcpy(c->d_fsrc_b.p, b.data(), b.size() * 8, cudaMemcpyHostToDevice));
    }
    HRN_CUDA(c, cudaMemcpy(c->d_ftab.p, c->h_ftab.data(), c->h_ftab.size() * 8, cudaMemcpyHostToDevice));
    return 0;
}

static int upload_receivers(hrn_ctx *c)
{
    if (c->neq == 0 || c->nshot == 0 || c->nrec3 == 0) {
        c->nslot_a = 0;
        if (c->neq) {
            std::vector<int32_t> slot(size_t(c->neq), -1);
            HRN_CUDA(c, c->d_slot_a.alloc(slot.size() * 4));
            HRN_CUDA(c, cudaMemcpy(c->d_slot_a.p, slot.data(), slot.size() * 4, cudaMemcpyHostToDevice));
        }
        return 0;
    }
    std::map<int32_t, std::vector<int32_t>> lists;
    for (int q = 0; q < c->nrec3; ++q) {
        const int32_t e = c->h_eqdis[q];
        if (e < 0 || e >= c->neq) return set_error(c, HRN_EARG, "receiver equation out of range");
        if (c->h_eqdis_map[q] < 0 || c->h_eqdis_map[q] >= c->nstore) return set_error(c, HRN_EARG, "receiver history position out of range");
        lists[e].push_back(q);
    }
    std::vector<int32_t> ptr(1, 0), ql, seq;
    std::vector<int32_t> slot(size_t(c->neq), -1);
    for (auto &kv : lists) {
        slot[kv.first] = int32_t(seq.size());
        seq.push_back(kv.first);
        for (int32_t q : kv.second) ql.push_back(q);
        ptr.push_back(int32_t(ql.size()));
    }
    c->nslot_a = int(seq.size());
    const int S = c->nshot;
    HRN_CUDA(c, c->d_slot_a.alloc(slot.size() * 4));
    HRN_CUDA(c, c->d_aslot_ptr.alloc(ptr.size() * 4));
    HRN_CUDA(c, c->d_aslot_q.alloc(ql.size() * 4));
    HRN_CUDA(c, c->d_aslot_eq.alloc(seq.size() * 4));
    HRN_CUDA(c, c->d_eqdis_map.alloc(size_t(c->nrec3) * 4));
    HRN_CUDA(c, c->d_srcv_a.alloc(size_t(4) * c->nslot_a * S * c->elem_bytes()));
    HRN_CUDA(c, cudaMemcpy(c->d_slot_a.p, slot.data(), slot.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_aslot_ptr.p, ptr.data(), ptr.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_aslot_q.p, ql.data(), ql.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_aslot_eq.p, seq.data(), seq.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_eqdis_map.p, c->h_eqdis_map.data(), size_t(c->nrec3) * 4, cudaMemcpyHostToDevice));
    std::vector<int32_t> iota(size_t(c->nrec3));
    for (int q = 0; q < c->nrec3; ++q) iota[q] = q;
    HRN_CUDA(c, c->d_eqdis.alloc(size_t(c->nrec3) * 4));
    HRN_CUDA(c, c->d_iota.alloc(size_t(c->nrec3) * 4));
    HRN_CUDA(c, cudaMemcpy(c->d_eqdis.p, c->h_eqdis.data(), size_t(c->nrec3) * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_iota.p, iota.data(), size_t(c->nrec3) * 4, cudaMemcpyHostToDevice));
    return 0;
}

static int ensure_state(hrn_ctx *c)
{
    const size_t S = size_t(c->nshot), eb = c->elem_bytes();
    HRN_CUDA(c, c->d_X.alloc(2 * 3 * size_t(c->neq) * S * eb));
    HRN_CUDA(c, c->d_KB.alloc(3 * size_t(c->neq) * S * eb));
    HRN_CUDA(c, c->d_MB.alloc(2 * 3 * size_t(c->neq) * S * eb));
    if (c->ckpt > 0) {
        // forward states every ckpt steps, one segment of history, all receiver traces
        c->d_hist.release();
        const size_t nck = size_t(c->nstep / c->ckpt) + 1;
        HRN_CUDA(c, c->d_ckpt.alloc(nck * 3 * size_t(c->neq) * S * eb));
        HRN_CUDA(c, c->d_ckseg.alloc(std::max<size_t>(size_t(c->ckpt) * c->nstore * S * eb, 1)));
        HRN_CUDA(c, c->d_traces.alloc(std::max<size_t>(size_t(c->nstep + 1) * c->nrec3 * S * eb, 1)));
        HRN_CUDA(c, c->d_Xr.alloc(2 * 3 * size_t(c->neq) * S * eb));
    } else {
        c->d_ckpt.release();
        c->d_ckseg.release();
        c->d_traces.release();
        c->d_Xr.release();
        HRN_CUDA(c, c->d_hist.alloc(std::max<size_t>(size_t(c->nstep + 1) * c->nstore * S * eb, 1)));
    }
    return 0;
}

static int check_ready(hrn_ctx *c, bool need_mesh)
{
    if (!c->have_operator) return set_error(c, HRN_ESTATE, "no operator: call hrn_set_operator_csr or hrn_assemble first");
    if (c->nshot == 0) return set_error(c, HRN_ESTATE, "no shots: call hrn_set_shots first");
    if (c->nstore == 0) return set_error(c, HRN_ESTATE, "no history equations: call hrn_set_history first");
    if (need_mesh && !c->have_mesh) return set_error(c, HRN_ESTATE, "no mesh: call hrn_set_mesh first");
    return 0;
}

// (Re)bind everything that depends on neq once an operator exists.
static int rebind(hrn_ctx *c)
{
    if (int rc = upload_store_pos(c)) return rc;
    if (int rc = upload_sources(c)) return rc;
    if (int rc = upload_receivers(c)) return rc;
    return 0;
}

}  // namespace hrn

using namespace hrn;

extern "C" {

int hrn_version(void) { return 100; }

int hrn_create(int device, int precision, hrn_ctx **out)
{
    if (!out) return HRN_EARG;
    *out = nullptr;
    if (precision != HRN_FP64 && precision != HRN_FP32) return HRN_EARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return HRN_ECUDA; }
    if (device < 0 || device >= ndev) return HRN_EARG;
    hrn_ctx *c = new (std::nothrow) hrn_ctx();
    if (!c) return HRN_EOOM;
    c->device = device;
    c->precision = precision;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return HRN_ECUDA;
    }
    c->stream = c->own_stream;
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (c->d_step_err.alloc(16) != cudaSuccess || cudaMemset(c->d_step_err.p, 0, 16) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return HRN_EOOM;
    }
    *out = c;
    return HRN_OK;
}

int hrn_destroy(hrn_ctx *c)
{
    if (!c) return HRN_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
    if (c->side_stream) {
        cudaStreamSynchronize(c->side_stream);
        cudaStreamDestroy(c->side_stream);
        cudaEventDestroy(c->ev_fork);
        cudaEventDestroy(c->ev_join);
    }
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return HRN_OK;
}

const char *hrn_last_error(const hrn_ctx *c) { return c ? c->err.c_str() : "null context"; }

int hrn_set_stream(hrn_ctx *c, void *stream)
{
    if (!c) return HRN_EARG;
    ++c->epoch;
    c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own_stream;
    return HRN_OK;
}

int hrn_set_graphs(hrn_ctx *c, int32_t enable)
{
    if (!c) return HRN_EARG;
    c->graphs = enable != 0;
    if (!c->graphs) {
        cudaSetDevice(c->device);
        c->gfwd.reset();
        c->gadj.reset();
    }
    return HRN_OK;
}

int hrn_graph_stats(hrn_ctx *c, int64_t *captures, int64_t *replays)
{
    if (!c) return HRN_EARG;
    if (captures) *captures = c->graph_captures;
    if (replays) *replays = c->graph_replays;
    return HRN_OK;
}

int hrn_set_timing(hrn_ctx *c, int32_t enable)
{
    if (!c) return HRN_EARG;
    c->timing = enable != 0;
    if (c->timing) {
        c->acc_stage_ms = 0.0;
        c->acc_stage_launches = 0;
    }
    return HRN_OK;
}

int hrn_last_timing(hrn_ctx *c, double *total_ms, double *stage_kernel_ms, int64_t *stage_launches)
{
    if (!c) return HRN_EARG;
    if (total_ms) *total_ms = c->last_total_ms;
    if (stage_kernel_ms) *stage_kernel_ms = c->acc_stage_ms;
    if (stage_launches) *stage_launches = c->acc_stage_launches;
    return HRN_OK;
}

int hrn_set_operator_csr(hrn_ctx *c, int32_t neq, const int32_t *c_ia, const int32_t *c_ja, const double *c_a,
                         const int32_t *k_ia, const int32_t *k_ja, const double *k_a, const int32_t *g_ia,
                         const int32_t *g_ja, const double *g_a, const double *diag_m)
{
    if (!c) return HRN_EARG;
    ++c->epoch;
    if (c->mf_only) return set_error(c, HRN_ESTATE, "the context is in matrix-free operator mode");
    if (neq <= 0 || !c_ia || !k_ia || !g_ia || !diag_m) return set_error(c, HRN_EARG, "bad operator arguments");
    if (c->have_mesh && neq != c->neq) return set_error(c, HRN_EARG, "neq differs from the mesh");
    cudaSetDevice(c->device);
    const int32_t *ia[3] = {c_ia, k_ia, g_ia}, *ja[3] = {c_ja, k_ja, g_ja};
    const double *aa[3] = {c_a, k_a, g_a};
    if (int rc = build_pattern(c, neq, ia, ja)) return rc;
    std::vector<double> raw(size_t(std::max<int64_t>(c->nnz, 1)));
    int64_t k = 0;
    for (int32_t i = 0; i < neq; ++i)
        for (int w = 0; w < 3; ++w)
            for (int32_t p = ia[w][i]; p < ia[w][i + 1]; ++p) {
                if (!std::isfinite(aa[w][p])) return set_error(c, HRN_ENAN, "non-finite operator value");
                raw[k++] = aa[w][p];
            }
    HRN_CUDA(c, cudaMemcpy(c->d_raw.p, raw.data(), size_t(c->nnz) * 8, cudaMemcpyHostToDevice));
    if (int rc = set_mass(c, diag_m, false)) return rc;
    if (int rc = launch_scale_operator(c)) return rc;
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    c->have_operator = true;
    c->op_from_mesh = false;
    if (c->lanes_f >= 90 && c->lanes_f <= 105) c->lanes_f = 0;   // matrix-free needs an assembled operator: tune again
    if (c->lanes_a >= 90 && c->lanes_a <= 105) c->lanes_a = 0;
    c->have_forward = false;
    return rebind(c);
}

int hrn_set_mesh(hrn_ctx *c, int32_t nj, int32_t nel, int32_t neq, const double *xyz, const int32_t *inod,
                 const int32_t *mtel, const int32_t *id, const double *rho_el, const double *pml_param)
{
    if (!c) return HRN_EARG;
    ++c->epoch;
    if (nj <= 0 || nel <= 0 || neq <= 0 || !xyz || !inod || !mtel || !id || !rho_el || !pml_param)
        return set_error(c, HRN_EARG, "bad mesh arguments");
    if ((c->have_pattern || (c->mf_only && c->have_operator)) && neq != c->neq)
        return set_error(c, HRN_EARG, "neq differs from the operator");
    for (int64_t k = 0; k < int64_t(nel) * 27; ++k)
        if (inod[k] < 0 || inod[k] >= nj) return set_error(c, HRN_EARG, "INOD entry out of range");
    for (int64_t k = 0; k < int64_t(nj) * 9; ++k)
        if (id[k] < -1 || id[k] >= neq) return set_error(c, HRN_EARG, "ID entry out of range");
    for (int e = 0; e < nel; ++e)
        if (mtel[e] != 1 && mtel[e] != 2) return set_error(c, HRN_EARG, "MTEL must be 1 (RD) or 2 (PML)");
    cudaSetDevice(c->device);
    c->have_elem = false;
    c->op_from_mesh = false;
    c->nj = nj;
    c->nel = nel;
    c->neq = neq;
    c->h_xyz.assign(xyz, xyz + size_t(nj) * 3);
    c->h_inod.assign(inod, inod + size_t(nel) * 27);
    c->h_mtel.assign(mtel, mtel + nel);
    c->h_id.assign(id, id + size_t(nj) * 9);
    c->h_rho.assign(rho_el, rho_el + nel);
    c->h_pml.assign(pml_param, pml_param + 24);
    HRN_CUDA(c, c->d_xyz.alloc(c->h_xyz.size() * 8));
    HRN_CUDA(c, c->d_inod.alloc(c->h_inod.size() * 4));
    HRN_CUDA(c, c->d_id.alloc(c->h_id.size() * 4));
    HRN_CUDA(c, c->d_rho.alloc(c->h_rho.size() * 8));
    HRN_CUDA(c, c->d_pml.alloc(24 * 8));
    HRN_CUDA(c, c->d_g.alloc(size_t(2) * nj * 8));
    HRN_CUDA(c, cudaMemcpy(c->d_xyz.p, c->h_xyz.data(), c->h_xyz.size() * 8, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_inod.p, c->h_inod.data(), c->h_inod.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_id.p, c->h_id.data(), c->h_id.size() * 4, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_rho.p, c->h_rho.data(), c->h_rho.size() * 8, cudaMemcpyHostToDevice));
    HRN_CUDA(c, cudaMemcpy(c->d_pml.p, c->h_pml.data(), 24 * 8, cudaMemcpyHostToDevice));
    if (int rc = build_rd_geometry(c)) return rc;
    c->have_mesh = true;
    return HRN_OK;
}

static int assemble_common(hrn_ctx *c, const double *lambda, const double *mu, bool device_src)
{
    if (!c) return HRN_EARG;
    if (!c->have_mesh) return set_error(c, HRN_ESTATE, "no mesh: call hrn_set_mesh first");
    if (!lambda || !mu) return set_error(c, HRN_EARG, "null material");
    cudaSetDevice(c->device);
    HRN_CUDA(c, c->d_lam.alloc(size_t(c->nj) * 8));
    HRN_CUDA(c, c->d_mu.alloc(size_t(c->nj) * 8));
    if (device_src) {
        HRN_CUDA(c, cudaMemcpyAsync(c->d_lam.p, lambda, size_t(c->nj) * 8, cudaMemcpyDeviceToDevice, c->stream));
        HRN_CUDA(c, cudaMemcpyAsync(c->d_mu.p, mu, size_t(c->nj) * 8, cudaMemcpyDeviceToDevice, c->stream));
    } else {
        for (int i = 0; i < c->nj; ++i)
            if (!std::isfinite(lambda[i]) || !std::isfinite(mu[i])) return set_error(c, HRN_ENAN, "non-finite material");
        HRN_CUDA(c, cudaMemcpyAsync(c->d_lam.p, lambda, size_t(c->nj) * 8, cudaMemcpyHostToDevice, c->stream));
        HRN_CUDA(c, cudaMemcpyAsync(c->d_mu.p, mu, size_t(c->nj) * 8, cudaMemcpyHostToDevice, c->stream));
    }
    const bool first = c->mf_only ? !c->have_operator : !c->have_pattern;
    if (int rc = assemble_device(c, !c->mf_only && first)) return rc;
    c->have_operator = true;
    c->op_from_mesh = true;
    c->have_forward = false;
    if (first) return rebind(c);
    return HRN_OK;
}

int hrn_set_operator_mode(hrn_ctx *c, int32_t matrix_free_only)
{
    if (!c) return HRN_EARG;
    ++c->epoch;
    if (!c->have_mesh) return set_error(c, HRN_ESTATE, "no mesh: call hrn_set_mesh first");
    const bool mf = matrix_free_only != 0;
    if (mf == c->mf_only) return HRN_OK;
    if (c->have_operator) return set_error(c, HRN_ESTATE, "choose the operator mode before the first assembly");
    c->mf_only = mf;
    return HRN_OK;
}

int hrn_assemble(hrn_ctx *c, const double *lambda, const double *mu) { return assemble_common(c, lambda, mu, false); }

int hrn_assemble_device(hrn_ctx *c, const double *d_lambda, const double *d_mu)
{
    return assemble_common(c, d_lambda, d_mu, true);
}

int hrn_get_operator_csr(hrn_ctx *c, int32_t which, int32_t *ia, int32_t *ja, double *a, int64_t *nnz)
{
    if (!c) return HRN_EARG;
    if (!c->have_operator) return set_error(c, HRN_ESTATE, "no operator");
    if (which < 0 || which > 2) return set_error(c, HRN_EARG, "which must be 0 (C), 1 (K) or 2 (G)");
    cudaSetDevice(c->device);
    if (nnz) *nnz = c->nnz_w[which];
    if (!ia && !ja && !a) return HRN_OK;
    if (c->mf_only) return set_error(c, HRN_ESTATE, "a matrix-free operator has no stored entries");
    std::vector<double> raw(size_t(std::max<int64_t>(c->nnz, 1)));
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    HRN_CUDA(c, cudaMemcpy(raw.data(), c->d_raw.p, size_t(c->nnz) * 8, cudaMemcpyDeviceToHost));
    int64_t k = 0;
    if (ia) ia[0] = 0;
    for (int32_t i = 0; i < c->neq; ++i) {
        for (int32_t p = c->h_rowptr[i]; p < c->h_rowptr[i + 1]; ++p) {
            if ((c->h_colx[p] >> kTagBits) != uint32_t(which)) continue;
            if (ja) ja[k] = int32_t(c->h_colx[p] & kColMask);
            if (a) a[k] = raw[p];
            ++k;
        }
        if (ia) ia[i + 1] = int32_t(k);
    }
    return HRN_OK;
}

int hrn_apply_operator(hrn_ctx *c, int32_t which, int32_t adjoint, const double *x, double *y)
{
    if (!c || !x || !y) return HRN_EARG;
    if (!c->have_operator) return set_error(c, HRN_ESTATE, "no operator");
    if (which < 0 || which > 2) return set_error(c, HRN_EARG, "which must be 0 (C), 1 (K) or 2 (G)");
    if (c->mf_only) return set_error(c, HRN_ESTATE, "a matrix-free operator has no stored entries");
    cudaSetDevice(c->device);
    DevBuf dx, dy;
    const size_t vb = size_t(c->neq) * 8;
    HRN_CUDA(c, dx.alloc(vb));
    HRN_CUDA(c, dy.alloc(vb));
    HRN_CUDA(c, cudaMemcpyAsync(dx.p, x, vb, cudaMemcpyHostToDevice, c->stream));
    if (int rc = run_apply_operator(c, which, adjoint != 0, dx.as<double>(), dy.as<double>())) return rc;
    HRN_CUDA(c, cudaMemcpyAsync(y, dy.p, vb, cudaMemcpyDeviceToHost, c->stream));
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    return HRN_OK;
}

int hrn_assemble_face_force(hrn_ctx *c, const int32_t *nface, double *b)
{
    if (!c || !nface) return HRN_EARG;
    if (!c->have_mesh) return set_error(c, HRN_ESTATE, "no mesh: call hrn_set_mesh first");
    cudaSetDevice(c->device);
    if (int rc = face_force(c, nface)) return rc;
    if (b) {
        HRN_CUDA(c, cudaMemcpyAsync(b, c->d_face_b.p, size_t(c->neq) * 8, cudaMemcpyDeviceToHost, c->stream));
        HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    return HRN_OK;
}

int hrn_set_shots_face_force(hrn_ctx *c, int32_t nshot, int32_t nstep, double dt, const double *ftab)
{
    if (!c || !ftab) return HRN_EARG;
    if (!c->have_face_b) return set_error(c, HRN_ESTATE, "no face force: call hrn_assemble_face_force first");
    if (nshot < 1 || nshot > HRN_MAX_SHOTS) return set_error(c, HRN_EARG, "nshot must be 1..HRN_MAX_SHOTS");
    cudaSetDevice(c->device);
    std::vector<double> bvec(size_t(c->neq));
    HRN_CUDA(c, cudaMemcpyAsync(bvec.data(), c->d_face_b.p, size_t(c->neq) * 8, cudaMemcpyDeviceToHost, c->stream));
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    // the entries of B that load the system; every shot carries the same B
    std::vector<int32_t> eq;
    std::vector<double> vals;
    for (int32_t i = 0; i < c->neq; ++i)
        if (bvec[i] != 0.0) {
            eq.push_back(i);
            for (int s = 0; s < nshot; ++s) vals.push_back(bvec[i]);
        }
    return hrn_set_shots(c, nshot, nstep, dt, int32_t(eq.size()), eq.empty() ? nullptr : eq.data(),
                         vals.empty() ? nullptr : vals.data(), ftab);
}

int hrn_get_diag_m(hrn_ctx *c, double *diag_m)
{
    if (!c || !diag_m) return HRN_EARG;
    if (!c->have_operator) return set_error(c, HRN_ESTATE, "no operator");
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    HRN_CUDA(c, cudaMemcpy(diag_m, c->d_diag_m.p, size_t(c->neq) * 8, cudaMemcpyDeviceToHost));
    return HRN_OK;
}

int hrn_set_history(hrn_ctx *c, int32_t nstore, const int32_t *store_eq)
{
    if (!c) return HRN_EARG;
    ++c->epoch;
    if (nstore <= 0 || !store_eq) return set_error(c, HRN_EARG, "bad history arguments");
    c->nstore = nstore;
    c->h_store_eq.assign(store_eq, store_eq + nstore);
    c->have_rd_store = false;
    c->have_forward = false;
    cudaSetDevice(c->device);
    return upload_store_pos(c);
}

int hrn_set_shots(hrn_ctx *c, int32_t nshot, int32_t nstep, double dt, int32_t nsrc, const int32_t *src_eq,
                  const double *src_b, const double *ftab)
{
    if (!c) return HRN_EARG;
    ++c->epoch;
    if (nshot < 1 || nshot > HRN_MAX_SHOTS) return set_error(c, HRN_EARG, "nshot must be 1..HRN_MAX_SHOTS");
    if (nstep < 1 || !(dt > 0.0) || nsrc < 0 || (nsrc > 0 && (!src_eq || !src_b)) || !ftab)
        return set_error(c, HRN_EARG, "bad shot arguments");
    c->nshot = nshot;
    c->nstep = nstep;
    c->dt = dt;
    c->h_src_eq.assign(src_eq, src_eq + nsrc);
    c->h_src_b.assign(src_b, src_b + size_t(nsrc) * nshot);
    c->h_ftab.assign(ftab, ftab + size_t(nshot) * (nstep + 1) * 3);
    c->h_shot_nstep.clear();
    c->h_rec_mask.clear();
    c->have_data = false;
    for (double v : c->h_ftab)
        if (!std::isfinite(v)) return set_error(c, HRN_ENAN, "non-finite time function sample");
    c->have_forward = false;
    cudaSetDevice(c->device);
    HRN_CUDA(c, c->d_mis_terms.alloc(size_t(nshot) * (nstep + 1) * 8));
    HRN_CUDA(c, c->d_cost.alloc(size_t(1 + nshot) * 8));
    if (int rc = upload_sources(c)) return rc;
    return upload_receivers(c);
}

int hrn_set_receivers(hrn_ctx *c, int32_t nrec3, const int32_t *eqdis, const int32_t *eqdis_map)
{
    if (!c) return HRN_EARG;
    ++c->epoch;
    if (nrec3 < 0 || (nrec3 > 0 && (!eqdis || !eqdis_map))) return set_error(c, HRN_EARG, "bad receiver arguments");
    c->nrec3 = nrec3;
    c->h_eqdis.assign(eqdis, eqdis + nrec3);
    c->h_eqdis_map.assign(eqdis_map, eqdis_map + nrec3);
    c->h_rec_mask.clear();
    cudaSetDevice(c->device);
    return upload_receivers(c);
}

int hrn_set_shot_records(hrn_ctx *c, const int32_t *nstep_shot, const uint8_t *rec_mask)
{
    if (!c) return HRN_EARG;
    ++c->epoch;
    if (c->nshot < 1) return set_error(c, HRN_ESTATE, "call hrn_set_shots first");
    cudaSetDevice(c->device);
    c->h_shot_nstep.clear();
    c->h_rec_mask.clear();
    if (nstep_shot) {
        bool uneven = false;
        for (int s = 0; s < c->nshot; ++s) {
            if (nstep_shot[s] < 1 || nstep_shot[s] > c->nstep)
                return set_error(c, HRN_EARG, "a shot's record length must be 1..nstep of hrn_set_shots");
            uneven |= nstep_shot[s] != c->nstep;
        }
        if (uneven) {
            c->h_shot_nstep.assign(nstep_shot, nstep_shot + c->nshot);
            HRN_CUDA(c, c->d_shot_nstep.alloc(size_t(c->nshot) * 4));
            HRN_CUDA(c, cudaMemcpy(c->d_shot_nstep.p, c->h_shot_nstep.data(), size_t(c->nshot) * 4, cudaMemcpyHostToDevice));
        }
    }
    if (rec_mask && c->nrec3 > 0) {
        const size_t nm = size_t(c->nshot) * c->nrec3;
        bool all = true;
        for (size_t i = 0; i < nm; ++i) all &= rec_mask[i] != 0;
        if (!all) {
            c->h_rec_mask.resize(nm);
            for (size_t i = 0; i < nm; ++i) c->h_rec_mask[i] = rec_mask[i] ? 1 : 0;
            HRN_CUDA(c, c->d_rec_mask.alloc(nm));
            HRN_CUDA(c, cudaMemcpy(c->d_rec_mask.p, c->h_rec_mask.data(), nm, cudaMemcpyHostToDevice));
        }
    }
    return HRN_OK;
}

int hrn_forward(hrn_ctx *c)
{
    if (!c) return HRN_EARG;
    if (int rc = check_ready(c, false)) return rc;
    cudaSetDevice(c->device);
    if (int rc = ensure_state(c)) return rc;
    return run_forward(c);
}

int hrn_get_state(hrn_ctx *c, int32_t step, int32_t shot, double *x1, double *x2, double *x3)
{
    if (!c) return HRN_EARG;
    if (!c->have_forward) return set_error(c, HRN_ESTATE, "no forward state: call hrn_forward first");
    if (c->ckpt <= 0) return set_error(c, HRN_ESTATE, "states are kept only with checkpointing (hrn_set_checkpointing)");
    if (step < 0 || step > c->nstep || step % c->ckpt != 0)
        return set_error(c, HRN_EARG, "step must be a multiple of the checkpoint interval within 0..nstep");
    if (shot < 0 || shot >= c->nshot) return set_error(c, HRN_EARG, "shot out of range");
    const size_t S = c->nshot, vn = size_t(c->neq) * S, eb = c->elem_bytes();
    std::vector<unsigned char> h(3 * vn * eb);
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    HRN_CUDA(c, cudaMemcpy(h.data(), static_cast<const unsigned char *>(c->d_ckpt.p) + size_t(step / c->ckpt) * 3 * vn * eb,
                           h.size(), cudaMemcpyDeviceToHost));
    double *out[3] = {x1, x2, x3};
    for (int k = 0; k < 3; ++k) {
        if (!out[k]) continue;
        for (int i = 0; i < c->neq; ++i) {
            const size_t at = size_t(k) * vn + size_t(i) * S + size_t(shot);
            out[k][i] = c->precision == HRN_FP64 ? reinterpret_cast<const double *>(h.data())[at]
                                                 : double(reinterpret_cast<const float *>(h.data())[at]);
        }
    }
    return HRN_OK;
}

int hrn_get_history(hrn_ctx *c, int32_t shot, double *u_store)
{
    if (!c || !u_store) return HRN_EARG;
    if (!c->have_forward) return set_error(c, HRN_ESTATE, "no forward history");
    if (c->ckpt > 0) return set_error(c, HRN_ESTATE, "the forward history is not kept with checkpointing (receiver traces are)");
    if (shot < 0 || shot >= c->nshot) return set_error(c, HRN_EARG, "shot out of range");
    const size_t S = c->nshot, n = size_t(c->nstep + 1) * c->nstore;
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    if (c->precision == HRN_FP64) {
        std::vector<double> h(n * S);
        HRN_CUDA(c, cudaMemcpy(h.data(), c->d_hist.p, h.size() * 8, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; ++i) u_store[i] = h[i * S + shot];
    } else {
        std::vector<float> h(n * S);
        HRN_CUDA(c, cudaMemcpy(h.data(), c->d_hist.p, h.size() * 4, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; ++i) u_store[i] = h[i * S + shot];
    }
    return HRN_OK;
}

int hrn_get_adjoint_history(hrn_ctx *c, int32_t shot, double *p_store)
{
    if (!c || !p_store) return HRN_EARG;
    if (!c->have_phist) return set_error(c, HRN_ESTATE, "no adjoint history (run hrn_adjoint_gradient with keep_p)");
    if (shot < 0 || shot >= c->nshot) return set_error(c, HRN_EARG, "shot out of range");
    const size_t S = c->nshot, n = size_t(c->nstep + 1) * c->nstore;
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    if (c->precision == HRN_FP64) {
        std::vector<double> h(n * S);
        HRN_CUDA(c, cudaMemcpy(h.data(), c->d_phist.p, h.size() * 8, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; ++i) p_store[i] = h[i * S + shot];
    } else {
        std::vector<float> h(n * S);
        HRN_CUDA(c, cudaMemcpy(h.data(), c->d_phist.p, h.size() * 4, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; ++i) p_store[i] = h[i * S + shot];
    }
    return HRN_OK;
}

int hrn_get_traces(hrn_ctx *c, double *traces)
{
    if (!c || !traces) return HRN_EARG;
    if (!c->have_forward) return set_error(c, HRN_ESTATE, "no forward history");
    const size_t S = c->nshot, T1 = size_t(c->nstep) + 1, eb = c->elem_bytes();
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    // one strided 2D copy per receiver pulls its S values at every step
    std::vector<char> buf(T1 * S * eb);
    const RecView rv = rec_view(c);
    for (int q = 0; q < c->nrec3; ++q) {
        const int pos = c->ckpt > 0 ? q : c->h_eqdis_map[q];
        const char *src = static_cast<const char *>(rv.hist) + size_t(pos) * S * eb;
        HRN_CUDA(c, cudaMemcpy2D(buf.data(), S * eb, src, size_t(rv.stride) * S * eb, S * eb, T1, cudaMemcpyDeviceToHost));
        for (size_t s = 0; s < S; ++s)
            for (size_t n = 0; n < T1; ++n) {
                double v = eb == 8 ? reinterpret_cast<const double *>(buf.data())[n * S + s]
                                   : double(reinterpret_cast<const float *>(buf.data())[n * S + s]);
                traces[(s * c->nrec3 + q) * T1 + n] = v;
            }
    }
    return HRN_OK;
}

static int upload_dis(hrn_ctx *c, const double *dis_meas, bool device_src = false)
{
    const size_t n = size_t(c->nshot) * c->nrec3 * (c->nstep + 1);
    if (!dis_meas) {
        if (n && !c->have_data) return set_error(c, HRN_ESTATE, "no measured data: pass dis_meas or call hrn_set_data");
        return HRN_OK;
    }
    if (n == 0) return HRN_OK;
    HRN_CUDA(c, c->d_dis.alloc(n * 8));
    HRN_CUDA(c, cudaMemcpyAsync(c->d_dis.p, dis_meas, n * 8, device_src ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                c->stream));
    c->have_data = true;
    return HRN_OK;
}

int hrn_set_data(hrn_ctx *c, const double *dis_meas, int32_t on_device)
{
    if (!c || !dis_meas) return HRN_EARG;
    if (c->nshot == 0) return set_error(c, HRN_ESTATE, "no shots: call hrn_set_shots first");
    cudaSetDevice(c->device);
    return upload_dis(c, dis_meas, on_device != 0);
}

int hrn_get_gradient_device(hrn_ctx *c, double *d_g_lambda, double *d_g_mu)
{
    if (!c) return HRN_EARG;
    if (!c->have_mesh || !c->d_g.p) return set_error(c, HRN_ESTATE, "no gradient");
    if (d_g_lambda) HRN_CUDA(c, cudaMemcpyAsync(d_g_lambda, c->d_g.p, size_t(c->nj) * 8, cudaMemcpyDeviceToDevice, c->stream));
    if (d_g_mu)
        HRN_CUDA(c, cudaMemcpyAsync(d_g_mu, c->d_g.as<double>() + c->nj, size_t(c->nj) * 8, cudaMemcpyDeviceToDevice, c->stream));
    return HRN_OK;
}

int hrn_set_variant(hrn_ctx *c, int32_t forward, int32_t adjoint)
{
    if (!c) return HRN_EARG;
    ++c->epoch;
    auto ok = [](int v) {
        return v == 0 || v == 40 || v == 80 || v == 160 || v == 41 || v == 81 || v == 161 || v == 42 || v == 43 || v == 82 ||
               v == 83 || hrn::is_gt_variant(v) || (v >= 90 && v <= 95) || (v >= 100 && v <= 105);
    };
    if (!ok(forward) || !ok(adjoint))
        return set_error(c, HRN_EARG, "variant must be 0 (tune), lanes*10 + mat + tiled (lanes 4/8/16, mat 0/1, tiled 0/2/4; "
                                      "tiled only with lanes 4/8) or 90-95 / 100-105 (matrix-free with materialized / rebuilt stage inputs: "
                                      "slots even, atomics odd; 1, 2, 4 shots per thread)");
    c->lanes_f = forward;
    c->lanes_a = adjoint;
    return HRN_OK;
}

int hrn_get_variant(hrn_ctx *c, int32_t *forward, int32_t *adjoint)
{
    if (!c) return HRN_EARG;
    if (forward) *forward = c->lanes_f;
    if (adjoint) *adjoint = c->lanes_a;
    return HRN_OK;
}

int hrn_set_checkpointing(hrn_ctx *c, int32_t interval)
{
    if (!c) return HRN_EARG;
    ++c->epoch;
    if (interval < 0) return set_error(c, HRN_EARG, "checkpoint interval must be >= 0");
    c->ckpt = interval;
    c->have_forward = false;
    c->have_phist = false;
    return HRN_OK;
}

int hrn_time_stage(hrn_ctx *c, int32_t adjoint, int32_t nsteps, double *avg_stage_ms)
{
    if (!c || !avg_stage_ms || nsteps < 1) return HRN_EARG;
    if (int rc = check_ready(c, false)) return rc;
    cudaSetDevice(c->device);
    return run_time_stage(c, adjoint != 0, nsteps, avg_stage_ms);
}

int hrn_launch_count(hrn_ctx *c, int64_t *n)
{
    if (!c || !n) return HRN_EARG;
    *n = c->launches;
    return HRN_OK;
}

int hrn_misfit(hrn_ctx *c, const double *dis_meas, double *cost)
{
    if (!c || !cost) return HRN_EARG;
    if (!c->have_forward) return set_error(c, HRN_ESTATE, "no forward history");
    cudaSetDevice(c->device);
    if (int rc = upload_dis(c, dis_meas)) return rc;
    std::vector<double> out(size_t(1 + c->nshot));
    if (int rc = run_misfit(c, out.data())) return rc;
    if (!std::isfinite(out[0])) return set_error(c, HRN_ENAN, "non-finite misfit");
    *cost = out[0];
    return HRN_OK;
}

int hrn_adjoint_gradient(hrn_ctx *c, const double *dis_meas, int32_t lambda_2mu, int32_t keep_p, double *g_lambda,
                         double *g_mu)
{
    if (!c) return HRN_EARG;
    if (int rc = check_ready(c, true)) return rc;
    if (!c->have_forward) return set_error(c, HRN_ESTATE, "no forward history: call hrn_forward first");
    cudaSetDevice(c->device);
    if (int rc = upload_dis(c, dis_meas)) return rc;
    if (int rc = run_adjoint_gradient(c, lambda_2mu, keep_p)) return rc;
    if (g_lambda) HRN_CUDA(c, cudaMemcpyAsync(g_lambda, c->d_g.p, size_t(c->nj) * 8, cudaMemcpyDeviceToHost, c->stream));
    if (g_mu) HRN_CUDA(c, cudaMemcpyAsync(g_mu, c->d_g.as<double>() + c->nj, size_t(c->nj) * 8, cudaMemcpyDeviceToHost, c->stream));
    if (g_lambda || g_mu) HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    return HRN_OK;
}

}  // extern "C"
