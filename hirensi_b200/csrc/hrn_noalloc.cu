// hrn_noalloc.cu -- the misfit of the current forward history for callers that
// cannot allocate device memory (hrn_misfit_noalloc, include/hirensi_b200.h).
//
// hrn_misfit keeps its per-step terms in a buffer the context allocates.  Some
// callers cannot let a library call cudaMalloc at that point:
// * cudaMalloc and cudaFree synchronize the whole device;
// * the allocation fails when another framework's caching pool already holds
//   the free memory, for example a Fortran driver that reserved its HBM budget
//   up front, or a PyTorch process whose allocator cached most of the device.
// This variant takes the measured data as a device pointer the caller owns and
// keeps its scratch in a fixed file-scope device array, so it allocates
// nothing.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "hrn_internal.h"
#include "hrn_misfit.cuh"

namespace hrn {

// Scratch of hrn_misfit_noalloc: per-(shot, step) terms, then the costs.
// Maximum: nshot * (nstep + 1) <= kNoAllocMaxTerms = 131072 (1 MiB of FP64
// terms: 8 shots of 16383 steps).  Every device on which the library's module
// is loaded holds this array until the process exits.
constexpr int kNoAllocMaxTerms = 1 << 17;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxTerms + 1 + HRN_MAX_SHOTS];

template <typename T>
__global__ void k_noalloc_terms(int nshot, int nstep, int nstore, int nrec3, int nslot, const int32_t *__restrict__ ptr,
                                const int32_t *__restrict__ qlist, const int32_t *__restrict__ emap, const T *__restrict__ hist,
                                const double *__restrict__ dis, double *__restrict__ terms,
                                const int32_t *__restrict__ shot_nstep, const uint8_t *__restrict__ mask)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (nstep + 1) * nshot) return;
    const int s = t % nshot, n = t / nshot;
    terms[size_t(s) * (nstep + 1) + n] =
        misfit_term<T>(nshot, s, n, nstep, nstore, nrec3, nslot, ptr, qlist, emap, hist, dis, shot_nstep, mask);
}

// cost[0] = total, cost[1 + s] = shot s; the reference's order n = nstep..1
__global__ void k_noalloc_sum(int nshot, int nstep, double dt, const double *__restrict__ terms, double *__restrict__ cost)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    misfit_sum(nshot, nstep, dt, terms, cost);
}

// Device address of the scratch array, looked up once per device with that
// device current (in host code the symbol is only a host-side stand-in).  The
// address belongs to the device's primary context: after a cudaDeviceReset the
// cached value is stale, so the entry must not be used across one.
static int scratch_address(hrn_ctx *c, double **out)
{
    static std::mutex mu;
    static double *addr[64] = {nullptr};
    if (c->device < 0 || c->device >= 64) return set_error(c, HRN_EARG, "device index out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[c->device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_error(c, e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        addr[c->device] = static_cast<double *>(p);
    }
    *out = addr[c->device];
    return 0;
}

}  // namespace hrn

using namespace hrn;

extern "C" int hrn_misfit_noalloc(hrn_ctx *c, const double *d_dis_meas, double *cost)
{
    if (!c || !cost) return HRN_EARG;
    const long long nterms = (long long)c->nshot * (c->nstep + 1);
    if (nterms > kNoAllocMaxTerms)
        return set_error(c, HRN_EARG, "nshot * (nstep + 1) exceeds the 131072 terms of the static scratch of hrn_misfit_noalloc");
    if (!c->have_forward) return set_error(c, HRN_ESTATE, "no forward history: call hrn_forward first");
    if (c->nrec3 > 0 && !d_dis_meas) return set_error(c, HRN_EARG, "null measured data");
    HRN_CUDA(c, cudaSetDevice(c->device));
    if (c->nrec3 > 0) {
        // hrn_misfit takes a host pointer of the same C type: refuse host memory and
        // other devices' memory here rather than fault in the kernel
        cudaPointerAttributes at{};
        cudaError_t e = cudaPointerGetAttributes(&at, d_dis_meas);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return set_error(c, HRN_EARG, "d_dis_meas is not a device pointer");
        }
        if ((at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) || at.device != c->device)
            return set_error(c, HRN_EARG, "d_dis_meas must point to device (or managed) memory of the context's device");
    }
    double *scratch = nullptr;
    if (int rc = scratch_address(c, &scratch)) return rc;
    double *terms = scratch, *out = scratch + kNoAllocMaxTerms;
    const int th = 128, nb = int((nterms + th - 1) / th);
    if (c->nslot_a > 0) {
        const RecView rv = rec_view(c);
        if (c->precision == HRN_FP64)
            k_noalloc_terms<double><<<nb, th, 0, c->stream>>>(c->nshot, c->nstep, rv.stride, c->nrec3, c->nslot_a,
                                                              c->d_aslot_ptr.as<int32_t>(), c->d_aslot_q.as<int32_t>(), rv.map,
                                                              static_cast<const double *>(rv.hist), d_dis_meas, terms,
                                                              shot_nstep_ptr(c), rec_mask_ptr(c));
        else
            k_noalloc_terms<float><<<nb, th, 0, c->stream>>>(c->nshot, c->nstep, rv.stride, c->nrec3, c->nslot_a,
                                                             c->d_aslot_ptr.as<int32_t>(), c->d_aslot_q.as<int32_t>(), rv.map,
                                                             static_cast<const float *>(rv.hist), d_dis_meas, terms,
                                                             shot_nstep_ptr(c), rec_mask_ptr(c));
        ++c->launches;
    } else {
        // no receivers: every term is zero (the scratch keeps the last call's contents)
        HRN_CUDA(c, cudaMemsetAsync(terms, 0, size_t(nterms) * sizeof(double), c->stream));
    }
    k_noalloc_sum<<<1, 1, 0, c->stream>>>(c->nshot, c->nstep, c->dt, terms, out);
    ++c->launches;
    HRN_CUDA(c, cudaGetLastError());
    HRN_CUDA(c, cudaMemcpyAsync(cost, out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    HRN_CUDA(c, cudaStreamSynchronize(c->stream));
    if (!std::isfinite(*cost)) return set_error(c, HRN_ENAN, "non-finite misfit");
    return HRN_OK;
}
