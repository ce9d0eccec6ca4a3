// Device arithmetic of the misfit, shared by hrn_misfit (shot count fixed at
// compile time) and hrn_misfit_noalloc (shot count at run time), so that both
// entries keep one copy of the reference's sum order and masking.
//
// Reference: Compute_Misfit, S4/Solver_PETSc_Inverse.F90:591-657 -- J = sum over
// shots of sum_{n=nstep..1} 0.5 * dt * |u(x_r, t_n) - d(x_r, t_n)|^2, receivers
// listed on the same equation adding their residuals before the square.
#pragma once
#include <stdint.h>

namespace hrn {

// Squared residual of shot s at step n over the receiver slots (sl: one slot per
// distinct equation, ptr/qlist its receivers).  Shots of uneven record length add
// nothing past their last step; masked receivers are skipped.
template <typename T>
__device__ __forceinline__ double misfit_term(int nshot, int s, int n, int nstep, int nstore, int nrec3, int nslot,
                                             const int32_t *__restrict__ ptr, const int32_t *__restrict__ qlist,
                                             const int32_t *__restrict__ emap, const T *__restrict__ hist,
                                             const double *__restrict__ dis, const int32_t *__restrict__ shot_nstep,
                                             const uint8_t *__restrict__ mask)
{
    double d = 0.0;
    for (int sl = 0; sl < nslot && !(shot_nstep && n > shot_nstep[s]); ++sl) {
        double r = 0.0;
        for (int k = ptr[sl]; k < ptr[sl + 1]; ++k) {
            const int q = qlist[k];
            if (mask && !mask[size_t(s) * nrec3 + q]) continue;
            r += double(hist[(size_t(n) * nstore + emap[q]) * nshot + s]) - dis[(size_t(s) * nrec3 + q) * (nstep + 1) + n];
        }
        d += r * r;
    }
    return d;
}

// cost[0] = total, cost[1 + s] = shot s, each shot summed in the reference's
// order n = nstep..1 (one thread).
__device__ __forceinline__ void misfit_sum(int nshot, int nstep, double dt, const double *__restrict__ terms,
                                           double *__restrict__ cost)
{
    double total = 0.0;
    for (int s = 0; s < nshot; ++s) {
        double c = 0.0;
        for (int n = nstep; n >= 1; --n) c = c + 0.5 * terms[size_t(s) * (nstep + 1) + n] * dt;
        cost[1 + s] = c;
        total += c;
    }
    cost[0] = total;
}

}  // namespace hrn
