// Pair terms shared by more than one kernel.
#pragma once

#include "ctx.h"

namespace capac {

// Force on the metal atom from the permanent charge q of a non-metal atom at
// metal - atom separation r (nm); the atom receives the opposite force.
// cpff.c:604-702.  Returns through f[3]; also gives const_a0 for energy [11].
__device__ __forceinline__ void cpim_charge_pair(const DevParams &P, const double r[3], double r2, double q_perm,
                                                 double q_ind, const double p_ind[3], double f[3], double &a0,
                                                 double &ec_out)
{
    const double rr = sqrt(r2);
    double ec = 0.0, eg = 0.0;
    if (P.use_coulomb == 1) {
        ec = erfc(P.w_alpha * rr);
        eg = exp(-P.w_alpha * P.w_alpha * r2);
        a0 = (ec / r2 + P.w_a2_sqrtpi * eg / rr - P.w_const) / rr;
    } else {
        a0 = 1.0 / (r2 * rr);
    }
    ec_out = ec;
#pragma unroll
    for (int a = 0; a < 3; ++a) f[a] = a0 * r[a] * kFQQ * q_perm * q_ind;
    if (P.use_coulomb == 1) {
        const double al3 = P.w_alpha * P.w_alpha * P.w_alpha;
        const double a1 = 1.0 / (rr * rr * rr * rr * rr) * (ec + P.w_a2_sqrtpi * rr * eg);
        const double b1 = 4.0 * kInvSqrtPi * al3 / r2 * eg;
        const double c1 = P.w_const / (rr * rr * rr);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const double dab = a == b ? 1.0 : 0.0;
                f[b] += -(a1 * (3.0 * r[a] * r[b] - dab * r2) + b1 * r[a] * r[b] - c1 * (r[a] * r[b] - dab * r2)) *
                        kFQQ * q_perm * p_ind[a] / kNm2Bohr;
            }
    } else {
        const double ir5 = 1.0 / (rr * rr * rr * rr * rr);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const double dab = a == b ? 1.0 : 0.0;
                f[b] += -((3.0 * r[a] * r[b] - dab * r2) * ir5) * kFQQ * q_perm * p_ind[a] / kNm2Bohr;
            }
    }
}

}  // namespace capac
