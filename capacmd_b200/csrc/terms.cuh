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

// The 4x4 CPIM block of the ordered metal pair (i, j) in FP64, entries
// e[4*row + col] over (p_x, p_y, p_z, q): mpi_cpff_mat_relay_COO,
// cpff.c:245-436.  r = r_j - r_i (pbc_12) in Bohr; diagonal block when same.
// Entries with |e| <= 1e-15 are dropped as in the reference (typedef.h:89-93).
__device__ __forceinline__ void cpim_block(const DevParams &P, const double4 &pi, const double4 &pj, bool same,
                                           double e[16])
{
#pragma unroll
    for (int k = 0; k < 16; ++k) e[k] = 0.0;
    if (same) {
        e[0] = e[5] = e[10] = keep_entry(P.inv_polar);
        e[15] = keep_entry(-P.inv_capac);
        return;
    }
    double r[3] = {pj.x - pi.x, pj.y - pi.y, pj.z - pi.z};
    image(r[0], r[1], r[2], P.box);
    r[0] *= kNm2Bohr;
    r[1] *= kNm2Bohr;
    r[2] *= kNm2Bohr;
    const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2], rr = sqrt(r2);
    const double ipp = P.inv_r_pp, ipq = P.inv_r_pq;
    const double gpp = exp(-(r2 * ipp * ipp));
    const double c1 = 1.0 / (r2 * r2 * rr) * (erf(rr * ipp) - 2.0 * kInvSqrtPi * ipp * rr * gpp);
    const double c2 = 4.0 * kInvSqrtPi * (ipp * ipp * ipp) / r2 * gpp;
    const double gpq = exp(-(r2 * ipq * ipq));
    const double c3 = 1.0 / (r2 * rr) * (erf(rr * ipq) - 2.0 * kInvSqrtPi * ipq * rr * gpq);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const double dab = a == b ? 1.0 : 0.0;
            e[4 * a + b] = keep_entry(-(c1 * (3.0 * r[a] * r[b] - dab * r2) - c2 * r[a] * r[b]));
        }
        e[4 * a + 3] = keep_entry(c3 * r[a]);
        e[12 + a] = keep_entry(-c3 * r[a]);
    }
    e[15] = keep_entry(-erf(rr * P.inv_r_qq) / rr);
}

}  // namespace capac
