// Nonbonded pair forces over the full neighbour list, FP64.
//
// Per pair this is compute_nonbonded / compute_erf_vdw / compute_morse /
// compute_buckingham (force.c:591-816) as dispatched by mpi_nonb_pair
// (force.c:1476-1528): LJ shifted force + damped shifted force Coulomb
// (funct 1), Buckingham (2), Morse (3), erf-damped vdW (4).
//
// One warp owns atom i and walks its list; every pair is visited from both
// ends, so forces need no atomics and each end adds half of the pair energy
// and virial.  The cut-off test uses the reference's r^2 rounding.
//
// The same traversal adds, on each charged non-metal atom, the force from the
// induced charges and dipoles of metal neighbours inside the cut-off: the
// water side of the metal-water loop of mpi_cpff_force (cpff.c:578-724).  The
// metal side, with energies [10],[11] and the virial, is k_cpim_metal.
#include "terms.cuh"

namespace capac {

namespace {

// Force factor (force on j = f * rvec) and energies of one nonbonded pair.
__device__ __forceinline__ double pair_term(const DevParams &P, int k, double qi, double qj, double r2,
                                            double &e_qq, double &e_vdw)
{
    const int fn = P.nb_funct[k];
    const double4 pr = P.nb_par[k];  // (c6, c12, a, b)
    const double r = sqrt(r2);
    if (fn == 4) {  // compute_erf_vdw, force.c:591-632
        if (pr.x != 0.0 || pr.y != 0.0) {
            const double r6 = r2 * r2 * r2, r12 = r6 * r6;
            const double a12 = pr.y / r12, a6 = pr.x / r6, u = r / pr.z, eu = erf(u);
            e_vdw += (a12 - a6) * eu;
            return ((12.0 * a12 - 6.0 * a6) / r * eu - (a12 - a6) * 2.0 * kInvSqrtPi * exp(-u * u) / pr.z) / r;
        }
        return 0.0;
    }
    if (fn == 3) {  // compute_morse, force.c:639-667 (D = A, a = B, R = C6)
        const double e1 = exp(-pr.w * (r - pr.x)), e2 = e1 * e1;
        e_vdw += pr.z * (e2 - 2.0 * e1);
        return 2.0 * pr.z * pr.w * (e2 - e1) / r;
    }
    if (fn == 2) {  // compute_buckingham, force.c:674-703 (A, B, C6)
        const double r6 = r2 * r2 * r2, r8 = r6 * r2, eb = exp(-pr.w * r);
        e_vdw += pr.z * eb - pr.x / r6;
        return pr.z * eb * pr.w / r - 6.0 * pr.x / r8;
    }
    // funct 1: compute_nonbonded, force.c:710-816 (not a 1-4 pair)
    double f = 0.0;
    if (pr.x != 0.0 || pr.y != 0.0) {
        const double r6 = r2 * r2 * r2, r12 = r6 * r6;
        if (P.use_vdw == 1) {
            const double fr = 12.0 * pr.y / r12 - 6.0 * pr.x / r6;
            const double fc = 12.0 * pr.y * P.inv_rc12 - 6.0 * pr.x * P.inv_rc6;
            f = (fr - fc) / r2;
            e_vdw += (pr.y / r12 - pr.x / r6) + (r - P.rc) * fc / P.rc - (pr.y * P.inv_rc12 - pr.x * P.inv_rc6);
        } else {
            f = (pr.y * 2.0 / r12 - pr.x / r6) * 6.0 / r2;
            e_vdw += pr.y / r12 - pr.x / r6;
        }
    }
    if (qi != 0.0 && qj != 0.0) {
        if (P.use_coulomb == 1) {
            const double a = P.w_alpha, ec = erfc(a * r);
            f += kFQQ * qi * qj * ((ec / r2 + P.w_a2_sqrtpi * exp(-a * a * r2) / r) - P.w_const) / r;
            e_qq += kFQQ * qi * qj * (ec / r - P.w_erfc_arcut + P.w_const * (r - P.rc));
        } else {
            f += kFQQ * qi * qj / (r2 * r);
            e_qq += kFQQ * qi * qj / r;
        }
    }
    return f;
}

}  // namespace

template <bool NONBONDED, bool CPIM>
__global__ void __launch_bounds__(256) k_pair_f64(DevParams P, const double4 *__restrict__ pos4,
                                                  const uint32_t *__restrict__ nbr, const int *__restrict__ nnb,
                                                  int cap, const double *__restrict__ vec_pq,
                                                  double *__restrict__ fx, double *__restrict__ fy,
                                                  double *__restrict__ fz, double *__restrict__ partials)
{
    __shared__ double sh[32 * 11];
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    double acc[11] = {0.0};  // fx fy fz e_qq e_vdw vir[9] -> packed below
    double f3[3] = {0.0, 0.0, 0.0};
    if (i < P.N) {
        const double4 pi = pos4[i];
        const int ti = P.type[i];
        const bool metal_i = P.is_metal[i] != 0;
        const int n = nnb[i];
        const uint32_t *row = nbr + (size_t)i * cap;
        for (int k = lane; k < n; k += 32) {
            const uint32_t e = row[k];
            const int j = nb_index(e);
            const double4 pj = pos4[j];
            double dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
            image(dx, dy, dz, P.box);
            const double r2 = norm2_exact(dx, dy, dz);
            if (r2 >= P.rc2) continue;
            if (NONBONDED) {
                const double f = pair_term(P, ti * P.n_types + nb_type(e), pi.w, pj.w, r2, acc[0], acc[1]);
                f3[0] -= f * dx;
                f3[1] -= f * dy;
                f3[2] -= f * dz;
                // virial -= r_a (f r_b), half per visit
                const double fjx = f * dx, fjy = f * dy, fjz = f * dz;
                acc[2] -= 0.5 * dx * fjx; acc[3] -= 0.5 * dx * fjy; acc[4] -= 0.5 * dx * fjz;
                acc[5] -= 0.5 * dy * fjx; acc[6] -= 0.5 * dy * fjy; acc[7] -= 0.5 * dy * fjz;
                acc[8] -= 0.5 * dz * fjx; acc[9] -= 0.5 * dz * fjy; acc[10] -= 0.5 * dz * fjz;
            }
            if (CPIM && !metal_i && pi.w != 0.0 && P.is_metal[j]) {
                const int jm = j - P.metal_min;
                const double r[3] = {dx, dy, dz};  // metal - atom
                const double pind[3] = {vec_pq[3 * jm], vec_pq[3 * jm + 1], vec_pq[3 * jm + 2]};
                double f[3], a0, ec;
                cpim_charge_pair(P, r, r2, pi.w, vec_pq[3 * P.M + jm], pind, f, a0, ec);
                f3[0] -= f[0];
                f3[1] -= f[1];
                f3[2] -= f[2];
            }
        }
        f3[0] = warp_sum(f3[0]);
        f3[1] = warp_sum(f3[1]);
        f3[2] = warp_sum(f3[2]);
        if (lane == 0) {
            fx[i] += f3[0];
            fy[i] += f3[1];
            fz[i] += f3[2];
        }
        acc[0] *= 0.5;
        acc[1] *= 0.5;
    }
    if (NONBONDED) block_partials<11>(acc, sh, partials);
}

void launch_pair_forces(capac_ctx *c, int mode)
{
    const unsigned grid = grid_for((long)c->N * 32, 256);
    if (mode == 0) {
        {
            ProfScope ps(c, K_PAIR);
            if (c->M > 0 && c->use_cpff)
                k_pair_f64<true, true><<<grid, 256, 0, c->stream>>>(c->P, c->pos4, c->nbr, c->nnb, c->cap,
                                                                    c->vec_pq, c->fx, c->fy, c->fz, c->partials);
            else
                k_pair_f64<true, false><<<grid, 256, 0, c->stream>>>(c->P, c->pos4, c->nbr, c->nnb, c->cap,
                                                                     c->vec_pq, c->fx, c->fy, c->fz, c->partials);
        }
        ++c->launches;
        static const int pot_slots[11] = {7, 8, -1, -1, -1, -1, -1, -1, -1, -1, -1};
        static const int vir_slots[11] = {-1, -1, 0, 1, 2, 3, 4, 5, 6, 7, 8};
        launch_finalize(c, (int)grid, 11, pot_slots, vir_slots);
    } else {
        ProfScope ps(c, K_PAIR);
        k_pair_f64<false, true><<<grid, 256, 0, c->stream>>>(c->P, c->pos4, c->nbr, c->nnb, c->cap, c->vec_pq,
                                                             c->fx, c->fy, c->fz, c->partials);
        ++c->launches;
    }
}

}  // namespace capac
