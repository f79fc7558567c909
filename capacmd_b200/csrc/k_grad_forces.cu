// Directional derivative of the forces along a displacement of the
// positions, at fixed induced vector: dF/de (r + e w) at e = 0, i.e. minus
// the Hessian of the energy times w.  The force-matching position gradient
// needs it (k_grad.cu).  Each force term of the step is recomputed on dual
// numbers from the neighbour list and the dense metal set, mirroring the
// FP64 kernels term by term:
//   * nonbonded pairs and the water side of the metal - permanent charge
//     CPIM terms: k_pair.cu (force.c:591-816, cpff.c:578-724);
//   * Sutton-Chen: both passes (force.c:385-542), with the densities on
//     dual numbers;
//   * the metal side of CPIM: k_cpim_metal (cpff.c:578-926).
// The external field acts on charges with a force independent of the
// positions and has no derivative.
#include "dual.cuh"
#include "terms.cuh"

namespace capac {

namespace {

// pair_term (k_pair.cu) on scalar type T: the force on j is f * (r_j - r_i).
template <class T>
__device__ __forceinline__ T pair_term_t(const DevParams &P, int k, double qi, double qj, T r2)
{
    const int fn = P.nb_funct[k];
    const double4 pr = P.nb_par[k];  // (c6, c12, a, b)
    const T r = sqrt(r2), rinv = 1.0 / r, r2inv = rinv * rinv;
    if (fn == 4) {  // compute_erf_vdw, force.c:591-632
        if (pr.x != 0.0 || pr.y != 0.0) {
            const T r6inv = r2inv * r2inv * r2inv;
            const T a12 = pr.y * (r6inv * r6inv), a6 = pr.x * r6inv, u = r / pr.z, eu = erf(u);
            return ((12.0 * a12 - 6.0 * a6) * rinv * eu - (a12 - a6) * (2.0 * kInvSqrtPi) * exp(-(u * u)) / pr.z) * rinv;
        }
        return zero<T>();
    }
    if (fn == 3) {  // compute_morse, force.c:639-667
        const T e1 = exp(-pr.w * (r - pr.x)), e2 = e1 * e1;
        return (2.0 * pr.z * pr.w) * (e2 - e1) * rinv;
    }
    if (fn == 2) {  // compute_buckingham, force.c:674-703
        const T r6inv = r2inv * r2inv * r2inv, eb = exp(-pr.w * r);
        return pr.z * eb * pr.w * rinv - (6.0 * pr.x) * r6inv * r2inv;
    }
    T f = zero<T>();
    if (pr.x != 0.0 || pr.y != 0.0) {  // compute_nonbonded, force.c:710-816
        const T r6inv = r2inv * r2inv * r2inv, r12inv = r6inv * r6inv;
        if (P.use_vdw == 1) {
            const T fr = (12.0 * pr.y) * r12inv - (6.0 * pr.x) * r6inv;
            const double fc = 12.0 * pr.y * P.inv_rc12 - 6.0 * pr.x * P.inv_rc6;
            f = (fr - fc) * r2inv;
        } else {
            f = (pr.y * 2.0 * r12inv - pr.x * r6inv) * 6.0 * r2inv;
        }
    }
    if (qi != 0.0 && qj != 0.0) {
        const double qq = kFQQ * qi * qj;
        if (P.use_coulomb == 1) {
            const double a = P.w_alpha;
            const T ec = erfc(a * r);
            f = f + qq * ((ec * r2inv + P.w_a2_sqrtpi * exp(-(a * a) * r2) * rinv) - P.w_const) * rinv;
        } else {
            f = f + qq * r2inv * rinv;
        }
    }
    return f;
}

// cpim_charge_pair (terms.cuh) on scalar type T: force on the metal atom
// (r = metal - atom) from a permanent charge and the induced (q, p).
template <class T>
__device__ __forceinline__ void cpim_charge_pair_t(const DevParams &P, const T (&r)[3], T r2, double q_perm,
                                                   double q_ind, const double p[3], T (&f)[3])
{
    const T rr = sqrt(r2);
    T a0, ec = zero<T>(), eg = zero<T>();
    if (P.use_coulomb == 1) {
        ec = erfc(P.w_alpha * rr);
        eg = exp(-(P.w_alpha * P.w_alpha) * r2);
        a0 = (ec / r2 + P.w_a2_sqrtpi * eg / rr - P.w_const) / rr;
    } else {
        a0 = 1.0 / (r2 * rr);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) f[a] = a0 * r[a] * (kFQQ * q_perm * q_ind);
    const double sp = kFQQ * q_perm / kNm2Bohr;
    if (P.use_coulomb == 1) {
        const double al3 = P.w_alpha * P.w_alpha * P.w_alpha;
        const T a1 = (ec + P.w_a2_sqrtpi * rr * eg) / (r2 * r2 * rr);
        const T b1 = (4.0 * kInvSqrtPi * al3) * eg / r2;
        const T c1 = P.w_const / (r2 * rr);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                T rab = r[a] * r[b];
                T t = a1 * (3.0 * rab) + b1 * rab - c1 * rab;
                if (a == b) t = t - a1 * r2 + c1 * r2;
                f[b] = f[b] - t * (sp * p[a]);
            }
    } else {
        const T ir5 = 1.0 / (r2 * r2 * rr);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                T t = 3.0 * r[a] * r[b];
                if (a == b) t = t - r2;
                f[b] = f[b] - t * ir5 * (sp * p[a]);
            }
    }
}

// Nonbonded pairs and the water side of the CPIM charge terms, warp per atom.
__global__ void __launch_bounds__(256) k_pair_dual(DevParams P, const double4 *__restrict__ pos4,
                                                   const double *__restrict__ wdir, const uint32_t *__restrict__ nbr,
                                                   const int *__restrict__ nnb, int cap, const double *__restrict__ pq,
                                                   int cpim, double *dfx, double *dfy, double *dfz)
{
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < P.N; i += nwarps) {
        Dual ri[3];
        load_pos(pos4, wdir, i, ri);
        const double qi = pos4[i].w;
        const bool cpim_i = cpim && P.is_metal[i] == 0 && qi != 0.0;
        const int trow = P.type[i] * P.n_types;
        const uint32_t *row = nbr + (size_t)i * cap;
        double a[3] = {0.0, 0.0, 0.0};
        for (int k = lane; k < nnb[i]; k += 32) {
            const uint32_t e = row[k];
            const int j = nb_index(e);
            Dual rj[3];
            load_pos(pos4, wdir, j, rj);
            Dual d[3] = {rj[0] - ri[0], rj[1] - ri[1], rj[2] - ri[2]};
            image_t(d[0], d[1], d[2], P.box);
            if (norm2_exact(d[0].v, d[1].v, d[2].v) >= P.rc2) continue;
            const Dual r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            const Dual f = pair_term_t<Dual>(P, trow + nb_type(e), qi, pos4[j].w, r2);
#pragma unroll
            for (int c = 0; c < 3; ++c) a[c] -= (f * d[c]).d;
            if (cpim_i && P.is_metal[j]) {
                const int jm = j - P.metal_min;
                const double p[3] = {pq[3 * jm], pq[3 * jm + 1], pq[3 * jm + 2]};
                Dual g[3];
                cpim_charge_pair_t(P, d, r2, qi, pq[3 * P.M + jm], p, g);
#pragma unroll
                for (int c = 0; c < 3; ++c) a[c] -= g[c].d;
            }
        }
        const double s0 = warp_sum(a[0]), s1 = warp_sum(a[1]), s2 = warp_sum(a[2]);
        if (lane == 0) {
            dfx[i] += s0;
            dfy[i] += s1;
            dfz[i] += s2;
        }
    }
}

// Sutton-Chen density on dual numbers, warp per metal atom: 1/sqrt(rho_i).
__global__ void __launch_bounds__(256) k_qsc_density_dual(DevParams P, const double4 *__restrict__ pos4,
                                                          const double *__restrict__ wdir, double *isd_v,
                                                          double *isd_d)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= P.M) return;
    Dual ri[3];
    load_pos(pos4, wdir, P.metal_min + i, ri);
    Dual rho = zero<Dual>();
    for (int j = lane; j < P.M; j += 32) {
        if (j == i) continue;
        Dual rj[3];
        load_pos(pos4, wdir, P.metal_min + j, rj);
        Dual d[3] = {rj[0] - ri[0], rj[1] - ri[1], rj[2] - ri[2]};
        image_t(d[0], d[1], d[2], P.box);
        if (norm2_exact(d[0].v, d[1].v, d[2].v) >= P.rc2) continue;
        rho += pow(P.qsc_a / sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), P.qsc_m);
    }
    rho = warp_sum_t(rho);
    if (lane == 0) {
        const Dual s = rho.v > 0.0 ? 1.0 / sqrt(rho) : zero<Dual>();
        isd_v[i] = s.v;
        isd_d[i] = s.d;
    }
}

// Sutton-Chen forces on dual numbers (k_qsc_force), warp per metal atom.
__global__ void __launch_bounds__(256) k_qsc_force_dual(DevParams P, const double4 *__restrict__ pos4,
                                                        const double *__restrict__ wdir,
                                                        const double *__restrict__ isd_v,
                                                        const double *__restrict__ isd_d, double *dfx, double *dfy,
                                                        double *dfz)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= P.M) return;
    Dual ri[3];
    load_pos(pos4, wdir, P.metal_min + i, ri);
    const double cm2 = P.qsc_c * P.qsc_m / 2.0;
    double a[3] = {0.0, 0.0, 0.0};
    for (int j = lane; j < P.M; j += 32) {
        if (j == i) continue;
        Dual rj[3];
        load_pos(pos4, wdir, P.metal_min + j, rj);
        Dual d[3] = {rj[0] - ri[0], rj[1] - ri[1], rj[2] - ri[2]};
        image_t(d[0], d[1], d[2], P.box);
        if (norm2_exact(d[0].v, d[1].v, d[2].v) >= P.rc2) continue;
        const Dual r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        const Dual ar = P.qsc_a / sqrt(r2);
        const Dual an = pow(ar, P.qsc_n), am = pow(ar, P.qsc_m);
        const Dual isum = Dual{isd_v[i] + isd_v[j], isd_d[i] + isd_d[j]};
        const Dual f = P.qsc_eps * (P.qsc_n * an - cm2 * isum * am) / r2;
#pragma unroll
        for (int c = 0; c < 3; ++c) a[c] -= (f * d[c]).d;
    }
    const double s0 = warp_sum(a[0]), s1 = warp_sum(a[1]), s2 = warp_sum(a[2]);
    if (lane == 0) {
        const int im = P.metal_min + i;
        dfx[im] += s0;
        dfy[im] += s1;
        dfz[im] += s2;
    }
}

// Metal side of CPIM on dual numbers (k_cpim_metal), block per metal atom.
__global__ void __launch_bounds__(256) k_cpim_metal_dual(DevParams P, const double4 *__restrict__ pos4,
                                                         const double *__restrict__ wdir,
                                                         const uint32_t *__restrict__ nbr,
                                                         const int *__restrict__ nnb, int cap,
                                                         const double *__restrict__ pq, double *dfx, double *dfy,
                                                         double *dfz)
{
    __shared__ double sh[32 * 3];
    const int i = blockIdx.x, M = P.M, im = P.metal_min + i;
    Dual ri[3];
    load_pos(pos4, wdir, im, ri);
    const double qi = pq[3 * M + i];
    const double pi[3] = {pq[3 * i], pq[3 * i + 1], pq[3 * i + 2]};
    double acc[3] = {0.0, 0.0, 0.0};
    // metal - permanent charge (cpff.c:578-724)
    const uint32_t *row = nbr + (size_t)im * cap;
    for (int k = threadIdx.x; k < nnb[im]; k += blockDim.x) {
        const int j = nb_index(row[k]);
        if (P.is_metal[j]) continue;
        const double qw = pos4[j].w;
        if (qw == 0.0) continue;
        Dual rj[3];
        load_pos(pos4, wdir, j, rj);
        Dual r[3] = {ri[0] - rj[0], ri[1] - rj[1], ri[2] - rj[2]};
        image_t(r[0], r[1], r[2], P.box);
        if (norm2_exact(r[0].v, r[1].v, r[2].v) >= P.rc2) continue;
        const Dual r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        Dual f[3];
        cpim_charge_pair_t(P, r, r2, qw, qi, pi, f);
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[c] += f[c].d;
    }
    // metal - metal, atomic units (cpff.c:752-926)
    const double iqq = P.inv_r_qq, ipq = P.inv_r_pq, ipp = P.inv_r_pp;
    const double ipq3 = ipq * ipq * ipq, ipp3 = ipp * ipp * ipp, ipp5 = ipp3 * ipp * ipp;
    for (int j = threadIdx.x; j < M; j += blockDim.x) {
        if (j == i) continue;
        Dual rj[3];
        load_pos(pos4, wdir, P.metal_min + j, rj);
        Dual r[3] = {rj[0] - ri[0], rj[1] - ri[1], rj[2] - ri[2]};
        image_t(r[0], r[1], r[2], P.box);
        r[0] = r[0] * kNm2Bohr;
        r[1] = r[1] * kNm2Bohr;
        r[2] = r[2] * kNm2Bohr;
        const Dual r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2], rr = sqrt(r2);
        const Dual ir3 = 1.0 / (r2 * rr), ir5 = ir3 / r2, ir7 = ir5 / r2;
        const double qj = pq[3 * M + j];
        const double pj[3] = {pq[3 * j], pq[3 * j + 1], pq[3 * j + 2]};
        Dual f[3] = {zero<Dual>(), zero<Dual>(), zero<Dual>()};
        const Dual gqq = exp(-(r2 * (iqq * iqq))), erq = erf(rr * iqq);
        const Dual A0 = ir3 * (erq - (2.0 * kInvSqrtPi * iqq) * rr * gqq);
#pragma unroll
        for (int a = 0; a < 3; ++a) f[a] = f[a] + A0 * r[a] * (kFqqAu2 * qi * qj);
        const Dual gpq = exp(-(r2 * (ipq * ipq)));
        const Dual tpq = erf(rr * ipq) - (2.0 * kInvSqrtPi * ipq) * rr * gpq;
        const Dual A1 = ir5 * tpq, B1 = (4.0 * kInvSqrtPi * ipq3) * gpq / r2;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                Dual T = A1 * (3.0 * r[a] * r[b]) - B1 * r[a] * r[b];
                if (a == b) T = T - A1 * r2;
                f[b] = f[b] + T * (kFqqAu2 * (qj * pi[a] - qi * pj[a]));
            }
        const Dual gpp = exp(-(r2 * (ipp * ipp))), erp = erf(rr * ipp);
        const Dual A2 = ir7 * (3.0 * erp - (6.0 * kInvSqrtPi * ipp) * rr * gpp -
                               (4.0 * kInvSqrtPi * ipp3) * (r2 * rr) * gpp);
        const Dual B2 = (8.0 * kInvSqrtPi * ipp5) * gpp / r2;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const double w = kFqqAu2 * pi[a] * pj[b];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    Dual t = 5.0 * r[a] * r[b] * r[c];
                    if (b == c) t = t - r2 * r[a];
                    if (c == a) t = t - r2 * r[b];
                    if (a == b) t = t - r2 * r[c];
                    f[c] = f[c] - (A2 * t - B2 * r[a] * r[b] * r[c]) * w;
                }
            }
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[c] -= f[c].d;
    }
    block_sum<3>(acc, sh);
    if (threadIdx.x == 0) {
        dfx[im] += acc[0];
        dfy[im] += acc[1];
        dfz[im] += acc[2];
    }
}

}  // namespace

// dF/de along wdir (interleaved, 3 per atom) at fixed induced vector, added
// to (dfx, dfy, dfz); isd_v and isd_d are scratch of n_metal doubles each.
void launch_force_derivative(capac_ctx *c, const double *wdir, double *dfx, double *dfy, double *dfz, double *isd_v,
                             double *isd_d)
{
    ensure_full_atom_list(c);  // the dual pair kernel walks every atom's row
    cudaStream_t s = c->stream;
    const bool cpim = c->M > 0 && c->use_cpff;
    const unsigned pair_blocks = grid_for((long)c->N * 32, 256);
    k_pair_dual<<<pair_blocks, 256, 0, s>>>(c->P, c->pos4, wdir, c->nbr, c->nnb, c->cap, c->vec_pq, cpim ? 1 : 0,
                                            dfx, dfy, dfz);
    ++c->launches;
    if (c->M > 0) {
        const unsigned mb = grid_for((long)c->M * 32, 256);
        k_qsc_density_dual<<<mb, 256, 0, s>>>(c->P, c->pos4, wdir, isd_v, isd_d);
        k_qsc_force_dual<<<mb, 256, 0, s>>>(c->P, c->pos4, wdir, isd_v, isd_d, dfx, dfy, dfz);
        c->launches += 2;
    }
    if (cpim) {
        k_cpim_metal_dual<<<c->M, 256, 0, s>>>(c->P, c->pos4, wdir, c->nbr, c->nnb, c->cap, c->vec_pq, dfx, dfy,
                                               dfz);
        ++c->launches;
    }
}

}  // namespace capac
