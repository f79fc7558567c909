// Gradients of the total potential energy and of a force-matching loss with
// respect to the positions and the metal's parameters, and parameter
// get/set for fitting.
//
// Parameters.  The reference has one metal type (file.c:533-549):
// Sutton-Chen (eps, c, a, n, m; force.c:385-542) and CPIM (capacitance C,
// polarizability alpha; the Gaussian widths R_q = sqrt(2/pi) C and
// R_p = (sqrt(2/pi) alpha / 3)^(1/3), mpi-main.c:315-323, which may be
// decoupled and varied on their own).
//
// Energy.  E(r, theta, x) is the sum of the reference's energy terms
// potential[1..14]; x = (p, q, lambda) solves A(r, theta) x = b(r) (the CPIM
// system, cpff.c:43-519).  The reference's forces are the explicit gradient
// -dE/dr at fixed x (cpff.c:526-950), but E is not stationary in x at the
// solution: the charge rows of A carry -H_qq q + H_qp p while the energy's
// charge-dipole term enters with the other sign, and the energy of the
// external field on the induced dipoles (cpff.c:941-947) is scaled by
// 1 Bohr/nm relative to the field in b (cpff.c:176-183).  So the total
// derivative needs the adjoint of the solve: with g = dE/dx and A mu = g
// (A is symmetric),
//     dE/dtheta = dE/dtheta|_x - mu^T (dA/dtheta) x,
//     dE/dr     = -F - d/dr [mu^T (A(r) x - b(r))]   (mu, x fixed).
// g is dense over the metal atoms plus the list terms of the permanent
// charges; the last term is a bilinear "force" of mu and x, recomputed from
// positions (dense metal-metal Gaussian-damped T0/T1/T2 derivatives, and the
// DSF field of the permanent charges from the neighbour list).
//
// Force matching.  L = sum_k (F_k - F_target,k)^2 / (3N); with
// w = 2 (F - F_target) / (3N) and Psi = w . dE/dr|_x,
//     dL/dtheta = -dPsi/dtheta = -(dPsi/dtheta|_x - nu^T (dA/dtheta) x),
//     A nu = dPsi/dx.
// dPsi/dx and dPsi/dtheta|_x are directional derivatives along w of g and of
// the explicit parameter derivatives: the same kernels evaluated on dual
// numbers (dual.cuh), exact to rounding.
//
// Adjoint solves use FP64 iterative refinement around the context's own
// BiCGSTAB (FP64 residual recomputed from positions each sweep) to a relative
// residual of 1e-12.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "dual.cuh"
#include "terms.cuh"

namespace capac {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kAdjointTol = 1.0e-12;
constexpr int kAdjointSweeps = 24;

// block_sum over T values; `sh` needs 32 * K * width<T>() doubles.
template <class T, int K>
__device__ __forceinline__ void block_sum_t(T (&v)[K], double *sh)
{
    if constexpr (std::is_same<T, Dual>::value) {
        double d[2 * K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            d[k] = v[k].v;
            d[K + k] = v[k].d;
        }
        block_sum<2 * K>(d, sh);
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = Dual{d[k], d[K + k]};
    } else {
        block_sum<K>(v, sh);
    }
}

// Block partials: the K values, then (for Dual) the K derivatives.
template <class T, int K>
__device__ __forceinline__ void block_partials_t(T (&v)[K], double *sh, double *partials)
{
    block_sum_t<T, K>(v, sh);
    if (threadIdx.x == 0) {
        constexpr int W = width<T>();
        double *out = partials + (size_t)blockIdx.x * K * W;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            out[k] = val(v[k]);
            if (W == 2) out[K + k] = der(v[k]);
        }
    }
}

// The 4x4 CPIM block (i, j) of cpff.c:255-440 on scalar type T, as the
// energy has it: without the solver's drop of entries |e| <= 1e-15
// (typedef.h:89-93), which would also drop the derivative of an entry that
// vanishes by symmetry (r_a = 0) but not in a neighbourhood.
template <class T>
__device__ __forceinline__ void cpim_block_t(const DevParams &P, const T (&ri)[3], const T (&rj)[3], bool same,
                                             T (&e)[16])
{
#pragma unroll
    for (int k = 0; k < 16; ++k) e[k] = zero<T>();
    if (same) {
        e[0] = e[5] = e[10] = lift<T>(P.inv_polar, 0.0);
        e[15] = lift<T>(-P.inv_capac, 0.0);
        return;
    }
    T r[3] = {rj[0] - ri[0], rj[1] - ri[1], rj[2] - ri[2]};
    image_t(r[0], r[1], r[2], P.box);
    r[0] = r[0] * kNm2Bohr;
    r[1] = r[1] * kNm2Bohr;
    r[2] = r[2] * kNm2Bohr;
    const T r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2], rr = sqrt(r2);
    const double ipp = P.inv_r_pp, ipq = P.inv_r_pq;
    const T gpp = exp(-(r2 * (ipp * ipp)));
    const T c1 = (erf(rr * ipp) - 2.0 * kInvSqrtPi * ipp * rr * gpp) / (r2 * r2 * rr);
    const T c2 = 4.0 * kInvSqrtPi * (ipp * ipp * ipp) * gpp / r2;
    const T gpq = exp(-(r2 * (ipq * ipq)));
    const T c3 = (erf(rr * ipq) - 2.0 * kInvSqrtPi * ipq * rr * gpq) / (r2 * rr);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            T t = 3.0 * r[a] * r[b];
            if (a == b) t = t - r2;
            e[4 * a + b] = -(c1 * t - c2 * r[a] * r[b]);
        }
        e[4 * a + 3] = c3 * r[a];
        e[12 + a] = -(c3 * r[a]);
    }
    e[15] = -(erf(rr * P.inv_r_qq) / rr);
}

// g = dE/dx for the induced dipoles and charge of metal atom i (block i);
// the neutrality rows have g = 0.  With T = Dual, gd receives the derivative
// along wdir.
template <class T>
__global__ void __launch_bounds__(256) k_cpim_dx(DevParams P, const double4 *__restrict__ pos4,
                                                 const double *__restrict__ wdir, const uint32_t *__restrict__ nbr,
                                                 const int *__restrict__ nnb, int cap, const double *__restrict__ x,
                                                 double *__restrict__ g, double *__restrict__ gd)
{
    __shared__ double sh[32 * 8 * 2];
    const int i = blockIdx.x, M = P.M, im = P.metal_min + i;
    T ri[3];
    load_pos(pos4, wdir, im, ri);
    // 0..2: (H_pp p + H_pq q)_i, 3: (H_qq q + H_qp p)_i (the A blocks with the
    // sign of the energy), 4..6 and 7: linear coefficients of p_i and q_i
    T acc[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[k] = zero<T>();
    for (int j = threadIdx.x; j < M; j += blockDim.x) {
        T rj[3];
        load_pos(pos4, wdir, P.metal_min + j, rj);
        T e[16];
        cpim_block_t(P, ri, rj, i == j, e);
        const double qj = x[3 * M + j], p0 = x[3 * j], p1 = x[3 * j + 1], p2 = x[3 * j + 2];
#pragma unroll
        for (int a = 0; a < 3; ++a) acc[a] += e[4 * a] * p0 + e[4 * a + 1] * p1 + e[4 * a + 2] * p2 + e[4 * a + 3] * qj;
        acc[3] += e[12] * p0 + e[13] * p1 + e[14] * p2 - e[15] * qj;
    }
    // permanent charges within the cut-off (cpff.c:578-724, energies [10] [11])
    const uint32_t *row = nbr + (size_t)im * cap;
    for (int k = threadIdx.x; k < nnb[im]; k += blockDim.x) {
        const int j = nb_index(row[k]);
        if (P.is_metal[j]) continue;
        const double qw = pos4[j].w;
        if (qw == 0.0) continue;
        T rj[3];
        load_pos(pos4, wdir, j, rj);
        T r[3] = {ri[0] - rj[0], ri[1] - rj[1], ri[2] - rj[2]};
        image_t(r[0], r[1], r[2], P.box);
        if (norm2_exact(val(r[0]), val(r[1]), val(r[2])) >= P.rc2) continue;
        const T r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2], rr = sqrt(r2);
        T phi, a0;
        if (P.use_coulomb == 1) {
            const T ec = erfc(P.w_alpha * rr), eg = exp(-(P.w_alpha * P.w_alpha) * r2);
            a0 = (ec / r2 + P.w_a2_sqrtpi * eg / rr - P.w_const) / rr;
            phi = ec / rr - P.w_erfc_arcut + P.w_const * (rr - P.rc);
        } else {
            a0 = 1.0 / (r2 * rr);
            phi = 1.0 / rr;
        }
        acc[7] += (kFQQ * qw) * phi;
#pragma unroll
        for (int a = 0; a < 3; ++a) acc[4 + a] += (-kFQQ * qw / kNm2Bohr) * (a0 * r[a]);
    }
    block_sum_t<T, 8>(acc, sh);
    if (threadIdx.x == 0) {
        // external field on the induced charge and dipole (cpff.c:930-948, energy [9])
        acc[7] -= P.efield[0] * ri[0] + P.efield[1] * ri[1] + P.efield[2] * ri[2];
        T out[4];
#pragma unroll
        for (int a = 0; a < 3; ++a) out[a] = kFqqAu1 * acc[a] + acc[4 + a] - P.efield[a];
        out[3] = kFqqAu1 * acc[3] + acc[7];
#pragma unroll
        for (int a = 0; a < 3; ++a) g[3 * i + a] = val(out[a]);
        g[3 * M + i] = val(out[3]);
        if (gd) {
#pragma unroll
            for (int a = 0; a < 3; ++a) gd[3 * i + a] = der(out[a]);
            gd[3 * M + i] = der(out[3]);
        }
    }
}

// Sutton-Chen sums, warp per metal atom i: S1 = 1/2 sum_j (a/r)^n,
// S2 = sqrt(rho_i), S3 = 1/2 sum_j (a/r)^n ln(a/r),
// S4 = sum_j (a/r)^m ln(a/r) / (2 sqrt(rho_i)).  E_SC = eps (S1 - c S2);
// dE/deps = S1 - c S2, dE/dc = -eps S2, dE/da = eps (n S1 - c m S2 / 2) / a,
// dE/dn = eps S3, dE/dm = -eps c S4.
template <class T>
__global__ void __launch_bounds__(256) k_qsc_param_sums(DevParams P, const double4 *__restrict__ pos4,
                                                        const double *__restrict__ wdir, double *partials)
{
    __shared__ double sh[32 * 4 * 2];
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    T acc[4] = {zero<T>(), zero<T>(), zero<T>(), zero<T>()};
    if (i < P.M) {
        T ri[3];
        load_pos(pos4, wdir, P.metal_min + i, ri);
        T sn = zero<T>(), ln = zero<T>(), rho = zero<T>(), lm = zero<T>();
        for (int j = lane; j < P.M; j += 32) {
            if (j == i) continue;
            T rj[3];
            load_pos(pos4, wdir, P.metal_min + j, rj);
            T d[3] = {rj[0] - ri[0], rj[1] - ri[1], rj[2] - ri[2]};
            image_t(d[0], d[1], d[2], P.box);
            if (norm2_exact(val(d[0]), val(d[1]), val(d[2])) >= P.rc2) continue;
            const T ar = P.qsc_a / sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), lar = log(ar);
            const T an = pow(ar, P.qsc_n), am = pow(ar, P.qsc_m);
            sn += an;
            ln += an * lar;
            rho += am;
            lm += am * lar;
        }
        sn = warp_sum_t(sn);
        ln = warp_sum_t(ln);
        rho = warp_sum_t(rho);
        lm = warp_sum_t(lm);
        if (lane == 0) {
            acc[0] = 0.5 * sn;
            acc[2] = 0.5 * ln;
            if (val(rho) > 0.0) {
                const T sr = sqrt(rho);
                acc[1] = sr;
                acc[3] = lm / (2.0 * sr);
            }
        }
    }
    block_partials_t<T, 4>(acc, sh, partials);
}

// CPIM parameter sums, block per metal atom i over j != i (ordered pairs):
//   0..2  explicit dE/du (u = 1/R_qq, 1/R_pq, 1/R_pp) of the energy terms
//         [12] [13] [14] at fixed x, without the Hartree factor;
//   3..5  mu^T (dA/du) x;
//   6..9  1/2 q_i^2, 1/2 |p_i|^2, mu_q,i q_i, mu_p,i . p_i.
// The u-derivatives: d/du erf(r u)/r = 2/sqrt(pi) e, and with
// c3 = [erf(r u) - 2/sqrt(pi) u r e] / r^3, c1 = c3 / r^2,
// c2 = 4/sqrt(pi) u^3 e / r^2 (e = exp(-r^2 u^2)):
//   dc3/du = 4/sqrt(pi) u^2 e, dc1/du = 4/sqrt(pi) u^2 e / r^2,
//   dc2/du = 4/sqrt(pi) (3 u^2 - 2 r^2 u^4) e / r^2.
template <class T>
__global__ void __launch_bounds__(256) k_cpim_param_sums(DevParams P, const double4 *__restrict__ pos4,
                                                         const double *__restrict__ wdir,
                                                         const double *__restrict__ x, const double *__restrict__ mu,
                                                         double *partials)
{
    __shared__ double sh[32 * 10 * 2];
    const int i = blockIdx.x, M = P.M;
    T ri[3];
    load_pos(pos4, wdir, P.metal_min + i, ri);
    const double qi = x[3 * M + i], pi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
    const double mqi = mu[3 * M + i], mpi[3] = {mu[3 * i], mu[3 * i + 1], mu[3 * i + 2]};
    const double uqq = P.inv_r_qq, upq = P.inv_r_pq, upp = P.inv_r_pp;
    T acc[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) acc[k] = zero<T>();
    for (int j = threadIdx.x; j < M; j += blockDim.x) {
        if (j == i) continue;
        T rj[3];
        load_pos(pos4, wdir, P.metal_min + j, rj);
        T r[3] = {rj[0] - ri[0], rj[1] - ri[1], rj[2] - ri[2]};
        image_t(r[0], r[1], r[2], P.box);
        r[0] = r[0] * kNm2Bohr;
        r[1] = r[1] * kNm2Bohr;
        r[2] = r[2] * kNm2Bohr;
        const T r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        const double qj = x[3 * M + j], pj[3] = {x[3 * j], x[3 * j + 1], x[3 * j + 2]};
        const T pir = pi[0] * r[0] + pi[1] * r[1] + pi[2] * r[2];
        const T pjr = pj[0] * r[0] + pj[1] * r[1] + pj[2] * r[2];
        const T mpir = mpi[0] * r[0] + mpi[1] * r[1] + mpi[2] * r[2];
        const double pipj = pi[0] * pj[0] + pi[1] * pj[1] + pi[2] * pj[2];
        const double mpipj = mpi[0] * pj[0] + mpi[1] * pj[1] + mpi[2] * pj[2];
        const T eqq = exp(-(r2 * (uqq * uqq))), epq = exp(-(r2 * (upq * upq))), epp = exp(-(r2 * (upp * upp)));
        const T dqq = (2.0 * kInvSqrtPi) * eqq;
        const T dc3 = (4.0 * kInvSqrtPi * upq * upq) * epq;
        const T dc1 = (4.0 * kInvSqrtPi * upp * upp) * epp / r2;
        const T dc2 = 4.0 * kInvSqrtPi * (3.0 * upp * upp - 2.0 * r2 * (upp * upp * upp * upp)) * epp / r2;
        acc[0] += (0.5 * qi * qj) * dqq;
        acc[1] += 0.5 * (qj * pir - qi * pjr) * dc3;
        acc[2] += -0.5 * ((3.0 * pir * pjr - r2 * pipj) * dc1 - pir * pjr * dc2);
        acc[3] += -(mqi * qj) * dqq;
        acc[4] += dc3 * (mpir * qj - mqi * pjr);
        acc[5] += -((3.0 * mpir * pjr - r2 * mpipj) * dc1 - mpir * pjr * dc2);
    }
    if (threadIdx.x == 0) {
        acc[6] = lift<T>(0.5 * qi * qi, 0.0);
        acc[7] = lift<T>(0.5 * (pi[0] * pi[0] + pi[1] * pi[1] + pi[2] * pi[2]), 0.0);
        acc[8] = lift<T>(mqi * qi, 0.0);
        acc[9] = lift<T>(mpi[0] * pi[0] + mpi[1] * pi[1] + mpi[2] * pi[2], 0.0);
    }
    block_partials_t<T, 10>(acc, sh, partials);
}

// Gradient with respect to r (Bohr, r = r_j - r_i) of the bilinear form
// B(a, b, r) = a_p . A_pp(r) b_p + (a_p . r) c3 b_q - a_q c3 (r . b_p)
//              - a_q b_q erf(r u_qq) / r
// of one off-diagonal CPIM block (a a row vector, b a column vector).
__device__ __forceinline__ void grad_block_form(const DevParams &P, const double ap[3], double aq,
                                                const double bp[3], double bq, const double r[3], double out[3])
{
    const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2], rr = sqrt(r2);
    const double uqq = P.inv_r_qq, upq = P.inv_r_pq, upp = P.inv_r_pp;
    // charge - charge: grad erf(r u)/r = -A0 r
    const double eqq = exp(-(r2 * uqq * uqq));
    const double A0 = (erf(rr * uqq) - 2.0 * kInvSqrtPi * uqq * rr * eqq) / (r2 * rr);
    // charge - dipole: grad (c3 (a . r)) = -T a, T = A1 (3 r r - r^2 I) - B1 r r
    const double epq = exp(-(r2 * upq * upq));
    const double A1 = (erf(rr * upq) - 2.0 * kInvSqrtPi * upq * rr * epq) / (r2 * r2 * rr);
    const double B1 = 4.0 * kInvSqrtPi * upq * upq * upq * epq / r2;
    const double rap = r[0] * ap[0] + r[1] * ap[1] + r[2] * ap[2];
    const double rbp = r[0] * bp[0] + r[1] * bp[1] + r[2] * bp[2];
    // dipole - dipole: S = c1 (3 (a.r)(b.r) - r^2 a.b) - c2 (a.r)(b.r), A_pp form = -S;
    // (1/r) dc1/dr = 4/sqrt(pi) u^3 e / r^4 - 5 c1 / r^2, (1/r) dc2/dr = -2 u^2 c2 - 2 c2 / r^2
    const double epp = exp(-(r2 * upp * upp));
    const double c1 = (erf(rr * upp) - 2.0 * kInvSqrtPi * upp * rr * epp) / (r2 * r2 * rr);
    const double c2 = 4.0 * kInvSqrtPi * upp * upp * upp * epp / r2;
    const double D1 = 4.0 * kInvSqrtPi * upp * upp * upp * epp / (r2 * r2) - 5.0 * c1 / r2;
    const double D2 = -2.0 * upp * upp * c2 - 2.0 * c2 / r2;
    const double ab = ap[0] * bp[0] + ap[1] * bp[1] + ap[2] * bp[2];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double Ta = A1 * (3.0 * r[k] * rap - r2 * ap[k]) - B1 * r[k] * rap;
        const double Tb = A1 * (3.0 * r[k] * rbp - r2 * bp[k]) - B1 * r[k] * rbp;
        const double gS = c1 * (3.0 * ap[k] * rbp + 3.0 * bp[k] * rap - 2.0 * r[k] * ab) +
                          D1 * r[k] * (3.0 * rap * rbp - r2 * ab) - c2 * (ap[k] * rbp + bp[k] * rap) -
                          D2 * r[k] * rap * rbp;
        out[k] = aq * bq * A0 * r[k] - bq * Ta + aq * Tb - gS;
    }
}

// Adds -scale d/dr [mu^T (A(r) x - b(r))] to (gx, gy, gz): block per metal atom i;
// the metal atom's own entry is written by its block, the permanent charges
// within its cut-off receive theirs by atomic adds.
__global__ void __launch_bounds__(256) k_cpim_adjoint_positions(DevParams P, const double4 *__restrict__ pos4,
                                                                const uint32_t *__restrict__ nbr,
                                                                const int *__restrict__ nnb, int cap,
                                                                const double *__restrict__ x,
                                                                const double *__restrict__ mu, double scale,
                                                                double *gx, double *gy, double *gz)
{
    __shared__ double sh[32 * 3];
    const int i = blockIdx.x, M = P.M, im = P.metal_min + i;
    const double4 pi4 = pos4[im];
    const double xpi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]}, xqi = x[3 * M + i];
    const double mpi[3] = {mu[3 * i], mu[3 * i + 1], mu[3 * i + 2]}, mqi = mu[3 * M + i];
    double acc[3] = {0.0, 0.0, 0.0};  // d Phi / d r_i
    for (int j = threadIdx.x; j < M; j += blockDim.x) {
        if (j == i) continue;
        const double4 pj4 = pos4[P.metal_min + j];
        double r[3] = {pj4.x - pi4.x, pj4.y - pi4.y, pj4.z - pi4.z};
        image(r[0], r[1], r[2], P.box);
        r[0] *= kNm2Bohr;
        r[1] *= kNm2Bohr;
        r[2] *= kNm2Bohr;
        const double nr[3] = {-r[0], -r[1], -r[2]};
        const double xpj[3] = {x[3 * j], x[3 * j + 1], x[3 * j + 2]}, xqj = x[3 * M + j];
        const double mpj[3] = {mu[3 * j], mu[3 * j + 1], mu[3 * j + 2]}, mqj = mu[3 * M + j];
        double g1[3], g2[3];
        grad_block_form(P, mpi, mqi, xpj, xqj, r, g1);   // block (i, j): r = r_j - r_i
        grad_block_form(P, mpj, mqj, xpi, xqi, nr, g2);  // block (j, i): r_i - r_j
#pragma unroll
        for (int k = 0; k < 3; ++k) acc[k] += kNm2Bohr * (g2[k] - g1[k]);
    }
    // -mu^T b: the DSF field and potential of the permanent charges
    // (cpff.c:43-198); d(mu^T b)/dr_i = kConvV f with f the charge-pair force
    // of cpim_charge_pair for (q_ind, p_ind) = (-mu_q, mu_p)
    const uint32_t *row = nbr + (size_t)im * cap;
    const double neg_mq = -mqi;
    for (int k = threadIdx.x; k < nnb[im]; k += blockDim.x) {
        const int j = nb_index(row[k]);
        if (P.is_metal[j]) continue;
        const double4 pj = pos4[j];
        if (pj.w == 0.0) continue;
        double r[3] = {pi4.x - pj.x, pi4.y - pj.y, pi4.z - pj.z};
        image(r[0], r[1], r[2], P.box);
        const double r2 = norm2_exact(r[0], r[1], r[2]);
        if (r2 >= P.rc2) continue;
        double f[3], a0, ec;
        cpim_charge_pair(P, r, r2, pj.w, neg_mq, mpi, f, a0, ec);
#pragma unroll
        for (int a = 0; a < 3; ++a) acc[a] -= kConvV * f[a];
        // dPhi/dr_j = +kConvV f; the gradient takes -dPhi/dr_j
        atomicAdd(gx + j, -scale * kConvV * f[0]);
        atomicAdd(gy + j, -scale * kConvV * f[1]);
        atomicAdd(gz + j, -scale * kConvV * f[2]);
    }
    block_sum<3>(acc, sh);
    if (threadIdx.x == 0) {
        // b_q includes -E_ext . r_i (cpff.c:176-183)
#pragma unroll
        for (int a = 0; a < 3; ++a) acc[a] += kConvV * mqi * P.efield[a];
        gx[im] -= scale * acc[0];
        gy[im] -= scale * acc[1];
        gz[im] -= scale * acc[2];
    }
}

// g = -F (positions gradient of E at fixed x)
__global__ void __launch_bounds__(256) k_neg_forces(int N, const double *__restrict__ fx,
                                                    const double *__restrict__ fy, const double *__restrict__ fz,
                                                    double *gx, double *gy, double *gz)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    gx[k] = -fx[k];
    gy[k] = -fy[k];
    gz[k] = -fz[k];
}

// w = 2 (F - F_target) / (3N) interleaved, partials of sum (F - F_target)^2
__global__ void __launch_bounds__(256) k_force_match_dir(int N, const double *__restrict__ fx,
                                                         const double *__restrict__ fy,
                                                         const double *__restrict__ fz,
                                                         const double *__restrict__ tf, double *wdir,
                                                         double *partials)
{
    __shared__ double sh[32];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double s[1] = {0.0};
    if (k < N) {
        const double d0 = fx[k] - tf[k], d1 = fy[k] - tf[N + k], d2 = fz[k] - tf[2 * (size_t)N + k];
        const double sc = 2.0 / (3.0 * (double)N);
        wdir[3 * k] = sc * d0;
        wdir[3 * k + 1] = sc * d1;
        wdir[3 * k + 2] = sc * d2;
        s[0] = d0 * d0 + d1 * d1 + d2 * d2;
    }
    block_partials<1>(s, sh, partials);
}

// r = b - Ax and partials of (r, r) and (b, b)
__global__ void __launch_bounds__(256) k_adj_residual(int n, const double *__restrict__ b,
                                                      const double *__restrict__ Ax, double *__restrict__ r,
                                                      double *partials)
{
    __shared__ double sh[32 * 2];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double s[2] = {0.0, 0.0};
    if (k < n) {
        const double v = b[k] - Ax[k];
        r[k] = v;
        s[0] = v * v;
        s[1] = b[k] * b[k];
    }
    block_partials<2>(s, sh, partials);
}

__global__ void __launch_bounds__(256) k_adj_axpy(int n, const double *__restrict__ d, double *__restrict__ x)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) x[k] += d[k];
}

// Sum rows of a [rows][k] partials array on the host in a fixed order.
std::vector<double> host_sums(const double *d_partials, int rows, int k, cudaStream_t s)
{
    std::vector<double> h((size_t)rows * k), out(k, 0.0);
    CAPAC_CUDA(cudaMemcpyAsync(h.data(), d_partials, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s));
    CAPAC_CUDA(cudaStreamSynchronize(s));
    for (int r = 0; r < rows; ++r)
        for (int q = 0; q < k; ++q) out[q] += h[(size_t)r * k + q];
    return out;
}

void need_ctx(capac_ctx *c)
{
    if (!c) throw Error(CAPAC_ERR_INVALID, "null context");
}

void need_state(capac_ctx *c)
{
    if (!c->grad_ready)
        throw Error(CAPAC_ERR_INVALID,
                    "gradients need a force evaluation with a solve after the last change of positions, "
                    "induced vector or parameters");
}

void need_partials(capac_ctx *c, size_t doubles)
{
    if (doubles > c->partials_cap) throw Error(CAPAC_ERR_CAPACITY, "partials buffer too small for the gradient sums");
}

void set_widths(capac_ctx *c)
{
    c->c.inv_r_qq = 1.0 / sqrt(2.0 * c->rq * c->rq);
    c->c.inv_r_pq = 1.0 / sqrt(c->rp * c->rp + c->rq * c->rq);
    c->c.inv_r_pp = 1.0 / sqrt(2.0 * c->rp * c->rp);
    c->P.inv_r_qq = c->c.inv_r_qq;
    c->P.inv_r_pq = c->c.inv_r_pq;
    c->P.inv_r_pp = c->c.inv_r_pp;
}

void upload_diag(capac_ctx *c)
{
    const int M = c->M, n = c->n_mat;
    std::vector<double> diag(n, 1.0);
    for (int i = 0; i < M; ++i) {
        diag[3 * i] = diag[3 * i + 1] = diag[3 * i + 2] = c->c.inv_polar;
        diag[3 * M + i] = -c->c.inv_capac;
    }
    CAPAC_CUDA(cudaMemcpyAsync(c->diag, diag.data(), sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
    CAPAC_CUDA(cudaStreamSynchronize(c->stream));
}

// Solver chunks captured as CUDA graphs hold the parameters they were
// launched with: drop them so the next solve captures afresh.
void drop_graphs(capac_ctx *c)
{
    CAPAC_CUDA(cudaStreamSynchronize(c->stream));
    for (auto &g : c->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        for (auto &e : g.ev)
            if (e) cudaEventDestroy(e);
    }
    c->graphs.clear();
}

// Workspace: 7 vectors of n_mat (g, gd, mu, nu, r, d, Ax) and 2 of 3N
// (direction or position gradient, force targets), allocated at the first
// gradient call.
enum { GW_G = 0, GW_GD, GW_MU, GW_NU, GW_R, GW_D, GW_AX, GW_NVEC };
double *gw_vec(capac_ctx *c, int k) { return c->gw + (size_t)k * c->n_mat; }
double *gw_dir(capac_ctx *c) { return c->gw + (size_t)GW_NVEC * c->n_mat; }
double *gw_target(capac_ctx *c) { return gw_dir(c) + (size_t)3 * c->N; }

void ensure_workspace(capac_ctx *c)
{
    if (c->gw) return;
    const size_t doubles = (size_t)GW_NVEC * c->n_mat + (size_t)6 * c->N;
    CAPAC_CUDA(cudaMalloc(&c->gw, sizeof(double) * doubles));
    CAPAC_CUDA(cudaMemsetAsync(c->gw, 0, sizeof(double) * doubles, c->stream));
}

// Solve A y = rhs in FP64 by iterative refinement around the context's
// BiCGSTAB (FP64 residual from positions each sweep).  Returns the sweeps.
int adjoint_solve(capac_ctx *c, const double *rhs, double *y)
{
    const int n = c->n_mat, nbv = (int)grid_for(n, 256);
    cudaStream_t s = c->stream;
    need_partials(c, (size_t)nbv * 2);
    double *r = gw_vec(c, GW_R), *d = gw_vec(c, GW_D), *Ax = gw_vec(c, GW_AX);
    CAPAC_CUDA(cudaMemsetAsync(y, 0, sizeof(double) * n, s));
    for (int sweep = 0;; ++sweep) {
        spmv_free(c, y, Ax);
        k_adj_residual<<<nbv, 256, 0, s>>>(n, rhs, Ax, r, c->partials);
        ++c->launches;
        const std::vector<double> rb = host_sums(c->partials, nbv, 2, s);
        if (rb[1] == 0.0 || rb[0] <= kAdjointTol * kAdjointTol * rb[1]) return sweep;
        if (sweep == kAdjointSweeps) {
            char msg[160];
            snprintf(msg, sizeof msg, "adjoint solve stopped at relative residual %.3e", sqrt(rb[0] / rb[1]));
            throw Error(CAPAC_ERR_NOT_CONVERGED, msg);
        }
        CAPAC_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * n, s));
        bicgstab_core(c, r, d, 1.0e-10, 1.0e-300);  // reduce the residual by 1e-5
        k_adj_axpy<<<nbv, 256, 0, s>>>(n, d, y);
        ++c->launches;
    }
}

// The parameter gradient from the primitive derivatives
// prim = d/d(u_qq, u_pq, u_pp, 1/C, 1/alpha): out = d/d(C, alpha, R_q, R_p).
// R_q follows C and R_p follows alpha unless they were set on their own.
void chain_cpim(const capac_ctx *c, const double prim[5], double out[4])
{
    const double uqq = c->P.inv_r_qq, upq = c->P.inv_r_pq, upp = c->P.inv_r_pp;
    const double upq3 = upq * upq * upq;
    const double d_rq = prim[0] * (-uqq / c->rq) + prim[1] * (-c->rq * upq3);
    const double d_rp = prim[2] * (-upp / c->rp) + prim[1] * (-c->rp * upq3);
    out[2] = d_rq;
    out[3] = d_rp;
    out[0] = prim[3] * (-1.0 / (c->capac * c->capac)) + (c->rq_tied ? d_rq * sqrt(2.0 / kPi) : 0.0);
    out[1] = prim[4] * (-1.0 / (c->polar * c->polar)) + (c->rp_tied ? d_rp * c->rp / (3.0 * c->polar) : 0.0);
}

// dE/d(eps, c, a, n, m) from the Sutton-Chen sums (or their derivatives).
void qsc_grad(const capac_ctx *c, const double S[4], double out[5])
{
    const double eps = c->P.qsc_eps, cc = c->P.qsc_c, a = c->P.qsc_a, nn = c->P.qsc_n, mm = c->P.qsc_m;
    out[0] = S[0] - cc * S[1];
    out[1] = -eps * S[1];
    out[2] = eps * (nn * S[0] - 0.5 * cc * mm * S[1]) / a;
    out[3] = eps * S[2];
    out[4] = -eps * cc * S[3];
}

// Sutton-Chen sums (4 values, then 4 derivatives along the direction when dual)
std::vector<double> qsc_sums(capac_ctx *c, bool dual)
{
    const unsigned grid = grid_for((long)c->M * 32, 256);
    const int k = dual ? 8 : 4;
    need_partials(c, (size_t)grid * k);
    if (dual)
        k_qsc_param_sums<Dual><<<grid, 256, 0, c->stream>>>(c->P, c->pos4, gw_dir(c), c->partials);
    else
        k_qsc_param_sums<double><<<grid, 256, 0, c->stream>>>(c->P, c->pos4, nullptr, c->partials);
    ++c->launches;
    return host_sums(c->partials, (int)grid, k, c->stream);
}

std::vector<double> cpim_sums(capac_ctx *c, const double *mu, bool dual)
{
    const int k = dual ? 20 : 10;
    need_partials(c, (size_t)c->M * k);
    if (dual)
        k_cpim_param_sums<Dual><<<c->M, 256, 0, c->stream>>>(c->P, c->pos4, gw_dir(c), c->vec_pq, mu, c->partials);
    else
        k_cpim_param_sums<double><<<c->M, 256, 0, c->stream>>>(c->P, c->pos4, nullptr, c->vec_pq, mu, c->partials);
    ++c->launches;
    return host_sums(c->partials, c->M, k, c->stream);
}

void launch_dx(capac_ctx *c, bool dual)
{
    double *g = gw_vec(c, GW_G), *gd = gw_vec(c, GW_GD);
    const size_t n = c->n_mat;
    CAPAC_CUDA(cudaMemsetAsync(g, 0, sizeof(double) * n, c->stream));
    CAPAC_CUDA(cudaMemsetAsync(gd, 0, sizeof(double) * n, c->stream));
    if (dual)
        k_cpim_dx<Dual><<<c->M, 256, 0, c->stream>>>(c->P, c->pos4, gw_dir(c), c->nbr, c->nnb, c->cap, c->vec_pq,
                                                     g, gd);
    else
        k_cpim_dx<double><<<c->M, 256, 0, c->stream>>>(c->P, c->pos4, nullptr, c->nbr, c->nnb, c->cap, c->vec_pq,
                                                       g, nullptr);
    ++c->launches;
}

}  // namespace

void param_defaults(capac_ctx *c, const capac_desc *d)
{
    c->capac = d->cpff_capac;
    c->polar = d->cpff_polar;
    c->rq = sqrt(2.0 / kPi) * d->cpff_capac;
    c->rp = pow(sqrt(2.0 / kPi) * d->cpff_polar / 3.0, 1.0 / 3.0);
    c->rq_tied = c->rp_tied = true;
}

}  // namespace capac

using namespace capac;

extern "C" {

int capac_param_get(capac_ctx *c, const char *name, double *value)
{
    return guard([&] {
        need_ctx(c);
        if (!name || !value) throw Error(CAPAC_ERR_INVALID, "null argument");
        const std::string n(name);
        if (n == "cpff_capac") *value = c->capac;
        else if (n == "cpff_polar") *value = c->polar;
        else if (n == "cpim_rq") *value = c->rq;
        else if (n == "cpim_rp") *value = c->rp;
        else if (n == "cpim_rq_tied") *value = c->rq_tied ? 1.0 : 0.0;
        else if (n == "cpim_rp_tied") *value = c->rp_tied ? 1.0 : 0.0;
        else if (n == "qsc_eps") *value = c->P.qsc_eps;
        else if (n == "qsc_c") *value = c->P.qsc_c;
        else if (n == "qsc_a") *value = c->P.qsc_a;
        else if (n == "qsc_n") *value = c->P.qsc_n;
        else if (n == "qsc_m") *value = c->P.qsc_m;
        else throw Error(CAPAC_ERR_INVALID, "unknown parameter " + n);
    });
}

int capac_param_set(capac_ctx *c, const char *name, double value)
{
    return guard([&] {
        need_ctx(c);
        if (!name) throw Error(CAPAC_ERR_INVALID, "null argument");
        if (!std::isfinite(value)) throw Error(CAPAC_ERR_INVALID, "parameter value is not finite");
        const std::string n(name);
        const bool cpim = n == "cpff_capac" || n == "cpff_polar" || n == "cpim_rq" || n == "cpim_rp";
        const bool width = n == "cpim_rq" || n == "cpim_rp";
        if (cpim && c->M == 0) throw Error(CAPAC_ERR_INVALID, "no metal atoms");
        if (cpim && (value < 0.0 || (value == 0.0 && !width)))
            throw Error(CAPAC_ERR_INVALID, n + (width ? " must not be negative" : " must be positive"));
        if (n == "cpff_capac") {  // a tied width follows, as the reference derives it
            c->capac = value;
            c->c.inv_capac = c->P.inv_capac = 1.0 / value;
            if (c->rq_tied) c->rq = sqrt(2.0 / kPi) * value;
            set_widths(c);
            upload_diag(c);
        } else if (n == "cpff_polar") {
            c->polar = value;
            c->c.inv_polar = c->P.inv_polar = 1.0 / value;
            if (c->rp_tied) c->rp = pow(sqrt(2.0 / kPi) * value / 3.0, 1.0 / 3.0);
            set_widths(c);
            upload_diag(c);
        } else if (n == "cpim_rq") {  // a width decouples from C; 0 ties it again
            c->rq_tied = value == 0.0;
            c->rq = c->rq_tied ? sqrt(2.0 / kPi) * c->capac : value;
            set_widths(c);
        } else if (n == "cpim_rp") {
            c->rp_tied = value == 0.0;
            c->rp = c->rp_tied ? pow(sqrt(2.0 / kPi) * c->polar / 3.0, 1.0 / 3.0) : value;
            set_widths(c);
        } else if (n == "qsc_eps") c->P.qsc_eps = value;
        else if (n == "qsc_c") c->P.qsc_c = value;
        else if (n == "qsc_a") c->P.qsc_a = value;
        else if (n == "qsc_n") c->P.qsc_n = value;
        else if (n == "qsc_m") c->P.qsc_m = value;
        else throw Error(CAPAC_ERR_INVALID, "unknown parameter " + n);
        c->precond_age = 0;  // the matrix changed: fresh preconditioner blocks
        c->grad_ready = false;
        drop_graphs(c);
    });
}

int capac_energy_grad(capac_ctx *c, double *grad, double *gx, double *gy, double *gz)
{
    return guard([&] {
        need_ctx(c);
        need_state(c);
        const bool pos = gx && gy && gz;
        if (!grad && !pos) throw Error(CAPAC_ERR_INVALID, "nothing requested");
        ensure_workspace(c);
        cudaStream_t s = c->stream;
        double *dgx = gw_dir(c), *dgy = dgx + c->N, *dgz = dgy + c->N;  // device gradient (3 planes)
        if (pos) {
            k_neg_forces<<<grid_for(c->N, 256), 256, 0, s>>>(c->N, c->fx, c->fy, c->fz, dgx, dgy, dgz);
            ++c->launches;
        }
        double out[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (c->M > 0) {
            const std::vector<double> S = qsc_sums(c, false);
            qsc_grad(c, S.data(), out + 4);
        }
        if (c->M > 0 && c->use_cpff) {
            launch_dx(c, false);
            double *mu = gw_vec(c, GW_MU);
            adjoint_solve(c, gw_vec(c, GW_G), mu);
            if (grad) {
                const std::vector<double> v = cpim_sums(c, mu, false);
                const double prim[5] = {kFqqAu1 * v[0] - v[3], kFqqAu1 * v[1] - v[4], kFqqAu1 * v[2] - v[5],
                                        kFqqAu1 * v[6] + v[8], kFqqAu1 * v[7] - v[9]};
                chain_cpim(c, prim, out);
            }
            if (pos) {
                k_cpim_adjoint_positions<<<c->M, 256, 0, s>>>(c->P, c->pos4, c->nbr, c->nnb, c->cap, c->vec_pq, mu,
                                                              1.0, dgx, dgy, dgz);
                ++c->launches;
            }
        }
        if (grad)
            for (int k = 0; k < 9; ++k) grad[k] = out[k];
        if (pos) {
            const size_t bytes = sizeof(double) * c->N;
            CAPAC_CUDA(cudaMemcpyAsync(gx, dgx, bytes, cudaMemcpyDeviceToHost, s));
            CAPAC_CUDA(cudaMemcpyAsync(gy, dgy, bytes, cudaMemcpyDeviceToHost, s));
            CAPAC_CUDA(cudaMemcpyAsync(gz, dgz, bytes, cudaMemcpyDeviceToHost, s));
            CAPAC_CUDA(cudaStreamSynchronize(s));
        }
    });
}

int capac_force_match_grad(capac_ctx *c, const double *tfx, const double *tfy, const double *tfz, double *loss,
                           double *grad, double *gx, double *gy, double *gz)
{
    return guard([&] {
        need_ctx(c);
        need_state(c);
        if (!tfx || !tfy || !tfz || !loss) throw Error(CAPAC_ERR_INVALID, "null argument");
        const bool pos = gx && gy && gz;
        ensure_workspace(c);
        cudaStream_t s = c->stream;
        const int N = c->N;
        double *tf = gw_target(c);
        const size_t bytes = sizeof(double) * N;
        CAPAC_CUDA(cudaMemcpyAsync(tf, tfx, bytes, cudaMemcpyHostToDevice, s));
        CAPAC_CUDA(cudaMemcpyAsync(tf + N, tfy, bytes, cudaMemcpyHostToDevice, s));
        CAPAC_CUDA(cudaMemcpyAsync(tf + 2 * (size_t)N, tfz, bytes, cudaMemcpyHostToDevice, s));
        const unsigned nb = grid_for(N, 256);
        need_partials(c, nb);
        k_force_match_dir<<<nb, 256, 0, s>>>(N, c->fx, c->fy, c->fz, tf, gw_dir(c), c->partials);
        ++c->launches;
        *loss = host_sums(c->partials, (int)nb, 1, s)[0] / (3.0 * N);
        double out[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (grad && c->M > 0) {
            const std::vector<double> S = qsc_sums(c, true);  // [4..7]: derivatives along w
            qsc_grad(c, S.data() + 4, out + 4);
            for (int k = 4; k < 9; ++k) out[k] = -out[k];
        }
        const bool cpim = c->M > 0 && c->use_cpff;
        double *nu = gw_vec(c, GW_NU);
        if (cpim) {
            launch_dx(c, true);  // GW_GD = dPsi/dx
            adjoint_solve(c, gw_vec(c, GW_GD), nu);
        }
        if (grad && cpim) {
            const std::vector<double> v = cpim_sums(c, nu, true);  // [0..9] values with nu, [10..19] derivatives
            // dPsi/dphi = dPsi/dphi|_x - nu^T (dA/dphi) x; dL/dphi = -dPsi/dphi
            const double dpsi[5] = {kFqqAu1 * v[10] - v[3], kFqqAu1 * v[11] - v[4], kFqqAu1 * v[12] - v[5], v[8],
                                    -v[9]};
            double prim[5];
            for (int k = 0; k < 5; ++k) prim[k] = -dpsi[k];
            chain_cpim(c, prim, out);
        }
        if (grad)
            for (int k = 0; k < 9; ++k) grad[k] = out[k];
        if (pos) {
            // dL/dr = -dPsi/dr|_x + d/dr [nu^T (A x - b)] = dF/de (along w) + dPhi_nu/dr;
            // the targets are no longer needed: their planes take the gradient
            double *dgx = tf, *dgy = tf + N, *dgz = tf + 2 * (size_t)N;
            CAPAC_CUDA(cudaMemsetAsync(tf, 0, sizeof(double) * 3 * (size_t)N, s));
            launch_force_derivative(c, gw_dir(c), dgx, dgy, dgz, gw_vec(c, GW_R), gw_vec(c, GW_D));
            if (cpim) {
                k_cpim_adjoint_positions<<<c->M, 256, 0, s>>>(c->P, c->pos4, c->nbr, c->nnb, c->cap, c->vec_pq, nu,
                                                              -1.0, dgx, dgy, dgz);
                ++c->launches;
            }
            CAPAC_CUDA(cudaMemcpyAsync(gx, dgx, bytes, cudaMemcpyDeviceToHost, s));
            CAPAC_CUDA(cudaMemcpyAsync(gy, dgy, bytes, cudaMemcpyDeviceToHost, s));
            CAPAC_CUDA(cudaMemcpyAsync(gz, dgz, bytes, cudaMemcpyDeviceToHost, s));
            CAPAC_CUDA(cudaStreamSynchronize(s));
        }
    });
}

}  // extern "C"
