// Nonbonded pair forces over the full neighbour list (FP64 and mixed).
//
// Per pair this is compute_nonbonded / compute_erf_vdw / compute_morse /
// compute_buckingham (force.c:591-816) as dispatched by mpi_nonb_pair
// (force.c:1476-1528): LJ shifted force + damped shifted force Coulomb
// (funct 1), Buckingham (2), Morse (3), erf-damped vdW (4).
//
// One warp owns an atom i at a time (grid-stride over atoms) and walks its
// list; every pair is visited from both ends, so forces need no atomics and
// each end adds half of the pair energy and virial.  The cut-off test is done
// in FP64 with the reference's r^2 rounding, so both precisions keep exactly
// the reference's pair set.  Candidates that pass it are compacted into a
// per-warp queue in shared memory and the pair math runs on full warps.
//
// The same traversal adds, on each charged non-metal atom, the force from the
// induced charges and dipoles of metal neighbours inside the cut-off: the
// water side of the metal-water loop of mpi_cpff_force (cpff.c:578-724).  The
// metal side, with energies [10],[11] and the virial, is k_cpim_metal.
//
// Mixed path: coordinate differences and the cut-off in FP64, the pair terms
// in FP32, force sums per lane with Kahan compensation, energies and virial
// gathered per atom in FP32 and summed across atoms in FP64.
#include <algorithm>

#include "terms.cuh"

namespace capac {

namespace {

constexpr int kPairWarps = 8;  // warps per block

// FP32 constants of the run.
struct PairConstsF {
    float rc, inv_rc, inv_rc12, inv_rc6, alpha, a2_sqrtpi, w_const, w_erfc_arcut, fqq, rc2;
    int use_vdw, use_coulomb;
};

// One type pair in FP32, with the shifted-force constants of funct 1
// precomputed: fc = 12 c12 / rc^12 - 6 c6 / rc^6, es = c12 / rc^12 - c6 / rc^6.
struct TypePairF {
    float c6, c12, a, b, fc, es;
    int fn, pad;
};

__device__ __forceinline__ TypePairF make_type_pair_f(const DevParams &P, const PairConstsF &K, int k)
{
    const double4 pd = P.nb_par[k];
    TypePairF t;
    t.c6 = (float)pd.x;
    t.c12 = (float)pd.y;
    t.a = (float)pd.z;
    t.b = (float)pd.w;
    t.fc = (float)(12.0 * pd.y * P.inv_rc12 - 6.0 * pd.x * P.inv_rc6);
    t.es = (float)(pd.y * P.inv_rc12 - pd.x * P.inv_rc6);
    t.fn = P.nb_funct[k];
    t.pad = 0;
    return t;
}

// 1/x by the hardware approximation (rcp.approx.ftz.f32, within about one
// ulp); 1 <= x <= 3.5 here.
__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// erfc(x) for 0 <= x in FP32 as exp(-x^2) R(x), with R(x) = erfc(x) exp(x^2)
// (the scaled complementary error function) fitted on [0, 5] by a degree-9
// polynomial in t = 1 / (1 + x / 2), least squares in relative error
// (relative error of R below 4e-8 in exact arithmetic, 3e-7 in FP32).  The
// caller has exp(-x^2) already, for the Gaussian term of the same pair.
// Beyond x = 5 the library erfcf.
__device__ __forceinline__ float erfc_from_gauss_f(float x, float gauss)
{
    if (x >= 5.0f) return erfcf(x);
    const float t = rcp_approx(fmaf(0.5f, x, 1.0f));
    float r = -3.71903017e-02f;
    r = fmaf(r, t, 1.64898831e-01f);
    r = fmaf(r, t, -2.03180485e-01f);
    r = fmaf(r, t, -1.05265965e-01f);
    r = fmaf(r, t, 2.97262422e-01f);
    r = fmaf(r, t, 2.51787793e-02f);
    r = fmaf(r, t, 3.06175054e-01f);
    r = fmaf(r, t, 2.68365236e-01f);
    r = fmaf(r, t, 2.83852814e-01f);
    r = fmaf(r, t, -9.64172679e-05f);
    return gauss * r;
}

// FP64 pair term (force on j = f * rvec), reference formulas with the
// divisions by r, r^2, r^6, r^12 turned into products with 1/r.
__device__ __forceinline__ double pair_term(const DevParams &P, int k, double qi, double qj, double r2,
                                            double &e_qq, double &e_vdw)
{
    const int fn = P.nb_funct[k];
    const double4 pr = P.nb_par[k];  // (c6, c12, a, b)
    const double r = sqrt(r2), rinv = 1.0 / r, r2inv = rinv * rinv;
    if (fn == 4) {  // compute_erf_vdw, force.c:591-632 (width = a)
        if (pr.x != 0.0 || pr.y != 0.0) {
            const double r6inv = r2inv * r2inv * r2inv;
            const double a12 = pr.y * r6inv * r6inv, a6 = pr.x * r6inv, u = r / pr.z, eu = erf(u);
            e_vdw += (a12 - a6) * eu;
            return ((12.0 * a12 - 6.0 * a6) * rinv * eu - (a12 - a6) * 2.0 * kInvSqrtPi * exp(-u * u) / pr.z) * rinv;
        }
        return 0.0;
    }
    if (fn == 3) {  // compute_morse, force.c:639-667 (D = A, a = B, R = C6)
        const double e1 = exp(-pr.w * (r - pr.x)), e2 = e1 * e1;
        e_vdw += pr.z * (e2 - 2.0 * e1);
        return 2.0 * pr.z * pr.w * (e2 - e1) * rinv;
    }
    if (fn == 2) {  // compute_buckingham, force.c:674-703 (A, B, C6)
        const double r6inv = r2inv * r2inv * r2inv, eb = exp(-pr.w * r);
        e_vdw += pr.z * eb - pr.x * r6inv;
        return pr.z * eb * pr.w * rinv - 6.0 * pr.x * r6inv * r2inv;
    }
    // funct 1: compute_nonbonded, force.c:710-816 (not a 1-4 pair)
    double f = 0.0;
    if (pr.x != 0.0 || pr.y != 0.0) {
        const double r6inv = r2inv * r2inv * r2inv, r12inv = r6inv * r6inv;
        if (P.use_vdw == 1) {
            const double fr = 12.0 * pr.y * r12inv - 6.0 * pr.x * r6inv;
            const double fc = 12.0 * pr.y * P.inv_rc12 - 6.0 * pr.x * P.inv_rc6;
            f = (fr - fc) * r2inv;
            e_vdw += (pr.y * r12inv - pr.x * r6inv) + (r - P.rc) * fc / P.rc - (pr.y * P.inv_rc12 - pr.x * P.inv_rc6);
        } else {
            f = (pr.y * 2.0 * r12inv - pr.x * r6inv) * 6.0 * r2inv;
            e_vdw += pr.y * r12inv - pr.x * r6inv;
        }
    }
    if (qi != 0.0 && qj != 0.0) {
        const double qq = kFQQ * qi * qj;
        if (P.use_coulomb == 1) {
            const double a = P.w_alpha, ec = erfc(a * r);
            f += qq * ((ec * r2inv + P.w_a2_sqrtpi * exp(-a * a * r2) * rinv) - P.w_const) * rinv;
            e_qq += qq * (ec * rinv - P.w_erfc_arcut + P.w_const * (r - P.rc));
        } else {
            f += qq * r2inv * rinv;
            e_qq += qq * rinv;
        }
    }
    return f;
}

// The same terms in FP32, from the FP32 type pair.
__device__ __forceinline__ float pair_term_f(const PairConstsF &K, const TypePairF &tp, float qi, float qj, float r2,
                                             float &e_qq, float &e_vdw)
{
    const int fn = tp.fn;
    const float c6 = tp.c6, c12 = tp.c12, pa = tp.a, pb = tp.b;
    const float rinv = rsqrtf(r2), r = r2 * rinv, r2inv = rinv * rinv;
    if (fn == 4) {
        if (c6 != 0.f || c12 != 0.f) {
            const float r6inv = r2inv * r2inv * r2inv;
            const float a12 = c12 * r6inv * r6inv, a6 = c6 * r6inv, u = r / pa, eu = erff(u);
            e_vdw += (a12 - a6) * eu;
            return ((12.f * a12 - 6.f * a6) * rinv * eu - (a12 - a6) * 2.f * (float)kInvSqrtPi * expf(-u * u) / pa) *
                   rinv;
        }
        return 0.f;
    }
    if (fn == 3) {
        const float e1 = expf(-pb * (r - c6)), e2 = e1 * e1;
        e_vdw += pa * (e2 - 2.f * e1);
        return 2.f * pa * pb * (e2 - e1) * rinv;
    }
    if (fn == 2) {
        const float r6inv = r2inv * r2inv * r2inv, eb = expf(-pb * r);
        e_vdw += pa * eb - c6 * r6inv;
        return pa * eb * pb * rinv - 6.f * c6 * r6inv * r2inv;
    }
    float f = 0.f;
    if (c6 != 0.f || c12 != 0.f) {
        const float r6inv = r2inv * r2inv * r2inv, r12inv = r6inv * r6inv;
        if (K.use_vdw == 1) {
            const float fr = 12.f * c12 * r12inv - 6.f * c6 * r6inv;
            f = (fr - tp.fc) * r2inv;
            e_vdw += (c12 * r12inv - c6 * r6inv) + (r - K.rc) * tp.fc * K.inv_rc - tp.es;
        } else {
            f = (c12 * 2.f * r12inv - c6 * r6inv) * 6.f * r2inv;
            e_vdw += c12 * r12inv - c6 * r6inv;
        }
    }
    if (qi != 0.f && qj != 0.f) {
        const float qq = K.fqq * qi * qj;
        if (K.use_coulomb == 1) {
            const float ar = K.alpha * r, eg = expf(-ar * ar), ec = erfc_from_gauss_f(ar, eg);
            f += qq * ((ec * r2inv + K.a2_sqrtpi * eg * rinv) - K.w_const) * rinv;
            e_qq += qq * (ec * rinv - K.w_erfc_arcut + K.w_const * (r - K.rc));
        } else {
            f += qq * r2inv * rinv;
            e_qq += qq * rinv;
        }
    }
    return f;
}

// CPIM force on a metal atom from a permanent charge (the atom receives the
// opposite), FP32; r = metal - atom (cpim_charge_pair in FP32).
__device__ __forceinline__ void cpim_charge_pair_f(const PairConstsF &K, const float r[3], float r2, float q_perm,
                                                   float q_ind, const float p[3], float f[3])
{
    const float rinv = rsqrtf(r2), rr = r2 * rinv, r2inv = rinv * rinv;
    float a0, ec = 0.f, eg = 0.f;
    if (K.use_coulomb == 1) {
        const float ar = K.alpha * rr;
        eg = expf(-ar * ar);
        ec = erfc_from_gauss_f(ar, eg);
        a0 = (ec * r2inv + K.a2_sqrtpi * eg * rinv - K.w_const) * rinv;
    } else {
        a0 = r2inv * rinv;
    }
    const float s = K.fqq * q_perm;
#pragma unroll
    for (int a = 0; a < 3; ++a) f[a] = a0 * r[a] * s * q_ind;
    const float pr = p[0] * r[0] + p[1] * r[1] + p[2] * r[2];
    const float sp = s / (float)kNm2Bohr;
    const float ir3 = r2inv * rinv, ir5 = ir3 * r2inv;
    if (K.use_coulomb == 1) {
        const float al3 = K.alpha * K.alpha * K.alpha;
        const float a1 = ir5 * (ec + K.a2_sqrtpi * rr * eg);
        const float b1 = 4.f * (float)kInvSqrtPi * al3 * r2inv * eg;
        const float c1 = K.w_const * ir3;
        // sum_a T_ab p_a, T_ab = a1 (3 r_a r_b - d_ab r^2) + b1 r_a r_b - c1 (r_a r_b - d_ab r^2)
#pragma unroll
        for (int b = 0; b < 3; ++b)
            f[b] -= (a1 * (3.f * pr * r[b] - p[b] * r2) + b1 * pr * r[b] - c1 * (pr * r[b] - p[b] * r2)) * sp;
    } else {
#pragma unroll
        for (int b = 0; b < 3; ++b) f[b] -= (3.f * pr * r[b] - p[b] * r2) * ir5 * sp;
    }
}

// Per-lane force accumulator: plain FP64, or Kahan-compensated FP32.
template <typename Real>
struct Acc;
template <>
struct Acc<double> {
    double s = 0.0;
    __device__ __forceinline__ void add(double v) { s += v; }
    __device__ __forceinline__ double value() const { return s; }
};
template <>
struct Acc<float> {
    float s = 0.f, c = 0.f;
    __device__ __forceinline__ void add(float v)
    {
        const float y = v - c;
        const float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

// A candidate inside the cut-off, parked in the warp's queue: FP64 record
// (48 B) for the FP64 path, FP32 record (24 B) for the mixed path.
template <typename Real>
struct Cand;
template <>
struct Cand<double> {
    double dx, dy, dz, r2, qj;
    uint32_t e;
    int pad;
};
template <>
struct Cand<float> {
    float dx, dy, dz, r2, qj;
    uint32_t e;
};

// Type-pair tables staged in shared memory when the type count allows.
constexpr int kSmemTypes = 16;

// Candidate chunks of 32 whose list entries and positions are loaded before
// any is tested: more loads in flight per warp.
template <typename Real>
struct Batch {
    static constexpr int N = 2;
};

// One warp per atom i (grid-stride); see the file comment.
template <typename Real, bool NONBONDED, bool CPIM>
__global__ void __launch_bounds__(kPairWarps * 32, sizeof(Real) == 4 ? 3 : 2) k_pair(DevParams P, PairConstsF K, const double4 *__restrict__ pos4,
                                                           const uint32_t *__restrict__ nbr,
                                                           const int *__restrict__ nnb, int cap,
                                                           const double *__restrict__ vec_pq, double *__restrict__ fx,
                                                           double *__restrict__ fy, double *__restrict__ fz,
                                                           double *__restrict__ partials)
{
    constexpr int NB = Batch<Real>::N;
    __shared__ Cand<Real> queue[kPairWarps][64];
    __shared__ double sh[32 * 11];
    __shared__ double wacc[kPairWarps][8];  // per warp: e_qq, e_vdw, virial xx xy xz yy yz zz
    // type-pair table: double4 parameters (FP64) or TypePairF records (mixed), 32 B each
    __shared__ __align__(16) unsigned char s_tab[kSmemTypes * kSmemTypes * 32];
    __shared__ int s_fn[kSmemTypes * kSmemTypes];
    __shared__ unsigned char s_metal[kSmemTypes];
    double4 *s_par = reinterpret_cast<double4 *>(s_tab);
    TypePairF *s_tpf = reinterpret_cast<TypePairF *>(s_tab);
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    Cand<Real> *Q = queue[wib];
    if (lane < 8) wacc[wib][lane] = 0.0;
    const bool smem_types = P.n_types <= kSmemTypes;
    if (smem_types) {
        const int nt2 = P.n_types * P.n_types;
        for (int k = threadIdx.x; k < nt2; k += blockDim.x) {
            if constexpr (sizeof(Real) == 8) s_par[k] = P.nb_par[k];
            else s_tpf[k] = make_type_pair_f(P, K, k);
            s_fn[k] = P.nb_funct[k];
        }
        for (int k = threadIdx.x; k < P.n_types; k += blockDim.x) s_metal[k] = P.type_metal[k];
    }
    __syncthreads();
    // the type-pair table as the pair terms read it
    DevParams Pt = P;
    if (smem_types) {
        Pt.nb_par = s_par;
        Pt.nb_funct = s_fn;
    }
    const bool metal_by_type = smem_types && P.metal_by_type;
    const int stride = gridDim.x * kPairWarps;
    for (int i = blockIdx.x * kPairWarps + wib; i < P.N; i += stride) {
        const double4 pi = pos4[i];
        const int trow = P.type[i] * P.n_types;
        const bool cpim_i = CPIM && P.is_metal[i] == 0 && pi.w != 0.0;
        const int n = nnb[i];
        const uint32_t *row = nbr + (size_t)i * cap;
        Acc<Real> f0, f1, f2;
        Real e_qq = 0, e_vdw = 0;
        Real v[6];  // the pair virial is symmetric: xx xy xz yy yz zz
#pragma unroll
        for (int q = 0; q < 6; ++q) v[q] = 0;

        auto process = [&](const Cand<Real> &c) {
            const Real dx = c.dx, dy = c.dy, dz = c.dz;
            if (NONBONDED) {
                Real f;
                if constexpr (sizeof(Real) == 8)
                    f = pair_term(Pt, trow + nb_type(c.e), pi.w, c.qj, c.r2, e_qq, e_vdw);
                else
                    f = pair_term_f(K, smem_types ? s_tpf[trow + nb_type(c.e)] : make_type_pair_f(P, K, trow + nb_type(c.e)),
                                    (float)pi.w, c.qj, c.r2, e_qq, e_vdw);
                const Real gx = f * dx, gy = f * dy, gz = f * dz;
                f0.add(-gx);
                f1.add(-gy);
                f2.add(-gz);
                v[0] -= dx * gx; v[1] -= dx * gy; v[2] -= dx * gz;
                v[3] -= dy * gy; v[4] -= dy * gz; v[5] -= dz * gz;
            }
            if (cpim_i) {
                const int j = nb_index(c.e);
                const bool mj = metal_by_type ? s_metal[nb_type(c.e)] != 0 : P.is_metal[j] != 0;
                if (mj) {
                    const int jm = j - P.metal_min;
                    if constexpr (sizeof(Real) == 8) {
                        const double r[3] = {c.dx, c.dy, c.dz};  // metal - atom
                        const double p[3] = {vec_pq[3 * jm], vec_pq[3 * jm + 1], vec_pq[3 * jm + 2]};
                        double g[3], a0, ec;
                        cpim_charge_pair(P, r, c.r2, pi.w, vec_pq[3 * P.M + jm], p, g, a0, ec);
                        f0.add(-g[0]);
                        f1.add(-g[1]);
                        f2.add(-g[2]);
                    } else {
                        const float r[3] = {c.dx, c.dy, c.dz};
                        const float p[3] = {(float)vec_pq[3 * jm], (float)vec_pq[3 * jm + 1],
                                            (float)vec_pq[3 * jm + 2]};
                        float g[3];
                        cpim_charge_pair_f(K, r, c.r2, (float)pi.w, (float)vec_pq[3 * P.M + jm], p, g);
                        f0.add(-g[0]);
                        f1.add(-g[1]);
                        f2.add(-g[2]);
                    }
                }
            }
        };

        int qn = 0;  // queue fill, warp-uniform
        // list entries are loaded one batch ahead (the list streams from
        // HBM once per step, evict-first)
        uint32_t nxt[NB];
#pragma unroll
        for (int u = 0; u < NB; ++u) {
            const int k = u * 32 + lane;
            nxt[u] = k < n ? __ldcs(row + k) : 0u;
        }
        for (int base = 0; base < n; base += 32 * NB) {
            uint32_t ev[NB];
            bool valid[NB];
#pragma unroll
            for (int u = 0; u < NB; ++u) {
                valid[u] = base + u * 32 + lane < n;
                ev[u] = nxt[u];
                const int k = base + (NB + u) * 32 + lane;
                nxt[u] = k < n ? __ldcs(row + k) : 0u;
            }
            double4 pj[NB];
#pragma unroll
            for (int u = 0; u < NB; ++u)
                if (valid[u]) pj[u] = pos4[nb_index(ev[u])];
#pragma unroll
            for (int u = 0; u < NB; ++u) {
                bool ok = false;
                Cand<Real> c;
                if (valid[u]) {
                    double dx = pj[u].x - pi.x, dy = pj[u].y - pi.y, dz = pj[u].z - pi.z;
                    image(dx, dy, dz, P.box);
                    if constexpr (sizeof(Real) == 8) {
                        // the reference's rounding of r^2: the FP64 pair set is the reference's
                        const double r2 = norm2_exact(dx, dy, dz);
                        ok = r2 < P.rc2;
                        c.r2 = r2;
                    } else {
                        // mixed: r^2 and the cut-off in FP32 from the FP64 minimum-image
                        // difference; pairs within rounding of the cut-off contribute
                        // nothing (shifted force and energy vanish there)
                        const float fx = (float)dx, fy = (float)dy, fz = (float)dz;
                        const float r2 = fmaf(fz, fz, fmaf(fy, fy, fx * fx));
                        ok = r2 < K.rc2;
                        c.r2 = r2;
                    }
                    c.dx = (Real)dx;
                    c.dy = (Real)dy;
                    c.dz = (Real)dz;
                    c.qj = (Real)pj[u].w;
                    c.e = ev[u];
                }
                const unsigned ballot = __ballot_sync(0xffffffffu, ok);
                if (ok) Q[qn + __popc(ballot & lt_mask)] = c;
                qn += __popc(ballot);
                __syncwarp();
                if (qn >= 32) {
                    process(Q[lane]);
                    __syncwarp();
                    if (lane < qn - 32) Q[lane] = Q[lane + 32];
                    __syncwarp();
                    qn -= 32;
                }
            }
        }
        if (lane < qn) process(Q[lane]);
        __syncwarp();

        const double s0 = warp_sum(f0.value()), s1 = warp_sum(f1.value()), s2 = warp_sum(f2.value());
        if (lane == 0) {
            fx[i] += s0;
            fy[i] += s1;
            fz[i] += s2;
        }
        if (NONBONDED) {
            const double t[8] = {warp_sum((double)e_qq), warp_sum((double)e_vdw), warp_sum((double)v[0]),
                                 warp_sum((double)v[1]), warp_sum((double)v[2]), warp_sum((double)v[3]),
                                 warp_sum((double)v[4]), warp_sum((double)v[5])};
            if (lane == 0) {
#pragma unroll
                for (int q = 0; q < 8; ++q) wacc[wib][q] += 0.5 * t[q];
            }
        }
    }
    if (NONBONDED) {
        __syncthreads();
        // acc: e_qq, e_vdw, virial[9] (mirrored from the symmetric six)
        double acc[11] = {0.0};
        if (threadIdx.x < kPairWarps) {
            const double *w = wacc[threadIdx.x];
            acc[0] = w[0];
            acc[1] = w[1];
            acc[2] = w[2]; acc[3] = w[3]; acc[4] = w[4];
            acc[5] = w[3]; acc[6] = w[5]; acc[7] = w[6];
            acc[8] = w[4]; acc[9] = w[6]; acc[10] = w[7];
        }
        block_partials<11>(acc, sh, partials);
    }
}

// Mixed path on the cluster list (k_list.cu): one warp per cluster of up to
// four atoms.  Each entry (a j atom, its type, the mask of members it is a
// list neighbour of) is loaded once; j's minimum-image difference from the
// cluster centroid is formed in FP64 and rounded once, and the members' FP32
// offsets from the centroid give each member's difference and r^2 in FP32,
// cut as in k_pair.  The survivors go through the same per-warp queue and
// pair terms as k_pair, tagged with their member.  Each lane adds its pair's
// force in FP64 to its own slot of a shared-memory accumulator per member
// and axis; at the end of the cluster the 32 slots are summed in a fixed
// order, so the FP32 pair forces are summed without loss and run to run
// identically.  Pair energies are summed per lane in FP64 too.  Per chunk of
// 32 entries the four member tests run in straight-line code and append up to
// 128 pairs to the warp's queue (dynamic shared memory, kClQueue entries);
// full flushes of 32 follow at one site, which keeps the pair terms in the
// code once.
//
// HALF (pair_list 0, the default, or 2): the list holds every pair once (k_list.cu), so each
// survivor's force goes to both ends: the member's slot as above, the
// neighbour's by FP64 atomic adds, and energies and virial count in full.
// The CPIM force on a charged water atom from a metal atom is taken from
// whichever end holds the metal.  The atomic adds make the order of the
// neighbour-side sums vary from run to run (FP64 rounding of FP32 terms).
constexpr int kClQueue = 160;  // < 32 left over + 4 x 32 appended
constexpr int kClWarps = 8;      // warps per block of the cluster kernel
constexpr int kClMinBlocks = 2;  // resident blocks per SM the register budget allows
constexpr size_t kClQueueBytes = (size_t)kClWarps * kClQueue * (sizeof(float4) + sizeof(uint32_t));
// A warp's queue as two arrays: the neighbour's FP32 difference from the
// cluster centroid with its charge, and the list entry with the member
// index in its mask bits; the flush forms the member's difference from them
// by the same operations as the member test, so the pair's r^2 is the one
// the test accepted.  An append or a read is one 16-byte and one 4-byte
// shared-memory access.
struct ClQueue {
    float4 *a;
    uint32_t *b;
};
template <bool NONBONDED, bool CPIM, bool HALF>
__global__ void __launch_bounds__(kClWarps * 32, kClMinBlocks) k_pair_cl(DevParams P, PairConstsF K, const double4 *__restrict__ pos4,
                                                              const int4 *__restrict__ cl_atoms,
                                                              const int *__restrict__ n_cl,
                                                              const uint32_t *__restrict__ nbr,
                                                              const int *__restrict__ nnb,
                                                              const unsigned char *__restrict__ cl_metal, int cap,
                                                              const double *__restrict__ vec_pq,
                                                              double *__restrict__ fx, double *__restrict__ fy,
                                                              double *__restrict__ fz, double *__restrict__ partials,
                                                              int *__restrict__ next, const int *__restrict__ sel)
{
    constexpr int NB = 2;
    extern __shared__ __align__(16) unsigned char s_dyn[];  // the warps' queues
    __shared__ float4 s_mem[kClWarps][4];  // member offset from the centroid, charge
    __shared__ int s_trow[kClWarps][4];    // member type * n_types
    __shared__ unsigned char s_cpim[kClWarps][4];  // the member takes the CPIM force of metal neighbours
    __shared__ int s_mmetal[kClWarps][4];          // half list: the member's metal index, -1 not metal
    __shared__ double s_acc[kClWarps][12][32];  // force on (member, axis) per lane slot
    __shared__ double sh[32 * 11];
    __shared__ double wacc[kClWarps][8];
    __shared__ __align__(16) TypePairF s_tpf[kSmemTypes * kSmemTypes];
    __shared__ unsigned char s_metal[kSmemTypes];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    ClQueue Q;
    Q.a = reinterpret_cast<float4 *>(s_dyn) + wib * kClQueue;
    Q.b = reinterpret_cast<uint32_t *>(s_dyn + (size_t)kClWarps * kClQueue * sizeof(float4)) + wib * kClQueue;
    if (lane < 8) wacc[wib][lane] = 0.0;
    const bool smem_types = P.n_types <= kSmemTypes;
    if (smem_types) {
        const int nt2 = P.n_types * P.n_types;
        for (int k = threadIdx.x; k < nt2; k += blockDim.x) s_tpf[k] = make_type_pair_f(P, K, k);
        for (int k = threadIdx.x; k < P.n_types; k += blockDim.x) s_metal[k] = P.type_metal[k];
    }
    __syncthreads();
    const bool metal_by_type = smem_types && P.metal_by_type;
    const double L[3] = {P.box.L[0], P.box.L[1], P.box.L[2]};
    const double iL[3] = {1.0 / L[0], 1.0 / L[1], 1.0 / L[2]};
    const int ncl = *n_cl;
    // next (the half list): a resident grid whose warps take the next cluster
    // from the counter (zeroed before the launch) until none is left, so
    // list lengths that differ from cluster to cluster leave no warp idle at
    // the end; else the fixed grid-stride order, which keeps the energy and
    // virial sums in the same order from run to run
    // sel: only the listed clusters (n_cl then counts them)
    for (int k = 0;; ++k) {
        int ci = blockIdx.x * kClWarps + wib + k * gridDim.x * kClWarps;
        if (next) {
            if (lane == 0) ci = atomicAdd(next, 1);
            ci = __shfl_sync(0xffffffffu, ci, 0);
        }
        if (ci >= ncl) break;
        const int cl = sel ? __ldg(sel + ci) : ci;
        const int4 A = cl_atoms[cl];
        const int nk = 1 + (A.y >= 0) + (A.z >= 0) + (A.w >= 0);
        const int mine = lane == 0 ? A.x : lane == 1 ? A.y : lane == 2 ? A.z : A.w;
        double4 pm = make_double4(0.0, 0.0, 0.0, 0.0);
        if (lane < nk) pm = pos4[mine];
        const double x0 = __shfl_sync(0xffffffffu, pm.x, 0), y0 = __shfl_sync(0xffffffffu, pm.y, 0),
                     z0 = __shfl_sync(0xffffffffu, pm.z, 0);
        double ox = 0.0, oy = 0.0, oz = 0.0;
        if (lane < nk) {
            ox = min_image(pm.x - x0, L[0], iL[0]);
            oy = min_image(pm.y - y0, L[1], iL[1]);
            oz = min_image(pm.z - z0, L[2], iL[2]);
        }
        // member mean offset: lanes 0..3 hold the offsets, the others zero
        double sx = ox, sy = oy, sz = oz;
#pragma unroll
        for (int o = 1; o <= 2; o <<= 1) {
            sx += __shfl_xor_sync(0xffffffffu, sx, o);
            sy += __shfl_xor_sync(0xffffffffu, sy, o);
            sz += __shfl_xor_sync(0xffffffffu, sz, o);
        }
        const double inv_nk = 1.0 / nk;
        const double mx = __shfl_sync(0xffffffffu, sx, 0) * inv_nk, my = __shfl_sync(0xffffffffu, sy, 0) * inv_nk,
                     mz = __shfl_sync(0xffffffffu, sz, 0) * inv_nk;
        const double cx = x0 + mx, cy = y0 + my, cz = z0 + mz;
        if (lane < nk) {
            s_mem[wib][lane] = make_float4((float)(ox - mx), (float)(oy - my), (float)(oz - mz), (float)pm.w);
            s_trow[wib][lane] = P.type[mine] * P.n_types;
            s_cpim[wib][lane] = CPIM && P.is_metal[mine] == 0 && pm.w != 0.0;
            s_mmetal[wib][lane] = HALF && P.is_metal[mine] != 0 ? mine - P.metal_min : -1;
        }
#pragma unroll
        for (int q = 0; q < 12; ++q) s_acc[wib][q][lane] = 0.0;
        __syncwarp();
        const bool cpim_cl = CPIM && cl_metal[cl] != 0;
        const int n = nnb[cl];
        const uint32_t *row = nbr + (size_t)cl * cap;
        double e_qq = 0.0, e_vdw = 0.0;  // per pair in FP64: a cluster's lane sums ~100 pairs
        float v[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) v[q] = 0.f;

        // pair terms of the queue entries head .. head + cnt - 1 into the
        // lanes' slots
        auto flush = [&](int head, int cnt) {
            float hj0 = 0.f, hj1 = 0.f, hj2 = 0.f;  // half list: the neighbour's force of this lane's pair
            int jj = -1;
            if (lane < cnt) {
                float g0 = 0.f, g1 = 0.f, g2 = 0.f;
                float n0 = 0.f, n1 = 0.f, n2 = 0.f;  // the pair force on the member (reversed on the half list)
                const float4 bq4 = Q.a[head + lane];
                Cand<float> c;
                c.e = Q.b[head + lane];
                const int k = (int)((c.e >> kClMaskShift) & 3u);
                const int tj = (int)(c.e >> kClTypeShift);
                const float4 mk = s_mem[wib][k];
                c.dx = bq4.x - mk.x;
                c.dy = bq4.y - mk.y;
                c.dz = bq4.z - mk.z;
                c.r2 = fmaf(c.dz, c.dz, fmaf(c.dy, c.dy, c.dx * c.dx));
                c.qj = bq4.w;
                if (NONBONDED) {
                    const int tp = s_trow[wib][k] + tj;
                    float eq = 0.f, ev = 0.f;
                    const float f = pair_term_f(K, smem_types ? s_tpf[tp] : make_type_pair_f(P, K, tp), mk.w, c.qj,
                                                c.r2, eq, ev);
                    e_qq += (double)eq;
                    e_vdw += (double)ev;
                    const float gx = f * c.dx, gy = f * c.dy, gz = f * c.dz;
                    g0 = n0 = -gx;
                    g1 = n1 = -gy;
                    g2 = n2 = -gz;
                    v[0] -= c.dx * gx; v[1] -= c.dx * gy; v[2] -= c.dx * gz;
                    v[3] -= c.dy * gy; v[4] -= c.dy * gz; v[5] -= c.dz * gz;
                }
                if (cpim_cl && s_cpim[wib][k]) {
                    const int j = (int)(c.e & kClIdxMask);
                    const bool mj = metal_by_type ? s_metal[tj] != 0 : P.is_metal[j] != 0;
                    if (mj) {
                        const int jm = j - P.metal_min;
                        const float r[3] = {c.dx, c.dy, c.dz};  // metal - atom
                        const float p[3] = {(float)vec_pq[3 * jm], (float)vec_pq[3 * jm + 1],
                                            (float)vec_pq[3 * jm + 2]};
                        float g[3];
                        cpim_charge_pair_f(K, r, c.r2, mk.w, (float)vec_pq[3 * P.M + jm], p, g);
                        g0 -= g[0];
                        g1 -= g[1];
                        g2 -= g[2];
                    }
                }
                s_acc[wib][3 * k][lane] += (double)g0;
                s_acc[wib][3 * k + 1][lane] += (double)g1;
                s_acc[wib][3 * k + 2][lane] += (double)g2;
                if (HALF) {
                    // the neighbour's side: the pair force reversed, and the
                    // CPIM force on it when the member is the metal atom
                    float h0 = -n0, h1 = -n1, h2 = -n2;
                    const int mm = s_mmetal[wib][k];
                    if (CPIM && cpim_cl && mm >= 0 && c.qj != 0.f) {
                        const int j = (int)(c.e & kClIdxMask);
                        const bool mj = metal_by_type ? s_metal[tj] != 0 : P.is_metal[j] != 0;
                        if (!mj) {
                            const float r[3] = {-c.dx, -c.dy, -c.dz};  // metal - atom
                            const float p[3] = {(float)vec_pq[3 * mm], (float)vec_pq[3 * mm + 1],
                                                (float)vec_pq[3 * mm + 2]};
                            float g[3];
                            cpim_charge_pair_f(K, r, c.r2, c.qj, (float)vec_pq[3 * P.M + mm], p, g);
                            h0 -= g[0];
                            h1 -= g[1];
                            h2 -= g[2];
                        }
                    }
                    hj0 = h0;
                    hj1 = h1;
                    hj2 = h2;
                    jj = (int)(c.e & kClIdxMask);
                }
            }
            if (HALF) {
                // a neighbour's pairs are adjacent (at most four): sum them
                // into the first lane of the run, which adds them to the atom
                const int jl = lane < cnt ? jj : -1 - lane;
#pragma unroll
                for (int o = 1; o < 4; o <<= 1) {
                    const float t0 = __shfl_down_sync(0xffffffffu, hj0, o);
                    const float t1 = __shfl_down_sync(0xffffffffu, hj1, o);
                    const float t2 = __shfl_down_sync(0xffffffffu, hj2, o);
                    const int tj = __shfl_down_sync(0xffffffffu, jl, o);
                    if (lane + o < 32 && tj == jl) {
                        hj0 += t0;
                        hj1 += t1;
                        hj2 += t2;
                    }
                }
                const int prev = __shfl_up_sync(0xffffffffu, jl, 1);
                if (lane < cnt && (lane == 0 || prev != jl) && (hj0 != 0.f || hj1 != 0.f || hj2 != 0.f)) {
                    atomicAdd(fx + jl, (double)hj0);
                    atomicAdd(fy + jl, (double)hj1);
                    atomicAdd(fz + jl, (double)hj2);
                }
            }
        };

        int qn = 0;  // queue fill, warp-uniform
        uint32_t nxt[NB];
#pragma unroll
        for (int u = 0; u < NB; ++u) {
            const int k = u * 32 + lane;
            nxt[u] = k < n ? __ldcs(row + k) : 0u;
        }
        for (int base = 0; base < n; base += 32 * NB) {
            uint32_t ev[NB];
            bool valid[NB];
#pragma unroll
            for (int u = 0; u < NB; ++u) {
                valid[u] = base + u * 32 + lane < n;
                ev[u] = nxt[u];
                const int k = base + (NB + u) * 32 + lane;
                nxt[u] = k < n ? __ldcs(row + k) : 0u;
            }
            double4 pj[NB];
#pragma unroll
            for (int u = 0; u < NB; ++u)
                if (valid[u]) pj[u] = pos4[ev[u] & kClIdxMask];
            static_assert(NB == 2, "the member loop selects between two chunks");
            float dxc[NB], dyc[NB], dzc[NB], qj[NB];
            unsigned mask[NB];
            uint32_t keep[NB];
#pragma unroll
            for (int u = 0; u < NB; ++u) {
                dxc[u] = dyc[u] = dzc[u] = qj[u] = 0.f;
                mask[u] = 0;
                if (valid[u]) {
                    dxc[u] = (float)min_image(pj[u].x - cx, L[0], iL[0]);
                    dyc[u] = (float)min_image(pj[u].y - cy, L[1], iL[1]);
                    dzc[u] = (float)min_image(pj[u].z - cz, L[2], iL[2]);
                    qj[u] = (float)pj[u].w;
                    mask[u] = (ev[u] >> kClMaskShift) & 15u;
                }
                keep[u] = ev[u] & ~(15u << kClMaskShift);
            }
            // per chunk: the member tests in straight-line code (mask bits
            // exist only for members < nk), the survivors appended to the
            // queue, then the full flushes and the remainder moved to the front
#pragma unroll 1
            for (int u = 0; u < NB; ++u) {
                const bool hi = u == 1;
                const float bx = hi ? dxc[1] : dxc[0], by = hi ? dyc[1] : dyc[0], bz = hi ? dzc[1] : dzc[0];
                const float bq = hi ? qj[1] : qj[0];
                const unsigned bm = hi ? mask[1] : mask[0];
                const uint32_t bk = hi ? keep[1] : keep[0];
                if (HALF) {
                    // each entry's survivors appended next to each other (the
                    // flush sums a neighbour's pairs before its atomic adds)
                    unsigned smask = 0;
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        const float4 mk = s_mem[wib][kk];
                        const float dx = bx - mk.x, dy = by - mk.y, dz = bz - mk.z;
                        const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                        if (((bm >> kk) & 1u) && r2 < K.rc2) smask |= 1u << kk;
                    }
                    const int cnt = __popc(smask);
                    int incl = cnt;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int t = __shfl_up_sync(0xffffffffu, incl, o);
                        if (lane >= o) incl += t;
                    }
                    int pos = qn + incl - cnt;
#pragma unroll
                    const float4 b4 = make_float4(bx, by, bz, bq);
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        if ((smask >> kk) & 1u) {
                            Q.a[pos] = b4;
                            Q.b[pos] = bk | ((uint32_t)kk << kClMaskShift);
                            ++pos;
                        }
                    }
                    qn += __shfl_sync(0xffffffffu, incl, 31);
                } else {
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        const float4 mk = s_mem[wib][kk];
                        const float dx = bx - mk.x, dy = by - mk.y, dz = bz - mk.z;
                        const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                        const bool ok = ((bm >> kk) & 1u) && r2 < K.rc2;
                        const unsigned ballot = __ballot_sync(0xffffffffu, ok);
                        if (ok) {
                            const int at = qn + __popc(ballot & lt_mask);
                            Q.a[at] = make_float4(bx, by, bz, bq);
                            Q.b[at] = bk | ((uint32_t)kk << kClMaskShift);
                        }
                        qn += __popc(ballot);
                    }
                }
                __syncwarp();
                int head = 0;
                while (qn - head >= 32) {
                    flush(head, 32);
                    head += 32;
                }
                if (head > 0) {
                    const int rest = qn - head;
                    float4 ta;
                    uint32_t tb = 0;
                    if (lane < rest) {
                        ta = Q.a[head + lane];
                        tb = Q.b[head + lane];
                    }
                    __syncwarp();
                    if (lane < rest) {
                        Q.a[lane] = ta;
                        Q.b[lane] = tb;
                    }
                    __syncwarp();
                    qn = rest;
                }
            }
        }
        if (qn > 0) flush(0, qn);
        __syncwarp();

        // member forces: lane 3 k + a sums the 32 slots of (k, a), starting
        // at its own slot (no bank conflicts), in a fixed order
        if (lane < 3 * nk) {
            const int k = lane / 3, a = lane - 3 * k;
            double s = 0.0;
#pragma unroll 8
            for (int q = 0; q < 32; ++q) s += s_acc[wib][lane][(q + lane) & 31];
            const int atom = k == 0 ? A.x : k == 1 ? A.y : k == 2 ? A.z : A.w;
            double *f = a == 0 ? fx : (a == 1 ? fy : fz);
            if (HALF)
                atomicAdd(f + atom, s);  // other clusters add to this atom as a neighbour
            else
                f[atom] += s;
        }
        if (NONBONDED) {
            const double t[8] = {warp_sum(e_qq), warp_sum(e_vdw), warp_sum((double)v[0]),
                                 warp_sum((double)v[1]), warp_sum((double)v[2]), warp_sum((double)v[3]),
                                 warp_sum((double)v[4]), warp_sum((double)v[5])};
            if (lane == 0) {
#pragma unroll
                for (int q = 0; q < 8; ++q) wacc[wib][q] += (HALF ? 1.0 : 0.5) * t[q];
            }
        }
        __syncwarp();
    }
    if (NONBONDED) {
        __syncthreads();
        double acc[11] = {0.0};
        if (threadIdx.x < kClWarps) {
            const double *w = wacc[threadIdx.x];
            acc[0] = w[0];
            acc[1] = w[1];
            acc[2] = w[2]; acc[3] = w[3]; acc[4] = w[4];
            acc[5] = w[3]; acc[6] = w[5]; acc[7] = w[6];
            acc[8] = w[4]; acc[9] = w[6]; acc[10] = w[7];
        }
        block_partials<11>(acc, sh, partials);
    }
}

// Mixed path on the cluster-pair list (pair_list 4, k_list.cu): one warp per
// cluster I at a time (taken from a counter, as on the half cluster list),
// two entries (clusters J) per step.  Lane l works on member k = l & 3 of I
// with member m = (l >> 2) & 3 of entry h = l >> 4: the 32 lanes cover the
// 2 x 16 member pairs with no compaction, and a pair that is masked at the
// build or outside the cut-off now contributes nothing.  I's member stays in
// the lane's registers for the whole list; each step a lane loads J's
// centroid, its member's offset and charge, and its atom and type (the four
// lanes of one J member read the same addresses).  The pair difference is
// the FP64 minimum image of the centroid difference, rounded once, plus the
// FP32 offsets; the FP32 cut-off decides the pair as in k_pair.  Each pair
// counts once: the force on I's member accumulates in FP64 in the lane (the
// eight lanes of a member summed at the end, then added with FP64 atomic
// adds, since other clusters add to the same atom), the force on J's member
// is summed over its four lanes by shuffles and added with FP64 atomic adds;
// pair energies are summed per lane in FP64, the virial per lane in FP32 per
// cluster.  CPIM: on entries where either cluster has a metal member, the
// CPIM force on a charged non-metal atom from a metal atom of the pair,
// whichever end holds the metal.
constexpr int kCpWarps = 8;
constexpr int kCpMinBlocks = 2;
template <bool NONBONDED, bool CPIM>
__global__ void __launch_bounds__(kCpWarps * 32, kCpMinBlocks)
    k_pair_cp(DevParams P, PairConstsF K, const double4 *__restrict__ cent, const float4 *__restrict__ off,
              const int *__restrict__ ti, const uint2 *__restrict__ list, const int *__restrict__ cnt, int cap,
              int ncl, const double *__restrict__ vec_pq, double *__restrict__ fx, double *__restrict__ fy,
              double *__restrict__ fz, double *__restrict__ partials, int *__restrict__ next)
{
    __shared__ double sh[32 * 11];
    __shared__ double wacc[kCpWarps][8];
    __shared__ __align__(16) TypePairF s_tpf[kSmemTypes * kSmemTypes];
    __shared__ unsigned char s_metal[kSmemTypes];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ki = lane & 3, mj = (lane >> 2) & 3, h = lane >> 4;
    if (lane < 8) wacc[wib][lane] = 0.0;
    const bool smem_types = P.n_types <= kSmemTypes;
    if (smem_types) {
        const int nt2 = P.n_types * P.n_types;
        for (int k = threadIdx.x; k < nt2; k += blockDim.x) s_tpf[k] = make_type_pair_f(P, K, k);
        for (int k = threadIdx.x; k < P.n_types; k += blockDim.x) s_metal[k] = P.type_metal[k];
    }
    __syncthreads();
    const bool metal_by_type = smem_types && P.metal_by_type;
    const double L[3] = {P.box.L[0], P.box.L[1], P.box.L[2]};
    const double iL[3] = {1.0 / L[0], 1.0 / L[1], 1.0 / L[2]};
    for (;;) {
        int ic = 0;
        if (lane == 0) ic = atomicAdd(next, 1);
        ic = __shfl_sync(0xffffffffu, ic, 0);
        if (ic >= ncl) break;
        const double4 ci = cent[ic];
        const float4 oi = off[4 * ic + ki];
        const int tii = ti[4 * ic + ki];
        const bool vi = tii >= 0;
        const int ai = tii & kCpIdxMask;
        const int tyi = vi ? (tii >> kCpTypeShift) : 0;
        const int trow = tyi * P.n_types;
        const bool metal_i = vi && (metal_by_type ? s_metal[tyi] != 0 : P.is_metal[ai] != 0);
        const int mi = metal_i ? ai - P.metal_min : 0;
        const bool water_i = CPIM && vi && !metal_i && oi.w != 0.f;  // takes the CPIM force of metal atoms
        double fix = 0.0, fiy = 0.0, fiz = 0.0, e_qq = 0.0, e_vdw = 0.0;
        float v[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) v[q] = 0.f;
        const int n = cnt[ic];
        const uint2 *row = list + (size_t)ic * cap;
        for (int q0 = 0; q0 < n; q0 += 2) {
            const int q = q0 + h;
            const bool ve = q < n;
            const uint2 e = ve ? row[q] : make_uint2((uint32_t)ic, 0u);
            const int jc = (int)e.x;
            const double4 cj = cent[jc];
            const float4 oj = off[4 * jc + mj];
            const int tij = ti[4 * jc + mj];
            const float dcx = (float)min_image(cj.x - ci.x, L[0], iL[0]);
            const float dcy = (float)min_image(cj.y - ci.y, L[1], iL[1]);
            const float dcz = (float)min_image(cj.z - ci.z, L[2], iL[2]);
            const float dx = dcx + (oj.x - oi.x), dy = dcy + (oj.y - oi.y), dz = dcz + (oj.z - oi.z);
            const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            const bool act = ((e.y >> (4 * ki + mj)) & 1u) && r2 < K.rc2;
            float gx = 0.f, gy = 0.f, gz = 0.f;  // force on I's member
            float hx = 0.f, hy = 0.f, hz = 0.f;  // force on J's member
            if (act) {
                const int aj = tij & kCpIdxMask, tyj = tij >> kCpTypeShift;
                if (NONBONDED) {
                    const int tp = trow + tyj;
                    float eq = 0.f, ev = 0.f;
                    const float f = pair_term_f(K, smem_types ? s_tpf[tp] : make_type_pair_f(P, K, tp), oi.w, oj.w,
                                                r2, eq, ev);
                    e_qq += (double)eq;
                    e_vdw += (double)ev;
                    hx = f * dx;
                    hy = f * dy;
                    hz = f * dz;
                    gx = -hx;
                    gy = -hy;
                    gz = -hz;
                    v[0] -= dx * hx; v[1] -= dx * hy; v[2] -= dx * hz;
                    v[3] -= dy * hy; v[4] -= dy * hz; v[5] -= dz * hz;
                }
                if (CPIM && (e.y & kCpMetalBit)) {
                    const bool metal_j = metal_by_type ? s_metal[tyj] != 0 : P.is_metal[aj] != 0;
                    if (water_i && metal_j) {
                        const int jm = aj - P.metal_min;
                        const float r[3] = {dx, dy, dz};  // metal - atom
                        const float p[3] = {(float)vec_pq[3 * jm], (float)vec_pq[3 * jm + 1], (float)vec_pq[3 * jm + 2]};
                        float g[3];
                        cpim_charge_pair_f(K, r, r2, oi.w, (float)vec_pq[3 * P.M + jm], p, g);
                        gx -= g[0];
                        gy -= g[1];
                        gz -= g[2];
                    } else if (metal_i && !metal_j && oj.w != 0.f) {
                        const float r[3] = {-dx, -dy, -dz};  // metal - atom
                        const float p[3] = {(float)vec_pq[3 * mi], (float)vec_pq[3 * mi + 1], (float)vec_pq[3 * mi + 2]};
                        float g[3];
                        cpim_charge_pair_f(K, r, r2, oj.w, (float)vec_pq[3 * P.M + mi], p, g);
                        hx -= g[0];
                        hy -= g[1];
                        hz -= g[2];
                    }
                }
            }
            fix += (double)gx;
            fiy += (double)gy;
            fiz += (double)gz;
            // J's member: the four lanes of (h, m) summed, added by the first
#pragma unroll
            for (int o = 1; o <= 2; o <<= 1) {
                hx += __shfl_xor_sync(0xffffffffu, hx, o);
                hy += __shfl_xor_sync(0xffffffffu, hy, o);
                hz += __shfl_xor_sync(0xffffffffu, hz, o);
            }
            if (ki == 0 && (hx != 0.f || hy != 0.f || hz != 0.f)) {
                const int aj = tij & kCpIdxMask;
                atomicAdd(fx + aj, (double)hx);
                atomicAdd(fy + aj, (double)hy);
                atomicAdd(fz + aj, (double)hz);
            }
        }
        // I's member: its eight lanes summed in a fixed order
#pragma unroll
        for (int o = 4; o < 32; o <<= 1) {
            fix += __shfl_xor_sync(0xffffffffu, fix, o);
            fiy += __shfl_xor_sync(0xffffffffu, fiy, o);
            fiz += __shfl_xor_sync(0xffffffffu, fiz, o);
        }
        if (lane < 4 && vi && (fix != 0.0 || fiy != 0.0 || fiz != 0.0)) {
            atomicAdd(fx + ai, fix);
            atomicAdd(fy + ai, fiy);
            atomicAdd(fz + ai, fiz);
        }
        if (NONBONDED) {
            const double t[8] = {warp_sum(e_qq), warp_sum(e_vdw), warp_sum((double)v[0]),
                                 warp_sum((double)v[1]), warp_sum((double)v[2]), warp_sum((double)v[3]),
                                 warp_sum((double)v[4]), warp_sum((double)v[5])};
            if (lane == 0) {
#pragma unroll
                for (int q = 0; q < 8; ++q) wacc[wib][q] += t[q];
            }
        }
        __syncwarp();
    }
    if (NONBONDED) {
        __syncthreads();
        double acc[11] = {0.0};
        if (threadIdx.x < kCpWarps) {
            const double *w = wacc[threadIdx.x];
            acc[0] = w[0];
            acc[1] = w[1];
            acc[2] = w[2]; acc[3] = w[3]; acc[4] = w[4];
            acc[5] = w[3]; acc[6] = w[5]; acc[7] = w[6];
            acc[8] = w[4]; acc[9] = w[6]; acc[10] = w[7];
        }
        block_partials<11>(acc, sh, partials);
    }
}

PairConstsF pair_consts_f(const capac_ctx *c)
{
    PairConstsF K;
    K.rc = (float)c->P.rc;
    K.inv_rc = (float)(1.0 / c->P.rc);
    K.inv_rc12 = (float)c->P.inv_rc12;
    K.inv_rc6 = (float)c->P.inv_rc6;
    K.alpha = (float)c->P.w_alpha;
    K.a2_sqrtpi = (float)c->P.w_a2_sqrtpi;
    K.w_const = (float)c->P.w_const;
    K.w_erfc_arcut = (float)c->P.w_erfc_arcut;
    K.fqq = (float)kFQQ;
    K.rc2 = (float)c->P.rc2;
    K.use_vdw = c->P.use_vdw;
    K.use_coulomb = c->P.use_coulomb;
    return K;
}

template <typename Real>
void launch_pair_t(capac_ctx *c, int mode, unsigned grid)
{
    const PairConstsF K = pair_consts_f(c);
    const bool cpim = c->M > 0 && c->use_cpff;
    ProfScope ps(c, K_PAIR);
    if (mode == 0 && cpim)
        k_pair<Real, true, true><<<grid, kPairWarps * 32, 0, c->stream>>>(c->P, K, c->pos4, c->nbr, c->nnb, c->cap,
                                                                          c->vec_pq, c->fx, c->fy, c->fz, c->partials);
    else if (mode == 0)
        k_pair<Real, true, false><<<grid, kPairWarps * 32, 0, c->stream>>>(c->P, K, c->pos4, c->nbr, c->nnb, c->cap,
                                                                           c->vec_pq, c->fx, c->fy, c->fz, c->partials);
    else
        k_pair<Real, false, true><<<grid, kPairWarps * 32, 0, c->stream>>>(c->P, K, c->pos4, c->nbr, c->nnb, c->cap,
                                                                           c->vec_pq, c->fx, c->fy, c->fz, c->partials);
    ++c->launches;
}

// The cluster pair kernel on stream st, its block partials to `partials`;
// sel: only the clusters with a metal member or neighbour.
template <bool NONBONDED, bool CPIM, bool HALF>
void launch_pair_cl_t(capac_ctx *c, unsigned grid, cudaStream_t st, double *partials, bool sel)
{
    // the queues and the static arrays together exceed the default 48 KB
    CAPAC_CUDA(cudaFuncSetAttribute(k_pair_cl<NONBONDED, CPIM, HALF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kClQueueBytes));
    if (HALF) CAPAC_CUDA(cudaMemsetAsync(c->cl_next, 0, sizeof(int), st));
    k_pair_cl<NONBONDED, CPIM, HALF><<<grid, kClWarps * 32, kClQueueBytes, st>>>(
        c->P, pair_consts_f(c), c->pos4, c->cl_atoms, sel ? c->n_cl_sel : c->cl_cell_start + c->n_cells, c->cl_nbr,
        c->cl_nnb, c->cl_metal, c->cl_cap, c->vec_pq, c->fx, c->fy, c->fz, partials, HALF ? c->cl_next : nullptr,
        sel ? c->cl_sel : nullptr);
}

template <bool NONBONDED, bool CPIM>
void launch_pair_cp_t(capac_ctx *c, unsigned grid)
{
    CAPAC_CUDA(cudaMemsetAsync(c->cl_next, 0, sizeof(int), c->stream));
    k_pair_cp<NONBONDED, CPIM><<<grid, kCpWarps * 32, 0, c->stream>>>(
        c->P, pair_consts_f(c), c->cp_cent, c->cp_off, c->cp_ti, c->cp_list, c->cp_n, c->cp_cap, c->n_clusters,
        c->vec_pq, c->fx, c->fy, c->fz, c->partials, c->cl_next);
}

// The cluster frames of the current positions, then the cluster-pair kernel.
void launch_pair_cpairs(capac_ctx *c, int mode, unsigned grid)
{
    const bool cpim = c->M > 0 && c->use_cpff;
    ProfScope ps(c, K_PAIR);
    launch_cluster_frames(c, false);
    if (mode == 0 && cpim)
        launch_pair_cp_t<true, true>(c, grid);
    else if (mode == 0)
        launch_pair_cp_t<true, false>(c, grid);
    else
        launch_pair_cp_t<false, true>(c, grid);
    ++c->launches;
}

void launch_pair_clusters(capac_ctx *c, int mode, unsigned grid)
{
    const bool cpim = c->M > 0 && c->use_cpff;
    ProfScope ps(c, K_PAIR);
    if (c->cl_half) {
        if (mode == 0 && cpim && c->pair_split) {
            // the pair terms without the CPIM branches, then the water-side
            // CPIM term over the clusters with a metal member or neighbour
            launch_pair_cl_t<true, false, true>(c, grid, c->stream, c->partials, false);
            launch_pair_cl_t<false, true, true>(c, grid, c->stream, c->partials, true);
            ++c->launches;
        } else if (mode == 0 && cpim)
            launch_pair_cl_t<true, true, true>(c, grid, c->stream, c->partials, false);
        else if (mode == 0)
            launch_pair_cl_t<true, false, true>(c, grid, c->stream, c->partials, false);
        else
            launch_pair_cl_t<false, true, true>(c, grid, c->stream, c->partials, false);
    } else if (mode == 0 && cpim)
        launch_pair_cl_t<true, true, false>(c, grid, c->stream, c->partials, false);
    else if (mode == 0)
        launch_pair_cl_t<true, false, false>(c, grid, c->stream, c->partials, false);
    else
        launch_pair_cl_t<false, true, false>(c, grid, c->stream, c->partials, false);
    ++c->launches;
}

}  // namespace

// Blocks of the pair launch: one warp per atom (or per cluster), at most 16
// blocks per SM (grid-stride beyond); on the half cluster list the resident
// blocks only (its warps take clusters from a counter).
unsigned pair_grid(const capac_ctx *c)
{
    if (c->cpairs) return (unsigned)c->num_sms * kCpMinBlocks;
    const long units = c->clusters ? c->n_clusters : c->N;
    const int warps = c->clusters ? kClWarps : kPairWarps;
    const long need = (units + warps - 1) / warps;
    const long cap = (long)c->num_sms * (c->clusters && c->cl_half ? kClMinBlocks : 16);
    return (unsigned)std::max(1L, std::min(need, cap));
}

// Overlap, first half (on stream2, once `stream` has reached this point):
// the nonbonded terms of the half cluster list, one block per SM so that the
// CPIM solve's blocks find room beside it; energies and virial into
// partials2.  The forces go to fx, fy, fz by atomic adds only, so the
// kernels that run meanwhile on `stream` must leave them alone (the CPIM
// right-hand side, matrix and solve do).
void launch_pair_nonbonded_async(capac_ctx *c)
{
    CAPAC_CUDA(cudaEventRecord(c->ev_fork, c->stream));
    CAPAC_CUDA(cudaStreamWaitEvent(c->stream2, c->ev_fork, 0));
    c->work_stream = c->stream2;
    {
        ProfScope ps(c, K_PAIR);
        // one block per SM, and no more blocks than warps have clusters to take
        c->async_grid = std::min((unsigned)c->num_sms, pair_grid(c));
        launch_pair_cl_t<true, false, true>(c, c->async_grid, c->stream2, c->partials2, false);
    }
    c->work_stream = nullptr;
    ++c->launches;
    CAPAC_CUDA(cudaEventRecord(c->ev_join, c->stream2));
}

// Overlap, second half (on `stream`, after the solve): wait for the first,
// sum its energies and virial, then the CPIM forces on water atoms from the
// solved induced vector over the clusters with a metal member or neighbour.
void launch_pair_join(capac_ctx *c)
{
    CAPAC_CUDA(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
    static const int pot_slots[11] = {7, 8, -1, -1, -1, -1, -1, -1, -1, -1, -1};
    static const int vir_slots[11] = {-1, -1, 0, 1, 2, 3, 4, 5, 6, 7, 8};
    launch_finalize(c, (int)c->async_grid, 11, pot_slots, vir_slots, c->partials2);
    {
        ProfScope ps(c, K_PAIR);
        launch_pair_cl_t<false, true, true>(c, pair_grid(c), c->stream, c->partials, true);
    }
    ++c->launches;
}

void launch_pair_forces(capac_ctx *c, int mode)
{
    const unsigned grid = pair_grid(c);
    if (c->cpairs)
        launch_pair_cpairs(c, mode, grid);
    else if (c->clusters)
        launch_pair_clusters(c, mode, grid);
    else if (c->opt.precision == CAPAC_PREC_MIXED)
        launch_pair_t<float>(c, mode, grid);
    else
        launch_pair_t<double>(c, mode, grid);
    if (mode == 0) {
        static const int pot_slots[11] = {7, 8, -1, -1, -1, -1, -1, -1, -1, -1, -1};
        static const int vir_slots[11] = {-1, -1, 0, 1, 2, 3, 4, 5, 6, 7, 8};
        launch_finalize(c, (int)grid, 11, pot_slots, vir_slots);
    }
}

}  // namespace capac
