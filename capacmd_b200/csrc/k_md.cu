// Velocity-Verlet MD step pieces on the device (mpi-main.c:874-1013):
// Nose-Hoover chain, half kicks, drift, RATTLE, kinetic energy, COM-velocity
// removal, apply_pbc and the force diagnostics.  Scalars (thermostat chain,
// kinetic energy, temperature) stay in device memory.
#include "ctx.h"

namespace capac {

namespace {

struct MdParams {
    int N, n_mols, fix_metal, ndf;
    double dt, dt_2, q_mass;
    Box box;
};

MdParams md_params(const capac_ctx *c)
{
    MdParams m;
    m.N = c->N;
    m.n_mols = c->n_mols;
    m.fix_metal = c->fix_metal;
    m.ndf = c->c.ndf;
    m.dt = c->dt;
    m.dt_2 = c->c.dt_2;
    m.q_mass = c->c.q_mass;
    m.box = c->P.box;
    return m;
}

// Heating ramp of the reference temperature (mpi-main.c:879-891).
__global__ void k_heating(ThermoState *th, long step, int n_heating)
{
    if (step < n_heating)
        th->ref_temp = th->first_temp + (th->ext_temp - th->first_temp) * step / n_heating;
    else
        th->ref_temp = th->ext_temp;
    th->kT = kBoltz * th->ref_temp;
}

// nose_hoover_chain, thermostat.c:117-191: 10 links, Nc = 5, 5th-order
// Suzuki-Yoshida weights; the velocity scale is left in th->scale.
__global__ void k_nhc(ThermoState *th, MdParams m)
{
    const int Nc = 5, L = kNhc;
    const double w1 = 0.41449077179437571194, w3 = -0.65796308717750284778;
    const double w[5] = {w1, w1, w3, w1, w1};
    const double Q = m.q_mass, kT = th->kT, NkT = kT * m.ndf, dt = m.dt, ek = th->eksum;
    // the chain in registers (every index is fixed once the loops unroll),
    // written back at the end
    double vQ[kNhc], aQ[kNhc], scale = 1.0;
#pragma unroll
    for (int k = 0; k < L; ++k) vQ[k] = th->vQ[k];
    aQ[0] = (ek - NkT) / Q;
#pragma unroll
    for (int k = 0; k < L - 1; ++k) aQ[k + 1] = (Q * vQ[k] * vQ[k] - kT) / Q;
    for (int c = 0; c < Nc; ++c) {
#pragma unroll
        for (int y = 0; y < 5; ++y) {
            const double h4 = w[y] * dt / (4 * Nc), h8 = w[y] * dt / (8 * Nc), h2 = w[y] * dt / (2 * Nc);
            vQ[L - 1] += aQ[L - 1] * h4;
#pragma unroll
            for (int k = 0; k < L - 1; ++k) {
                const double e = exp(-h8 * vQ[L - (k + 1)]);
                vQ[L - 1 - (k + 1)] = vQ[L - 1 - (k + 1)] * e * e + h4 * aQ[L - 1 - (k + 1)] * e;
            }
            scale *= exp(-h2 * vQ[0]);
            aQ[0] = (ek * scale * scale - NkT) / Q;
#pragma unroll
            for (int k = 0; k < L - 1; ++k) {
                const double e = exp(-h8 * vQ[k + 1]);
                vQ[k] = vQ[k] * e * e + h4 * aQ[k] * e;
                aQ[k + 1] = (Q * vQ[k] * vQ[k] - kT) / Q;
            }
            vQ[L - 1] += aQ[L - 1] * h4;
        }
    }
#pragma unroll
    for (int k = 0; k < L; ++k) {
        th->vQ[k] = vQ[k];
        th->aQ[k] = aQ[k];
    }
    th->scale = scale;
    th->eksum = ek * (scale * scale);
    th->inst_temp *= scale * scale;
}

// Berendsen weak coupling (no counterpart in the reference, whose only
// thermostat is the Nose-Hoover chain): lambda = sqrt(1 + dt/tau (T0/T - 1))
// from the temperature after the second RATTLE (Berendsen et al., J. Chem.
// Phys. 81, 3684 (1984)), lambda^2 held to [0.64, 1.5625] and lambda = 1 at
// T = 0; the scale is left in th->scale for k_scale_velocities.
__global__ void k_berendsen(ThermoState *th, double dt_over_tau)
{
    const double T = th->inst_temp;
    double s2 = 1.0;
    if (T > 0.0) s2 = fmin(fmax(1.0 + dt_over_tau * (th->ref_temp / T - 1.0), 0.64), 1.5625);
    const double s = sqrt(s2);
    th->scale = s;
    th->eksum *= s * s;
    th->inst_temp *= s * s;
}

// Optional thermostat scaling of every velocity, then v += dt/2 F/m for
// atoms that move (mpi-main.c:900-913).
__global__ void k_half_kick(MdParams m, const unsigned char *is_metal, const double *inv_mass,
                            const double *fx, const double *fy, const double *fz, double *vx, double *vy,
                            double *vz, const ThermoState *th, int apply_scale)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.N) return;
    double a = vx[i], b = vy[i], c = vz[i];
    if (apply_scale) {
        const double s = th->scale;
        a *= s; b *= s; c *= s;
    }
    if (!(m.fix_metal == 1 && is_metal[i])) {
        const double im = inv_mass[i];
        a += m.dt_2 * fx[i] * im;
        b += m.dt_2 * fy[i] * im;
        c += m.dt_2 * fz[i] * im;
    }
    vx[i] = a; vy[i] = b; vz[i] = c;
}

__global__ void k_scale_velocities(int N, const ThermoState *th, double *vx, double *vy, double *vz)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double s = th->scale;
    vx[i] *= s; vy[i] *= s; vz[i] *= s;
}

// old_r = r; r += dt v (mpi-main.c:917-932).
__global__ void k_drift(MdParams m, const unsigned char *is_metal, double *rx, double *ry, double *rz,
                        const double *vx, const double *vy, const double *vz, double *ox, double *oy, double *oz)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.N) return;
    if (m.fix_metal == 1 && is_metal[i]) return;
    ox[i] = rx[i]; oy[i] = ry[i]; oz[i] = rz[i];
    rx[i] += m.dt * vx[i];
    ry[i] += m.dt * vy[i];
    rz[i] += m.dt * vz[i];
}

struct CstrView {
    const int *mol_first, *mol_type, *off, *cnt, *ci, *cj;
    const double *len;
    const double *inv_mass;
    const int *mol_atoms;  // atoms per molecule type
};

// Three-atom molecules with at most three constraints (the 3-site waters)
// iterate on a copy of their atoms held in registers, written back once: the
// same operations in the same order as on the global arrays, without a round
// trip to L2 per constraint and iteration.  Mol3 reads and updates atom a of
// a molecule with selects, so the values never leave registers.
struct Mol3 {
    double v0, v1, v2;
    __device__ __forceinline__ double get(int a) const { return a == 0 ? v0 : (a == 1 ? v1 : v2); }
    __device__ __forceinline__ void add(int a, double x)
    {
        if (a == 0) v0 += x;
        else if (a == 1) v1 += x;
        else v2 += x;
    }
    __device__ __forceinline__ void load(const double *p, int first)
    {
        v0 = p[first];
        v1 = p[first + 1];
        v2 = p[first + 2];
    }
    __device__ __forceinline__ void store(double *p, int first) const
    {
        p[first] = v0;
        p[first + 1] = v1;
        p[first + 2] = v2;
    }
};

// rattle_1st, force.c:1907-1997: one thread per molecule.
__global__ void __launch_bounds__(256, 2) k_rattle1(MdParams m, CstrView cv, double *rx, double *ry, double *rz, const double *ox,
                          const double *oy, const double *oz, double *vx, double *vy, double *vz, int *flags)
{
    const int im = blockIdx.x * blockDim.x + threadIdx.x;
    if (im >= m.n_mols) return;
    const int first = cv.mol_first[im], mt = cv.mol_type[first];
    const int nc = cv.cnt[mt], c0 = cv.off[mt];
    if (nc == 0) return;
    const double tol2 = 2.0e-05, inv_dt = 1.0 / m.dt;  // the velocity update multiplies by 1/dt
    int iter = 0, done = 0;
    if (cv.mol_atoms[mt] == 3 && nc <= 3) {
        Mol3 X, Y, Z, VX, VY, VZ, OX, OY, OZ, IM;
        X.load(rx, first); Y.load(ry, first); Z.load(rz, first);
        VX.load(vx, first); VY.load(vy, first); VZ.load(vz, first);
        OX.load(ox, first); OY.load(oy, first); OZ.load(oz, first);
        IM.load(cv.inv_mass, first);
        int ca[3] = {0, 0, 0}, cb[3] = {0, 0, 0};
        double l2[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (k < nc) {
                ca[k] = cv.ci[c0 + k];
                cb[k] = cv.cj[c0 + k];
                l2[k] = cv.len[c0 + k] * cv.len[c0 + k];
            }
        while (!done) {
            done = 1;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (k >= nc) continue;
                const int a = ca[k], b = cb[k];
                const double len2 = l2[k];
                const double px = wrap1(X.get(a) - X.get(b), m.box.L[0]);
                const double py = wrap1(Y.get(a) - Y.get(b), m.box.L[1]);
                const double pz = wrap1(Z.get(a) - Z.get(b), m.box.L[2]);
                const double diff = len2 - (px * px + py * py + pz * pz);
                if (fabs(diff) > len2 * tol2) {
                    const double qx = wrap1(OX.get(a) - OX.get(b), m.box.L[0]);
                    const double qy = wrap1(OY.get(a) - OY.get(b), m.box.L[1]);
                    const double qz = wrap1(OZ.get(a) - OZ.get(b), m.box.L[2]);
                    const double ma = IM.get(a), mb = IM.get(b);
                    const double g = diff / (2.0 * (ma + mb) * (qx * px + qy * py + qz * pz));
                    double dx = qx * g, dy = qy * g, dz = qz * g;
                    X.add(a, ma * dx); Y.add(a, ma * dy); Z.add(a, ma * dz);
                    X.add(b, -(mb * dx)); Y.add(b, -(mb * dy)); Z.add(b, -(mb * dz));
                    dx *= inv_dt; dy *= inv_dt; dz *= inv_dt;
                    VX.add(a, ma * dx); VY.add(a, ma * dy); VZ.add(a, ma * dz);
                    VX.add(b, -(mb * dx)); VY.add(b, -(mb * dy)); VZ.add(b, -(mb * dz));
                    done = 0;
                }
            }
            if (++iter > kMaxIter) break;
        }
        X.store(rx, first); Y.store(ry, first); Z.store(rz, first);
        VX.store(vx, first); VY.store(vy, first); VZ.store(vz, first);
        if (!done) atomicOr(&flags[2], 1);
        return;
    }
    while (!done) {
        done = 1;
        for (int k = 0; k < nc; ++k) {
            const int a = first + cv.ci[c0 + k], b = first + cv.cj[c0 + k];
            const double len2 = cv.len[c0 + k] * cv.len[c0 + k];
            const double px = wrap1(rx[a] - rx[b], m.box.L[0]);
            const double py = wrap1(ry[a] - ry[b], m.box.L[1]);
            const double pz = wrap1(rz[a] - rz[b], m.box.L[2]);
            const double diff = len2 - (px * px + py * py + pz * pz);
            if (fabs(diff) > len2 * tol2) {
                const double qx = wrap1(ox[a] - ox[b], m.box.L[0]);
                const double qy = wrap1(oy[a] - oy[b], m.box.L[1]);
                const double qz = wrap1(oz[a] - oz[b], m.box.L[2]);
                const double ma = cv.inv_mass[a], mb = cv.inv_mass[b];
                const double g = diff / (2.0 * (ma + mb) * (qx * px + qy * py + qz * pz));
                double dx = qx * g, dy = qy * g, dz = qz * g;
                rx[a] += ma * dx; ry[a] += ma * dy; rz[a] += ma * dz;
                rx[b] -= mb * dx; ry[b] -= mb * dy; rz[b] -= mb * dz;
                dx *= inv_dt; dy *= inv_dt; dz *= inv_dt;
                vx[a] += ma * dx; vy[a] += ma * dy; vz[a] += ma * dz;
                vx[b] -= mb * dx; vy[b] -= mb * dy; vz[b] -= mb * dz;
                done = 0;
            }
        }
        if (++iter > kMaxIter) break;
    }
    if (!done) atomicOr(&flags[2], 1);
}

// rattle_2nd, force.c:2004-2090: one thread per molecule; the constraint
// virial goes to per-block partials.
__global__ void __launch_bounds__(256) k_rattle2(MdParams m, CstrView cv, const double *rx, const double *ry,
                                                 const double *rz, double *vx, double *vy, double *vz,
                                                 int *flags, double *partials)
{
    __shared__ double sh[32 * 9];
    double vir[9] = {0.0};
    const int im = blockIdx.x * blockDim.x + threadIdx.x;
    if (im < m.n_mols) {
        const int first = cv.mol_first[im], mt = cv.mol_type[first];
        const int nc = cv.cnt[mt], c0 = cv.off[mt];
        // 1/(dt/2) and, per constraint of a three-atom molecule, the
        // reciprocal of its fixed denominator (m_a + m_b) len^2 taken once:
        // the iterations multiply where the reference divides (equal to
        // within a rounding of each product)
        const double tol = 1.0e-05, inv_hdt = 2.0 / m.dt;
        int iter = 0, done = nc == 0;
        const bool fast = !done && cv.mol_atoms[mt] == 3 && nc <= 3;
        if (fast) {
            Mol3 X, Y, Z, VX, VY, VZ, IM;
            X.load(rx, first); Y.load(ry, first); Z.load(rz, first);
            VX.load(vx, first); VY.load(vy, first); VZ.load(vz, first);
            IM.load(cv.inv_mass, first);
            int ca[3] = {0, 0, 0}, cb[3] = {0, 0, 0};
            double inv_den[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int k = 0; k < 3; ++k)
                if (k < nc) {
                    ca[k] = cv.ci[c0 + k];
                    cb[k] = cv.cj[c0 + k];
                    const double len = cv.len[c0 + k];
                    inv_den[k] = 1.0 / ((IM.get(ca[k]) + IM.get(cb[k])) * (len * len));
                }
            while (!done) {
                done = 1;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    if (k >= nc) continue;
                    const int a = ca[k], b = cb[k];
                    const double ux = VX.get(a) - VX.get(b), uy = VY.get(a) - VY.get(b), uz = VZ.get(a) - VZ.get(b);
                    const double px = wrap1(X.get(a) - X.get(b), m.box.L[0]);
                    const double py = wrap1(Y.get(a) - Y.get(b), m.box.L[1]);
                    const double pz = wrap1(Z.get(a) - Z.get(b), m.box.L[2]);
                    const double ma = IM.get(a), mb = IM.get(b);
                    const double g = -(px * ux + py * uy + pz * uz) * inv_den[k];
                    if (fabs(g) > tol) {
                        double dx = px * g, dy = py * g, dz = pz * g;
                        VX.add(a, ma * dx); VY.add(a, ma * dy); VZ.add(a, ma * dz);
                        VX.add(b, -(mb * dx)); VY.add(b, -(mb * dy)); VZ.add(b, -(mb * dz));
                        dx *= inv_hdt; dy *= inv_hdt; dz *= inv_hdt;
                        vir[0] -= px * dx; vir[1] -= px * dy; vir[2] -= px * dz;
                        vir[3] -= py * dx; vir[4] -= py * dy; vir[5] -= py * dz;
                        vir[6] -= pz * dx; vir[7] -= pz * dy; vir[8] -= pz * dz;
                        done = 0;
                    }
                }
                if (++iter > kMaxIter) break;
            }
            VX.store(vx, first); VY.store(vy, first); VZ.store(vz, first);
        }
        while (!fast && !done) {
            done = 1;
            for (int k = 0; k < nc; ++k) {
                const int a = first + cv.ci[c0 + k], b = first + cv.cj[c0 + k];
                const double len2 = cv.len[c0 + k] * cv.len[c0 + k];
                const double ux = vx[a] - vx[b], uy = vy[a] - vy[b], uz = vz[a] - vz[b];
                const double px = wrap1(rx[a] - rx[b], m.box.L[0]);
                const double py = wrap1(ry[a] - ry[b], m.box.L[1]);
                const double pz = wrap1(rz[a] - rz[b], m.box.L[2]);
                const double ma = cv.inv_mass[a], mb = cv.inv_mass[b];
                const double g = -(px * ux + py * uy + pz * uz) / ((ma + mb) * len2);
                if (fabs(g) > tol) {
                    double dx = px * g, dy = py * g, dz = pz * g;
                    vx[a] += ma * dx; vy[a] += ma * dy; vz[a] += ma * dz;
                    vx[b] -= mb * dx; vy[b] -= mb * dy; vz[b] -= mb * dz;
                    dx *= inv_hdt; dy *= inv_hdt; dz *= inv_hdt;
                    vir[0] -= px * dx; vir[1] -= px * dy; vir[2] -= px * dz;
                    vir[3] -= py * dx; vir[4] -= py * dy; vir[5] -= py * dz;
                    vir[6] -= pz * dx; vir[7] -= pz * dy; vir[8] -= pz * dz;
                    done = 0;
                }
            }
            if (++iter > kMaxIter) break;
        }
        if (!done) atomicOr(&flags[2], 2);
    }
    block_partials<9>(vir, sh, partials);
}

// partials of sum m v^2 per axis (kinetic_energy, thermostat.c:34-63)
__global__ void __launch_bounds__(256) k_kinetic(int N, const double *mass, const double *vx, const double *vy,
                                                 const double *vz, double *partials)
{
    __shared__ double sh[32 * 3];
    double v[3] = {0.0, 0.0, 0.0};
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) {
        const double mm = mass[i];
        if (mm > 0.0) {
            v[0] = mm * vx[i] * vx[i];
            v[1] = mm * vy[i] * vy[i];
            v[2] = mm * vz[i] * vz[i];
        }
    }
    block_partials<3>(v, sh, partials);
}

__global__ void k_kinetic_final(const double *partials, int nb, int ndf, ThermoState *th)
{
    __shared__ double sh[32 * 3];
    double v[3] = {0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        v[0] += partials[3 * b];
        v[1] += partials[3 * b + 1];
        v[2] += partials[3 * b + 2];
    }
    block_sum<3>(v, sh);
    if (threadIdx.x == 0) {
        th->eksum = v[0] + v[1] + v[2];
        th->inst_temp = th->eksum / (kBoltz * ndf);
    }
}

// remove_comm, thermostat.c:69-108
__global__ void __launch_bounds__(256) k_momentum(int N, const double *mass, const double *vx, const double *vy,
                                                  const double *vz, double *partials)
{
    __shared__ double sh[32 * 4];
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) {
        const double mm = mass[i];
        if (mm > 0.0) {
            v[0] = vx[i] * mm;
            v[1] = vy[i] * mm;
            v[2] = vz[i] * mm;
            v[3] = mm;
        }
    }
    block_partials<4>(v, sh, partials);
}

__global__ void k_momentum_final(const double *partials, int nb, ThermoState *th)
{
    __shared__ double sh[32 * 4];
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
        for (int k = 0; k < 4; ++k) v[k] += partials[4 * b + k];
    block_sum<4>(v, sh);
    if (threadIdx.x == 0) {
        th->vcom[0] = v[0] / v[3];
        th->vcom[1] = v[1] / v[3];
        th->vcom[2] = v[2] / v[3];
        th->vcom[3] = v[3];
    }
}

__global__ void k_sub_com(int N, const double *mass, const ThermoState *th, double *vx, double *vy, double *vz)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N || !(mass[i] > 0.0)) return;
    vx[i] -= th->vcom[0];
    vy[i] -= th->vcom[1];
    vz[i] -= th->vcom[2];
}

// apply_pbc, force.c:127-165: one thread per molecule.
__global__ void k_apply_pbc(MdParams m, const int *mol_first, const int *mol_last, double *rx, double *ry,
                            double *rz)
{
    const int im = blockIdx.x * blockDim.x + threadIdx.x;
    if (im >= m.n_mols) return;
    const int lo = mol_first[im], hi = mol_last[im], mid = (lo + hi) / 2;
    double *r[3] = {rx, ry, rz};
    const double h[3] = {0.5 * m.box.L[0], 0.5 * m.box.L[1], 0.5 * m.box.L[2]};
    for (int a = 0; a < 3; ++a) {
        if (r[a][mid] > m.box.L[a]) r[a][mid] -= m.box.L[a];
        else if (r[a][mid] < 0.0) r[a][mid] += m.box.L[a];
    }
    for (int i = lo; i <= hi; ++i) {
        if (i == mid) continue;
        for (int a = 0; a < 3; ++a) {
            if (r[a][i] - r[a][mid] > h[a]) r[a][i] -= m.box.L[a];
            else if (r[a][i] - r[a][mid] < -h[a]) r[a][i] += m.box.L[a];
        }
    }
}

// get_fmax_rms, force.c:361-378
__global__ void __launch_bounds__(256) k_fmax(int N, const double *fx, const double *fy, const double *fz,
                                              double *partials)
{
    __shared__ double sh[32 * 2];
    __shared__ double shm[8];
    double v[2] = {0.0, 0.0};
    double mx = 0.0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) {
        const double f2 = fx[i] * fx[i] + fy[i] * fy[i] + fz[i] * fz[i];
        v[0] = f2;
        mx = f2;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) shm[threadIdx.x >> 5] = mx;
    block_sum<2>(v, sh);
    if (threadIdx.x == 0) {
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) mx = fmax(mx, shm[w]);
        partials[2 * blockIdx.x] = v[0];
        partials[2 * blockIdx.x + 1] = mx;
    }
}

__global__ void k_fmax_final(const double *partials, int nb, int N, ThermoState *th)
{
    __shared__ double sh[32 * 2];
    __shared__ double shm[32];
    double v[2] = {0.0, 0.0};
    double mx = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        v[0] += partials[2 * b];
        mx = fmax(mx, partials[2 * b + 1]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) shm[threadIdx.x >> 5] = mx;
    block_sum<2>(v, sh);
    if (threadIdx.x == 0) {
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) mx = fmax(mx, shm[w]);
        th->fmax = sqrt(mx);
        th->frms = sqrt(v[0] / N);
    }
}

// Energy minimisation step (mpi-main.c:730-756): old_r = r for every atom;
// r += s / f_max * em_length except for fixed metal atoms.
__global__ void k_em_move(MdParams m, const unsigned char *is_metal, const ThermoState *th, double em_length,
                          const double *__restrict__ sx, const double *__restrict__ sy,
                          const double *__restrict__ sz, double *rx, double *ry, double *rz, double *ox, double *oy,
                          double *oz)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.N) return;
    ox[i] = rx[i];
    oy[i] = ry[i];
    oz[i] = rz[i];
    if (m.fix_metal == 1 && is_metal[i]) return;
    const double fmax = th->fmax;
    rx[i] += sx[i] / fmax * em_length;
    ry[i] += sy[i] / fmax * em_length;
    rz[i] += sz[i] / fmax * em_length;
}

// s = F + gamma s, old F = F (mpi-main.c:843-852).
__global__ void k_em_direction(int N, double gamma, const double *__restrict__ fx, const double *__restrict__ fy,
                               const double *__restrict__ fz, double *sx, double *sy, double *sz, double *gx,
                               double *gy, double *gz)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    sx[i] = fx[i] + gamma * sx[i];
    sy[i] = fy[i] + gamma * sy[i];
    sz[i] = fz[i] + gamma * sz[i];
    gx[i] = fx[i];
    gy[i] = fy[i];
    gz[i] = fz[i];
}

// Partials of g22 = (F, F), g12 = (F_old, F), g11 = (F_old, F_old) for the
// conjugate-gradient gamma (mpi-main.c:823-840).
__global__ void __launch_bounds__(256) k_em_dots(int N, const double *__restrict__ fx, const double *__restrict__ fy,
                                                 const double *__restrict__ fz, const double *__restrict__ gx,
                                                 const double *__restrict__ gy, const double *__restrict__ gz,
                                                 double *partials)
{
    __shared__ double sh[32 * 3];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[3] = {0.0, 0.0, 0.0};
    if (i < N) {
        acc[0] = fx[i] * fx[i] + fy[i] * fy[i] + fz[i] * fz[i];
        acc[1] = gx[i] * fx[i] + gy[i] * fy[i] + gz[i] * fz[i];
        acc[2] = gx[i] * gx[i] + gy[i] * gy[i] + gz[i] * gz[i];
    }
    block_partials<3>(acc, sh, partials);
}

__global__ void k_sum_potential(double *pot)
{
    double s = 0.0;
    for (int k = 1; k < 15; ++k) s += pot[k];
    pot[0] = s;
}

CstrView cstr_view(const capac_ctx *c)
{
    CstrView v;
    v.mol_first = c->mol_first;
    v.mol_type = c->mol_type;
    v.off = c->cstr_off;
    v.cnt = c->cstr_cnt;
    v.ci = c->cstr_i;
    v.cj = c->cstr_j;
    v.len = c->cstr_r;
    v.inv_mass = c->inv_mass;
    v.mol_atoms = c->mol_atoms;
    return v;
}

}  // namespace

void launch_heating(capac_ctx *c, long step)
{
    k_heating<<<1, 1, 0, c->stream>>>(c->th, step, c->n_heating);
    ++c->launches;
}

void launch_nhc(capac_ctx *c)
{
    k_nhc<<<1, 1, 0, c->stream>>>(c->th, md_params(c));
    ++c->launches;
}

void launch_berendsen(capac_ctx *c)
{
    k_berendsen<<<1, 1, 0, c->stream>>>(c->th, c->dt_over_tau);
    ++c->launches;
}

void launch_md_half_kick(capac_ctx *c, bool with_nhc_scale)
{
    k_half_kick<<<grid_for(c->N, 256), 256, 0, c->stream>>>(md_params(c), c->is_metal, c->inv_mass, c->fx, c->fy,
                                                           c->fz, c->vx, c->vy, c->vz, c->th,
                                                           with_nhc_scale ? 1 : 0);
    ++c->launches;
}

void launch_scale_velocities(capac_ctx *c)
{
    k_scale_velocities<<<grid_for(c->N, 256), 256, 0, c->stream>>>(c->N, c->th, c->vx, c->vy, c->vz);
    ++c->launches;
}

void launch_md_drift(capac_ctx *c)
{
    k_drift<<<grid_for(c->N, 256), 256, 0, c->stream>>>(md_params(c), c->is_metal, c->rx, c->ry, c->rz, c->vx,
                                                       c->vy, c->vz, c->ox, c->oy, c->oz);
    ++c->launches;
}

void launch_rattle(capac_ctx *c, int second)
{
    if (!c->has_cstr) return;
    const unsigned grid = grid_for(c->n_mols, 256);
    if (!second) {
        k_rattle1<<<grid, 256, 0, c->stream>>>(md_params(c), cstr_view(c), c->rx, c->ry, c->rz, c->ox, c->oy, c->oz,
                                               c->vx, c->vy, c->vz, c->flags);
        ++c->launches;
    } else {
        k_rattle2<<<grid, 256, 0, c->stream>>>(md_params(c), cstr_view(c), c->rx, c->ry, c->rz, c->vx, c->vy, c->vz,
                                               c->flags, c->partials);
        ++c->launches;
        static const int pot_slots[9] = {-1, -1, -1, -1, -1, -1, -1, -1, -1};
        static const int vir_slots[9] = {0, 1, 2, 3, 4, 5, 6, 7, 8};
        launch_finalize(c, (int)grid, 9, pot_slots, vir_slots);
    }
}

void launch_kinetic(capac_ctx *c)
{
    const unsigned grid = grid_for(c->N, 256);
    k_kinetic<<<grid, 256, 0, c->stream>>>(c->N, c->mass, c->vx, c->vy, c->vz, c->partials);
    k_kinetic_final<<<1, 256, 0, c->stream>>>(c->partials, (int)grid, c->c.ndf, c->th);
    c->launches += 2;
}

void launch_remove_com(capac_ctx *c)
{
    const unsigned grid = grid_for(c->N, 256);
    k_momentum<<<grid, 256, 0, c->stream>>>(c->N, c->mass, c->vx, c->vy, c->vz, c->partials);
    k_momentum_final<<<1, 256, 0, c->stream>>>(c->partials, (int)grid, c->th);
    k_sub_com<<<grid, 256, 0, c->stream>>>(c->N, c->mass, c->th, c->vx, c->vy, c->vz);
    c->launches += 3;
}

void launch_apply_pbc(capac_ctx *c)
{
    k_apply_pbc<<<grid_for(c->n_mols, 256), 256, 0, c->stream>>>(md_params(c), c->mol_first, c->mol_last, c->rx,
                                                                c->ry, c->rz);
    ++c->launches;
}

void launch_fmax_rms(capac_ctx *c)
{
    const unsigned grid = grid_for(c->N, 256);
    k_fmax<<<grid, 256, 0, c->stream>>>(c->N, c->fx, c->fy, c->fz, c->partials);
    k_fmax_final<<<1, 256, 0, c->stream>>>(c->partials, (int)grid, c->N, c->th);
    c->launches += 2;
}

void launch_sum_potential(capac_ctx *c)
{
    k_sum_potential<<<1, 1, 0, c->stream>>>(c->pot);
    ++c->launches;
}

// em_buf layout: sx sy sz | old fx fy fz, N each
void launch_em_move(capac_ctx *c)
{
    const size_t N = c->N;
    k_em_move<<<grid_for(c->N, 256), 256, 0, c->stream>>>(md_params(c), c->is_metal, c->th, c->em_length, c->em_buf,
                                                         c->em_buf + N, c->em_buf + 2 * N, c->rx, c->ry, c->rz,
                                                         c->ox, c->oy, c->oz);
    ++c->launches;
}

void launch_em_direction(capac_ctx *c, double gamma)
{
    const size_t N = c->N;
    double *b = c->em_buf;
    k_em_direction<<<grid_for(c->N, 256), 256, 0, c->stream>>>(c->N, gamma, c->fx, c->fy, c->fz, b, b + N,
                                                              b + 2 * N, b + 3 * N, b + 4 * N, b + 5 * N);
    ++c->launches;
}

void launch_em_dots(capac_ctx *c)
{
    const size_t N = c->N;
    const double *b = c->em_buf;
    k_em_dots<<<grid_for(c->N, 256), 256, 0, c->stream>>>(c->N, c->fx, c->fy, c->fz, b + 3 * N, b + 4 * N,
                                                         b + 5 * N, c->partials);
    ++c->launches;
}

}  // namespace capac
