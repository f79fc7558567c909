// Bonded terms and virtual sites (force.c:822-1347, 1582-1900).
//
// One thread per molecule walks its molecule type's terms in the reference's
// order (bonds, 1-4 pairs, angles, dihedrals), as mpi_bonded does; atoms
// belong to one molecule, so the forces need no atomics and the sums keep
// the reference's order within a molecule.  Energies go to potential[2]
// (bonds, Urey-Bradley), [3] (angles), [4] (dihedrals), [7] and [8] (1-4
// Coulomb and LJ); the virial follows each term's own convention (the RB
// dihedral's uses the PBC-treated absolute positions, force.c:1205-1230).
// Virtual sites (funct 4): positions built before the force evaluation
// (build_vsites, force.c:1582-1629), their forces distributed to the three
// constructing atoms after it (mpi_vsites, force.c:1636-1690).
#include "terms.cuh"

namespace capac {

namespace {

constexpr double kPiB = 3.14159265358979323846;  // M_PI

struct V3 {
    double x, y, z;
};

__device__ __forceinline__ V3 wrapped(double dx, double dy, double dz, const Box &b)
{
    return V3{wrap1(dx, b.L[0]), wrap1(dy, b.L[1]), wrap1(dz, b.L[2])};
}
__device__ __forceinline__ double dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 scale3(double s, V3 v) { return V3{s * v.x, s * v.y, s * v.z}; }
__device__ __forceinline__ V3 cross3(V3 a, V3 b)
{
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// vir[a][b] -= r_a f_b
__device__ __forceinline__ void vir_sub(double *vir, V3 r, V3 f)
{
    const double rr[3] = {r.x, r.y, r.z}, ff[3] = {f.x, f.y, f.z};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) vir[3 * a + b] -= rr[a] * ff[b];
}

// acc: 0 bond, 1 angle, 2 dihedral, 3 Coulomb 1-4, 4 LJ 1-4, 5..13 virial
constexpr int kAcc = 14;

// compute_bond_1 (force.c:822-862): returns the force on j (i gets minus it)
__device__ V3 bond_harmonic(V3 ri, V3 rj, double b0, double kb, const Box &box, double *acc)
{
    const V3 r = wrapped(rj.x - ri.x, rj.y - ri.y, rj.z - ri.z, box);
    const double rij = sqrt(norm2_exact(r.x, r.y, r.z));
    const double fij = kb * (b0 - rij) / rij;
    const V3 fj = scale3(fij, r);
    acc[0] += 0.5 * kb * (b0 - rij) * (b0 - rij);
    vir_sub(acc + 5, r, fj);
    return fj;
}

// compute_bond_3 (force.c:867-910), Morse
__device__ V3 bond_morse(V3 ri, V3 rj, double b0, double D, double beta, const Box &box, double *acc)
{
    const V3 r = wrapped(rj.x - ri.x, rj.y - ri.y, rj.z - ri.z, box);
    const double rij = sqrt(norm2_exact(r.x, r.y, r.z));
    const double e = exp(-beta * (rij - b0));
    const double fij = -2.0 * D * beta * e * (1.0 - e) / rij;
    const V3 fj = scale3(fij, r);
    acc[0] += D * ((1.0 - e) * (1.0 - e));
    vir_sub(acc + 5, r, fj);
    return fj;
}

// compute_angle_1 (force.c:956-1016): forces on i and k (j gets minus both)
__device__ void angle_harmonic(V3 ri, V3 rj, V3 rk, double a0, double ka, const Box &box, double *acc, V3 &fi,
                               V3 &fk)
{
    const V3 r21 = wrapped(ri.x - rj.x, ri.y - rj.y, ri.z - rj.z, box);
    const double d21 = sqrt(norm2_exact(r21.x, r21.y, r21.z));
    const V3 u21 = scale3(1.0 / d21, r21);
    const V3 r32 = wrapped(rj.x - rk.x, rj.y - rk.y, rj.z - rk.z, box);
    const double d32 = sqrt(norm2_exact(r32.x, r32.y, r32.z));
    const V3 u32 = scale3(1.0 / d32, r32);
    const double cs = -dot3(u21, u32);
    const double theta = acos(cs), sn = sin(theta);
    const double delta = a0 * kPiB / 180.0 - theta;
    const double f = ka * delta;
    fi = V3{(cs * u21.x + u32.x) / (sn * d21) * f, (cs * u21.y + u32.y) / (sn * d21) * f,
            (cs * u21.z + u32.z) / (sn * d21) * f};
    fk = V3{-(cs * u32.x + u21.x) / (sn * d32) * f, -(cs * u32.y + u21.y) / (sn * d32) * f,
            -(cs * u32.z + u21.z) / (sn * d32) * f};
    acc[1] += 0.5 * ka * delta * delta;
    vir_sub(acc + 5, r21, fi);
    vir_sub(acc + 5, V3{-r32.x, -r32.y, -r32.z}, fk);
}

// compute_dihedral_3 (force.c:1100-1233), RB form: forces on i, j, k, l
__device__ void dihedral_rb(V3 ri, V3 rj, V3 rk, V3 rl, const double *c, const Box &box, double *acc, V3 &fi,
                            V3 &fj, V3 &fk, V3 &fl)
{
    const V3 r21 = wrapped(ri.x - rj.x, ri.y - rj.y, ri.z - rj.z, box);
    const double d21 = sqrt(norm2_exact(r21.x, r21.y, r21.z));
    const V3 u21 = scale3(1.0 / d21, r21);
    const V3 r32 = wrapped(rj.x - rk.x, rj.y - rk.y, rj.z - rk.z, box);
    const double d32 = sqrt(norm2_exact(r32.x, r32.y, r32.z));
    const V3 u32 = scale3(1.0 / d32, r32);
    const V3 r43 = wrapped(rk.x - rl.x, rk.y - rl.y, rk.z - rl.z, box);
    const double d43 = sqrt(norm2_exact(r43.x, r43.y, r43.z));
    const V3 u43 = scale3(1.0 / d43, r43);
    const double cs123 = -dot3(u21, u32), sn123 = sin(acos(cs123));
    const double cs234 = -dot3(u32, u43), sn234 = sin(acos(cs234));
    const double cp = (cs123 * cs234 - dot3(u21, u43)) / (sn123 * sn234);
    const double cp2 = cp * cp, cp3 = cp2 * cp, cp4 = cp3 * cp, cp5 = cp4 * cp;
    // polymer convention: psi = phi - 180, the signs of odd terms flipped
    acc[2] += c[0] - c[1] * cp + c[2] * cp2 - c[3] * cp3 + c[4] * cp4 - c[5] * cp5;
    const double f = -(-c[1] + c[2] * 2.0 * cp - c[3] * 3.0 * cp2 + c[4] * 4.0 * cp3 - c[5] * 5.0 * cp4);
    const V3 x2132 = cross3(u21, u32), x4332 = cross3(u43, u32);
    const double s123_3 = sn123 * sn123 * sn123, s234_3 = sn234 * sn234 * sn234;
    const double k1 = dot3(u43, x2132) / (d21 * s123_3 * sn234);
    const double k4 = dot3(u43, x2132) / (d43 * s234_3 * sn123);
    const double c123 = d21 * cs123 / d32 - 1.0, b432 = d43 * cs234 / d32;
    fi = V3{-k1 * x2132.x * f, -k1 * x2132.y * f, -k1 * x2132.z * f};
    fl = V3{-k4 * x4332.x * f, -k4 * x4332.y * f, -k4 * x4332.z * f};
    fj = V3{c123 * fi.x - b432 * fl.x, c123 * fi.y - b432 * fl.y, c123 * fi.z - b432 * fl.z};
    fk = V3{-fi.x - fj.x - fl.x, -fi.y - fj.y - fl.y, -fi.z - fj.z - fl.z};
    V3 rv = ri;
    vir_sub(acc + 5, rv, fi);
    rv = V3{rv.x - r21.x, rv.y - r21.y, rv.z - r21.z};
    vir_sub(acc + 5, rv, fj);
    rv = V3{rv.x - r32.x, rv.y - r32.y, rv.z - r32.z};
    vir_sub(acc + 5, rv, fk);
    rv = V3{rv.x - r43.x, rv.y - r43.y, rv.z - r43.z};
    vir_sub(acc + 5, rv, fl);
}

// compute_nonbonded with is_14_pair = 1 (force.c:710-816): plain LJ and
// Coulomb scaled by scaleLJ / scaleQQ; returns the force on j
__device__ V3 pair_14(V3 ri, V3 rj, double c6, double c12, double qi, double qj, double slj, double sqq,
                      const Box &box, double *acc)
{
    const V3 r = wrapped(rj.x - ri.x, rj.y - ri.y, rj.z - ri.z, box);
    const double r2 = norm2_exact(r.x, r.y, r.z), rij = sqrt(r2);
    V3 f{0.0, 0.0, 0.0};
    if (c6 != 0.0 || c12 != 0.0) {
        const double r6 = r2 * r2 * r2, r12 = r6 * r6;
        const double fij = (c12 * 2.0 / r12 - c6 / r6) * 6.0 / r2 * slj;
        acc[4] += (c12 / r12 - c6 / r6) * slj;
        f = scale3(fij, r);
    }
    if (qi != 0.0 && qj != 0.0) {
        const double fij = sqq * kFQQ * qi * qj / (r2 * rij);
        acc[3] += sqq * kFQQ * qi * qj / rij;
        f = V3{f.x + fij * r.x, f.y + fij * r.y, f.z + fij * r.z};
    }
    vir_sub(acc + 5, r, f);
    return f;
}

__device__ __forceinline__ void add_force(double *fx, double *fy, double *fz, int a, V3 f)
{
    fx[a] += f.x;
    fy[a] += f.y;
    fz[a] += f.z;
}
__device__ __forceinline__ V3 neg(V3 v) { return V3{-v.x, -v.y, -v.z}; }
__device__ __forceinline__ V3 at(const double *rx, const double *ry, const double *rz, int a)
{
    return V3{rx[a], ry[a], rz[a]};
}

__global__ void __launch_bounds__(128) k_bonded(DevParams P, BondedView B, const double *__restrict__ rx,
                                                const double *__restrict__ ry, const double *__restrict__ rz,
                                                double *fx, double *fy, double *fz, double *partials)
{
    __shared__ double sh[32 * kAcc];
    const int im = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[kAcc];
#pragma unroll
    for (int k = 0; k < kAcc; ++k) acc[k] = 0.0;
    if (im < B.n_mols) {
        const int first = B.mol_first[im], mt = P.mol_type[first];
        const int t0 = B.bt_offset[mt], nt = B.bt_count[mt];
        for (int t = t0; t < t0 + nt; ++t) {
            const int *ai = B.bt_atoms + 4 * (size_t)t;
            const double *p = B.bt_par + 6 * (size_t)t;
            const int i = first + ai[0], j = first + ai[1], k = first + ai[2], l = first + ai[3];
            const V3 ri = at(rx, ry, rz, i), rj = at(rx, ry, rz, j);
            switch (B.bt_kind[t]) {
            case CAPAC_BT_BOND_HARMONIC: {
                const V3 f = bond_harmonic(ri, rj, p[0], p[1], P.box, acc);
                add_force(fx, fy, fz, i, neg(f));
                add_force(fx, fy, fz, j, f);
                break;
            }
            case CAPAC_BT_BOND_MORSE: {
                const V3 f = bond_morse(ri, rj, p[0], p[1], p[2], P.box, acc);
                add_force(fx, fy, fz, i, neg(f));
                add_force(fx, fy, fz, j, f);
                break;
            }
            case CAPAC_BT_PAIR_14:
            case CAPAC_BT_PAIR_USER: {
                double c6, c12, qi, qj, slj, sqq;
                if (B.bt_kind[t] == CAPAC_BT_PAIR_14) {
                    const double4 np = P.nb_par[P.type[i] * P.n_types + P.type[j]];
                    c6 = np.x;
                    c12 = np.y;
                    qi = P.charge[i];
                    qj = P.charge[j];
                    slj = B.scale_lj;
                    sqq = B.scale_qq;
                } else {
                    sqq = p[0];
                    qi = p[1];
                    qj = p[2];
                    c6 = p[3];
                    c12 = p[4];
                    slj = 1.0;
                }
                const V3 f = pair_14(ri, rj, c6, c12, qi, qj, slj, sqq, P.box, acc);
                add_force(fx, fy, fz, i, neg(f));
                add_force(fx, fy, fz, j, f);
                break;
            }
            case CAPAC_BT_ANGLE_HARMONIC:
            case CAPAC_BT_ANGLE_UB: {
                const V3 rk = at(rx, ry, rz, k);
                V3 fi, fk;
                angle_harmonic(ri, rj, rk, p[0], p[1], P.box, acc, fi, fk);
                const V3 fj = V3{-fi.x - fk.x, -fi.y - fk.y, -fi.z - fk.z};
                if (B.bt_kind[t] == CAPAC_BT_ANGLE_UB && p[3] > 0.0) {  // compute_angle_5, force.c:1021-1053
                    const V3 fb = bond_harmonic(ri, rk, p[2], p[3], P.box, acc);
                    fi = V3{fi.x - fb.x, fi.y - fb.y, fi.z - fb.z};
                    fk = V3{fk.x + fb.x, fk.y + fb.y, fk.z + fb.z};
                }
                add_force(fx, fy, fz, i, fi);
                add_force(fx, fy, fz, j, fj);
                add_force(fx, fy, fz, k, fk);
                break;
            }
            case CAPAC_BT_DIHEDRAL_RB: {
                const V3 rk = at(rx, ry, rz, k), rl = at(rx, ry, rz, l);
                V3 fi, fj, fk, fl;
                dihedral_rb(ri, rj, rk, rl, p, P.box, acc, fi, fj, fk, fl);
                add_force(fx, fy, fz, i, fi);
                add_force(fx, fy, fz, j, fj);
                add_force(fx, fy, fz, k, fk);
                add_force(fx, fy, fz, l, fl);
                break;
            }
            default:
                break;
            }
        }
    }
    block_partials<kAcc>(acc, sh, partials);
}

// build_vsites (force.c:1582-1629): r_s = r_i + a r_ij + b r_ik + c (r_ij x r_ik)
__global__ void __launch_bounds__(128) k_build_vsites(DevParams P, BondedView B, double *rx, double *ry, double *rz)
{
    const int im = blockIdx.x * blockDim.x + threadIdx.x;
    if (im >= B.n_mols) return;
    const int first = B.mol_first[im], mt = P.mol_type[first];
    for (int v = B.vs_offset[mt]; v < B.vs_offset[mt] + B.vs_count[mt]; ++v) {
        const int i = first + B.vs_atoms[4 * v], j = first + B.vs_atoms[4 * v + 1];
        const int k = first + B.vs_atoms[4 * v + 2], s = first + B.vs_atoms[4 * v + 3];
        const double a = B.vs_par[3 * v], b = B.vs_par[3 * v + 1], c = B.vs_par[3 * v + 2];
        const V3 rij = wrapped(rx[j] - rx[i], ry[j] - ry[i], rz[j] - rz[i], P.box);
        const V3 rik = wrapped(rx[k] - rx[i], ry[k] - ry[i], rz[k] - rz[i], P.box);
        const V3 x = cross3(rij, rik);
        rx[s] = rx[i] + a * rij.x + b * rik.x + c * x.x;
        ry[s] = ry[i] + a * rij.y + b * rik.y + c * x.y;
        rz[s] = rz[i] + a * rij.z + b * rik.z + c * x.z;
    }
}

// mpi_vsites with compute_vsite_4 (force.c:1060-1093, 1636-1690)
__global__ void __launch_bounds__(128) k_vsite_forces(DevParams P, BondedView B, const double *__restrict__ rx,
                                                      const double *__restrict__ ry, const double *__restrict__ rz,
                                                      double *fx, double *fy, double *fz)
{
    const int im = blockIdx.x * blockDim.x + threadIdx.x;
    if (im >= B.n_mols) return;
    const int first = B.mol_first[im], mt = P.mol_type[first];
    for (int v = B.vs_offset[mt]; v < B.vs_offset[mt] + B.vs_count[mt]; ++v) {
        const int i = first + B.vs_atoms[4 * v], j = first + B.vs_atoms[4 * v + 1];
        const int k = first + B.vs_atoms[4 * v + 2], s = first + B.vs_atoms[4 * v + 3];
        const double a = B.vs_par[3 * v], b = B.vs_par[3 * v + 1], c = B.vs_par[3 * v + 2];
        const V3 rij = wrapped(rx[j] - rx[i], ry[j] - ry[i], rz[j] - rz[i], P.box);
        const V3 rik = wrapped(rx[k] - rx[i], ry[k] - ry[i], rz[k] - rz[i], P.box);
        const double sx = fx[s], sy = fy[s], sz = fz[s];
        const V3 fj{a * sx - c * rik.z * sy + c * rik.y * sz, c * rik.z * sx + a * sy - c * rik.x * sz,
                    -c * rik.y * sx + c * rik.x * sy + a * sz};
        const V3 fk{b * sx + c * rij.z * sy - c * rij.y * sz, -c * rij.z * sx + b * sy + c * rij.x * sz,
                    c * rij.y * sx - c * rij.x * sy + b * sz};
        const V3 fi{sx - fj.x - fk.x, sy - fj.y - fk.y, sz - fj.z - fk.z};
        add_force(fx, fy, fz, i, fi);
        add_force(fx, fy, fz, j, fj);
        add_force(fx, fy, fz, k, fk);
        fx[s] = 0.0;
        fy[s] = 0.0;
        fz[s] = 0.0;
    }
}

}  // namespace

void launch_build_vsites(capac_ctx *c)
{
    if (!c->has_vsites) return;
    k_build_vsites<<<grid_for(c->n_mols, 128), 128, 0, c->stream>>>(c->P, c->bview, c->rx, c->ry, c->rz);
    ++c->launches;
}

void launch_bonded(capac_ctx *c)
{
    if (!c->has_bonded) return;
    const unsigned grid = grid_for(c->n_mols, 128);
    k_bonded<<<grid, 128, 0, c->stream>>>(c->P, c->bview, c->rx, c->ry, c->rz, c->fx, c->fy, c->fz, c->partials);
    ++c->launches;
    static const int pot_slots[kAcc] = {2, 3, 4, 7, 8, -1, -1, -1, -1, -1, -1, -1, -1, -1};
    static const int vir_slots[kAcc] = {-1, -1, -1, -1, -1, 0, 1, 2, 3, 4, 5, 6, 7, 8};
    launch_finalize(c, (int)grid, kAcc, pot_slots, vir_slots);
}

void launch_vsite_forces(capac_ctx *c)
{
    if (!c->has_vsites) return;
    k_vsite_forces<<<grid_for(c->n_mols, 128), 128, 0, c->stream>>>(c->P, c->bview, c->rx, c->ry, c->rz, c->fx,
                                                                    c->fy, c->fz);
    ++c->launches;
}

}  // namespace capac
