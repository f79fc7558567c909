/*
 * capac_oracle.c -- CPU restatement of CapacMD's per-timestep force-and-solve
 * path, used ONLY as a test oracle (by tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg).  Nothing in the product library calls it.
 *
 * Pinned against the reference itself: tests/golden/ holds outputs of the
 * reference sources compiled in place (oracle/Makefile target `ref`), made by
 * tests/golden/make_golden.py, and tests/test_oracle_golden.py checks this
 * file against them.
 *
 * Arithmetic is plain FP64 and follows the reference's expression order where
 * the result is discontinuous (cut-off tests use the reference's r^2 formula,
 * force.c:41-44, with the single conditional image shift, force.c:111-121).
 * The CPIM matrix is held dense (n_mat x n_mat) instead of COO; entries with
 * |e| <= 1e-15 are dropped as the reference does (typedef.h:89-93).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

#include "capacmd.h"

#define FQQ 138.935457696552          /* typedef.h:61 */
#define NM2BOHR 18.8972612456506      /* typedef.h:67 */
#define K_BOLTZ 0.00831446214546895   /* typedef.h:73 */
#define INV_SQRT_PI 0.564189583547756 /* typedef.h:44 */
#define MAX_ITER 1000                 /* typedef.h:85 */
#define THRSHD 1.0e-15                /* typedef.h:89-93 */
#define CONV_E 2.01552955019358e-05   /* cpff.c:72 */
#define CONV_V 3.80879884583368e-04   /* cpff.c:75 */
#define FQQ_AU2 49614.7526045429      /* cpff.c:758 */
#define FQQ_AU1 2625.49964037578      /* cpff.c:759 */
#define NHC_LEN 10                    /* mpi-main.c:514 */

typedef struct orc {
    const capac_desc *d;
    capac_consts c;
    int N, M, n_mat, step;
    double box[6];
    double *rx, *ry, *rz, *vx, *vy, *vz, *fx, *fy, *fz, *ox, *oy, *oz;
    double pot[15], vir[9];
    double *inv_sqrt_dens, *vec_ext, *vec_pq, *diag, *A;
    double *w; /* BiCGSTAB work vectors: Ax r0 r p v s t y z Kt K */
    double eksum, inst_temp, ref_temp, first_temp, ext_temp;
    double vQ[NHC_LEN], aQ[NHC_LEN];
    double solver_tol;
    int iterations;
    double f_max, f_rms;
    int error;
    int *sample; /* atoms whose nonbonded forces are formed when set (orc_set_sample) */
    int n_sample;
} orc;

/* ---------------------------------------------------------- geometry */

/* pbc_12, force.c:111-121: one conditional shift per axis. */
static void image(double *x, double *y, double *z, const double *box)
{
    if (*x < -box[3]) *x += box[0]; else if (*x > box[3]) *x -= box[0];
    if (*y < -box[4]) *y += box[1]; else if (*y > box[4]) *y -= box[1];
    if (*z < -box[5]) *z += box[2]; else if (*z > box[5]) *z -= box[2];
}

/* dist_2, force.c:41-44 */
static double norm2(double x, double y, double z) { return x * x + y * y + z * z; }

/* pbc, force.c:104-109 */
static double wrap1(double dx, double L)
{
    if (dx < -0.5 * L) dx += L; else if (dx > 0.5 * L) dx -= L;
    return dx;
}

static void acc_vir(double *v, double rx, double ry, double rz, double fx, double fy, double fz,
                    double s)
{
    v[0] -= rx * fx * s; v[1] -= rx * fy * s; v[2] -= rx * fz * s;
    v[3] -= ry * fx * s; v[4] -= ry * fy * s; v[5] -= ry * fz * s;
    v[6] -= rz * fx * s; v[7] -= rz * fy * s; v[8] -= rz * fz * s;
}

/* ---------------------------------------------------- nonbonded pairs */

/* Scalar force factor and energies of one pair at distance^2 r2 (force j
 * gets fij * rvec).  Follows compute_erf_vdw force.c:591-632, compute_morse
 * :639-667, compute_buckingham :674-703, compute_nonbonded :710-816 (non-1-4). */
static double pair_term(const orc *o, int ti, int tj, double qi, double qj, double r2, double *e_qq,
                        double *e_vdw)
{
    const capac_desc *d = o->d;
    const int k = ti * d->n_types + tj;
    const int fn = d->nb_funct[k];
    const double r = sqrt(r2);
    double f_vdw = 0.0, f_qq = 0.0;
    if (fn == 4) {
        const double c6 = d->nb_c6[k], c12 = d->nb_c12[k], w = d->nb_a[k];
        if (c6 != 0.0 || c12 != 0.0) {
            const double r6 = r2 * r2 * r2, r12 = r6 * r6;
            const double a12 = c12 / r12, a6 = c6 / r6, u = r / w, eu = erf(u);
            *e_vdw += (a12 - a6) * eu;
            f_vdw = ((12.0 * a12 - 6.0 * a6) / r * eu - (a12 - a6) * 2.0 * INV_SQRT_PI * exp(-u * u) / w) / r;
        }
        return f_vdw;
    }
    if (fn == 3) {
        const double D = d->nb_a[k], a = d->nb_b[k], R = d->nb_c6[k];
        const double e1 = exp(-a * (r - R)), e2 = e1 * e1;
        *e_vdw += D * (e2 - 2.0 * e1);
        return 2.0 * D * a * (e2 - e1) / r;
    }
    if (fn == 2) {
        const double A = d->nb_a[k], B = d->nb_b[k], c6 = d->nb_c6[k];
        const double r6 = r2 * r2 * r2, r8 = r6 * r2, eb = exp(-B * r);
        *e_vdw += A * eb - c6 / r6;
        return A * eb * B / r - 6.0 * c6 / r8;
    }
    /* funct 1: LJ plus Coulomb */
    const double c6 = d->nb_c6[k], c12 = d->nb_c12[k];
    if (c6 != 0.0 || c12 != 0.0) {
        const double r6 = r2 * r2 * r2, r12 = r6 * r6;
        if (d->use_vdw == 1) {
            const double fr = 12.0 * c12 / r12 - 6.0 * c6 / r6;
            const double fc = 12.0 * c12 * o->c.inv_rc12 - 6.0 * c6 * o->c.inv_rc6;
            f_vdw = (fr - fc) / r2;
            *e_vdw += (c12 / r12 - c6 / r6) + (r - d->r_cut) * fc / d->r_cut -
                      (c12 * o->c.inv_rc12 - c6 * o->c.inv_rc6);
        } else {
            f_vdw = (c12 * 2.0 / r12 - c6 / r6) * 6.0 / r2;
            *e_vdw += c12 / r12 - c6 / r6;
        }
    }
    if (qi != 0.0 && qj != 0.0) {
        if (d->use_coulomb == 1) {
            const double a = d->w_alpha, ec = erfc(a * r);
            f_qq = FQQ * qi * qj * ((ec / r2 + o->c.w_a2_sqrtpi * exp(-a * a * r2) / r) - o->c.w_const) / r;
            *e_qq += FQQ * qi * qj * (ec / r - o->c.w_erfc_arcut + o->c.w_const * (r - d->r_cut));
        } else {
            f_qq = FQQ * qi * qj / (r2 * r);
            *e_qq += FQQ * qi * qj / r;
        }
    }
    return f_vdw + f_qq;
}

static int excluded(const capac_desc *d, int i, int j)
{
    if (d->mol_id[i] != d->mol_id[j]) return 0;
    const int m = d->mol_type[i], na = d->mol_atoms[m];
    return d->excl[d->excl_offset[m] + d->atom_in_mol[i] * na + d->atom_in_mol[j]] != 0;
}

/* Cells of edge >= rc over the box, for traversals that must visit exactly
 * the reference's pairs without its N(N-1)/2 loop.  Positions wrapped into the
 * box pick a cell; two atoms that pbc_12 puts within rc are within rc of each
 * other's minimum image, so they lie in neighbouring cells, and with three or
 * more cells per edge the 27 cells around a cell are distinct, so each pair
 * is met once.  cells_build returns 0 (nothing allocated) for boxes with
 * fewer than three cells along an edge. */
typedef struct cells {
    int nc[3];
    int *cell;  /* [N] cell of each atom */
    int *start; /* [cells + 1] */
    int *atoms; /* [N] atoms in cell order, ascending index within a cell */
} cells;

static int cells_build(const orc *o, cells *c)
{
    const int N = o->N;
    for (int a = 0; a < 3; ++a) c->nc[a] = (int)floor(o->box[a] / o->d->r_cut);
    if (c->nc[0] < 3 || c->nc[1] < 3 || c->nc[2] < 3) return 0;
    const int ncell = c->nc[0] * c->nc[1] * c->nc[2];
    c->cell = (int *)malloc(sizeof(int) * (size_t)N);
    c->start = (int *)calloc((size_t)ncell + 1, sizeof(int));
    c->atoms = (int *)malloc(sizeof(int) * (size_t)N);
    int *fill = (int *)malloc(sizeof(int) * (size_t)ncell);
    const double *r[3] = {o->rx, o->ry, o->rz};
    for (int i = 0; i < N; ++i) {
        int k3[3];
        for (int a = 0; a < 3; ++a) {
            const double L = o->box[a];
            const double w = r[a][i] - L * floor(r[a][i] / L);
            const int k = (int)(w / L * c->nc[a]);
            k3[a] = k < 0 ? 0 : (k >= c->nc[a] ? c->nc[a] - 1 : k);
        }
        c->cell[i] = (k3[0] * c->nc[1] + k3[1]) * c->nc[2] + k3[2];
        ++c->start[c->cell[i] + 1];
    }
    for (int k = 0; k < ncell; ++k) c->start[k + 1] += c->start[k];
    memcpy(fill, c->start, sizeof(int) * (size_t)ncell);
    for (int i = 0; i < N; ++i) c->atoms[fill[c->cell[i]]++] = i;
    free(fill);
    return 1;
}

static void cells_free(cells *c)
{
    free(c->cell); free(c->start); free(c->atoms);
}

/* The k-th (0..26) cell around atom i's cell. */
static int cells_near(const cells *c, int i, int k)
{
    const int ci = c->cell[i], nz = c->nc[2], ny = c->nc[1];
    const int cz = ci % nz, cy = (ci / nz) % ny, cx = ci / (ny * nz);
    const int kx = (cx + k / 9 - 1 + c->nc[0]) % c->nc[0], ky = (cy + (k / 3) % 3 - 1 + ny) % ny,
              kz = (cz + k % 3 - 1 + nz) % nz;
    return (kx * ny + ky) * nz + kz;
}

/* Accumulators of the pair loop: forces (fx, fy, fz of N each), the
 * Coulomb and van der Waals energies, the virial. */
typedef struct nb_acc {
    double *fx, *fy, *fz;
    double e_qq, e_vdw;
    double vir[9];
} nb_acc;

/* One pair of mpi_nonb_pair's loop (force.c:1440-1538): i > j, r = r_j - r_i. */
static void nonbonded_pair(const orc *o, int i, int j, nb_acc *a)
{
    const capac_desc *d = o->d;
    const double rc = d->r_cut;
    if (excluded(d, i, j)) return;
    double x = o->rx[j] - o->rx[i], y = o->ry[j] - o->ry[i], z = o->rz[j] - o->rz[i];
    image(&x, &y, &z, o->box);
    if (x >= rc && y >= rc && z >= rc) return;
    const double r2 = norm2(x, y, z);
    if (r2 >= o->c.r_cut2) return;
    const double f = pair_term(o, d->atom_type[i], d->atom_type[j], d->charge[i], d->charge[j], r2, &a->e_qq,
                               &a->e_vdw);
    const double fjx = f * x, fjy = f * y, fjz = f * z;
    a->fx[i] -= fjx; a->fy[i] -= fjy; a->fz[i] -= fjz;
    a->fx[j] += fjx; a->fy[j] += fjy; a->fz[j] += fjz;
    acc_vir(a->vir, x, y, z, fjx, fjy, fjz, 1.0);
}

/* All pairs j < i of rows i = first, first + stride, ..., through cells when
 * c is set, else the reference's loop. */
static void nonbonded_rows(const orc *o, const cells *c, int first, int stride, nb_acc *a)
{
    for (int i = first; i < o->N; i += stride) {
        if (c) {
            for (int k = 0; k < 27; ++k) {
                const int cc = cells_near(c, i, k);
                for (int t = c->start[cc]; t < c->start[cc + 1]; ++t)
                    if (c->atoms[t] < i) nonbonded_pair(o, i, c->atoms[t], a);
            }
        } else {
            for (int j = 0; j < i; ++j) nonbonded_pair(o, i, j, a);
        }
    }
}

/* Host threads for the large-system loops: the online cores, at most 64. */
static int host_threads(void)
{
    const long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n < 1 ? 1 : (n > 64 ? 64 : (int)n);
}

typedef struct nb_job {
    const orc *o;
    const cells *c;
    int first, stride;
    nb_acc acc;
} nb_job;

static void *nb_thread(void *arg)
{
    nb_job *j = (nb_job *)arg;
    nonbonded_rows(j->o, j->c, j->first, j->stride, &j->acc);
    return NULL;
}

static void nonbonded_with(orc *o, const cells *c)
{
    const int N = o->N;
    const int nt = N >= 2048 ? host_threads() : 1;
    if (nt <= 1) {
        nb_acc a = {o->fx, o->fy, o->fz, 0.0, 0.0, {0}};
        nonbonded_rows(o, c, 0, 1, &a);
        o->pot[7] += a.e_qq;
        o->pot[8] += a.e_vdw;
        for (int k = 0; k < 9; ++k) o->vir[k] += a.vir[k];
        return;
    }
    nb_job *job = (nb_job *)calloc((size_t)nt, sizeof(nb_job));
    double *buf = (double *)calloc((size_t)nt * 3 * N, sizeof(double));
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nt);
    for (int t = 0; t < nt; ++t) {
        job[t].o = o;
        job[t].c = c;
        job[t].first = t;
        job[t].stride = nt;
        job[t].acc.fx = buf + (size_t)t * 3 * N;
        job[t].acc.fy = job[t].acc.fx + N;
        job[t].acc.fz = job[t].acc.fy + N;
        pthread_create(&th[t], NULL, nb_thread, &job[t]);
    }
    for (int t = 0; t < nt; ++t) pthread_join(th[t], NULL);
    for (int t = 0; t < nt; ++t) { /* in thread order: a fixed summation order */
        const nb_acc *a = &job[t].acc;
        for (int i = 0; i < N; ++i) { o->fx[i] += a->fx[i]; o->fy[i] += a->fy[i]; o->fz[i] += a->fz[i]; }
        o->pot[7] += a->e_qq;
        o->pot[8] += a->e_vdw;
        for (int k = 0; k < 9; ++k) o->vir[k] += a->vir[k];
    }
    free(th);
    free(buf);
    free(job);
}

/* mpi_nonb_pair, force.c:1402-1540, one rank, all j < i.  Systems of 2,048
 * atoms or more in boxes of four or more cells per edge visit the same pairs
 * through cells; systems of 2,048 atoms or more split the rows over the
 * host threads, each with its own accumulators, added in thread order
 * afterwards.  Both change only the order of the sums (rounding); smaller
 * systems take the reference's loop literally. */
static void nonbonded(orc *o)
{
    const int N = o->N;
    cells c;
    const int use_cells = N >= 2048 && cells_build(o, &c);
    if (use_cells && (c.nc[0] < 4 || c.nc[1] < 4 || c.nc[2] < 4)) {
        cells_free(&c);
        return nonbonded_with(o, NULL);
    }
    nonbonded_with(o, use_cells ? &c : NULL);
    if (use_cells) cells_free(&c);
}
/* Nonbonded forces on the atoms of a sample only: every pair that involves a
 * sampled atom s, taken in the reference's orientation (the larger index is
 * the outer atom i, r = r_j - r_i; force.c:1419-1473), so the cut-off decision
 * is the reference's to the bit.  The pairs' energies and virial are not
 * formed.  O(N) per sampled atom, for systems whose all-pairs loop is too slow
 * for a test; force_terms() uses it while a sample is set. */
static void nonbonded_sample(orc *o)
{
    const capac_desc *d = o->d;
    const double rc = d->r_cut, rc2 = o->c.r_cut2;
    double e_qq = 0.0, e_vdw = 0.0;
    for (int k = 0; k < o->n_sample; ++k) {
        const int s = o->sample[k];
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (int j = 0; j < o->N; ++j) {
            if (j == s) continue;
            const int i = s > j ? s : j, jj = s > j ? j : s;
            if (excluded(d, i, jj)) continue;
            double x = o->rx[jj] - o->rx[i], y = o->ry[jj] - o->ry[i], z = o->rz[jj] - o->rz[i];
            image(&x, &y, &z, o->box);
            if (x >= rc && y >= rc && z >= rc) continue;
            const double r2 = norm2(x, y, z);
            if (r2 >= rc2) continue;
            const double f = pair_term(o, d->atom_type[i], d->atom_type[jj], d->charge[i], d->charge[jj], r2,
                                       &e_qq, &e_vdw);
            if (s == i) { fx -= f * x; fy -= f * y; fz -= f * z; }
            else { fx += f * x; fy += f * y; fz += f * z; }
        }
        o->fx[s] += fx; o->fy[s] += fy; o->fz[s] += fz;
    }
}

/* Pair-set fingerprint: same traversal as nonbonded(), counting (i,j). */
static uint64_t mix64(uint64_t x)
{
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

/* ------------------------------------------------------- Sutton-Chen */

/* mpi_qsc_dens force.c:385-461 and mpi_qsc_force force.c:468-542. */
static void sutton_chen(orc *o)
{
    const capac_desc *d = o->d;
    const int lo = d->metal_min, hi = d->metal_max;
    const double rc2 = o->c.r_cut2;
    for (int i = lo; i <= hi; ++i) {
        double rho = 0.0;
        for (int j = lo; j <= hi; ++j) {
            if (j == i) continue;
            double x = o->rx[j] - o->rx[i], y = o->ry[j] - o->ry[i], z = o->rz[j] - o->rz[i];
            image(&x, &y, &z, o->box);
            const double r2 = norm2(x, y, z);
            if (r2 < rc2) rho += pow(d->qsc_a / sqrt(r2), d->qsc_m);
        }
        o->inv_sqrt_dens[i - lo] = 1.0 / sqrt(rho);
    }
    const double cm2 = d->qsc_c * d->qsc_m / 2.0;
    for (int i = lo; i <= hi; ++i) {
        for (int j = lo; j <= hi; ++j) {
            if (j == i) continue;
            double x = o->rx[j] - o->rx[i], y = o->ry[j] - o->ry[i], z = o->rz[j] - o->rz[i];
            image(&x, &y, &z, o->box);
            const double r2 = norm2(x, y, z);
            if (r2 >= rc2) continue;
            const double r = sqrt(r2), ar = d->qsc_a / r;
            const double an = pow(ar, d->qsc_n), am = pow(ar, d->qsc_m);
            const double s = o->inv_sqrt_dens[i - lo] + o->inv_sqrt_dens[j - lo];
            const double f = d->qsc_eps * (d->qsc_n * an - cm2 * s * am) / r2;
            o->fx[i] -= f * x; o->fy[i] -= f * y; o->fz[i] -= f * z;
            acc_vir(o->vir, x, y, z, f * x, f * y, f * z, 0.5);
            o->pot[1] += d->qsc_eps * an * 0.5;
        }
        o->pot[1] -= d->qsc_eps * d->qsc_c / o->inv_sqrt_dens[i - lo];
    }
}

/* ------------------------------------------------------------- CPIM */

/* mpi_cpff_vec_ext, cpff.c:43-198. */
static void cpim_rhs(orc *o)
{
    const capac_desc *d = o->d;
    const int M = o->M;
    const double rc = d->r_cut, rc2 = o->c.r_cut2, a = d->w_alpha;
    for (int im = d->metal_min; im <= d->metal_max; ++im) {
        double ex = 0.0, ey = 0.0, ez = 0.0, v = 0.0;
        for (int j = 0; j < o->N; ++j) {
            if (d->is_metal[j]) continue;
            const double qj = d->charge[j];
            if (qj == 0.0) continue;
            double x = o->rx[im] - o->rx[j], y = o->ry[im] - o->ry[j], z = o->rz[im] - o->rz[j];
            image(&x, &y, &z, o->box);
            const double r2 = norm2(x, y, z);
            double ef = 0.0, vf = 0.0;
            if (r2 < rc2) {
                const double r = sqrt(r2);
                if (d->use_coulomb == 1) {
                    const double ec = erfc(a * r), eg = exp(-a * a * r2);
                    ef = FQQ * qj * (ec / r2 + o->c.w_a2_sqrtpi * eg / r - o->c.w_const) / r;
                    vf = FQQ * qj * (ec / r - o->c.w_erfc_arcut + o->c.w_const * (r - rc));
                } else {
                    ef = FQQ * qj / (r2 * r);
                    vf = FQQ * qj / r;
                }
            }
            ex += ef * CONV_E * x; ey += ef * CONV_E * y; ez += ef * CONV_E * z;
            v += vf * CONV_V;
        }
        const int i = im - d->metal_min;
        o->vec_ext[3 * i + 0] = ex + d->efield[0] * CONV_E;
        o->vec_ext[3 * i + 1] = ey + d->efield[1] * CONV_E;
        o->vec_ext[3 * i + 2] = ez + d->efield[2] * CONV_E;
        const double vext = d->efield[0] * o->rx[im] + d->efield[1] * o->ry[im] + d->efield[2] * o->rz[im];
        o->vec_ext[3 * M + i] = v - vext * CONV_V;
    }
    for (int k = 0; k < d->n_nps; ++k) o->vec_ext[4 * M + k] = d->np_charge[k];
}

static double keep(double e) { return fabs(e) > THRSHD ? e : 0.0; }

/* mpi_cpff_mat_relay_COO, cpff.c:205-519, stored dense. */
static void cpim_matrix(orc *o)
{
    const capac_desc *d = o->d;
    const int M = o->M, n = o->n_mat;
    const double ipp = o->c.inv_r_pp, ipq = o->c.inv_r_pq, iqq = o->c.inv_r_qq;
    double *A = o->A;
    memset(A, 0, sizeof(double) * (size_t)n * n);
    for (int i = 0; i < M; ++i) {
        const int ia = d->metal_min + i;
        for (int j = 0; j < M; ++j) {
            const int ja = d->metal_min + j;
            if (j == i) {
                for (int a = 0; a < 3; ++a) {
                    A[(size_t)(3 * i + a) * n + 3 * i + a] = keep(o->c.inv_polar);
                    o->diag[3 * i + a] = o->c.inv_polar;
                }
                A[(size_t)(3 * M + i) * n + 3 * M + i] = keep(-o->c.inv_capac);
                o->diag[3 * M + i] = -o->c.inv_capac;
                continue;
            }
            double r[3] = {o->rx[ja] - o->rx[ia], o->ry[ja] - o->ry[ia], o->rz[ja] - o->rz[ia]};
            image(&r[0], &r[1], &r[2], o->box);
            r[0] *= NM2BOHR; r[1] *= NM2BOHR; r[2] *= NM2BOHR;
            const double r2 = norm2(r[0], r[1], r[2]), rr = sqrt(r2);
            const double gpp = exp(-(r2 * ipp * ipp));
            const double c1 = 1.0 / pow(rr, 5.0) * (erf(rr * ipp) - 2.0 * INV_SQRT_PI * ipp * rr * gpp);
            const double c2 = 4.0 * INV_SQRT_PI * pow(ipp, 3.0) / r2 * gpp;
            const double gpq = exp(-(r2 * ipq * ipq));
            const double c3 = 1.0 / pow(rr, 3.0) * (erf(rr * ipq) - 2.0 * INV_SQRT_PI * ipq * rr * gpq);
            for (int a = 0; a < 3; ++a) {
                for (int b = 0; b < 3; ++b) {
                    const double dab = a == b ? 1.0 : 0.0;
                    A[(size_t)(3 * i + a) * n + 3 * j + b] =
                        keep(-(c1 * (3.0 * r[a] * r[b] - dab * r2) - c2 * r[a] * r[b]));
                }
                A[(size_t)(3 * i + a) * n + 3 * M + j] = keep(c3 * r[a]);
                A[(size_t)(3 * M + i) * n + 3 * j + a] = keep(-c3 * r[a]);
            }
            A[(size_t)(3 * M + i) * n + 3 * M + j] = keep(-erf(rr * iqq) / rr);
        }
        for (int k = 0; k < d->n_nps; ++k) {
            if (d->metal_min + i >= d->np_start[k] && d->metal_min + i <= d->np_end[k]) {
                A[(size_t)(3 * M + i) * n + 4 * M + k] = 1.0;
                A[(size_t)(4 * M + k) * n + 3 * M + i] = 1.0;
            }
        }
    }
    for (int k = 0; k < d->n_nps; ++k) o->diag[4 * M + k] = 1.0;
}

/* Rows r0 .. r1 - 1 of y = A x (one row's sum in column order). */
static void matvec_rows(const orc *o, const double *x, double *y, int r0, int r1)
{
    const int n = o->n_mat;
    for (int r = r0; r < r1; ++r) {
        double s = 0.0;
        const double *row = o->A + (size_t)r * n;
        for (int c = 0; c < n; ++c) s += row[c] * x[c];
        y[r] = s;
    }
}

typedef struct mv_job {
    const orc *o;
    const double *x;
    double *y;
    int r0, r1;
} mv_job;

static void *mv_thread(void *arg)
{
    mv_job *j = (mv_job *)arg;
    matvec_rows(j->o, j->x, j->y, j->r0, j->r1);
    return NULL;
}

static void matvec(const orc *o, const double *x, double *y)
{
    const int n = o->n_mat;
    if (!o->A) { /* use_cpff 0: the reference's COO matrix stays empty */
        memset(y, 0, (size_t)n * sizeof(double));
        return;
    }
    if (n >= 1024) {
        const int nt = host_threads();
        mv_job *job = (mv_job *)malloc(sizeof(mv_job) * (size_t)nt);
        pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nt);
        for (int t = 0; t < nt; ++t) {
            job[t] = (mv_job){o, x, y, (int)((long)n * t / nt), (int)((long)n * (t + 1) / nt)};
            pthread_create(&th[t], NULL, mv_thread, &job[t]);
        }
        for (int t = 0; t < nt; ++t) pthread_join(th[t], NULL);
        free(th);
        free(job);
        return;
    }
    matvec_rows(o, x, y, 0, n);
}

static double dot(int n, const double *a, const double *b)
{
    double s = 0.0;
    for (int k = 0; k < n; ++k) s += a[k] * b[k];
    return s;
}

/* mpi_precon_bicg_stab_COO, bicg_stab.c:253-573 (Jacobi-preconditioned
 * BiCGSTAB, warm start from vec_pq).  Returns 0, or -1 when not converged. */
static int cpim_solve(orc *o)
{
    const int n = o->n_mat, M = o->M;
    double *Ax = o->w, *r0 = Ax + n, *r = r0 + n, *p = r + n, *v = p + n, *s = v + n, *t = s + n,
           *y = t + n, *z = y + n, *Kt = z + n, *K = Kt + n;
    double *x = o->vec_pq, *b = o->vec_ext;
    o->iterations = 0;
    const double bTb = dot(n, b, b);
    if (bTb < 1.0e-10) return 0;
    const double crit = bTb * o->solver_tol;
    /* A breakdown (alpha or omega zero or non-finite) restarts from the last
     * finite x; the reference has no such guard and would carry the NaN to
     * MAX_ITER.  It does not occur at the reference's own tolerance on the
     * golden inputs; tight-tolerance runs can reach it near the FP64 floor. */
    for (int start = 0; start < 8; ++start) {
        matvec(o, x, Ax);
        for (int k = 0; k < n; ++k) {
            r0[k] = b[k] - Ax[k];
            r[k] = r0[k];
            v[k] = p[k] = 0.0;
            K[k] = k < 4 * M ? 1.0 / o->diag[k] : 1.0;
        }
        double rho_old = 1.0, omega = 1.0, alpha = 1.0, rTr = dot(n, r, r);
        int iter = 0, broke = 0;
        for (;;) {
            const double rho = dot(n, r0, r);
            if (rho < 1.0e-10 && iter == 0 && start == 0) return 0;
            const double beta = (rho / rho_old) * (alpha / omega);
            for (int k = 0; k < n; ++k) {
                p[k] = r[k] + beta * (p[k] - omega * v[k]);
                y[k] = p[k] * K[k];
            }
            matvec(o, y, v);
            alpha = rho / dot(n, r0, v);
            if (!isfinite(alpha)) { broke = 1; break; }
            for (int k = 0; k < n; ++k) {
                s[k] = r[k] - alpha * v[k];
                z[k] = s[k] * K[k];
            }
            matvec(o, z, t);
            for (int k = 0; k < n; ++k) Kt[k] = t[k] * K[k];
            omega = dot(n, Kt, z) / dot(n, Kt, Kt);
            if (!isfinite(omega) || omega == 0.0) { broke = 1; break; }
            for (int k = 0; k < n; ++k) {
                x[k] += alpha * y[k] + omega * z[k];
                r[k] = s[k] - omega * t[k];
            }
            rho_old = rho;
            ++iter;
            ++o->iterations;
            rTr = dot(n, r, r);
            if (rTr < crit) return 0;
            if (iter > MAX_ITER) return rTr < crit * 100.0 ? 0 : -1;
        }
        if (broke && rTr < crit * 100.0) return 0;
    }
    return -1;
}

/* mpi_cpff_force, cpff.c:526-950 (metal atoms assumed first, as in every
 * reference input: the metal-metal loop there runs j_metal from 0). */
static void cpim_force(orc *o)
{
    const capac_desc *d = o->d;
    const int M = o->M;
    const double *pq = o->vec_pq;
    const double rc = d->r_cut, rc2 = o->c.r_cut2, al = d->w_alpha, al3 = pow(al, 3.0);
    const double ipp = o->c.inv_r_pp, ipq = o->c.inv_r_pq, iqq = o->c.inv_r_qq;
    const double ipp3 = pow(ipp, 3.0), ipq3 = pow(ipq, 3.0), ipp5 = pow(ipp, 5.0);
    for (int i = 0; i < M; ++i) {
        const int im = d->metal_min + i;
        /* metal - permanent charge, MD units */
        for (int j = 0; j < o->N; ++j) {
            if (d->is_metal[j] || d->charge[j] == 0.0) continue;
            double r[3] = {o->rx[im] - o->rx[j], o->ry[im] - o->ry[j], o->rz[im] - o->rz[j]};
            image(&r[0], &r[1], &r[2], o->box);
            const double r2 = norm2(r[0], r[1], r[2]);
            if (r2 >= rc2) continue;
            const double rr = sqrt(r2), qj = d->charge[j], qi = pq[3 * M + i];
            double f[3] = {0.0, 0.0, 0.0}, a0;
            double ec = 0.0, eg = 0.0;
            if (d->use_coulomb == 1) {
                ec = erfc(al * rr);
                eg = exp(-al * al * r2);
                a0 = (ec / r2 + o->c.w_a2_sqrtpi * eg / rr - o->c.w_const) / rr;
                o->pot[10] += FQQ * qj * qi * (ec / rr - o->c.w_erfc_arcut + o->c.w_const * (rr - rc));
            } else {
                a0 = 1.0 / (r2 * rr);
                o->pot[10] += FQQ * qj * qi / rr;
            }
            for (int a = 0; a < 3; ++a) f[a] += a0 * r[a] * FQQ * qj * qi;
            if (d->use_coulomb == 1) {
                const double a1 = 1.0 / pow(rr, 5.0) * (ec + o->c.w_a2_sqrtpi * rr * eg);
                const double b1 = 4.0 * INV_SQRT_PI * al3 / r2 * eg;
                const double c1 = o->c.w_const / pow(rr, 3.0);
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) {
                        const double dab = a == b ? 1.0 : 0.0;
                        f[b] += -(a1 * (3.0 * r[a] * r[b] - dab * r2) + b1 * r[a] * r[b] -
                                  c1 * (r[a] * r[b] - dab * r2)) * FQQ * qj * pq[3 * i + a] / NM2BOHR;
                    }
            } else {
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) {
                        const double dab = a == b ? 1.0 : 0.0;
                        f[b] += -((3.0 * r[a] * r[b] - dab * r2) / pow(rr, 5.0)) * FQQ * qj *
                                pq[3 * i + a] / NM2BOHR;
                    }
            }
            for (int a = 0; a < 3; ++a) o->pot[11] += -FQQ * qj * pq[3 * i + a] / NM2BOHR * a0 * r[a];
            o->fx[im] += f[0]; o->fy[im] += f[1]; o->fz[im] += f[2];
            o->fx[j] -= f[0]; o->fy[j] -= f[1]; o->fz[j] -= f[2];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) o->vir[3 * a + b] += -r[a] * f[b];
        }
        /* self terms */
        const double qi = pq[3 * M + i];
        o->pot[12] += 0.5 * FQQ * qi * qi * (o->c.inv_capac * NM2BOHR);
        for (int a = 0; a < 3; ++a)
            o->pot[14] += 0.5 * FQQ * pq[3 * i + a] * pq[3 * i + a] * (o->c.inv_polar * NM2BOHR);
        /* metal - metal, atomic units */
        for (int j = 0; j < M; ++j) {
            if (j == i) continue;
            const int jm = d->metal_min + j;
            double r[3] = {o->rx[jm] - o->rx[im], o->ry[jm] - o->ry[im], o->rz[jm] - o->rz[im]};
            image(&r[0], &r[1], &r[2], o->box);
            r[0] *= NM2BOHR; r[1] *= NM2BOHR; r[2] *= NM2BOHR;
            const double r2 = norm2(r[0], r[1], r[2]), rr = sqrt(r2);
            const double qj = pq[3 * M + j];
            const double *pi = pq + 3 * i, *pj = pq + 3 * j;
            double f[3] = {0.0, 0.0, 0.0};
            const double gqq = exp(-(r2 * iqq * iqq));
            const double A0 = 1.0 / pow(rr, 3.0) * (erf(rr * iqq) - 2.0 * INV_SQRT_PI * iqq * rr * gqq);
            for (int a = 0; a < 3; ++a) f[a] += A0 * r[a] * FQQ_AU2 * qi * qj;
            o->pot[12] += FQQ_AU1 * qi * qj * erf(rr * iqq) / rr * 0.5;
            const double gpq = exp(-(r2 * ipq * ipq));
            const double Apq0 = 1.0 / pow(rr, 3.0) * (erf(rr * ipq) - 2.0 * INV_SQRT_PI * ipq * rr * gpq);
            const double A1 = 1.0 / pow(rr, 5.0) * (erf(rr * ipq) - 2.0 * INV_SQRT_PI * ipq * rr * gpq);
            const double B1 = 4.0 * INV_SQRT_PI * ipq3 / r2 * gpq;
            for (int a = 0; a < 3; ++a) {
                for (int b = 0; b < 3; ++b) {
                    const double dab = a == b ? 1.0 : 0.0;
                    const double T = A1 * (3.0 * r[a] * r[b] - dab * r2) - B1 * r[a] * r[b];
                    f[b] += -T * FQQ_AU2 * qi * pj[a];
                    f[b] += T * FQQ_AU2 * qj * pi[a];
                }
                o->pot[13] += -FQQ_AU1 * qi * pj[a] * r[a] * Apq0 * 0.5;
                o->pot[13] += FQQ_AU1 * qj * pi[a] * r[a] * Apq0 * 0.5;
            }
            const double gpp = exp(-(r2 * ipp * ipp));
            const double App1 = 1.0 / pow(rr, 5.0) * (erf(rr * ipp) - 2.0 * INV_SQRT_PI * ipp * rr * gpp);
            const double Bpp1 = 4.0 * INV_SQRT_PI * ipp3 / r2 * gpp;
            const double A2 = 1.0 / pow(rr, 7.0) *
                              (3.0 * erf(rr * ipp) - 6.0 * INV_SQRT_PI * ipp * rr * gpp -
                               4.0 * pow(rr, 3.0) * INV_SQRT_PI * ipp3 * gpp);
            const double B2 = 8.0 * INV_SQRT_PI * ipp5 / r2 * gpp;
            for (int a = 0; a < 3; ++a) {
                for (int b = 0; b < 3; ++b) {
                    const double dab = a == b ? 1.0 : 0.0;
                    for (int c = 0; c < 3; ++c) {
                        const double dbc = b == c ? 1.0 : 0.0, dca = c == a ? 1.0 : 0.0;
                        f[c] += -(A2 * (5.0 * r[a] * r[b] * r[c] - r2 * (r[a] * dbc + r[b] * dca + r[c] * dab)) -
                                  B2 * r[a] * r[b] * r[c]) * FQQ_AU2 * pi[a] * pj[b];
                    }
                    o->pot[14] += -FQQ_AU1 * pi[a] * pj[b] *
                                  ((3.0 * r[a] * r[b] - dab * r2) * App1 - r[a] * r[b] * Bpp1) * 0.5;
                }
            }
            o->fx[im] -= f[0]; o->fy[im] -= f[1]; o->fz[im] -= f[2];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) o->vir[3 * a + b] += -r[a] * f[b] * 0.5;
        }
        /* external field on the induced charge and dipole */
        o->fx[im] += d->efield[0] * qi;
        o->fy[im] += d->efield[1] * qi;
        o->fz[im] += d->efield[2] * qi;
        o->pot[9] -= d->efield[0] * qi * o->rx[im] + d->efield[1] * qi * o->ry[im] +
                     d->efield[2] * qi * o->rz[im];
        o->pot[9] -= d->efield[0] * pq[3 * i] + d->efield[1] * pq[3 * i + 1] + d->efield[2] * pq[3 * i + 2];
    }
}

/* ------------------------------------------------------ mpi_force */

static void force_terms(orc *o, int solve)
{
    const capac_desc *d = o->d;
    memset(o->fx, 0, sizeof(double) * o->N);
    memset(o->fy, 0, sizeof(double) * o->N);
    memset(o->fz, 0, sizeof(double) * o->N);
    memset(o->pot, 0, sizeof o->pot);
    memset(o->vir, 0, sizeof o->vir);
    if (o->n_sample > 0) nonbonded_sample(o);
    else nonbonded(o);
    if (o->M > 0) {
        sutton_chen(o);
        if (d->use_cpff) {
            cpim_rhs(o);
            cpim_matrix(o);
            if (solve && cpim_solve(o) != 0) o->error = CAPAC_ERR_NOT_CONVERGED;
            cpim_force(o);
        }
    }
    for (int i = 0; i < o->N; ++i) { /* force.c:2251-2260 */
        const double q = d->charge[i];
        o->fx[i] += d->efield[0] * q;
        o->fy[i] += d->efield[1] * q;
        o->fz[i] += d->efield[2] * q;
        o->pot[9] -= d->efield[0] * q * o->rx[i] + d->efield[1] * q * o->ry[i] + d->efield[2] * q * o->rz[i];
    }
}

static void force(orc *o) { force_terms(o, 1); }

static void sum_potential(orc *o) /* force.c:322-331 */
{
    o->pot[0] = 0.0;
    for (int k = 1; k < 15; ++k) o->pot[0] += o->pot[k];
}

/* ------------------------------------------------------- integrator */

/* kinetic_energy, thermostat.c:34-63 */
static void kinetic(orc *o)
{
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int i = 0; i < o->N; ++i) {
        const double m = o->d->mass[i];
        if (m > 0.0) {
            sx += m * o->vx[i] * o->vx[i];
            sy += m * o->vy[i] * o->vy[i];
            sz += m * o->vz[i] * o->vz[i];
        }
    }
    o->eksum = sx + sy + sz;
    o->inst_temp = o->eksum / (K_BOLTZ * o->c.ndf);
}

/* remove_comm, thermostat.c:69-108 */
static void remove_com(orc *o)
{
    double px = 0.0, py = 0.0, pz = 0.0, ms = 0.0;
    for (int i = 0; i < o->N; ++i) {
        const double m = o->d->mass[i];
        if (m > 0.0) {
            px += o->vx[i] * m; py += o->vy[i] * m; pz += o->vz[i] * m;
            ms += m;
        }
    }
    px /= ms; py /= ms; pz /= ms;
    for (int i = 0; i < o->N; ++i)
        if (o->d->mass[i] > 0.0) { o->vx[i] -= px; o->vy[i] -= py; o->vz[i] -= pz; }
}

/* nose_hoover_chain, thermostat.c:117-191 (Nc = 5, 5th-order Suzuki-Yoshida) */
static void nhc(orc *o)
{
    const int Nc = 5, L = NHC_LEN;
    const double w1 = 0.41449077179437571194, w3 = -0.65796308717750284778;
    const double w[5] = {w1, w1, w3, w1, w1};
    const double Q = o->c.q_mass, kT = K_BOLTZ * o->ref_temp, NkT = kT * o->c.ndf, dt = o->d->dt;
    double *vQ = o->vQ, *aQ = o->aQ, scale = 1.0;
    aQ[0] = (o->eksum - NkT) / Q;
    for (int m = 0; m < L - 1; ++m) aQ[m + 1] = (Q * vQ[m] * vQ[m] - kT) / Q;
    for (int c = 0; c < Nc; ++c) {
        for (int y = 0; y < 5; ++y) {
            const double h4 = w[y] * dt / (4 * Nc), h8 = w[y] * dt / (8 * Nc), h2 = w[y] * dt / (2 * Nc);
            vQ[L - 1] += aQ[L - 1] * h4;
            for (int m = 0; m < L - 1; ++m) {
                const double e = exp(-h8 * vQ[L - (m + 1)]);
                vQ[L - 1 - (m + 1)] = vQ[L - 1 - (m + 1)] * e * e + h4 * aQ[L - 1 - (m + 1)] * e;
            }
            scale *= exp(-h2 * vQ[0]);
            aQ[0] = (o->eksum * scale * scale - NkT) / Q;
            for (int m = 0; m < L - 1; ++m) {
                const double e = exp(-h8 * vQ[m + 1]);
                vQ[m] = vQ[m] * e * e + h4 * aQ[m] * e;
                aQ[m + 1] = (Q * vQ[m] * vQ[m] - kT) / Q;
            }
            vQ[L - 1] += aQ[L - 1] * h4;
        }
    }
    for (int i = 0; i < o->N; ++i) { o->vx[i] *= scale; o->vy[i] *= scale; o->vz[i] *= scale; }
    o->eksum *= scale * scale;
    o->inst_temp *= scale * scale;
}

/* Berendsen weak coupling (Berendsen et al., J. Chem. Phys. 81, 3684 (1984));
 * no counterpart in the reference, which thermostats only with the chain
 * above: lambda = sqrt(1 + dt/tau (T0/T - 1)), lambda^2 held to
 * [0.64, 1.5625], lambda = 1 at T = 0, applied to every velocity. */
static void berendsen(orc *o)
{
    double s2 = 1.0;
    if (o->inst_temp > 0.0) {
        s2 = 1.0 + o->d->dt / o->d->tau_temp * (o->ref_temp / o->inst_temp - 1.0);
        s2 = s2 < 0.64 ? 0.64 : (s2 > 1.5625 ? 1.5625 : s2);
    }
    const double s = sqrt(s2);
    for (int i = 0; i < o->N; ++i) { o->vx[i] *= s; o->vy[i] *= s; o->vz[i] *= s; }
    o->eksum *= s * s;
    o->inst_temp *= s * s;
}

/* rattle_1st force.c:1907-1997 and rattle_2nd force.c:2004-2090. */
static int rattle(orc *o, int second)
{
    const capac_desc *d = o->d;
    const double dt = d->dt, hdt = 0.5 * dt, tol2 = 2.0e-05, tol = 1.0e-05;
    for (int im = 0; im < d->n_mols; ++im) {
        const int first = d->mol_first[im], mt = d->mol_type[first];
        const int nc = d->cstr_count[mt], c0 = d->cstr_offset[mt];
        if (nc == 0) continue;
        int iter = 0, done = 0;
        while (!done) {
            done = 1;
            for (int k = 0; k < nc; ++k) {
                const int a = first + d->cstr_i[c0 + k], b = first + d->cstr_j[c0 + k];
                const double len = d->cstr_r[c0 + k], len2 = len * len;
                const double ma = d->inv_mass[a], mb = d->inv_mass[b];
                if (!second) {
                    const double px = wrap1(o->rx[a] - o->rx[b], o->box[0]);
                    const double py = wrap1(o->ry[a] - o->ry[b], o->box[1]);
                    const double pz = wrap1(o->rz[a] - o->rz[b], o->box[2]);
                    const double diff = len2 - (px * px + py * py + pz * pz);
                    if (fabs(diff) > len2 * tol2) {
                        const double qx = wrap1(o->ox[a] - o->ox[b], o->box[0]);
                        const double qy = wrap1(o->oy[a] - o->oy[b], o->box[1]);
                        const double qz = wrap1(o->oz[a] - o->oz[b], o->box[2]);
                        const double g = diff / (2.0 * (ma + mb) * (qx * px + qy * py + qz * pz));
                        double dx = qx * g, dy = qy * g, dz = qz * g;
                        o->rx[a] += ma * dx; o->ry[a] += ma * dy; o->rz[a] += ma * dz;
                        o->rx[b] -= mb * dx; o->ry[b] -= mb * dy; o->rz[b] -= mb * dz;
                        dx /= dt; dy /= dt; dz /= dt;
                        o->vx[a] += ma * dx; o->vy[a] += ma * dy; o->vz[a] += ma * dz;
                        o->vx[b] -= mb * dx; o->vy[b] -= mb * dy; o->vz[b] -= mb * dz;
                        done = 0;
                    }
                } else {
                    const double vx = o->vx[a] - o->vx[b], vy = o->vy[a] - o->vy[b], vz = o->vz[a] - o->vz[b];
                    const double px = wrap1(o->rx[a] - o->rx[b], o->box[0]);
                    const double py = wrap1(o->ry[a] - o->ry[b], o->box[1]);
                    const double pz = wrap1(o->rz[a] - o->rz[b], o->box[2]);
                    const double g = -(px * vx + py * vy + pz * vz) / ((ma + mb) * len2);
                    if (fabs(g) > tol) {
                        double dx = px * g, dy = py * g, dz = pz * g;
                        o->vx[a] += ma * dx; o->vy[a] += ma * dy; o->vz[a] += ma * dz;
                        o->vx[b] -= mb * dx; o->vy[b] -= mb * dy; o->vz[b] -= mb * dz;
                        dx /= hdt; dy /= hdt; dz /= hdt;
                        o->vir[0] -= px * dx; o->vir[1] -= px * dy; o->vir[2] -= px * dz;
                        o->vir[3] -= py * dx; o->vir[4] -= py * dy; o->vir[5] -= py * dz;
                        o->vir[6] -= pz * dx; o->vir[7] -= pz * dy; o->vir[8] -= pz * dz;
                        done = 0;
                    }
                }
            }
            if (++iter > MAX_ITER) break;
        }
        if (!done) return CAPAC_ERR_RATTLE;
    }
    return 0;
}

/* apply_pbc, force.c:127-165 */
static void wrap_molecules(orc *o)
{
    const double *L = o->box;
    const double h[3] = {0.5 * L[0], 0.5 * L[1], 0.5 * L[2]};
    double *r[3] = {o->rx, o->ry, o->rz};
    for (int im = 0; im < o->d->n_mols; ++im) {
        const int lo = o->d->mol_first[im], hi = o->d->mol_last[im], mid = (lo + hi) / 2;
        for (int a = 0; a < 3; ++a) {
            if (r[a][mid] > L[a]) r[a][mid] -= L[a]; else if (r[a][mid] < 0.0) r[a][mid] += L[a];
        }
        for (int i = lo; i <= hi; ++i) {
            if (i == mid) continue;
            for (int a = 0; a < 3; ++a) {
                if (r[a][i] - r[a][mid] > h[a]) r[a][i] -= L[a];
                else if (r[a][i] - r[a][mid] < -h[a]) r[a][i] += L[a];
            }
        }
    }
}

/* get_fmax_rms, force.c:361-378 */
static void fmax_rms(orc *o)
{
    double m2 = 0.0, s = 0.0;
    for (int i = 0; i < o->N; ++i) {
        const double f2 = o->fx[i] * o->fx[i] + o->fy[i] * o->fy[i] + o->fz[i] * o->fz[i];
        s += f2;
        if (f2 > m2) m2 = f2;
    }
    o->f_max = sqrt(m2);
    o->f_rms = sqrt(s / o->N);
}

/* ------------------------------------------------------------- API */

/* Start-up constants, mpi-main.c:170-203 (DSF, LJ shifted force),
 * :315-323 (CPIM Gaussian widths), :548-562 (ndf, thermostat mass). */
static void derive_consts(const capac_desc *d, capac_consts *c)
{
    memset(c, 0, sizeof *c);
    const double rc = d->r_cut, a = d->w_alpha;
    c->r_cut2 = rc * rc;
    c->w_a2_sqrtpi = a * 2.0 * INV_SQRT_PI;
    c->w_const = erfc(a * rc) / c->r_cut2 + c->w_a2_sqrtpi * exp(-a * a * c->r_cut2) / rc;
    c->w_erfc_arcut = erfc(a * rc) / rc;
    c->inv_rc12 = 1.0 / pow(rc, 12.0);
    c->inv_rc6 = 1.0 / pow(rc, 6.0);
    if (d->n_metal > 0) {
        const double pi = 3.14159265358979323846;
        c->inv_polar = 1.0 / d->cpff_polar;
        c->inv_capac = 1.0 / d->cpff_capac;
        const double rq = sqrt(2.0 / pi) * d->cpff_capac;
        const double rp = pow(sqrt(2.0 / pi) * d->cpff_polar / 3.0, 1.0 / 3.0);
        c->inv_r_qq = 1.0 / sqrt(rq * rq + rq * rq);
        c->inv_r_pq = 1.0 / sqrt(rp * rp + rq * rq);
        c->inv_r_pp = 1.0 / sqrt(rp * rp + rp * rp);
    }
    c->ndf = 3 * (d->n_atoms - d->n_vsites_total) - 3 - d->n_cstr_total;
    c->kT = K_BOLTZ * d->ref_temp;
    c->q_mass = (double)c->ndf * c->kT * d->tau_temp * d->tau_temp;
    c->dt_2 = 0.5 * d->dt;
    c->n_mat = d->n_metal * 4 + d->n_nps;
}

orc *orc_create(const capac_desc *d, double solver_tol)
{
    orc *o = (orc *)calloc(1, sizeof(orc));
    if (!o) return NULL;
    o->d = d;
    derive_consts(d, &o->c);
    o->N = d->n_atoms;
    o->M = d->n_metal;
    o->n_mat = o->c.n_mat;
    o->solver_tol = solver_tol > 0.0 ? solver_tol : 1.0e-8;
    for (int a = 0; a < 3; ++a) { o->box[a] = d->box[a]; o->box[3 + a] = 0.5 * d->box[a]; }
    const size_t N = (size_t)o->N;
    double *block = (double *)calloc(N * 12, sizeof(double));
    double **slots[] = {&o->rx, &o->ry, &o->rz, &o->vx, &o->vy, &o->vz, &o->fx, &o->fy, &o->fz,
                        &o->ox, &o->oy, &o->oz};
    for (int k = 0; k < 12; ++k) *slots[k] = block + N * k;
    memcpy(o->rx, d->rx, N * sizeof(double)); memcpy(o->ry, d->ry, N * sizeof(double));
    memcpy(o->rz, d->rz, N * sizeof(double)); memcpy(o->vx, d->vx, N * sizeof(double));
    memcpy(o->vy, d->vy, N * sizeof(double)); memcpy(o->vz, d->vz, N * sizeof(double));
    const size_t n = (size_t)(o->n_mat > 0 ? o->n_mat : 1);
    o->inv_sqrt_dens = (double *)calloc(o->M > 0 ? o->M : 1, sizeof(double));
    o->vec_ext = (double *)calloc(n, sizeof(double));
    o->vec_pq = (double *)calloc(n, sizeof(double));
    o->diag = (double *)calloc(n, sizeof(double));
    for (size_t k = 0; k < n; ++k) o->diag[k] = 1.0;
    o->w = (double *)calloc(n * 11, sizeof(double));
    o->A = (o->M > 0 && d->use_cpff) ? (double *)calloc(n * n, sizeof(double)) : NULL;
    o->ref_temp = d->ref_temp;
    o->vQ[0] = d->vq0;
    return o;
}

void orc_destroy(orc *o)
{
    if (!o) return;
    free(o->rx); free(o->inv_sqrt_dens); free(o->vec_ext); free(o->vec_pq); free(o->diag);
    free(o->w); free(o->A); free(o->sample); free(o);
}

int orc_force(orc *o)
{
    o->error = 0;
    force(o);
    sum_potential(o);
    return o->error;
}

/* Every force term with the induced vector as currently held (no solve). */
int orc_force_given_pq(orc *o)
{
    o->error = 0;
    force_terms(o, 0);
    sum_potential(o);
    return o->error;
}

/* start-up after the first force call, mpi-main.c:627-655 */
void orc_md_init(orc *o)
{
    remove_com(o);
    kinetic(o);
    o->first_temp = o->inst_temp;
    o->ext_temp = o->d->ref_temp;
    fmax_rms(o);
}

/* MD loop, mpi-main.c:874-1013 */
int orc_md_steps(orc *o, int n)
{
    const capac_desc *d = o->d;
    const double dt = d->dt, h = o->c.dt_2;
    for (int k = 0; k < n; ++k) {
        const int step = ++o->step;
        if (step < d->n_heating)
            o->ref_temp = o->first_temp + (o->ext_temp - o->first_temp) * step / d->n_heating;
        else
            o->ref_temp = o->ext_temp;
        if (d->ensemble == CAPAC_NVT) nhc(o);
        for (int i = 0; i < o->N; ++i) {
            if (d->fix_metal == 1 && d->is_metal[i]) continue;
            const double im = d->inv_mass[i];
            o->vx[i] += h * o->fx[i] * im; o->vy[i] += h * o->fy[i] * im; o->vz[i] += h * o->fz[i] * im;
        }
        for (int i = 0; i < o->N; ++i) {
            if (d->fix_metal == 1 && d->is_metal[i]) continue;
            o->ox[i] = o->rx[i]; o->oy[i] = o->ry[i]; o->oz[i] = o->rz[i];
            o->rx[i] += dt * o->vx[i]; o->ry[i] += dt * o->vy[i]; o->rz[i] += dt * o->vz[i];
        }
        int rc = rattle(o, 0);
        if (rc) return rc;
        force(o);
        if (o->error) return o->error;
        sum_potential(o);
        for (int i = 0; i < o->N; ++i) {
            if (d->fix_metal == 1 && d->is_metal[i]) continue;
            const double im = d->inv_mass[i];
            o->vx[i] += h * o->fx[i] * im; o->vy[i] += h * o->fy[i] * im; o->vz[i] += h * o->fz[i] * im;
        }
        rc = rattle(o, 1);
        if (rc) return rc;
        kinetic(o);
        if (d->ensemble == CAPAC_NVT) nhc(o);
        else if (d->ensemble == CAPAC_BERENDSEN) berendsen(o);
        remove_com(o);
        kinetic(o);
        if (step % d->n_save == 0) {
            wrap_molecules(o);
            fmax_rms(o);
        }
    }
    return 0;
}

/* Stage entry points for stage-by-stage checks. */
void orc_zero(orc *o)
{
    memset(o->fx, 0, sizeof(double) * o->N);
    memset(o->fy, 0, sizeof(double) * o->N);
    memset(o->fz, 0, sizeof(double) * o->N);
    memset(o->pot, 0, sizeof o->pot);
    memset(o->vir, 0, sizeof o->vir);
}
void orc_nonbonded(orc *o) { nonbonded(o); }
void orc_qsc(orc *o) { if (o->M > 0) sutton_chen(o); }
void orc_cpff_vec_ext(orc *o) { if (o->M > 0) cpim_rhs(o); }
void orc_cpff_mat_relay(orc *o) { if (o->M > 0 && o->A) cpim_matrix(o); }
int orc_bicgstab(orc *o) { return (o->M > 0 && o->A) ? cpim_solve(o) : 0; }
void orc_cpff_force(orc *o) { if (o->M > 0) cpim_force(o); }
int orc_iterations(orc *o) { return o->iterations; }
int orc_step(orc *o) { return o->step; }

/* y = A x with the dense CPIM matrix in the reference vector layout. */
void orc_matvec(orc *o, const double *x, double *y) { matvec(o, x, y); }

void orc_pair_fingerprint(orc *o, long *count, unsigned long long *hash)
{
    const capac_desc *d = o->d;
    const double rc = d->r_cut, rc2 = o->c.r_cut2;
    long cnt = 0;
    uint64_t hs = 0;
    for (int i = 0; i < o->N; ++i) {
        for (int j = 0; j < i; ++j) {
            if (excluded(d, i, j)) continue;
            double x = o->rx[j] - o->rx[i], y = o->ry[j] - o->ry[i], z = o->rz[j] - o->rz[i];
            image(&x, &y, &z, o->box);
            if (x >= rc && y >= rc && z >= rc) continue;
            if (norm2(x, y, z) >= rc2) continue;
            ++cnt;
            hs += mix64(((uint64_t)(uint32_t)i << 32) | (uint32_t)j);
        }
    }
    *count = cnt;
    *hash = hs;
}

/* The same pair set as orc_pair_fingerprint, found through cells (see
 * cells_build) instead of all N(N-1)/2 pairs: each atom i tests the j < i of
 * the 27 cells around its own with the reference's image, early skip, r^2
 * formula and exclusions.  Boxes with fewer than three cells along an edge
 * take the all-pairs loop. */
void orc_pair_fingerprint_cells(orc *o, long *count, unsigned long long *hash)
{
    const capac_desc *d = o->d;
    const double rc = d->r_cut, rc2 = o->c.r_cut2;
    cells c;
    if (!cells_build(o, &c)) {
        orc_pair_fingerprint(o, count, hash);
        return;
    }
    long cnt = 0;
    uint64_t hs = 0;
    for (int i = 0; i < o->N; ++i)
        for (int k = 0; k < 27; ++k) {
            const int cc = cells_near(&c, i, k);
            for (int t = c.start[cc]; t < c.start[cc + 1]; ++t) {
                const int j = c.atoms[t];
                if (j >= i || excluded(d, i, j)) continue;
                double x = o->rx[j] - o->rx[i], y = o->ry[j] - o->ry[i], z = o->rz[j] - o->rz[i];
                image(&x, &y, &z, o->box);
                if (x >= rc && y >= rc && z >= rc) continue;
                if (norm2(x, y, z) >= rc2) continue;
                ++cnt;
                hs += mix64(((uint64_t)(uint32_t)i << 32) | (uint32_t)j);
            }
        }
    cells_free(&c);
    *count = cnt;
    *hash = hs;
}

/* Restrict the nonbonded pass of later force calls to the given atoms
 * (nonbonded_sample); n = 0 restores the full pass. */
int orc_set_sample(orc *o, const long *idx, int n)
{
    free(o->sample);
    o->sample = NULL;
    o->n_sample = 0;
    if (n <= 0) return 0;
    o->sample = (int *)malloc(sizeof(int) * (size_t)n);
    if (!o->sample) return -1;
    for (int k = 0; k < n; ++k) {
        if (idx[k] < 0 || idx[k] >= o->N) return -1;
        o->sample[k] = (int)idx[k];
    }
    o->n_sample = n;
    return 0;
}

int orc_get(orc *o, const char *what, double *out)
{
    const int N = o->N, n = o->M > 0 ? o->n_mat : 0;
    struct { const char *nm; const double *src; int cnt; } tab[] = {
        {"rx", o->rx, N}, {"ry", o->ry, N}, {"rz", o->rz, N}, {"vx", o->vx, N}, {"vy", o->vy, N},
        {"vz", o->vz, N}, {"fx", o->fx, N}, {"fy", o->fy, N}, {"fz", o->fz, N},
        {"potential", o->pot, 15}, {"virial", o->vir, 9}, {"vQ", o->vQ, NHC_LEN},
        {"vec_pq", o->vec_pq, n}, {"vec_ext", o->vec_ext, n}, {"diag_relay", o->diag, n},
        {"inv_sqrt_dens", o->inv_sqrt_dens, o->M}, {"box", o->box, 6},
    };
    for (size_t k = 0; k < sizeof tab / sizeof tab[0]; ++k) {
        if (0 == strcmp(what, tab[k].nm)) {
            if (tab[k].cnt > 0) memcpy(out, tab[k].src, sizeof(double) * tab[k].cnt);
            return tab[k].cnt;
        }
    }
    if (0 == strcmp(what, "thermo")) {
        out[0] = o->eksum; out[1] = o->inst_temp; out[2] = o->ref_temp; out[3] = o->c.ndf;
        return 4;
    }
    if (0 == strcmp(what, "fmax_rms")) {
        out[0] = o->f_max; out[1] = o->f_rms;
        return 2;
    }
    return -1;
}

int orc_set(orc *o, const char *what, const double *in)
{
    const int N = o->N, n = o->M > 0 ? o->n_mat : 0;
    struct { const char *nm; double *dst; int cnt; } tab[] = {
        {"rx", o->rx, N}, {"ry", o->ry, N}, {"rz", o->rz, N}, {"vx", o->vx, N}, {"vy", o->vy, N},
        {"vz", o->vz, N}, {"vec_pq", o->vec_pq, n}, {"fx", o->fx, N}, {"fy", o->fy, N}, {"fz", o->fz, N},
    };
    for (size_t k = 0; k < sizeof tab / sizeof tab[0]; ++k) {
        if (0 == strcmp(what, tab[k].nm)) {
            if (tab[k].cnt > 0) memcpy(tab[k].dst, in, sizeof(double) * tab[k].cnt);
            return tab[k].cnt;
        }
    }
    return -1;
}
