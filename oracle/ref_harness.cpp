// Oracle harness around the reference CapacMD sources (test infrastructure).
//
// The reference's physics (force.c, cpff.c, bicg_stab.c, thermostat.c, file.c)
// is compiled unmodified from its own source files by oracle/Makefile; this
// file replaces only its driver, mpi-main.c, with a single-rank set-up and MD
// loop exposed through a small extern "C" API so that Python tests can run it
// and read every intermediate array at full precision.
//
// The set-up follows mpi-main.c:97-626 and the MD loop mpi-main.c:874-1013
// (file output left out, apply_pbc kept because it changes positions).  One
// deliberate difference: the pair count is formed in 64-bit arithmetic; the
// reference evaluates `nAtoms * (nAtoms - 1) / 2` in int (mpi-main.c:406), which
// overflows for N >= 46342 and makes mpi_nonb_pair skip every pair.
#include <mpi.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include <vector>

#include "typedef.h"
#include "file.h"
#include "force.h"
#include "thermostat.h"

namespace {

struct RefSim {
    RunSet *rs = nullptr;
    Metal *metal = nullptr;
    Topol *topol = nullptr;
    Task *task = nullptr;
    System *sys = nullptr;
    Atom_Info *atom_info = nullptr;
    Mol_Info *mol_info = nullptr;
    Bicgstab *bcg = nullptr;
    double **time_used = nullptr;
    int n_atoms = 0, n_mols = 0, n_mat = 0, n_vsites = 0, n_cstrs = 0;
    int step = 0;
    bool has_metal = false;
};

template <class T>
T *zalloc(size_t n)
{
    void *p = calloc(n > 0 ? n : 1, sizeof(T));
    if (!p) { fprintf(stderr, "capref: out of memory\n"); abort(); }
    return static_cast<T *>(p);
}

double now_s()
{
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec + tv.tv_usec * 1.0e-6;
}

}  // namespace

// mpi_mat_vec_COO (bicg_stab.c:46-63) has no header declaration; it has C++
// linkage like every reference function; so do pbc_12 and dist_2 (force.c).
void mpi_mat_vec_COO(const int count_nnz, const int n_mat, Metal *p_metal, double *x, double *Ax);
void pbc_12(Vec_R *ptr_r, const double *box);
double dist_2(const Vec_R *ptr_r);

extern "C" {

void *capref_open_ex(const char *gro, const char *par, const char *mds, int first_force);

// Open a system from the three reference input files and evaluate the first
// force call exactly as the reference driver does before its MD loop.
void *capref_open(const char *gro, const char *par, const char *mds)
{
    return capref_open_ex(gro, par, mds, 1);
}

// Time one reference force call on a sample of the nonbonded pair loop: the
// pair range is restricted to the last `pair_frac` of the linear pair index,
// exactly the share one rank of a 1/pair_frac-rank run would own
// (Task.start_pair/end_pair, mpi-main.c:398-407, force.c:1405-1440); every
// other phase runs in full.  Returns wall seconds; per-phase seconds of this
// call go to phase[15] in the reference's time_used slots.
double capref_time_sampled_force(void *h, double pair_frac, double *phase)
{
    RefSim *s = static_cast<RefSim *>(h);
    Task *tk = s->task;
    const long P = (long)s->n_atoms * (long)(s->n_atoms - 1) / 2;
    long take = (long)(pair_frac * (double)P);
    if (take < 1) take = 1;
    if (take > P) take = P;
    const long s0 = tk->start_pair[0], e0 = tk->end_pair[0];
    tk->start_pair[0] = P - take;
    tk->end_pair[0] = P - 1;
    double before[15];
    memcpy(before, s->time_used[0], sizeof before);
    const double t0 = now_s();
    mpi_force(tk, s->topol, s->atom_info, s->mol_info, s->rs, s->metal, s->sys, s->bcg, 0, 1, s->time_used);
    const double t = now_s() - t0;
    tk->start_pair[0] = s0;
    tk->end_pair[0] = e0;
    for (int k = 0; k < 15; ++k) phase[k] = s->time_used[0][k] - before[k];
    return t;
}

void *capref_open_ex(const char *gro, const char *par, const char *mds, int first_force)
{
    RefSim *s = new RefSim();
    char gro_buf[MAX_STR_LEN], par_buf[MAX_STR_LEN], mds_buf[MAX_STR_LEN];
    snprintf(gro_buf, sizeof gro_buf, "%s", gro);
    snprintf(par_buf, sizeof par_buf, "%s", par);
    snprintf(mds_buf, sizeof mds_buf, "%s", mds);

    s->rs = zalloc<RunSet>(1);
    s->metal = new Metal();  // value-initialised: PODs zero, vectors constructed
    s->rs->external_efield = zalloc<double>(DIM);
    read_settings(mds_buf, s->rs, s->metal);

    RunSet *rs = s->rs;
    if (0 == strcmp(rs->coulomb_type, "cut_off")) rs->use_coulomb = 0;
    else if (0 == strcmp(rs->coulomb_type, "wolf_sum")) rs->use_coulomb = 1;
    else { fprintf(stderr, "capref: unknown coulomb_type %s\n", rs->coulomb_type); delete s; return nullptr; }

    rs->rCut2 = rs->rCut * rs->rCut;
    rs->w_a2_sqrtPI = rs->w_alpha * 2.0 * INV_SQRT_PI;
    rs->w_Const = erfc(rs->w_alpha * rs->rCut) / rs->rCut2 +
                  rs->w_a2_sqrtPI * exp(-rs->w_alpha * rs->w_alpha * rs->rCut2) / rs->rCut;
    rs->w_erfc_arCut = erfc(rs->w_alpha * rs->rCut) / rs->rCut;

    if (0 == strcmp(rs->vdw_type, "cut_off")) rs->use_vdw = 0;
    else if (0 == strcmp(rs->vdw_type, "shifted")) rs->use_vdw = 1;
    else { fprintf(stderr, "capref: unknown vdw_type %s\n", rs->vdw_type); delete s; return nullptr; }
    rs->inv_rc12 = 1.0 / pow(rs->rCut, 12.0);
    rs->inv_rc6 = 1.0 / pow(rs->rCut, 6.0);

    Topol *tp = s->topol = zalloc<Topol>(1);
    Metal *mt = s->metal;
    read_param_1(par_buf, tp, mt);

    mt->cpff_chg = zalloc<double>(mt->n_NPs);
    mt->start_NP = zalloc<int>(mt->n_NPs);
    mt->end_NP = zalloc<int>(mt->n_NPs);
    tp->atom_num = zalloc<int>(tp->mol_types);
    tp->mol_num = zalloc<int>(tp->mol_types);
    tp->atom_param = zalloc<AtomParam *>(tp->mol_types);

    NonbondedParam *nb = zalloc<NonbondedParam>((size_t)tp->n_types * tp->n_types);
    tp->nonbonded_param = zalloc<NonbondedParam *>(tp->n_types);
    for (int t = 0; t < tp->n_types; ++t) tp->nonbonded_param[t] = nb + (size_t)tp->n_types * t;

    int *counts = zalloc<int>((size_t)tp->mol_types * 6);
    tp->n_bonds = counts;
    tp->n_pairs = counts + tp->mol_types;
    tp->n_angles = counts + tp->mol_types * 2;
    tp->n_dihedrals = counts + tp->mol_types * 3;
    tp->n_vsites = counts + tp->mol_types * 4;
    tp->n_constraints = counts + tp->mol_types * 5;
    tp->vsite_funct = zalloc<int *>(tp->mol_types);
    tp->bond_param = zalloc<BondParam *>(tp->mol_types);
    tp->pair_param = zalloc<PairParam *>(tp->mol_types);
    tp->angle_param = zalloc<AngleParam *>(tp->mol_types);
    tp->dihedral_param = zalloc<DihedralParam *>(tp->mol_types);
    tp->vsite_4 = zalloc<VSite_4 *>(tp->mol_types);
    tp->constraint = zalloc<Constraint *>(tp->mol_types);
    tp->exclude = zalloc<int **>(tp->mol_types);

    s->has_metal = (mt->min >= 0 && mt->max >= mt->min);
    if (s->has_metal) mt->inv_sqrt_dens = zalloc<double>(mt->num);

    read_param_2(par_buf, tp, mt);
    s->n_atoms = tp->n_atoms;
    s->n_mols = tp->n_mols;
    for (int m = 0; m < tp->mol_types; ++m) {
        s->n_vsites += tp->n_vsites[m] * tp->mol_num[m];
        s->n_cstrs += tp->n_constraints[m] * tp->mol_num[m];
    }

    mt->inv_polar = 1.0 / mt->cpff_polar;
    mt->inv_capac = 1.0 / mt->cpff_capac;
    double R_q = sqrt(2.0 / M_PI) * mt->cpff_capac;
    double R_p = pow(sqrt(2.0 / M_PI) * mt->cpff_polar / 3.0, 1.0 / 3.0);
    mt->inv_R_qq = 1.0 / sqrt(R_q * R_q + R_q * R_q);
    mt->inv_R_pq = 1.0 / sqrt(R_p * R_p + R_q * R_q);
    mt->inv_R_pp = 1.0 / sqrt(R_p * R_p + R_p * R_p);

    // one rank owns everything
    Task *tk = s->task = zalloc<Task>(1);
    int *se = zalloc<int>(6);
    tk->start_mol = se + 0; tk->end_mol = se + 1;
    tk->start_atom = se + 2; tk->end_atom = se + 3;
    tk->start_metal = se + 4; tk->end_metal = se + 5;
    find_start_end(tk->start_mol, tk->end_mol, s->n_mols, 1);
    find_start_end(tk->start_atom, tk->end_atom, s->n_atoms, 1);
    find_start_end(tk->start_metal, tk->end_metal, mt->num, 1);
    long *sp = zalloc<long>(2);
    tk->start_pair = sp; tk->end_pair = sp + 1;
    long n_pairs = (long)s->n_atoms * (long)(s->n_atoms - 1) / 2;
    find_start_end_long(tk->start_pair, tk->end_pair, n_pairs, 1);

    s->atom_info = zalloc<Atom_Info>(s->n_atoms);
    s->mol_info = zalloc<Mol_Info>(s->n_mols);
    assign_indices(tp, mt, s->atom_info, s->mol_info);

    System *sy = s->sys = zalloc<System>(1);
    double *pot = zalloc<double>(30);
    sy->potential = pot; sy->partial_pot = pot + 15;
    sy->virial = zalloc<double *>(DIM);
    sy->partial_vir = zalloc<double *>(DIM);
    double *vir = zalloc<double>(DIM * DIM * 2);
    for (int i = 0; i < DIM; ++i) { sy->virial[i] = vir + DIM * i; sy->partial_vir[i] = vir + DIM * (DIM + i); }
    sy->box = zalloc<double>(6);
    size_t N = s->n_atoms;
    double *rvf = zalloc<double>(N * 21);
    double **slots[] = {&sy->rx, &sy->ry, &sy->rz, &sy->vx, &sy->vy, &sy->vz, &sy->fx, &sy->fy, &sy->fz,
                        &sy->partial_fx, &sy->partial_fy, &sy->partial_fz, &sy->old_rx, &sy->old_ry,
                        &sy->old_rz, &sy->old_fx, &sy->old_fy, &sy->old_fz, &sy->sx, &sy->sy, &sy->sz};
    for (int k = 0; k < 21; ++k) *slots[k] = rvf + N * k;

    sy->num_nhc = 10;
    sy->vQ = zalloc<double>(sy->num_nhc);
    sy->aQ = zalloc<double>(sy->num_nhc);
    int gro_n = 0;
    char gro_buf2[MAX_STR_LEN];
    snprintf(gro_buf2, sizeof gro_buf2, "%s", gro_buf);
    read_gro(gro_buf2, sy, &gro_n, s->atom_info);
    if (gro_n != s->n_atoms) {
        fprintf(stderr, "capref: gro has %d atoms, param has %d\n", gro_n, s->n_atoms);
        return nullptr;
    }
    sy->box[3] = sy->box[0] * 0.5;
    sy->box[4] = sy->box[1] * 0.5;
    sy->box[5] = sy->box[2] * 0.5;
    sy->volume = sy->box[0] * sy->box[1] * sy->box[2];
    sy->inv_volume = 1.0 / sy->volume;

    sy->ndf = 3 * (s->n_atoms - s->n_vsites) - 3 - s->n_cstrs;
    rs->kT = K_BOLTZ * rs->ref_temp;
    sy->qMass = (double)sy->ndf * rs->kT * rs->tau_temp * rs->tau_temp;
    rs->dt_2 = 0.5 * rs->dt;

    s->n_mat = mt->num * 4 + mt->n_NPs;
    if (s->has_metal) {
        double *rel = zalloc<double>((size_t)s->n_mat * 3);
        mt->vec_pq = rel;
        mt->vec_ext = rel + s->n_mat;
        mt->diag_relay = rel + 2 * s->n_mat;
        for (int k = 0; k < s->n_mat; ++k) mt->diag_relay[k] = 1.0;
    }
    double *bw = zalloc<double>((size_t)(s->n_mat > 0 ? s->n_mat : 1) * 11);
    Bicgstab *b = s->bcg = zalloc<Bicgstab>(1);
    double **bs[] = {&b->Ax, &b->r0, &b->r, &b->p, &b->v, &b->s, &b->t, &b->y, &b->z, &b->Kt, &b->K};
    for (int k = 0; k < 11; ++k) *bs[k] = bw + (size_t)s->n_mat * k;

    s->time_used = zalloc<double *>(1);
    s->time_used[0] = zalloc<double>(15);
    if (!first_force) return s;

    mpi_force(s->task, tp, s->atom_info, s->mol_info, rs, mt, sy, s->bcg, 0, 1, s->time_used);
    sum_potential(sy->potential);
    remove_comm(s->n_atoms, s->atom_info, sy);
    kinetic_energy(sy, s->n_atoms, s->atom_info);
    sy->first_temp = sy->inst_temp;
    sy->ext_temp = rs->ref_temp;
    get_fmax_rms(s->n_atoms, sy);
    return s;
}

// Re-evaluate mpi_force on the current state (positions may have been set).
void capref_force(void *h)
{
    RefSim *s = static_cast<RefSim *>(h);
    mpi_force(s->task, s->topol, s->atom_info, s->mol_info, s->rs, s->metal, s->sys, s->bcg, 0, 1,
              s->time_used);
    sum_potential(s->sys->potential);
}

// Advance n MD steps following the reference loop (mpi-main.c:874-1013).
void capref_md_steps(void *h, int n)
{
    RefSim *s = static_cast<RefSim *>(h);
    RunSet *rs = s->rs;
    System *sy = s->sys;
    Atom_Info *ai = s->atom_info;
    const int N = s->n_atoms;
    const bool nvt = (0 == strcmp(rs->ensemble, "nvt"));
    for (int k = 0; k < n; ++k) {
        const int step = ++s->step;
        if (step < rs->nHeating)
            rs->ref_temp = sy->first_temp + (sy->ext_temp - sy->first_temp) * step / rs->nHeating;
        else
            rs->ref_temp = sy->ext_temp;
        rs->kT = K_BOLTZ * rs->ref_temp;
        if (nvt) nose_hoover_chain(rs, sy, N);
        for (int i = 0; i < N; ++i) {
            if (1 == s->metal->fix_pos && 1 == ai[i].is_metal) continue;
            double im = ai[i].inv_mass;
            sy->vx[i] += rs->dt_2 * sy->fx[i] * im;
            sy->vy[i] += rs->dt_2 * sy->fy[i] * im;
            sy->vz[i] += rs->dt_2 * sy->fz[i] * im;
        }
        for (int i = 0; i < N; ++i) {
            if (1 == s->metal->fix_pos && 1 == ai[i].is_metal) continue;
            sy->old_rx[i] = sy->rx[i];
            sy->old_ry[i] = sy->ry[i];
            sy->old_rz[i] = sy->rz[i];
            sy->rx[i] += rs->dt * sy->vx[i];
            sy->ry[i] += rs->dt * sy->vy[i];
            sy->rz[i] += rs->dt * sy->vz[i];
        }
        rattle_1st(rs->dt, s->mol_info, ai, s->topol, sy);
        mpi_force(s->task, s->topol, ai, s->mol_info, rs, s->metal, sy, s->bcg, 0, 1, s->time_used);
        sum_potential(sy->potential);
        for (int i = 0; i < N; ++i) {
            if (1 == s->metal->fix_pos && 1 == ai[i].is_metal) continue;
            double im = ai[i].inv_mass;
            sy->vx[i] += rs->dt_2 * sy->fx[i] * im;
            sy->vy[i] += rs->dt_2 * sy->fy[i] * im;
            sy->vz[i] += rs->dt_2 * sy->fz[i] * im;
        }
        rattle_2nd(rs->dt, s->mol_info, ai, s->topol, sy);
        kinetic_energy(sy, N, ai);
        if (nvt) nose_hoover_chain(rs, sy, N);
        remove_comm(N, ai, sy);
        kinetic_energy(sy, N, ai);
        if (0 == step % rs->nSave) {
            apply_pbc(s->n_mols, s->mol_info, sy->rx, sy->ry, sy->rz, sy->box);
            get_fmax_rms(N, sy);
        }
    }
}

int capref_n_atoms(void *h) { return static_cast<RefSim *>(h)->n_atoms; }
int capref_n_metal(void *h) { return static_cast<RefSim *>(h)->metal->num; }
int capref_n_mat(void *h) { return static_cast<RefSim *>(h)->n_mat; }
int capref_step(void *h) { return static_cast<RefSim *>(h)->step; }
long capref_nnz(void *h) { return (long)static_cast<RefSim *>(h)->metal->vec_val.size(); }

// Copy a named array out.  Names: rx ry rz vx vy vz fx fy fz old_rx old_ry
// old_rz potential(15) virial(9) vec_pq vec_ext diag_relay(n_mat)
// inv_sqrt_dens(n_metal) vQ(10) thermo(4: eKsum inst_temp ref_temp ndf)
// time_used(15).  Returns the number of doubles written, -1 if unknown.
int capref_get(void *h, const char *what, double *out)
{
    RefSim *s = static_cast<RefSim *>(h);
    System *sy = s->sys;
    const int N = s->n_atoms;
    struct { const char *name; double *src; int n; } tab[] = {
        {"rx", sy->rx, N}, {"ry", sy->ry, N}, {"rz", sy->rz, N},
        {"vx", sy->vx, N}, {"vy", sy->vy, N}, {"vz", sy->vz, N},
        {"fx", sy->fx, N}, {"fy", sy->fy, N}, {"fz", sy->fz, N},
        {"old_rx", sy->old_rx, N}, {"old_ry", sy->old_ry, N}, {"old_rz", sy->old_rz, N},
        {"potential", sy->potential, 15}, {"vQ", sy->vQ, sy->num_nhc},
        {"vec_pq", s->metal->vec_pq, s->has_metal ? s->n_mat : 0},
        {"vec_ext", s->metal->vec_ext, s->has_metal ? s->n_mat : 0},
        {"diag_relay", s->metal->diag_relay, s->has_metal ? s->n_mat : 0},
        {"inv_sqrt_dens", s->metal->inv_sqrt_dens, s->has_metal ? s->metal->num : 0},
        {"time_used", s->time_used[0], 15},
    };
    for (auto &e : tab) {
        if (0 == strcmp(what, e.name)) {
            if (e.n > 0) memcpy(out, e.src, sizeof(double) * e.n);
            return e.n;
        }
    }
    if (0 == strcmp(what, "virial")) {
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) out[a * 3 + b] = sy->virial[a][b];
        return 9;
    }
    if (0 == strcmp(what, "thermo")) {
        out[0] = sy->eKsum; out[1] = sy->inst_temp; out[2] = s->rs->ref_temp; out[3] = sy->ndf;
        return 4;
    }
    if (0 == strcmp(what, "box")) {
        for (int k = 0; k < 6; ++k) out[k] = sy->box[k];
        return 6;
    }
    return -1;
}

// Overwrite a named per-atom array (rx ry rz vx vy vz) or vec_pq.
int capref_set(void *h, const char *what, const double *in)
{
    RefSim *s = static_cast<RefSim *>(h);
    System *sy = s->sys;
    const int N = s->n_atoms;
    struct { const char *name; double *dst; int n; } tab[] = {
        {"rx", sy->rx, N}, {"ry", sy->ry, N}, {"rz", sy->rz, N},
        {"vx", sy->vx, N}, {"vy", sy->vy, N}, {"vz", sy->vz, N},
        {"vec_pq", s->metal->vec_pq, s->has_metal ? s->n_mat : 0},
    };
    for (auto &e : tab) {
        if (0 == strcmp(what, e.name)) {
            if (e.n > 0) memcpy(e.dst, in, sizeof(double) * e.n);
            return e.n;
        }
    }
    return -1;
}

// Pair-set fingerprint of mpi_nonb_pair's traversal (force.c:1419-1473) on the
// current positions: the loop order and exclusion test are restated here, the
// image shift and r^2 are the reference's own pbc_12 and dist_2 (force.c:41,
// force.c:111).  Hash: sum of splitmix64(i << 32 | j) over the kept pairs.
static unsigned long long fp_mix(unsigned long long x)
{
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

void capref_pair_fingerprint(void *h, long *count, unsigned long long *hash)
{
    RefSim *s = static_cast<RefSim *>(h);
    System *sy = s->sys;
    Atom_Info *ai = s->atom_info;
    const double rc = s->rs->rCut, rc2 = s->rs->rCut2;
    long cnt = 0;
    unsigned long long hs = 0;
    for (int i = 0; i < s->n_atoms; ++i) {
        for (int j = 0; j < i; ++j) {
            if (ai[j].molID == ai[i].molID && 1 == s->topol->exclude[ai[i].iMol][ai[i].iAtom][ai[j].iAtom])
                continue;
            Vec_R r;
            r.x = sy->rx[j] - sy->rx[i];
            r.y = sy->ry[j] - sy->ry[i];
            r.z = sy->rz[j] - sy->rz[i];
            pbc_12(&r, sy->box);
            if (r.x >= rc && r.y >= rc && r.z >= rc) continue;
            if (dist_2(&r) >= rc2) continue;
            ++cnt;
            hs += fp_mix(((unsigned long long)(unsigned)i << 32) | (unsigned)j);
        }
    }
    *count = cnt;
    *hash = hs;
}

// y = A x with the reference COO matrix left by the last force call.
void capref_matvec(void *h, const double *x, double *y)
{
    RefSim *s = static_cast<RefSim *>(h);
    std::vector<double> xx(x, x + s->n_mat);
    mpi_mat_vec_COO((int)s->metal->vec_val.size(), s->n_mat, s->metal, xx.data(), y);
}

// Wall-clock seconds of n MD steps (CPU-baseline timing helper).
double capref_time_md_steps(void *h, int n)
{
    double t0 = now_s();
    capref_md_steps(h, n);
    return now_s() - t0;
}

}  // extern "C"
