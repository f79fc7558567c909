// Shared by the drop-in shims: a capac_desc built from the reference driver's
// own structures (the information read_settings, read_param_1/2,
// assign_indices and read_gro put there, file.c) and the one GPU context of
// the process.
//
// Compiled as C++ against the reference's headers (typedef.h pulls in
// std::vector), with the shims, by the drop-in targets of oracle/Makefile.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <initializer_list>
#include <string>
#include <vector>

#include "shim_desc.h"

namespace {

capac_ctx *g_ctx = nullptr;
bool g_full = false;  // the context knows the run settings and the metal
capac_desc g_desc;

// storage behind g_desc's pointers
std::vector<int> v_mol_num, v_mol_atoms, v_nb_funct, v_excl_offset, v_cstr_offset, v_cstr_count, v_cstr_i,
    v_cstr_j, v_atom_type, v_mol_id, v_mol_type, v_atom_in_mol, v_mol_first, v_mol_last;
std::vector<double> v_nb_c6, v_nb_c12, v_nb_a, v_nb_b, v_cstr_r, v_charge, v_mass, v_inv_mass;
std::vector<unsigned char> v_excl, v_is_metal;
std::vector<int> v_bt_offset, v_bt_count, v_bt_kind, v_bt_atoms, v_vs_offset, v_vs_count, v_vs_atoms;
std::vector<double> v_bt_par, v_vs_par;

void add_term(int kind, std::initializer_list<int> at, std::initializer_list<double> par)
{
    v_bt_kind.push_back(kind);
    int k = 0;
    for (int a : at) v_bt_atoms.push_back(a), ++k;
    for (; k < 4; ++k) v_bt_atoms.push_back(0);
    k = 0;
    for (double v : par) v_bt_par.push_back(v), ++k;
    for (; k < 6; ++k) v_bt_par.push_back(0.0);
}

// Bonded terms and virtual sites of molecule type mt in the order
// mpi_bonded (force.c:1694-1900) and build_vsites (force.c:1582-1629) use.
void add_bonded(const Topol *t, int mt)
{
    v_bt_offset[mt] = (int)v_bt_kind.size();
    for (int k = 0; k < t->n_bonds[mt]; ++k) {
        const BondParam &b = t->bond_param[mt][k];
        if (b.funct == 1) add_term(CAPAC_BT_BOND_HARMONIC, {b.atom_i, b.atom_j}, {b.b0, b.kb});
        else if (b.funct == 3) add_term(CAPAC_BT_BOND_MORSE, {b.atom_i, b.atom_j}, {b.b0, b.D, b.beta});
    }
    for (int k = 0; k < t->n_pairs[mt]; ++k) {
        const PairParam &p = t->pair_param[mt][k];
        if (p.funct == 1) {
            add_term(CAPAC_BT_PAIR_14, {p.atom_i, p.atom_j}, {});
        } else if (p.funct == 2) {
            const double sig_6 = pow(p.V, 6.0), eps_4 = 4.0 * p.W;
            const double c6 = eps_4 * sig_6, c12 = c6 * sig_6;
            add_term(CAPAC_BT_PAIR_USER, {p.atom_i, p.atom_j}, {p.scaleQQ, p.q_i, p.q_j, c6, c12});
        }
    }
    for (int k = 0; k < t->n_angles[mt]; ++k) {
        const AngleParam &a = t->angle_param[mt][k];
        if (a.funct == 1)
            add_term(CAPAC_BT_ANGLE_HARMONIC, {a.atom_i, a.atom_j, a.atom_k}, {a.a0, a.ka});
        else if (a.funct == 5)
            add_term(CAPAC_BT_ANGLE_UB, {a.atom_i, a.atom_j, a.atom_k}, {a.a0, a.ka, a.b0_ub, a.kb_ub});
    }
    for (int k = 0; k < t->n_dihedrals[mt]; ++k) {
        const DihedralParam &q = t->dihedral_param[mt][k];
        double c[6] = {q.c0, q.c1, q.c2, q.c3, q.c4, q.c5};
        if (q.funct != 3 && capac_dihedral_periodic_to_rb(q.phi0, q.kphi, q.n, c) != CAPAC_OK) {
            printf("<> Error: phi0 is not equal to 0 or pi, or n is not 1 to 4\n");
            exit(1);
        }
        add_term(CAPAC_BT_DIHEDRAL_RB, {q.atom_i, q.atom_j, q.atom_k, q.atom_l}, {c[0], c[1], c[2], c[3], c[4], c[5]});
    }
    v_bt_count[mt] = (int)v_bt_kind.size() - v_bt_offset[mt];
    v_vs_offset[mt] = (int)(v_vs_atoms.size() / 4);
    v_vs_count[mt] = t->n_vsites[mt];
    for (int k = 0; k < t->n_vsites[mt]; ++k) {
        const VSite_4 &v = t->vsite_4[mt][k];
        for (int a : {v.atom_i, v.atom_j, v.atom_k, v.atom_s}) v_vs_atoms.push_back(a);
        for (double x : {v.a, v.b, v.c}) v_vs_par.push_back(x);
    }
}


// capac_desc from the driver's structures (read_settings, read_param_*,
// assign_indices and read_gro have filled them: file.c).
void build_desc(const Topol *t, const Atom_Info *ai, const Mol_Info *mi, const RunSet *rs, const Metal *m,
                const System *s)
{
    capac_desc &d = g_desc;
    d = capac_desc{};
    d.run_type = CAPAC_RUN_MD;
    if (rs) {
        d.ensemble = std::string(rs->ensemble) == "nvt" ? CAPAC_NVT : CAPAC_NVE;
        d.n_steps = rs->nSteps;
        d.n_save = rs->nSave;
        d.n_heating = rs->nHeating;
        d.em_steps = rs->em_steps;
        d.dt = rs->dt;
        d.r_cut = rs->rCut;
        d.w_alpha = rs->w_alpha;
        d.ref_temp = rs->ref_temp;
        d.tau_temp = rs->tau_temp;
        d.em_length = rs->em_length;
        d.em_tol = rs->em_tol;
        d.use_vdw = rs->use_vdw;
        d.use_coulomb = rs->use_coulomb;
        for (int a = 0; a < 3; ++a) d.efield[a] = rs->external_efield[a];
    } else {  // a context for RATTLE alone: the force settings are never used
        d.ensemble = CAPAC_NVE;
        d.n_save = 1;
        d.dt = 0.001;
        d.r_cut = 1.0;
        d.w_alpha = 2.0;
        d.ref_temp = 300.0;
        d.tau_temp = 0.1;
        d.use_vdw = 1;
        d.use_coulomb = 1;
    }
    d.fix_metal = m ? m->fix_pos : 0;
    d.use_cpff = m ? m->use_cpff : 0;
    d.scale_lj = t->scaleLJ;
    d.scale_qq = t->scaleQQ;

    const int T = t->mol_types, NT = t->n_types, N = t->n_atoms;
    d.n_atoms = N;
    d.n_mols = t->n_mols;
    d.n_types = NT;
    d.mol_types = T;
    v_mol_num.assign(t->mol_num, t->mol_num + T);
    v_mol_atoms.assign(t->atom_num, t->atom_num + T);
    d.mol_num = v_mol_num.data();
    d.mol_atoms = v_mol_atoms.data();

    // nonbonded table: the reference fills [i][j] for j >= i (file.c:618-672)
    v_nb_funct.assign(NT * NT, 0);
    v_nb_c6.assign(NT * NT, 0.0);
    v_nb_c12.assign(NT * NT, 0.0);
    v_nb_a.assign(NT * NT, 0.0);
    v_nb_b.assign(NT * NT, 0.0);
    for (int i = 0; i < NT; ++i)
        for (int j = 0; j < NT; ++j) {
            const NonbondedParam &p = t->nonbonded_param[i < j ? i : j][i < j ? j : i];
            const int k = i * NT + j;
            v_nb_funct[k] = p.funct;
            v_nb_c6[k] = p.C6;
            v_nb_c12[k] = p.C12;
            v_nb_a[k] = p.A;
            v_nb_b[k] = p.B;
        }
    d.nb_funct = v_nb_funct.data();
    d.nb_c6 = v_nb_c6.data();
    d.nb_c12 = v_nb_c12.data();
    d.nb_a = v_nb_a.data();
    d.nb_b = v_nb_b.data();

    // exclusions and constraints per molecule type
    v_excl_offset.assign(T, 0);
    v_cstr_offset.assign(T, 0);
    v_cstr_count.assign(T, 0);
    v_excl.clear();
    v_cstr_i.clear();
    v_cstr_j.clear();
    v_cstr_r.clear();
    d.n_cstr_total = 0;
    d.n_bonded_terms = 0;
    d.n_vsites_total = 0;
    v_bt_offset.assign(T, 0);
    v_bt_count.assign(T, 0);
    v_vs_offset.assign(T, 0);
    v_vs_count.assign(T, 0);
    v_bt_kind.clear();
    v_bt_atoms.clear();
    v_bt_par.clear();
    v_vs_atoms.clear();
    v_vs_par.clear();
    for (int mt = 0; mt < T; ++mt) {
        const int na = t->atom_num[mt];
        v_excl_offset[mt] = (int)v_excl.size();
        for (int a = 0; a < na; ++a)
            for (int b = 0; b < na; ++b) v_excl.push_back(t->exclude[mt][a][b] ? 1 : 0);
        v_cstr_offset[mt] = (int)v_cstr_i.size();
        v_cstr_count[mt] = t->n_constraints[mt];
        for (int k = 0; k < t->n_constraints[mt]; ++k) {
            v_cstr_i.push_back(t->constraint[mt][k].atom_i);
            v_cstr_j.push_back(t->constraint[mt][k].atom_j);
            v_cstr_r.push_back(t->constraint[mt][k].r);
        }
        d.n_cstr_total += t->n_constraints[mt] * t->mol_num[mt];
        add_bonded(t, mt);
        d.n_bonded_terms += v_bt_count[mt] * t->mol_num[mt];
        d.n_vsites_total += t->n_vsites[mt] * t->mol_num[mt];
    }
    d.bt_offset = v_bt_offset.data();
    d.bt_count = v_bt_count.data();
    d.bt_kind = v_bt_kind.data();
    d.bt_atoms = v_bt_atoms.data();
    d.bt_par = v_bt_par.data();
    d.vs_offset = v_vs_offset.data();
    d.vs_count = v_vs_count.data();
    d.vs_atoms = v_vs_atoms.data();
    d.vs_par = v_vs_par.data();
    d.excl_offset = v_excl_offset.data();
    d.excl = v_excl.data();
    d.cstr_offset = v_cstr_offset.data();
    d.cstr_count = v_cstr_count.data();
    d.cstr_i = v_cstr_i.data();
    d.cstr_j = v_cstr_j.data();
    d.cstr_r = v_cstr_r.data();

    // metal and nanoparticles
    if (m) {
        d.metal_min = m->min;
        d.metal_max = m->max;
        d.n_metal = m->num;
        d.qsc_n = m->qsc_n;
        d.qsc_m = m->qsc_m;
        d.qsc_eps = m->qsc_eps;
        d.qsc_c = m->qsc_c;
        d.qsc_a = m->qsc_a;
        d.cpff_polar = m->cpff_polar;
        d.cpff_capac = m->cpff_capac;
        d.n_nps = m->n_NPs;
        d.np_start = m->start_NP;
        d.np_end = m->end_NP;
        d.np_charge = m->cpff_chg;
    } else {  // RATTLE alone: no metal terms
        d.metal_min = d.metal_max = -1;
        d.n_metal = 0;
    }

    // per atom (assign_indices, file.c:1031-1099)
    v_atom_type.resize(N);
    v_mol_id.resize(N);
    v_mol_type.resize(N);
    v_atom_in_mol.resize(N);
    v_is_metal.resize(N);
    v_charge.resize(N);
    v_mass.resize(N);
    v_inv_mass.resize(N);
    for (int i = 0; i < N; ++i) {
        v_atom_type[i] = ai[i].atomtype;
        v_mol_id[i] = ai[i].molID;
        v_mol_type[i] = ai[i].iMol;
        v_atom_in_mol[i] = ai[i].iAtom;
        v_is_metal[i] = ai[i].is_metal ? 1 : 0;
        v_charge[i] = ai[i].charge;
        v_mass[i] = ai[i].mass;
        v_inv_mass[i] = ai[i].inv_mass;
    }
    d.atom_type = v_atom_type.data();
    d.mol_id = v_mol_id.data();
    d.mol_type = v_mol_type.data();
    d.atom_in_mol = v_atom_in_mol.data();
    d.is_metal = v_is_metal.data();
    d.charge = v_charge.data();
    d.mass = v_mass.data();
    d.inv_mass = v_inv_mass.data();
    v_mol_first.assign(t->n_mols, N);
    v_mol_last.assign(t->n_mols, -1);
    if (mi) {
        for (int im = 0; im < t->n_mols; ++im) {
            v_mol_first[im] = mi[im].mini;
            v_mol_last[im] = mi[im].maxi;
        }
    } else {  // Mol_Info as assign_indices fills it (file.c:1031-1099): each molecule's atom range
        for (int i = 0; i < N; ++i) {
            const int im = ai[i].molID;
            if (im >= 0 && im < t->n_mols) {
                v_mol_first[im] = std::min(v_mol_first[im], i);
                v_mol_last[im] = std::max(v_mol_last[im], i);
            }
        }
    }
    d.mol_first = v_mol_first.data();
    d.mol_last = v_mol_last.data();

    // the state (positions are sent again on every call)
    for (int a = 0; a < 3; ++a) d.box[a] = s->box[a];
    d.rx = s->rx;
    d.ry = s->ry;
    d.rz = s->rz;
    d.vx = s->vx;
    d.vy = s->vy;
    d.vz = s->vz;
    d.vq0 = s->vQ[0];
    d.vp = s->vP;
}


}  // namespace

void shim_fail(const char *what)
{
    printf("GPU %s: %s\n", what, capac_last_error());
    exit(1);
}

capac_ctx *shim_existing() { return g_ctx; }

const capac_desc *shim_desc() { return g_ctx ? &g_desc : nullptr; }

capac_ctx *shim_context(const Topol *t, const Atom_Info *ai, const Mol_Info *mi, const RunSet *rs, const Metal *m,
                        const System *s)
{
    const bool full = rs != nullptr && m != nullptr;
    if (g_ctx && (g_full || !full)) return g_ctx;
    if (g_ctx) {  // a fuller description than the one the context was made from
        capac_destroy(g_ctx);
        g_ctx = nullptr;
    }
    build_desc(t, ai, mi, rs, m, s);
    capac_options o;
    capac_options_default(&o);  // FP64, the reference's solver rule
    if (const char *dev = getenv("CAPAC_DEVICE")) o.device = atoi(dev);
    if (capac_create(&g_desc, &o, &g_ctx)) shim_fail("create");
    g_full = full;
    return g_ctx;
}
