// Drop-in mpi_force for the reference CapacMD driver.
//
// Linked into the reference's own mpi-main with
//   -Wl,--wrap=_Z9mpi_forceP4TaskP5TopolP9Atom_InfoP8Mol_InfoP6RunSetP5MetalP6SystemP8BicgstabiiPPd
// so every call the driver makes to mpi_force (mpi-main.c:614, 765, 940)
// lands here instead of in force.c; everything else (input reading, the
// integrator, RATTLE, the thermostat, output) stays the reference's code.
//
// The first call builds a capac_desc from the driver's own structures (the
// same information the reference read from init.gro, param.txt and
// mdset.txt) and creates the GPU context; every call then runs
// capac_mpi_force on the current positions: positions and the vec_pq warm
// start go to the device, forces, potential[1..14], the virial and the CPIM
// vectors come back (force.h:100-103 semantics; potential[0] is the caller's,
// time_used is left as it is).  A failing call prints the library's message
// and exits, as the reference does on its own errors.
//
// Compiled as C++ against the reference's headers (typedef.h pulls in
// std::vector): the `dropin` target of oracle/Makefile links it with the
// reference's objects into oracle/_ref/mpi-main-gpu.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "capacmd.h"
#include "typedef.h"

namespace {

capac_ctx *g_ctx = nullptr;
capac_desc g_desc;

// storage behind g_desc's pointers
std::vector<int> v_mol_num, v_mol_atoms, v_nb_funct, v_excl_offset, v_cstr_offset, v_cstr_count, v_cstr_i,
    v_cstr_j, v_atom_type, v_mol_id, v_mol_type, v_atom_in_mol, v_mol_first, v_mol_last;
std::vector<double> v_nb_c6, v_nb_c12, v_nb_a, v_nb_b, v_cstr_r, v_charge, v_mass, v_inv_mass;
std::vector<unsigned char> v_excl, v_is_metal;

void fail(const char *what)
{
    printf("GPU mpi_force: %s: %s\n", what, capac_last_error());
    exit(1);
}

// capac_desc from the driver's structures (read_settings, read_param_*,
// assign_indices and read_gro have filled them: file.c).
void build_desc(const Topol *t, const Atom_Info *ai, const Mol_Info *mi, const RunSet *rs, const Metal *m,
                const System *s)
{
    capac_desc &d = g_desc;
    d = capac_desc{};
    d.run_type = CAPAC_RUN_MD;
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
    d.fix_metal = m->fix_pos;
    d.use_cpff = m->use_cpff;
    for (int a = 0; a < 3; ++a) d.efield[a] = rs->external_efield[a];
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
        d.n_bonded_terms += t->n_bonds[mt] + t->n_pairs[mt] + t->n_angles[mt] + t->n_dihedrals[mt];
        d.n_vsites_total += t->n_vsites[mt] * t->mol_num[mt];
    }
    d.excl_offset = v_excl_offset.data();
    d.excl = v_excl.data();
    d.cstr_offset = v_cstr_offset.data();
    d.cstr_count = v_cstr_count.data();
    d.cstr_i = v_cstr_i.data();
    d.cstr_j = v_cstr_j.data();
    d.cstr_r = v_cstr_r.data();

    // metal and nanoparticles
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
    v_mol_first.resize(t->n_mols);
    v_mol_last.resize(t->n_mols);
    for (int im = 0; im < t->n_mols; ++im) {
        v_mol_first[im] = mi[im].mini;
        v_mol_last[im] = mi[im].maxi;
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

// The driver's mpi_force(Task*, Topol*, Atom_Info*, Mol_Info*, RunSet*, Metal*,
// System*, Bicgstab*, int, int, double**), redirected here by --wrap.
extern "C" void __wrap__Z9mpi_forceP4TaskP5TopolP9Atom_InfoP8Mol_InfoP6RunSetP5MetalP6SystemP8BicgstabiiPPd(
    Task *, Topol *t, Atom_Info *ai, Mol_Info *mi, RunSet *rs, Metal *m, System *s, Bicgstab *, int, int,
    double **)
{
    if (!g_ctx) {
        build_desc(t, ai, mi, rs, m, s);
        capac_options o;
        capac_options_default(&o);  // FP64, the reference's solver rule
        if (const char *dev = getenv("CAPAC_DEVICE")) o.device = atoi(dev);
        if (capac_create(&g_desc, &o, &g_ctx)) fail("create");
    }
    double vir[9];
    // the driver allocates the CPIM vectors whenever there are metal atoms
    // (mpi-main.c:576-591) and inv_sqrt_dens with them (mpi-main.c:290)
    const bool metal = m->num > 0 && m->vec_pq != nullptr;
    if (capac_mpi_force(g_ctx, s->rx, s->ry, s->rz, s->fx, s->fy, s->fz, s->potential, vir,
                        metal ? m->vec_pq : nullptr, metal ? m->vec_ext : nullptr, metal ? m->diag_relay : nullptr,
                        metal ? m->inv_sqrt_dens : nullptr))
        fail("force");
    for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c) s->virial[a][c] = vir[3 * a + c];
}
