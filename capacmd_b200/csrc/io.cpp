// Input layer: the three CapacMD input files parsed into a capac_desc.
//
// Formats are the reference's (they have to be, to stay a drop-in):
//   mdset.txt  key/value lines                       (file.c:74-130)
//   .gro       title with "step N vQ x vP y", count,
//              fixed-column atom lines, box line      (file.c:138-203)
//   param.txt  sections in a fixed order              (file.c:286-562, 569-1023)
// followed by the per-atom bookkeeping of assign_indices (file.c:1031-1099) and
// the constants derived in the driver (mpi-main.c:170-203, 315-323, 548-552).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <string>
#include <vector>

#include "capacmd.h"
#include "capac_internal.h"

namespace capac {

namespace {

constexpr double kEv2KjMol = 96.4853363969351;  // typedef.h:64
constexpr double kBoltz = 0.00831446214546895;  // typedef.h:73
constexpr double kInvSqrtPi = 0.564189583547756; // typedef.h:44
constexpr double kPi = 3.14159265358979323846;
constexpr int kLine = 256;                       // MAX_STR_LEN, typedef.h:30

template <class T>
T *alloc_array(size_t n)
{
    T *p = static_cast<T *>(calloc(n > 0 ? n : 1, sizeof(T)));
    if (!p) throw Error(CAPAC_ERR_INVALID, "out of host memory");
    return p;
}

// Next non-blank line of the parameter file; its first word goes to `word`.
struct LineReader {
    FILE *f;
    std::string path;
    char line[kLine];
    char word[kLine];
    void next()
    {
        for (;;) {
            if (!fgets(line, kLine, f))
                throw Error(CAPAC_ERR_IO, "unexpected end of " + path);
            word[0] = '\0';
            sscanf(line, "%255s", word);
            if (word[0] != '\0') return;
        }
    }
    void expect(const std::string &name)
    {
        next();
        if (name != word)
            throw Error(CAPAC_ERR_IO, "in " + path + ": expected " + name + " in line: " + line);
    }
};

void read_mdset(const char *path, capac_desc *d)
{
    FILE *f = fopen(path, "r");
    if (!f) throw Error(CAPAC_ERR_IO, std::string("cannot open ") + path);
    // defaults for keys the file may omit
    d->run_type = CAPAC_RUN_MD;
    d->ensemble = CAPAC_NVE;
    d->n_save = 1;
    d->dt = 0.001;
    d->use_vdw = 1;
    d->use_coulomb = 1;
    d->tau_temp = 0.1;
    char line[kLine], key[kLine], val[kLine];
    while (fgets(line, kLine, f)) {
        key[0] = val[0] = '\0';
        if (sscanf(line, "%255s%255s", key, val) < 1) continue;
        std::string k(key);
        std::string v(val);
        if (k == "run_type") {
            if (v == "md") d->run_type = CAPAC_RUN_MD;
            else if (v == "em") d->run_type = CAPAC_RUN_EM;
            else if (v == "cg") d->run_type = CAPAC_RUN_CG;
            else throw Error(CAPAC_ERR_IO, "unknown run_type " + v);
        } else if (k == "ensemble") {
            if (v == "nvt") d->ensemble = CAPAC_NVT;
            else if (v == "berendsen") d->ensemble = CAPAC_BERENDSEN;  // no counterpart in the reference
            else d->ensemble = CAPAC_NVE;  // the reference thermostats only on "nvt"
        } else if (k == "em_steps") d->em_steps = atoi(val);
        else if (k == "em_length_in_nm") d->em_length = atof(val);
        else if (k == "em_tolerance") d->em_tol = atof(val);
        else if (k == "number_of_steps") d->n_steps = atoi(val);
        else if (k == "time_step_in_ps") d->dt = atof(val);
        else if (k == "save_step") d->n_save = atoi(val);
        else if (k == "vdw_type") {
            if (v == "cut_off") d->use_vdw = 0;
            else if (v == "shifted") d->use_vdw = 1;
            else throw Error(CAPAC_ERR_IO, "unknown vdw_type " + v);
        } else if (k == "coulomb_type") {
            if (v == "cut_off") d->use_coulomb = 0;
            else if (v == "wolf_sum") d->use_coulomb = 1;
            else throw Error(CAPAC_ERR_IO, "unknown coulomb_type " + v);
        } else if (k == "cut_off_radius") d->r_cut = atof(val);
        else if (k == "coulomb_alpha") d->w_alpha = atof(val);
        else if (k == "heating_steps") d->n_heating = atoi(val);
        else if (k == "ref_T_in_K") d->ref_temp = atof(val);
        else if (k == "tau_T_in_ps") d->tau_temp = atof(val);
        else if (k == "fix_metal") d->fix_metal = atoi(val);
        else if (k == "use_cpff") d->use_cpff = atoi(val);
        else if (k == "external_Ex") d->efield[0] = atof(val) * kEv2KjMol;
        else if (k == "external_Ey") d->efield[1] = atof(val) * kEv2KjMol;
        else if (k == "external_Ez") d->efield[2] = atof(val) * kEv2KjMol;
        else fprintf(stderr, "capacmd: warning: unknown option %s in %s\n", key, path);
    }
    fclose(f);
    if (d->n_save <= 0) throw Error(CAPAC_ERR_IO, "save_step must be positive");
}

void read_param(const char *path, capac_desc *d)
{
    FILE *f = fopen(path, "r");
    if (!f) throw Error(CAPAC_ERR_IO, std::string("cannot open param file ") + path);
    LineReader r{f, path, {0}, {0}};
    try {
        r.expect("SCALE_LJ_QQ");
        sscanf(r.line, "%*s%lf%lf", &d->scale_lj, &d->scale_qq);
        r.expect("MOLECULES");
        sscanf(r.line, "%*s%d", &d->mol_types);
        if (d->mol_types <= 0) throw Error(CAPAC_ERR_IO, "MOLECULES must be positive");
        const int T = d->mol_types;
        std::vector<std::string> names(T);
        d->mol_num = alloc_array<int>(T);
        d->mol_atoms = alloc_array<int>(T);
        for (int m = 0; m < T; ++m) {
            r.next();
            char nm[kLine];
            if (sscanf(r.line, "%255s%d", nm, &d->mol_num[m]) != 2)
                throw Error(CAPAC_ERR_IO, std::string("bad molecule line: ") + r.line);
            names[m] = nm;
        }
        // per molecule type: charge, mass, atom type of each atom
        std::vector<std::vector<double>> q(T), mass(T);
        std::vector<std::vector<int>> type(T);
        for (int m = 0; m < T; ++m) {
            r.expect(names[m] + "_ATOMS");
            sscanf(r.line, "%*s%d", &d->mol_atoms[m]);
            for (int a = 0; a < d->mol_atoms[m]; ++a) {
                r.next();
                double qq = 0, mm = 0;
                int tt = 0;
                if (sscanf(r.line, "%lf%lf%d", &qq, &mm, &tt) != 3)
                    throw Error(CAPAC_ERR_IO, std::string("bad atom line: ") + r.line);
                q[m].push_back(qq);
                mass[m].push_back(mm);
                type[m].push_back(tt);
            }
        }
        r.expect("NONBONDED");
        sscanf(r.line, "%*s%d", &d->n_types);
        const int NT = d->n_types;
        if (NT <= 0) throw Error(CAPAC_ERR_IO, "NONBONDED needs a positive type count");
        d->nb_funct = alloc_array<int>(NT * NT);
        d->nb_c6 = alloc_array<double>(NT * NT);
        d->nb_c12 = alloc_array<double>(NT * NT);
        d->nb_a = alloc_array<double>(NT * NT);
        d->nb_b = alloc_array<double>(NT * NT);
        for (int it = 0; it < NT; ++it) {
            for (int jt = it; jt < NT; ++jt) {
                r.next();
                int fn = 0;
                sscanf(r.line, "%d", &fn);
                const int k = it * NT + jt;
                double c6 = 0, c12 = 0, a = 0, b = 0;
                // column order per function type as in file.c:620-672
                if (fn == 1) sscanf(r.line, "%*d%le%le", &c6, &c12);
                else if (fn == 2 || fn == 3) sscanf(r.line, "%*d%le%le%le", &a, &b, &c6);
                else if (fn == 4) sscanf(r.line, "%*d%le%le%le", &c6, &c12, &a);
                else throw Error(CAPAC_ERR_IO, std::string("unsupported vdW type in line: ") + r.line);
                const int kt = jt * NT + it;
                d->nb_funct[k] = d->nb_funct[kt] = fn;
                d->nb_c6[k] = d->nb_c6[kt] = c6;
                d->nb_c12[k] = d->nb_c12[kt] = c12;
                d->nb_a[k] = d->nb_a[kt] = a;
                d->nb_b[k] = d->nb_b[kt] = b;
            }
        }
        // exclusions and constraints per molecule type
        d->excl_offset = alloc_array<int>(T);
        d->cstr_offset = alloc_array<int>(T);
        d->cstr_count = alloc_array<int>(T);
        size_t excl_total = 0;
        for (int m = 0; m < T; ++m) {
            d->excl_offset[m] = (int)excl_total;
            excl_total += (size_t)d->mol_atoms[m] * d->mol_atoms[m];
        }
        d->excl = alloc_array<unsigned char>(excl_total);
        std::vector<int> ci, cj;
        std::vector<double> cr;
        std::vector<int> bkind, batoms, vatoms;
        std::vector<double> bpar, vpar;
        d->bt_offset = alloc_array<int>(T);
        d->bt_count = alloc_array<int>(T);
        d->vs_offset = alloc_array<int>(T);
        d->vs_count = alloc_array<int>(T);
        auto add_term = [&](int kind, std::initializer_list<int> at, std::initializer_list<double> par) {
            bkind.push_back(kind);
            int k = 0;
            for (int a : at) batoms.push_back(a), ++k;
            for (; k < 4; ++k) batoms.push_back(0);
            k = 0;
            for (double v : par) bpar.push_back(v), ++k;
            for (; k < 6; ++k) bpar.push_back(0.0);
        };
        auto exclude = [&](int m, int a, int b) {
            const int na = d->mol_atoms[m];
            if (a < 0 || b < 0 || a >= na || b >= na)
                throw Error(CAPAC_ERR_IO, "atom index out of range in " + names[m]);
            d->excl[d->excl_offset[m] + a * na + b] = 1;
            d->excl[d->excl_offset[m] + b * na + a] = 1;
        };
        auto bad = [&](const char *what) {
            throw Error(CAPAC_ERR_UNSUPPORTED, std::string("unsupported ") + what + " in line: " + r.line);
        };
        for (int m = 0; m < T; ++m) {
            int n = 0;
            d->bt_offset[m] = (int)bkind.size();
            // bonds (file.c:715-765); every listed bond excludes its pair
            r.expect(names[m] + "_BONDS");
            sscanf(r.line, "%*s%d", &n);
            for (int k = 0; k < n; ++k) {
                r.next();
                int a = 0, b = 0, fn = 0;
                double p0 = 0, p1 = 0, p2 = 0;
                sscanf(r.line, "%d%d%d", &a, &b, &fn);
                if (fn == 1) {
                    sscanf(r.line, "%*d%*d%*d%le%le", &p0, &p1);
                    add_term(CAPAC_BT_BOND_HARMONIC, {a, b}, {p0, p1});
                } else if (fn == 3) {
                    sscanf(r.line, "%*d%*d%*d%le%le%le", &p0, &p1, &p2);
                    add_term(CAPAC_BT_BOND_MORSE, {a, b}, {p0, p1, p2});
                } else if (fn != 5) {  // 5: exclusion only
                    bad("bond function type");
                }
                exclude(m, a, b);
            }
            // 1-4 pairs (file.c:767-811)
            r.expect(names[m] + "_PAIRS");
            sscanf(r.line, "%*s%d", &n);
            for (int k = 0; k < n; ++k) {
                r.next();
                int a = 0, b = 0, fn = 0;
                sscanf(r.line, "%d%d%d", &a, &b, &fn);
                if (fn == 1) {
                    add_term(CAPAC_BT_PAIR_14, {a, b}, {});
                } else if (fn == 2) {
                    double sq = 0, qa = 0, qb = 0, V = 0, W = 0;
                    sscanf(r.line, "%*d%*d%*d%lf%lf%lf%le%le", &sq, &qa, &qb, &V, &W);
                    // sigma, epsilon -> C6, C12 as force.c:1783-1786
                    const double sig_6 = pow(V, 6.0), eps_4 = 4.0 * W;
                    const double c6 = eps_4 * sig_6, c12 = c6 * sig_6;
                    add_term(CAPAC_BT_PAIR_USER, {a, b}, {sq, qa, qb, c6, c12});
                } else {
                    bad("pair function type");
                }
                exclude(m, a, b);
            }
            // angles (file.c:813-864)
            r.expect(names[m] + "_ANGLES");
            sscanf(r.line, "%*s%d", &n);
            for (int k = 0; k < n; ++k) {
                r.next();
                int a = 0, b = 0, c = 0, fn = 0;
                double p0 = 0, p1 = 0, p2 = 0, p3 = 0;
                sscanf(r.line, "%d%d%d%d", &a, &b, &c, &fn);
                if (fn == 1) {
                    sscanf(r.line, "%*d%*d%*d%*d%le%le", &p0, &p1);
                    add_term(CAPAC_BT_ANGLE_HARMONIC, {a, b, c}, {p0, p1});
                } else if (fn == 5) {
                    sscanf(r.line, "%*d%*d%*d%*d%le%le%le%le", &p0, &p1, &p2, &p3);
                    add_term(CAPAC_BT_ANGLE_UB, {a, b, c}, {p0, p1, p2, p3});
                } else {
                    bad("angle function type");
                }
                exclude(m, a, b);
                exclude(m, a, c);
                exclude(m, b, c);
            }
            // dihedrals (file.c:866-928); the periodic form becomes the RB
            // coefficients compute_dihedral_9 derives (force.c:1236-1347)
            r.expect(names[m] + "_DIHEDRALS");
            sscanf(r.line, "%*s%d", &n);
            for (int k = 0; k < n; ++k) {
                r.next();
                int a = 0, b = 0, c = 0, e = 0, fn = 0;
                sscanf(r.line, "%d%d%d%d%d", &a, &b, &c, &e, &fn);
                double cc[6] = {0, 0, 0, 0, 0, 0};
                if (fn == 3) {
                    sscanf(r.line, "%*d%*d%*d%*d%*d%lf%lf%lf%lf%lf%lf", &cc[0], &cc[1], &cc[2], &cc[3], &cc[4],
                           &cc[5]);
                } else if (fn == 1 || fn == 4 || fn == 9) {
                    double phi0 = 0, kphi = 0;
                    int mult = 0;
                    sscanf(r.line, "%*d%*d%*d%*d%*d%lf%lf%d", &phi0, &kphi, &mult);
                    if (capac_dihedral_periodic_to_rb(phi0, kphi, mult, cc) != CAPAC_OK)
                        bad("periodic dihedral (phi0 0 or 180, multiplicity 1 to 4)");
                } else {
                    bad("dihedral function type");
                }
                add_term(CAPAC_BT_DIHEDRAL_RB, {a, b, c, e}, {cc[0], cc[1], cc[2], cc[3], cc[4], cc[5]});
                exclude(m, a, b); exclude(m, a, c); exclude(m, a, e);
                exclude(m, b, c); exclude(m, b, e); exclude(m, c, e);
            }
            d->bt_count[m] = (int)bkind.size() - d->bt_offset[m];
            d->n_bonded_terms += d->bt_count[m] * d->mol_num[m];
            // virtual sites (file.c:931-969)
            r.expect(names[m] + "_VSITES");
            sscanf(r.line, "%*s%d", &n);
            d->vs_offset[m] = (int)(vatoms.size() / 4);
            d->vs_count[m] = n;
            d->n_vsites_total += n * d->mol_num[m];
            for (int k = 0; k < n; ++k) {
                r.next();
                int a = 0, b = 0, c = 0, s = 0, fn = 0;
                double va = 0, vb = 0, vc = 0;
                sscanf(r.line, "%d%d%d%d%d%lf%lf%lf", &a, &b, &c, &s, &fn, &va, &vb, &vc);
                if (fn != 4) bad("virtual_sites function type");
                for (int x : {a, b, c, s}) vatoms.push_back(x);
                for (double v : {va, vb, vc}) vpar.push_back(v);
                exclude(m, s, a); exclude(m, s, b); exclude(m, s, c);
            }
            r.expect(names[m] + "_CSTRS");
            sscanf(r.line, "%*s%d", &n);
            d->cstr_offset[m] = (int)ci.size();
            d->cstr_count[m] = n;
            d->n_cstr_total += n * d->mol_num[m];
            for (int k = 0; k < n; ++k) {
                r.next();
                int a = 0, b = 0;
                double len = 0;
                if (sscanf(r.line, "%d%d%lf", &a, &b, &len) != 3)
                    throw Error(CAPAC_ERR_IO, std::string("bad constraint line: ") + r.line);
                exclude(m, a, b);
                ci.push_back(a);
                cj.push_back(b);
                cr.push_back(len);
            }
        }
        d->bt_kind = alloc_array<int>(bkind.size());
        d->bt_atoms = alloc_array<int>(batoms.size());
        d->bt_par = alloc_array<double>(bpar.size());
        d->vs_atoms = alloc_array<int>(vatoms.size());
        d->vs_par = alloc_array<double>(vpar.size());
        std::copy(bkind.begin(), bkind.end(), d->bt_kind);
        std::copy(batoms.begin(), batoms.end(), d->bt_atoms);
        std::copy(bpar.begin(), bpar.end(), d->bt_par);
        std::copy(vatoms.begin(), vatoms.end(), d->vs_atoms);
        std::copy(vpar.begin(), vpar.end(), d->vs_par);
        d->cstr_i = alloc_array<int>(ci.size());
        d->cstr_j = alloc_array<int>(ci.size());
        d->cstr_r = alloc_array<double>(ci.size());
        for (size_t k = 0; k < ci.size(); ++k) {
            d->cstr_i[k] = ci[k];
            d->cstr_j[k] = cj[k];
            d->cstr_r[k] = cr[k];
        }

        r.expect("MM_METAL");
        sscanf(r.line, "%*s%d%d", &d->metal_min, &d->metal_max);
        d->n_metal = (d->metal_min >= 0 && d->metal_max >= d->metal_min)
                         ? d->metal_max - d->metal_min + 1 : 0;
        r.expect("QSC_METAL");
        sscanf(r.line, "%*s%d%d%lf%lf%lf", &d->qsc_n, &d->qsc_m, &d->qsc_eps, &d->qsc_c, &d->qsc_a);
        r.expect("CPFF_METAL");
        sscanf(r.line, "%*s%lf%lf", &d->cpff_polar, &d->cpff_capac);
        r.expect("NANOPARTICLES");
        sscanf(r.line, "%*s%d", &d->n_nps);
        if (d->n_nps < 0) throw Error(CAPAC_ERR_IO, "negative NANOPARTICLES");
        d->np_start = alloc_array<int>(d->n_nps);
        d->np_end = alloc_array<int>(d->n_nps);
        d->np_charge = alloc_array<double>(d->n_nps);
        for (int k = 0; k < d->n_nps; ++k) {
            r.next();
            sscanf(r.line, "%*s%d%d%lf", &d->np_start[k], &d->np_end[k], &d->np_charge[k]);
        }
        fclose(f);
        f = nullptr;

        // assign_indices (file.c:1031-1099)
        int n_atoms = 0, n_mols = 0;
        for (int m = 0; m < T; ++m) {
            n_atoms += d->mol_num[m] * d->mol_atoms[m];
            n_mols += d->mol_num[m];
        }
        d->n_atoms = n_atoms;
        d->n_mols = n_mols;
        d->atom_type = alloc_array<int>(n_atoms);
        d->mol_id = alloc_array<int>(n_atoms);
        d->mol_type = alloc_array<int>(n_atoms);
        d->atom_in_mol = alloc_array<int>(n_atoms);
        d->is_metal = alloc_array<unsigned char>(n_atoms);
        d->charge = alloc_array<double>(n_atoms);
        d->mass = alloc_array<double>(n_atoms);
        d->inv_mass = alloc_array<double>(n_atoms);
        d->mol_first = alloc_array<int>(n_mols);
        d->mol_last = alloc_array<int>(n_mols);
        int i = 0, im = 0;
        for (int m = 0; m < T; ++m) {
            for (int k = 0; k < d->mol_num[m]; ++k) {
                d->mol_first[im] = i;
                for (int a = 0; a < d->mol_atoms[m]; ++a) {
                    d->mol_type[i] = m;
                    d->atom_in_mol[i] = a;
                    d->mol_id[i] = im;
                    d->charge[i] = q[m][a];
                    d->mass[i] = mass[m][a];
                    d->atom_type[i] = type[m][a];
                    d->inv_mass[i] = mass[m][a] > 0.0 ? 1.0 / mass[m][a] : 0.0;
                    if (type[m][a] < 0 || type[m][a] >= NT)
                        throw Error(CAPAC_ERR_IO, "atom type out of range in " + names[m]);
                    ++i;
                }
                d->mol_last[im] = i - 1;
                ++im;
            }
        }
        if (d->n_metal > 0) {
            if (d->metal_max >= n_atoms)
                throw Error(CAPAC_ERR_IO, "MM_METAL range beyond the last atom");
            for (int k = d->metal_min; k <= d->metal_max; ++k) d->is_metal[k] = 1;
        }
    } catch (...) {
        if (f) fclose(f);
        throw;
    }
}

void read_gro(const char *path, capac_desc *d)
{
    FILE *f = fopen(path, "r");
    if (!f) throw Error(CAPAC_ERR_IO, std::string("cannot open ") + path);
    char line[kLine], w1[kLine], w2[kLine], w3[kLine];
    int step = 0, n = 0;
    d->vq0 = 0.0;
    d->vp = 0.0;
    if (fgets(line, kLine, f))  // title: "step N vQ x vP y" (file.c:156-160)
        sscanf(line, "%255s%d%255s%lf%255s%lf", w1, &step, w2, &d->vq0, w3, &d->vp);
    if (!fgets(line, kLine, f) || sscanf(line, "%d", &n) != 1) {
        fclose(f);
        throw Error(CAPAC_ERR_IO, std::string("no atom count in ") + path);
    }
    if (n != d->n_atoms) {
        fclose(f);
        throw Error(CAPAC_ERR_IO, "groNAtoms(" + std::to_string(n) + ") not equal to nAtoms(" +
                                      std::to_string(d->n_atoms) + ")");
    }
    d->rx = alloc_array<double>(n); d->ry = alloc_array<double>(n); d->rz = alloc_array<double>(n);
    d->vx = alloc_array<double>(n); d->vy = alloc_array<double>(n); d->vz = alloc_array<double>(n);
    for (int i = 0; i < n; ++i) {
        if (!fgets(line, kLine, f)) {
            fclose(f);
            throw Error(CAPAC_ERR_IO, std::string("truncated atom list in ") + path);
        }
        // columns 0-19 hold residue id/name, atom name and number; numbers
        // start at column 20 in free format (file.c:181-190)
        if (strlen(line) <= 20 ||
            sscanf(line + 20, "%lf%lf%lf%lf%lf%lf", &d->rx[i], &d->ry[i], &d->rz[i], &d->vx[i],
                   &d->vy[i], &d->vz[i]) < 3) {
            fclose(f);
            throw Error(CAPAC_ERR_IO, std::string("bad atom line in ") + path + ": " + line);
        }
    }
    if (!fgets(line, kLine, f) || sscanf(line, "%lf%lf%lf", &d->box[0], &d->box[1], &d->box[2]) != 3) {
        fclose(f);
        throw Error(CAPAC_ERR_IO, std::string("no box line in ") + path);
    }
    fclose(f);
}

}  // namespace

void derive(const capac_desc *d, capac_consts *c)
{
    memset(c, 0, sizeof *c);
    const double rc = d->r_cut;
    c->r_cut2 = rc * rc;
    c->w_a2_sqrtpi = d->w_alpha * 2.0 * kInvSqrtPi;
    c->w_const = erfc(d->w_alpha * rc) / c->r_cut2 +
                 c->w_a2_sqrtpi * exp(-d->w_alpha * d->w_alpha * c->r_cut2) / rc;
    c->w_erfc_arcut = erfc(d->w_alpha * rc) / rc;
    c->inv_rc12 = 1.0 / pow(rc, 12.0);
    c->inv_rc6 = 1.0 / pow(rc, 6.0);
    if (d->n_metal > 0) {
        c->inv_polar = 1.0 / d->cpff_polar;
        c->inv_capac = 1.0 / d->cpff_capac;
        const double rq = sqrt(2.0 / kPi) * d->cpff_capac;
        const double rp = pow(sqrt(2.0 / kPi) * d->cpff_polar / 3.0, 1.0 / 3.0);
        c->inv_r_qq = 1.0 / sqrt(rq * rq + rq * rq);
        c->inv_r_pq = 1.0 / sqrt(rp * rp + rq * rq);
        c->inv_r_pp = 1.0 / sqrt(rp * rp + rp * rp);
    }
    c->ndf = 3 * (d->n_atoms - d->n_vsites_total) - 3 - d->n_cstr_total;
    c->kT = kBoltz * d->ref_temp;
    c->q_mass = (double)c->ndf * c->kT * d->tau_temp * d->tau_temp;
    c->dt_2 = 0.5 * d->dt;
    c->n_mat = d->n_metal * 4 + d->n_nps;
}

void desc_free(capac_desc *d)
{
    if (!d) return;
    void *arrays[] = {d->mol_num, d->mol_atoms, d->nb_funct, d->nb_c6, d->nb_c12, d->nb_a, d->nb_b,
                      d->excl_offset, d->excl, d->cstr_offset, d->cstr_count, d->cstr_i, d->cstr_j,
                      d->cstr_r, d->np_start, d->np_end, d->np_charge, d->atom_type, d->mol_id,
                      d->mol_type, d->atom_in_mol, d->is_metal, d->charge, d->mass, d->inv_mass,
                      d->mol_first, d->mol_last, d->rx, d->ry, d->rz, d->vx, d->vy, d->vz,
                      d->bt_offset, d->bt_count, d->bt_kind, d->bt_atoms, d->bt_par, d->vs_offset,
                      d->vs_count, d->vs_atoms, d->vs_par};
    for (void *p : arrays) free(p);
    free(d);
}

capac_desc *desc_load(const char *gro, const char *par, const char *mds)
{
    capac_desc *d = static_cast<capac_desc *>(calloc(1, sizeof(capac_desc)));
    if (!d) throw Error(CAPAC_ERR_INVALID, "out of host memory");
    try {
        read_mdset(mds, d);
        read_param(par, d);
        read_gro(gro, d);
    } catch (...) {
        desc_free(d);
        throw;
    }
    return d;
}

}  // namespace capac

extern "C" {

int capac_desc_load(const char *gro_path, const char *param_path, const char *mdset_path,
                    capac_desc **out)
{
    return capac::guard([&] {
        if (!gro_path || !param_path || !mdset_path || !out)
            throw capac::Error(CAPAC_ERR_INVALID, "null argument");
        *out = capac::desc_load(gro_path, param_path, mdset_path);
    });
}

void capac_desc_free(capac_desc *d) { capac::desc_free(d); }

int capac_dihedral_periodic_to_rb(double phi0, double kphi, int n, double c[6])
{
    if (!c) return CAPAC_ERR_INVALID;
    for (int k = 0; k < 6; ++k) c[k] = 0.0;
    const bool zero = phi0 == 0.0, pi = phi0 == 180.0;
    if (!zero && !pi) return CAPAC_ERR_UNSUPPORTED;
    if (n == 1) {
        c[0] = kphi;
        c[1] = zero ? kphi : kphi * (-1.0);
    } else if (n == 2) {
        if (zero) {
            c[2] = kphi * 2.0;
        } else {
            c[0] = kphi * 2.0;
            c[2] = kphi * (-2.0);
        }
    } else if (n == 3) {
        c[0] = kphi;
        c[1] = zero ? kphi * (-3.0) : kphi * 3.0;
        c[3] = zero ? kphi * 4.0 : kphi * (-4.0);
    } else if (n == 4) {
        if (zero) {
            c[0] = kphi * 2.0;
            c[2] = kphi * (-8.0);
            c[4] = kphi * 8.0;
        } else {
            c[2] = kphi * 8.0;
            c[4] = kphi * (-8.0);
        }
    } else {
        return CAPAC_ERR_UNSUPPORTED;
    }
    c[1] *= -1.0;
    c[3] *= -1.0;
    c[5] *= -1.0;
    return CAPAC_OK;
}

int capac_desc_derive(const capac_desc *d, capac_consts *out)
{
    return capac::guard([&] {
        if (!d || !out) throw capac::Error(CAPAC_ERR_INVALID, "null argument");
        capac::derive(d, out);
    });
}

int capac_desc_info(const capac_desc *d, int *n_atoms, int *n_mols, int *n_metal, int *n_nps, int *n_mat)
{
    if (!d) return CAPAC_ERR_INVALID;
    if (n_atoms) *n_atoms = d->n_atoms;
    if (n_mols) *n_mols = d->n_mols;
    if (n_metal) *n_metal = d->n_metal;
    if (n_nps) *n_nps = d->n_nps;
    if (n_mat) *n_mat = d->n_metal * 4 + d->n_nps;
    return CAPAC_OK;
}

int capac_desc_get(const capac_desc *d, const char *name, double *out)
{
    if (!d || !name || !out) return CAPAC_ERR_INVALID;
    const int n = d->n_atoms;
    struct { const char *nm; const double *src; int cnt; } tab[] = {
        {"rx", d->rx, n}, {"ry", d->ry, n}, {"rz", d->rz, n}, {"vx", d->vx, n},
        {"vy", d->vy, n}, {"vz", d->vz, n}, {"charge", d->charge, n}, {"mass", d->mass, n},
        {"box", d->box, 3},
    };
    for (auto &e : tab) {
        if (0 == strcmp(name, e.nm)) {
            memcpy(out, e.src, sizeof(double) * e.cnt);
            return e.cnt;
        }
    }
    if (0 == strcmp(name, "is_metal")) {
        for (int i = 0; i < n; ++i) out[i] = d->is_metal[i];
        return n;
    }
    if (0 == strcmp(name, "atom_type")) {
        for (int i = 0; i < n; ++i) out[i] = d->atom_type[i];
        return n;
    }
    if (0 == strcmp(name, "bonded_counts")) {  // terms in the system, virtual sites, constraints
        out[0] = d->n_bonded_terms;
        out[1] = d->n_vsites_total;
        out[2] = d->n_cstr_total;
        return 3;
    }
    if (0 == strcmp(name, "bonded_kinds")) {  // terms of each CAPAC_BT_* kind (1..7) in the system
        for (int k = 0; k < 8; ++k) out[k] = 0.0;
        if (d->bt_offset)
            for (int m = 0; m < d->mol_types; ++m)
                for (int t = d->bt_offset[m]; t < d->bt_offset[m] + d->bt_count[m]; ++t)
                    if (d->bt_kind[t] >= 0 && d->bt_kind[t] < 8) out[d->bt_kind[t]] += d->mol_num[m];
        return 8;
    }
    return CAPAC_ERR_INVALID;
}

}  // extern "C"
