// Input layer: the three CapacMD input files parsed into a capac_desc.
//
// Formats are the reference's (they have to be, to stay a drop-in):
//   mdset.txt  key/value lines                       (file.c:74-130)
//   .gro       title with "step N vQ x vP y", count,
//              fixed-column atom lines, box line      (file.c:138-203)
//   param.txt  sections in a fixed order              (file.c:286-562, 569-1023)
// followed by the per-atom bookkeeping of assign_indices (file.c:1031-1099) and
// the constants derived in the driver (mpi-main.c:170-203, 315-323, 548-552).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
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
        auto exclude = [&](int m, int a, int b) {
            const int na = d->mol_atoms[m];
            if (a < 0 || b < 0 || a >= na || b >= na)
                throw Error(CAPAC_ERR_IO, "atom index out of range in " + names[m]);
            d->excl[d->excl_offset[m] + a * na + b] = 1;
            d->excl[d->excl_offset[m] + b * na + a] = 1;
        };
        for (int m = 0; m < T; ++m) {
            int n = 0;
            // bonds: every listed bond excludes its pair (file.c:720-770)
            r.expect(names[m] + "_BONDS");
            sscanf(r.line, "%*s%d", &n);
            d->n_bonded_terms += n;
            for (int k = 0; k < n; ++k) {
                r.next();
                int a, b;
                sscanf(r.line, "%d%d", &a, &b);
                exclude(m, a, b);
            }
            r.expect(names[m] + "_PAIRS");
            sscanf(r.line, "%*s%d", &n);
            d->n_bonded_terms += n;
            for (int k = 0; k < n; ++k) {
                r.next();
                int a, b;
                sscanf(r.line, "%d%d", &a, &b);
                exclude(m, a, b);
            }
            r.expect(names[m] + "_ANGLES");
            sscanf(r.line, "%*s%d", &n);
            d->n_bonded_terms += n;
            for (int k = 0; k < n; ++k) {
                r.next();
                int a, b, c;
                sscanf(r.line, "%d%d%d", &a, &b, &c);
                exclude(m, a, b);
                exclude(m, a, c);
                exclude(m, b, c);
            }
            r.expect(names[m] + "_DIHEDRALS");
            sscanf(r.line, "%*s%d", &n);
            d->n_bonded_terms += n;
            for (int k = 0; k < n; ++k) {
                r.next();
                int a, b, c, e;
                sscanf(r.line, "%d%d%d%d", &a, &b, &c, &e);
                exclude(m, a, b); exclude(m, a, c); exclude(m, a, e);
                exclude(m, b, c); exclude(m, b, e); exclude(m, c, e);
            }
            r.expect(names[m] + "_VSITES");
            sscanf(r.line, "%*s%d", &n);
            d->n_vsites_total += n * d->mol_num[m];
            for (int k = 0; k < n; ++k) {
                r.next();
                int a, b, c, s;
                sscanf(r.line, "%d%d%d%d", &a, &b, &c, &s);
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
                      d->mol_first, d->mol_last, d->rx, d->ry, d->rz, d->vx, d->vy, d->vz};
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
    return CAPAC_ERR_INVALID;
}

}  // extern "C"
