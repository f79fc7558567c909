// Resident driver: the reference's command line, input files and output
// files, with the whole run on one GPU (mpi-main.c main loop).
//
//   capacmd-gpu -gro init.gro -par param.txt -mds mdset.txt
//               [-prec fp64|mixed] [-restart file] [-checkpoint file]
//
// run_type md: velocity Verlet with RATTLE and the Nose-Hoover chain as
// capac_md_steps runs them; every save_step steps the reference's status
// line and a traj.dat frame, every 10 save_step a traj.gro frame and a
// vec_pq.txt record (mpi-main.c:983-1003).  run_type em / cg: capac_em_step
// per step with a status line and a frame of each file per step
// (mpi-main.c:700-865).  The output formats are the reference's
// (file.c:212-278).  The state crosses to the host only at output.
// -restart loads a checkpoint after the start-up force call; -checkpoint
// writes one at the end (capac_checkpoint_save).
#include <sys/time.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "capacmd.h"

namespace {

void fail(const char *what)
{
    printf("Error: %s: %s\n", what, capac_last_error());
    exit(1);
}

// Residue numbers and names, atom names of the input .gro (read_gro, file.c:138-203).
struct GroNames {
    std::vector<int> res_id;
    std::vector<std::string> res_name, atom_name;
};

std::string field(const char *line, size_t from, size_t len)
{
    const size_t n = strlen(line);
    if (from >= n) return "";
    std::string s(line + from, std::min(len, n - from));
    const size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? "" : s.substr(a, b - a + 1);
}

GroNames read_names(const char *path, int n_atoms)
{
    GroNames g;
    FILE *f = fopen(path, "r");
    if (!f) {
        printf("Cannot open %s\n", path);
        exit(1);
    }
    char line[512];
    if (!fgets(line, sizeof line, f) || !fgets(line, sizeof line, f)) {
        printf("Cannot read %s\n", path);
        exit(1);
    }
    for (int i = 0; i < n_atoms; ++i) {
        if (!fgets(line, sizeof line, f)) {
            printf("Cannot read atom %d of %s\n", i + 1, path);
            exit(1);
        }
        g.res_id.push_back(atoi(field(line, 0, 5).c_str()));
        g.res_name.push_back(field(line, 5, 5));
        g.atom_name.push_back(field(line, 10, 5));
    }
    fclose(f);
    return g;
}

struct Host {
    int N, M, n_nps, n_mat;
    std::vector<double> rx, ry, rz, vx, vy, vz, pq, box, vq, pot, thermo, fm;
};

void fetch(capac_ctx *ctx, Host &h, bool velocities, bool pq)
{
    if (capac_get(ctx, "rx", h.rx.data()) < 0 || capac_get(ctx, "ry", h.ry.data()) < 0 ||
        capac_get(ctx, "rz", h.rz.data()) < 0 || capac_get(ctx, "box", h.box.data()) < 0 ||
        capac_get(ctx, "potential", h.pot.data()) < 0 || capac_get(ctx, "thermo", h.thermo.data()) < 0 ||
        capac_get(ctx, "fmax_rms", h.fm.data()) < 0 || capac_get(ctx, "vQ", h.vq.data()) < 0)
        fail("state transfer");
    if (velocities && (capac_get(ctx, "vx", h.vx.data()) < 0 || capac_get(ctx, "vy", h.vy.data()) < 0 ||
                       capac_get(ctx, "vz", h.vz.data()) < 0))
        fail("state transfer");
    if (pq && h.M > 0 && capac_get(ctx, "vec_pq", h.pq.data()) < 0) fail("state transfer");
}

// write_gro, file.c:212-229
void write_gro(FILE *f, const Host &h, const GroNames &g, int step, double vq0, double vp)
{
    fprintf(f, "step  %d  vQ  %lf  vP  %lf\n", step, vq0, vp);
    fprintf(f, "%5d\n", h.N);
    for (int i = 0; i < h.N; ++i)
        fprintf(f, "%5d%-5s%5s%5d%10.5f%10.5f%10.5f%10.6f%10.6f%10.6f\n", g.res_id[i], g.res_name[i].c_str(),
                g.atom_name[i].c_str(), i + 1, h.rx[i], h.ry[i], h.rz[i], h.vx[i], h.vy[i], h.vz[i]);
    fprintf(f, "%10.5f%10.5f%10.5f\n", h.box[0], h.box[1], h.box[2]);
}

// write_vec_pq, file.c:238-262
void write_vec_pq(FILE *f, const Host &h, int step)
{
    fprintf(f, "step %d", step);
    fprintf(f, "  lambda");
    for (int k = 0; k < h.n_nps; ++k) fprintf(f, " %.10f", h.pq[4 * h.M + k]);
    fprintf(f, "\n%5d\n", h.M);
    for (int i = 0; i < h.M; ++i)
        fprintf(f, "%15.8f%15.8f%15.8f%15.8f\n", h.pq[3 * i], h.pq[3 * i + 1], h.pq[3 * i + 2], h.pq[3 * h.M + i]);
}

// write_binary, file.c:270-278
void write_binary(FILE *f, const Host &h, int step)
{
    bool ok = fwrite(&h.N, sizeof(int), 1, f) == 1 && fwrite(&step, sizeof(int), 1, f) == 1 &&
              fwrite(h.box.data(), sizeof(double), 3, f) == 3;
    ok = ok && fwrite(h.rx.data(), sizeof(double), h.N, f) == (size_t)h.N &&
         fwrite(h.ry.data(), sizeof(double), h.N, f) == (size_t)h.N &&
         fwrite(h.rz.data(), sizeof(double), h.N, f) == (size_t)h.N;
    if (!ok) {
        printf("Cannot write to traj.dat!\n");
        exit(1);
    }
}

// print_potential, force.c:337-354
void print_potential(const double *p)
{
    printf("    Potential energies: \n");
    printf(" %15.6e   total energy                         \n", p[0]);
    printf(" %15.6e   metal quantum Sutton-Chen energy     \n", p[1]);
    printf(" %15.6e   non-metal bond stretching energy     \n", p[2]);
    printf(" %15.6e   non-metal angle bending energy       \n", p[3]);
    printf(" %15.6e   non-metal torsional energy           \n", p[4]);
    printf(" %15.6e   Long range Coulomb                   \n", p[6]);
    printf(" %15.6e   Coulomb energy (including 1-4)       \n", p[7]);
    printf(" %15.6e   vdW energy (including 1-4)           \n", p[8]);
    printf(" %15.6e   CPIM metal charge - non-metal charge \n", p[10]);
    printf(" %15.6e   CPIM metal dipole - non-metal charge \n", p[11]);
    printf(" %15.6e   CPIM metal charge - metal charge     \n", p[12]);
    printf(" %15.6e   CPIM metal charge - metal dipole     \n", p[13]);
    printf(" %15.6e   CPIM metal dipole - metal dipole     \n", p[14]);
    printf("\n");
}

FILE *open_out(const char *name, const char *mode)
{
    FILE *f = fopen(name, mode);
    if (!f) {
        printf("Cannot write to %s!\n", name);
        exit(1);
    }
    return f;
}

double now()
{
    timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec + tv.tv_usec * 1.0e-6;
}

}  // namespace

int main(int argc, char **argv)
{
    const char *gro = nullptr, *par = nullptr, *mds = nullptr, *restart = nullptr, *ckpt = nullptr;
    int precision = CAPAC_PREC_FP64;
    for (int a = 1; a + 1 < argc; a += 2) {
        const std::string k = argv[a];
        if (k == "-gro") gro = argv[a + 1];
        else if (k == "-par") par = argv[a + 1];
        else if (k == "-mds") mds = argv[a + 1];
        else if (k == "-restart") restart = argv[a + 1];
        else if (k == "-checkpoint") ckpt = argv[a + 1];
        else if (k == "-prec") precision = std::string(argv[a + 1]) == "mixed" ? CAPAC_PREC_MIXED : CAPAC_PREC_FP64;
        else {
            printf("Unknown option %s\n", argv[a]);
            return 1;
        }
    }
    if (!gro || !par || !mds) {
        printf("Usage: %s -gro init.gro -par param.txt -mds mdset.txt [-prec fp64|mixed] "
               "[-restart file] [-checkpoint file]\n", argv[0]);
        return 1;
    }
    const double t0 = now();
    capac_desc *d = nullptr;
    if (capac_desc_load(gro, par, mds, &d)) fail("reading the input");
    capac_options o;
    capac_options_default(&o);
    o.precision = precision;
    capac_ctx *ctx = nullptr;
    if (capac_create(d, &o, &ctx)) fail("creating the GPU context");
    const GroNames names = read_names(gro, d->n_atoms);

    int n_atoms, n_mols, n_metal, n_nps, n_mat;
    capac_desc_info(d, &n_atoms, &n_mols, &n_metal, &n_nps, &n_mat);
    Host h;
    h.N = n_atoms;
    h.M = n_metal;
    h.n_nps = n_nps;
    h.n_mat = n_mat;
    for (auto *v : {&h.rx, &h.ry, &h.rz, &h.vx, &h.vy, &h.vz}) v->assign(n_atoms, 0.0);
    h.pq.assign(n_mat > 0 ? n_mat : 1, 0.0);
    h.box.assign(6, 0.0);
    h.vq.assign(16, 0.0);
    h.pot.assign(15, 0.0);
    h.thermo.assign(4, 0.0);
    h.fm.assign(2, 0.0);

    printf("    %d atoms, %d molecules, %d metal atoms, %d nanoparticles; GPU %s path\n", n_atoms, n_mols, n_metal,
           n_nps, precision == CAPAC_PREC_MIXED ? "mixed-precision" : "FP64");
    // start-up (mpi-main.c:614-676)
    if (capac_md_init(ctx)) fail("first force evaluation");
    if (restart && capac_checkpoint_load(ctx, restart)) fail("loading the checkpoint");
    const bool em = d->run_type == CAPAC_RUN_EM || d->run_type == CAPAC_RUN_CG;
    double vp = em ? 0.0 : d->vp;
    FILE *fgro = open_out("traj.gro", "w"), *fdat = open_out("traj.dat", "wb");
    FILE *fpq = open_out("vec_pq.txt", "w");
    fetch(ctx, h, true, true);
    write_gro(fgro, h, names, 0, em ? 0.0 : h.vq[0], vp);
    write_binary(fdat, h, 0);
    if (n_metal > 0) write_vec_pq(fpq, h, 0);
    printf("              .---------------- start MD calculation ---------------.\n\n");
    if (em) {
        printf("    Step %-5d Fmax=%10.3e  E=%15.8e\n", 0, h.fm[0], h.pot[0]);
        if (capac_em_init(ctx)) fail("starting the minimisation");
        for (int step = 1; step <= d->em_steps; ++step) {
            capac_em_status st;
            if (capac_em_step(ctx, &st)) fail("minimisation step");
            printf("    Step %-5d Fmax=%10.3e  E=%15.8e\n", step, st.f_max, st.energy);
            fetch(ctx, h, true, true);
            write_gro(fgro, h, names, step, 0.0, 0.0);
            write_binary(fdat, h, step);
            if (n_metal > 0) write_vec_pq(fpq, h, step);
            if (st.converged) {
                printf("\n    F_max   (%13.6e) smaller than %e\n", st.f_max, d->em_tol);
                printf("    F_rms   (%13.6e) smaller than %e\n", st.f_rms, d->em_tol * 0.5);
                printf("    delta_E (%13.6e) smaller than %e\n\n", st.delta_pot, d->em_tol * 0.1);
                printf("    ===========  Optimization converged ============\n");
                break;
            }
        }
    } else {
        printf("  %10.3f  Fmax=%.2e  E=%.6e  T=%.3e\n", 0.0, h.fm[0], h.pot[0], h.thermo[1]);
        long step = 0;
        capac_stats stats;
        if (capac_get_stats(ctx, &stats) == 0) step = stats.md_step;
        const int save = d->n_save > 0 ? d->n_save : 1;
        while (step < d->n_steps) {
            const long next = std::min<long>(d->n_steps, (step / save + 1) * save);
            if (capac_md_steps(ctx, (int)(next - step))) fail("MD steps");
            step = next;
            if (step % save != 0) continue;
            const bool frame = step % (10L * save) == 0;
            fetch(ctx, h, frame, frame);
            printf("  %10.3f  Fmax=%.2e  E=%.6e  T=%.3e (%.1f)\n", d->dt * step, h.fm[0], h.pot[0], h.thermo[1],
                   h.thermo[2]);
            write_binary(fdat, h, (int)step);
            if (frame) {
                write_gro(fgro, h, names, (int)step, h.vq[0], vp);
                if (n_metal > 0) write_vec_pq(fpq, h, (int)step);
            }
        }
    }
    fclose(fdat);
    fclose(fpq);
    fclose(fgro);
    if (ckpt && capac_checkpoint_save(ctx, ckpt)) fail("writing the checkpoint");
    if (capac_get(ctx, "potential", h.pot.data()) < 0) fail("state transfer");
    printf("\n\n              .------------- final potential energies --------------.\n\n");
    print_potential(h.pot.data());
    const time_t end_t = time(nullptr);
    printf("    Calculation ended normally at %s", ctime(&end_t));
    printf("    %.3f seconds were used\n\n", now() - t0);
    capac_destroy(ctx);
    capac_desc_free(d);
    return 0;
}
