// Drop-in CPIM stages and RATTLE for the reference CapacMD driver.
//
// Linked into the reference's own mpi-main with -Wl,--wrap on the mangled
// names of
//   mpi_cpff_vec_ext         (cpff.h:30-33)
//   mpi_cpff_mat_relay_COO   (cpff.h:39-40)
//   mpi_precon_bicg_stab_COO (bicg_stab.h:58-59)
//   mpi_cpff_force           (cpff.h:46-48)
//   rattle_1st, rattle_2nd   (force.h:85-95)
// so the reference's own mpi_force (force.c:2097-2320) still runs its pair
// loop and Sutton-Chen on the host while every CPIM stage and both RATTLE
// half steps run on the GPU.  Each shim leaves the reference's structures
// as the reference function does:
//   * vec_ext: Metal.vec_ext[0 .. n_mat) from the current positions;
//   * mat_relay: Metal.vec_val / vec_row_ind / vec_col_ind in the
//     reference's entry order (rows of metal atom i, for each metal column j
//     the dipole rows with their dipole and charge columns, then the charge
//     row, then after the first column the neutrality couplings; the
//     Lagrange rows last), the vectors overwritten in place and grown only
//     when too short, diag_relay, and the entry count; the off-diagonal
//     values are the GPU's FP64 blocks (equal to the reference's to
//     rounding), the diagonal ones the Metal struct's own constants;
//   * bicgstab: reads that COO matrix, vec_ext and the vec_pq warm start,
//     solves with the reference's rule (rTr < 1e-8 bTb, bicg_stab.c:303) and
//     writes vec_pq; the Bicgstab work vectors are not written;
//   * cpff_force: adds the CPIM forces, energies [9..14] and virial to the
//     System's, for the induced vector it is given;
//   * rattle_1st / rattle_2nd: corrects the positions and velocities (and
//     adds the constraint virial) in place.
// A failure prints the library's message (the reference's own wording for
// RATTLE and BiCGSTAB) and exits, as the reference does.
//
// Compiled as C++ against the reference's headers: the `dropin` target of
// oracle/Makefile links it with shim_desc.cpp and the reference's objects
// into oracle/_ref/mpi-main-cpim.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <new>
#include <vector>

#include "shim_desc.h"

namespace {

capac_ctx *need_context(const char *what)
{
    capac_ctx *c = shim_existing();
    if (!c) {
        printf("GPU %s: called before any call that describes the system\n", what);
        exit(1);
    }
    return c;
}

void set_positions(capac_ctx *c, const System *s, const char *what)
{
    if (capac_set(c, "rx", s->rx) < 0 || capac_set(c, "ry", s->ry) < 0 || capac_set(c, "rz", s->rz) < 0)
        shim_fail(what);
}

// Metal.vec_val / vec_row_ind / vec_col_ind written as cpff.c does: entry k
// overwrites the k-th element, the vectors grow only past their size.
struct CooWriter {
    Metal *m = nullptr;
    long count = 0;
    void put(double e, double thr, long row, long col)
    {
        if (!(fabs(e) > thr)) return;
        if (count >= (long)m->vec_val.size()) {
            m->vec_val.push_back(e);
            m->vec_row_ind.push_back(row);
            m->vec_col_ind.push_back(col);
        } else {
            m->vec_val[count] = e;
            m->vec_row_ind[count] = row;
            m->vec_col_ind[count] = col;
        }
        ++count;
    }
};

constexpr double kThr = 1.0e-15;  // THRSHD_P, THRSHD_M, THRSHD_Q (typedef.h:89-93)

// One line on stderr the first time each shim runs, so a caller can see which
// reference functions the GPU replaced.
void announce(bool &done, const char *what)
{
    if (done) return;
    done = true;
    fprintf(stderr, "capacmd drop-in: %s on the GPU\n", what);
}
bool g_said[6];

}  // namespace

extern "C" void __wrap__Z16mpi_cpff_vec_extP4TaskP5MetalP6RunSetP9Atom_InfoP5TopolP6Systemi(
    Task *, Metal *m, RunSet *rs, Atom_Info *ai, Topol *t, System *s, int)
{
    announce(g_said[0], "mpi_cpff_vec_ext");
    capac_ctx *c = shim_context(t, ai, nullptr, rs, m, s);
    set_positions(c, s, "mpi_cpff_vec_ext");
    if (capac_cpff_vec_ext(c) || capac_get(c, "vec_ext", m->vec_ext) < 0) shim_fail("mpi_cpff_vec_ext");
}

extern "C" void __wrap__Z22mpi_cpff_mat_relay_COOP4TaskP5MetalP6SystemdiiPl(Task *, Metal *m, System *s, double, int,
                                                                            int, long *p_count_nnz)
{
    announce(g_said[1], "mpi_cpff_mat_relay_COO");
    capac_ctx *c = need_context("mpi_cpff_mat_relay_COO");
    // The driver allocates Metal with malloc (mpi-main.c:101) and never
    // constructs its std::vector members; the reference's own push_back works
    // only while that memory happens to be zero, which a process that has
    // loaded a large runtime before main does not guarantee.  The first call
    // constructs them (empty); later calls reuse them as cpff.c does.
    static bool constructed = false;
    if (!constructed) {
        new (&m->vec_val) std::vector<double>();
        new (&m->vec_row_ind) std::vector<long int>();
        new (&m->vec_col_ind) std::vector<long int>();
        constructed = true;
    }
    set_positions(c, s, "mpi_cpff_mat_relay_COO");
    const int M = m->num, nps = m->n_NPs;
    const long nM3 = 3L * M;
    const int chunk = std::max(1, std::min(M, (int)((64L << 20) / (8L * 16 * std::max(M, 1)))));
    std::vector<double> blk((size_t)chunk * M * 16);
    CooWriter w;
    w.m = m;
    for (int i0 = 0; i0 < M; i0 += chunk) {
        const int rows = std::min(chunk, M - i0);
        if (capac_cpim_blocks(c, i0, rows, blk.data())) shim_fail("mpi_cpff_mat_relay_COO");
        for (int i = i0; i < i0 + rows; ++i) {
            const int i_metal = m->min + i;
            for (int j = 0; j < M; ++j) {
                const double *B = &blk[((size_t)(i - i0) * M + j) * 16];
                for (int a = 0; a < 3; ++a) {
                    const long irow = 3L * i + a;
                    for (int b = 0; b < 3; ++b) {
                        if (j == i) {
                            if (b == a) {
                                m->diag_relay[irow] = m->inv_polar;
                                w.put(m->inv_polar, kThr, irow, 3L * j + b);
                            }
                        } else {
                            w.put(B[4 * a + b], kThr, irow, 3L * j + b);
                        }
                    }
                    if (j != i) w.put(B[4 * a + 3], kThr, irow, nM3 + j);
                }
                const long irow = nM3 + i;
                if (j != i)
                    for (int b = 0; b < 3; ++b) w.put(B[12 + b], kThr, irow, 3L * j + b);
                if (j == i) {
                    m->diag_relay[irow] = -m->inv_capac;
                    w.put(-m->inv_capac, kThr, irow, nM3 + j);
                } else {
                    w.put(B[15], kThr, irow, nM3 + j);
                }
                if (j == 0)
                    for (int k = 0; k < nps; ++k)
                        if (i_metal >= m->start_NP[k] && i_metal <= m->end_NP[k]) w.put(1.0, kThr, irow, 4L * M + k);
            }
        }
    }
    for (int k = 0; k < nps; ++k) {
        m->diag_relay[4L * M + k] = 1.0;
        for (int i = 0; i < M; ++i) {
            const int i_metal = m->min + i;
            if (i_metal >= m->start_NP[k] && i_metal <= m->end_NP[k]) w.put(1.0, kThr, 4L * M + k, nM3 + i);
        }
    }
    *p_count_nnz = w.count;
}

extern "C" void __wrap__Z24mpi_precon_bicg_stab_COOP4TaskP5MetaliiilP8Bicgstab(Task *, Metal *m, int, int, int,
                                                                              long count_nnz, Bicgstab *)
{
    announce(g_said[2], "mpi_precon_bicg_stab_COO");
    capac_ctx *c = need_context("mpi_precon_bicg_stab_COO");
    if (capac_cpim_set_coo(c, count_nnz, m->vec_val.data(), m->vec_row_ind.data(), m->vec_col_ind.data()) ||
        capac_set(c, "vec_ext", m->vec_ext) < 0 || capac_set(c, "vec_pq", m->vec_pq) < 0)
        shim_fail("mpi_precon_bicg_stab_COO");
    int it = 0;
    if (capac_bicgstab(c, &it)) {
        printf("%s\n", capac_last_error());
        exit(1);
    }
    if (capac_get(c, "vec_pq", m->vec_pq) < 0) shim_fail("mpi_precon_bicg_stab_COO");
}

extern "C" void __wrap__Z14mpi_cpff_forceP4TaskP5MetalP6RunSetP6SystemPdiP9Atom_Infoi(Task *, Metal *, RunSet *,
                                                                                    System *s, double *vec_pq,
                                                                                    int n_atoms, Atom_Info *, int)
{
    announce(g_said[3], "mpi_cpff_force");
    capac_ctx *c = need_context("mpi_cpff_force");
    set_positions(c, s, "mpi_cpff_force");
    std::vector<double> zero((size_t)n_atoms, 0.0), f((size_t)n_atoms);
    const double z15[15] = {0.0}, z9[9] = {0.0};
    if (capac_set(c, "vec_pq", vec_pq) < 0 || capac_set(c, "fx", zero.data()) < 0 ||
        capac_set(c, "fy", zero.data()) < 0 || capac_set(c, "fz", zero.data()) < 0 ||
        capac_set(c, "potential", z15) < 0 || capac_set(c, "virial", z9) < 0 || capac_cpff_force(c))
        shim_fail("mpi_cpff_force");
    const char *names[3] = {"fx", "fy", "fz"};
    double *dst[3] = {s->fx, s->fy, s->fz};
    for (int a = 0; a < 3; ++a) {
        if (capac_get(c, names[a], f.data()) < 0) shim_fail("mpi_cpff_force");
        for (int i = 0; i < n_atoms; ++i) dst[a][i] += f[i];
    }
    double pot[15], vir[9];
    if (capac_get(c, "potential", pot) < 0 || capac_get(c, "virial", vir) < 0) shim_fail("mpi_cpff_force");
    for (int k = 0; k < 15; ++k) s->potential[k] += pot[k];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) s->virial[a][b] += vir[3 * a + b];
}

extern "C" void __wrap__Z10rattle_1stdP8Mol_InfoP9Atom_InfoP5TopolP6System(double dt, Mol_Info *mi, Atom_Info *ai,
                                                                          Topol *t, System *s)
{
    announce(g_said[4], "rattle_1st");
    capac_ctx *c = shim_context(t, ai, mi, nullptr, nullptr, s);
    if (capac_rattle(c, 1, dt, s->rx, s->ry, s->rz, s->old_rx, s->old_ry, s->old_rz, s->vx, s->vy, s->vz, nullptr))
        shim_fail("rattle_1st");
}

extern "C" void __wrap__Z10rattle_2nddP8Mol_InfoP9Atom_InfoP5TopolP6System(double dt, Mol_Info *mi, Atom_Info *ai,
                                                                          Topol *t, System *s)
{
    announce(g_said[5], "rattle_2nd");
    capac_ctx *c = shim_context(t, ai, mi, nullptr, nullptr, s);
    double w[9] = {0.0};
    if (capac_rattle(c, 2, dt, s->rx, s->ry, s->rz, nullptr, nullptr, nullptr, s->vx, s->vy, s->vz, w))
        shim_fail("rattle_2nd");
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) s->virial[a][b] += w[3 * a + b];
}
