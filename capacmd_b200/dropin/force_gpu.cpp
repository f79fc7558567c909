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
// vectors come back (force.h:100-103 semantics; potential[0] is the caller's).
// time_used[my_id] receives the call's device phase times in the reference's
// slots (seconds, added as force.c:2134-2316 adds its own): 1 Sutton-Chen
// (density and force together), 4 nonbonded, 5 CPIM matrix, 6 CPIM vector,
// 7 CPIM solve, 8 CPIM force, 10 neighbour-list upkeep, and 11 the rest of
// the call's wall time (host<->device copies and host work), so the
// driver's own sum_time_used/analyze_time_used report shows where the GPU
// call spent its time.  A failing call prints the library's message and
// exits, as the reference does on its own errors.
//
// Compiled as C++ against the reference's headers (typedef.h pulls in
// std::vector): the `dropin` target of oracle/Makefile links it and
// shim_desc.cpp with the reference's objects into oracle/_ref/mpi-main-gpu.
#include <chrono>

#include "shim_desc.h"

// build_vsites is defined in the reference's force.c (force.c:1582), which the
// drop-in binary links; it has no header declaration there
void build_vsites(int mol_start, int mol_end, Mol_Info *mol_info, Atom_Info *atom_info, int *nVSites,
                  int **vsite_funct, VSite_4 **vsite_4, double *rx, double *ry, double *rz, double *box);

// The driver's mpi_force(Task*, Topol*, Atom_Info*, Mol_Info*, RunSet*, Metal*,
// System*, Bicgstab*, int, int, double**), redirected here by --wrap.
extern "C" void __wrap__Z9mpi_forceP4TaskP5TopolP9Atom_InfoP8Mol_InfoP6RunSetP5MetalP6SystemP8BicgstabiiPPd(
    Task *, Topol *t, Atom_Info *ai, Mol_Info *mi, RunSet *rs, Metal *m, System *s, Bicgstab *, int my_id, int,
    double **time_used)
{
    const auto t0 = std::chrono::steady_clock::now();
    capac_ctx *ctx = shim_context(t, ai, mi, rs, m, s);
    // the reference's mpi_force places the virtual sites in the caller's
    // positions first (force.c:2124-2129); the driver's own build_vsites does
    // the same here, and the GPU rebuilds them identically
    if (shim_desc()->n_vsites_total > 0)
        build_vsites(0, t->n_mols - 1, mi, ai, t->n_vsites, t->vsite_funct, t->vsite_4, s->rx, s->ry, s->rz, s->box);
    double vir[9];
    // the driver allocates the CPIM vectors whenever there are metal atoms
    // (mpi-main.c:576-591) and inv_sqrt_dens with them (mpi-main.c:290)
    const bool metal = m->num > 0 && m->vec_pq != nullptr;
    if (capac_mpi_force(ctx, s->rx, s->ry, s->rz, s->fx, s->fy, s->fz, s->potential, vir,
                        metal ? m->vec_pq : nullptr, metal ? m->vec_ext : nullptr, metal ? m->diag_relay : nullptr,
                        metal ? m->inv_sqrt_dens : nullptr))
        shim_fail("mpi_force");
    for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c) s->virial[a][c] = vir[3 * a + c];
    double ms[15];
    if (time_used && time_used[my_id] && capac_phase_times(ctx, ms) == CAPAC_OK) {
        const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        static const int slots[] = {1, 4, 5, 6, 7, 8, 10};
        for (int k : slots) time_used[my_id][k] += 1e-3 * ms[k];
        const double rest = wall - 1e-3 * ms[0];
        if (rest > 0.0) time_used[my_id][11] += rest;
    }
}
