/*
 * capacmd.h -- C ABI of the B200 (sm_100a) implementation of CapacMD's
 * per-timestep force-and-solve path.
 *
 * Every entry point takes plain pointers and sizes and returns an int status
 * (CAPAC_OK or a negative CAPAC_ERR_*); capac_last_error() gives the message
 * of the most recent failure on the calling thread.  The reference reports the
 * same failures with printf + exit(1); a caller that wants that behaviour
 * checks the status and exits.
 *
 * Reference interfaces replaced (paths inside the CapacMD project):
 *   system input      read_settings/read_gro/read_param_1/2/assign_indices
 *                     (file.h:30-80, file.c:74-203, file.c:286-1099)
 *                     -> capac_desc_load
 *   derived constants mpi-main.c:170-203, 315-323, 548-552 -> capac_desc_derive
 *   one force call    mpi_force (force.h:100-103)
 *                     -> capac_force (device-resident state) and
 *                        capac_mpi_force (host buffers in and out)
 *   CPIM stages       mpi_cpff_vec_ext (cpff.h:30-33) -> capac_cpff_vec_ext
 *                     mpi_cpff_mat_relay_COO (cpff.h:39-40) -> capac_cpff_mat_relay
 *                     mpi_precon_bicg_stab_COO (bicg_stab.h:58-59) -> capac_bicgstab
 *                     mpi_cpff_force (cpff.h:46-48) -> capac_cpff_force
 *   integrator        rattle_1st/rattle_2nd (force.h:85-95), apply_pbc
 *                     (force.h:37-38), get_fmax_rms (force.h:79),
 *                     kinetic_energy/remove_comm/nose_hoover_chain
 *                     (thermostat.h:31-45), MD loop (mpi-main.c:874-1013)
 *                     -> capac_md_steps and the per-stage entry points below.
 *
 * Units follow the reference: nm, ps, kJ/mol, e, amu; the CPIM vector is in
 * atomic units (e*Bohr for dipoles, e for charges).  The CPIM vector layout is
 * the reference's: [0,3M) dipoles x,y,z per metal atom, [3M,4M) charges,
 * [4M,4M+n_NPs) Lagrange multipliers (mpi-main.c:572-591).
 */
#ifndef CAPACMD_H
#define CAPACMD_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define CAPAC_OK 0
#define CAPAC_ERR_INVALID (-1)        /* bad argument or inconsistent input */
#define CAPAC_ERR_IO (-2)             /* input file missing or malformed */
#define CAPAC_ERR_CUDA (-3)           /* CUDA runtime failure */
#define CAPAC_ERR_NOT_CONVERGED (-4)  /* BiCGSTAB above 100x tolerance after MAX_ITER (bicg_stab.c:561-570) */
#define CAPAC_ERR_RATTLE (-5)         /* RATTLE did not converge (force.c:1990-1994, 2083-2087) */
#define CAPAC_ERR_UNSUPPORTED (-6)    /* input uses a function type the reference does not support either */
#define CAPAC_ERR_CAPACITY (-7)       /* a fixed-capacity buffer is too small for this input */
#define CAPAC_ERR_NO_DEVICE (-8)      /* no usable sm_100 device */

const char *capac_last_error(void);

/* ------------------------------------------------------- enumerations */
#define CAPAC_RUN_MD 0
#define CAPAC_RUN_EM 1
#define CAPAC_RUN_CG 2
/* bonded term kinds (force.c:822-1347 as mpi_bonded dispatches them, force.c:1694-1900) */
#define CAPAC_BT_BOND_HARMONIC 1  /* par: b0, kb                              (bond funct 1) */
#define CAPAC_BT_BOND_MORSE 2     /* par: b0, D, beta                         (bond funct 3) */
#define CAPAC_BT_PAIR_14 3        /* types, charges, SCALE_LJ_QQ of the atoms (pair funct 1) */
#define CAPAC_BT_PAIR_USER 4      /* par: scaleQQ, q_i, q_j, c6, c12          (pair funct 2) */
#define CAPAC_BT_ANGLE_HARMONIC 5 /* par: a0 (degrees), ka                    (angle funct 1) */
#define CAPAC_BT_ANGLE_UB 6       /* par: a0, ka, b0_ub, kb_ub                (angle funct 5) */
#define CAPAC_BT_DIHEDRAL_RB 7    /* par: c0..c5 (periodic funct 1/4/9 are given as their RB form) */
#define CAPAC_NVE 0
#define CAPAC_NVT 1
/* Berendsen weak coupling, "ensemble berendsen" in mdset.txt.  No counterpart
 * in the reference: its only thermostat is the Nose-Hoover chain
 * (thermostat.c:117-191), and its MD loop thermostats only on "nvt"
 * (mpi-main.c:894, 975).  Once a step, after the second RATTLE, every
 * velocity is scaled by lambda = sqrt(1 + dt/tau (T0/T - 1)) (Berendsen et
 * al., J. Chem. Phys. 81, 3684 (1984)), T the instantaneous temperature, T0
 * the reference temperature of the heating ramp, tau = tau_T_in_ps; lambda is
 * held to [0.8, 1.25], and to 1 when T is zero. */
#define CAPAC_BERENDSEN 2

#define CAPAC_PREC_FP64 0   /* plain FP64 path: reference arithmetic on the GPU */
#define CAPAC_PREC_MIXED 1  /* FP32 pair terms, FP32 CPIM matrix/SpMV, FP64 refinement */

/* ------------------------------------------------- system description
 * Everything the reference reads from mdset.txt, param.txt and the .gro file,
 * flattened into arrays.  Arrays are owned by whoever built the struct:
 * capac_desc_load allocates them (free with capac_desc_free); a caller that
 * fills the struct itself keeps ownership.
 */
typedef struct capac_desc {
    /* mdset.txt (RunSet, typedef.h:200-242; keys file.c:90-124) */
    int run_type;     /* CAPAC_RUN_* */
    int ensemble;     /* CAPAC_NVE / CAPAC_NVT / CAPAC_BERENDSEN */
    int n_steps, n_save, n_heating, em_steps;
    double dt, r_cut, w_alpha, ref_temp, tau_temp, em_length, em_tol;
    int use_vdw;      /* 1: shifted-force LJ ("shifted"), 0: plain cut-off */
    int use_coulomb;  /* 1: damped shifted force ("wolf_sum"), 0: plain cut-off */
    int fix_metal, use_cpff;
    double efield[3]; /* kJ mol^-1 nm^-1 e^-1 (input V/nm times 96.4853363969351) */

    /* param.txt (Topol, typedef.h:298-338; Metal, typedef.h:245-288) */
    double scale_lj, scale_qq;
    int n_atoms, n_mols, n_types, mol_types;
    int *mol_num;          /* [mol_types] molecules of each type */
    int *mol_atoms;        /* [mol_types] atoms per molecule of each type */
    int *nb_funct;         /* [n_types*n_types] 1 LJ, 2 Buckingham, 3 Morse, 4 erf-vdW */
    double *nb_c6, *nb_c12, *nb_a, *nb_b; /* [n_types*n_types] */
    int *excl_offset;      /* [mol_types] start of a mol_atoms^2 exclusion matrix */
    unsigned char *excl;   /* exclusion matrices, row-major */
    int *cstr_offset;      /* [mol_types] first constraint of the type */
    int *cstr_count;       /* [mol_types] constraints per molecule of the type */
    int *cstr_i, *cstr_j;  /* constraint atom indices within the molecule */
    double *cstr_r;        /* constraint lengths, nm */
    int n_cstr_total;      /* constraints in the whole system (for ndf) */
    int n_bonded_terms;    /* bonds+pairs+angles+dihedrals over all molecule types */
    int n_vsites_total;    /* virtual sites in the whole system */
    int metal_min, metal_max, n_metal;
    int qsc_n, qsc_m;
    double qsc_eps, qsc_c, qsc_a;
    double cpff_polar, cpff_capac; /* atomic units */
    int n_nps;
    int *np_start, *np_end;        /* [n_nps] atom index ranges, inclusive */
    double *np_charge;             /* [n_nps] total charge, e */

    /* per atom (Atom_Info, typedef.h:146-152; filled as assign_indices, file.c:1031-1099) */
    int *atom_type, *mol_id, *mol_type, *atom_in_mol;
    unsigned char *is_metal;
    double *charge, *mass, *inv_mass;
    int *mol_first, *mol_last;     /* [n_mols] Mol_Info */

    /* .gro (read_gro, file.c:138-203) */
    double box[3];
    double *rx, *ry, *rz, *vx, *vy, *vz;
    double vq0, vp;                /* thermostat velocities from the title line */

    /* bonded terms per molecule type, in the reference's order within a
     * molecule (bonds, pairs, angles, dihedrals; file.c:715-930) */
    int *bt_offset, *bt_count;     /* [mol_types] */
    int *bt_kind;                  /* [terms] CAPAC_BT_* */
    int *bt_atoms;                 /* [4 * terms] atom indices within the molecule */
    double *bt_par;                /* [6 * terms] */
    /* virtual sites per molecule type (funct 4, file.c:931-969):
     * r_s = r_i + a r_ij + b r_ik + c (r_ij x r_ik) */
    int *vs_offset, *vs_count;     /* [mol_types] */
    int *vs_atoms;                 /* [4 * sites] i, j, k, s */
    double *vs_par;                /* [3 * sites] a, b, c */
} capac_desc;

/* The RB coefficients compute_dihedral_9 (force.c:1236-1347) derives from a
 * periodic dihedral (phi0 0 or 180 degrees, multiplicity 1 to 4), signs of
 * c1, c3, c5 already flipped for the polymer convention; CAPAC_ERR_UNSUPPORTED
 * otherwise (where the reference exits). */
int capac_dihedral_periodic_to_rb(double phi0, double kphi, int n, double c[6]);

/* Constants the reference derives at start-up. */
typedef struct capac_consts {
    double r_cut2, w_a2_sqrtpi, w_const, w_erfc_arcut; /* mpi-main.c:170-178 */
    double inv_rc12, inv_rc6;                          /* mpi-main.c:202-203 */
    double inv_polar, inv_capac, inv_r_qq, inv_r_pq, inv_r_pp; /* mpi-main.c:315-323 */
    int ndf;                                           /* mpi-main.c:548 */
    double kT, q_mass, dt_2;                           /* mpi-main.c:551-562 */
    int n_mat;                                         /* 4*n_metal + n_nps */
} capac_consts;

/* Parse the three reference input files.  On success *out owns all arrays. */
int capac_desc_load(const char *gro_path, const char *param_path, const char *mdset_path,
                    capac_desc **out);
void capac_desc_free(capac_desc *d);
int capac_desc_derive(const capac_desc *d, capac_consts *out);
/* Copy a named per-system array of a description into out (doubles).  Names:
 * rx ry rz vx vy vz charge mass box.  Returns the count written or <0. */
int capac_desc_get(const capac_desc *d, const char *name, double *out);
/* capac_desc_get names: rx ry rz vx vy vz charge mass is_metal atom_type
 * (n_atoms), box (3), bonded_counts (3: terms, virtual sites, constraints in
 * the system), bonded_kinds (8: terms of each CAPAC_BT_* kind). */
/* Sizes of a description: atoms, molecules, metal atoms, NPs, n_mat. */
int capac_desc_info(const capac_desc *d, int *n_atoms, int *n_mols, int *n_metal, int *n_nps, int *n_mat);

/* ------------------------------------------------------- GPU context */
typedef struct capac_options {
    int precision;          /* CAPAC_PREC_FP64 or CAPAC_PREC_MIXED */
    int device;             /* CUDA device ordinal */
    double skin;            /* neighbour-list skin, nm (default 0.2) */
    int list_every;         /* forced list rebuild interval in steps, 0 = displacement only */
    int max_neighbors;      /* 0 = estimate from density */
    double solver_tol;      /* rTr < solver_tol * bTb; 0 = reference 1e-8 (bicg_stab.c:303) */
    double refine_tol;      /* mixed path: FP64 relative residual target (default 1e-10; an
                               ill-conditioned metal cluster may need 1e-11 to keep the induced
                               charges within 1e-8 of the FP64 solution) */
    int matrix_layout;      /* CPIM matrix: 0 symmetric packed 4x4 blocks (default), 1 full 4x4 blocks */
    int predictor;          /* mixed path warm start: polynomial extrapolation of the last solutions of
                               order 0 (last solution), 1 (linear), 2 (quadratic) or 3 (cubic, default) */
    int solver_kernel;      /* BiCGSTAB on the symmetric layout: 0 one persistent cooperative launch per
                               solve when the device supports it (default), 1 a launch per vector step */
    int inner_precond;      /* mixed path, persistent solver: preconditioner of the inner solves,
                               0 the reference's Jacobi, 1 block-Jacobi on 32-atom groups,
                               2 block-Jacobi with a coarse correction on each group's total charge
                               and the nanoparticle constraints, 3 (default) the same with the
                               groups' dipole sums as well (up to 384 coarse columns, about 3,000
                               metal atoms; beyond, as 1) */
    int pair_list;          /* mixed path nonbonded list: 0 (default) or 2 clusters of four atoms
                               sharing each neighbour's load, where the box is large enough, with
                               every pair listed once (Newton's third law: the neighbour's force by
                               FP64 atomic adds, so its summation order varies from run to run);
                               3 the same clusters with every pair listed from both ends (fixed
                               summation order, run-to-run identical); 1 one list per atom; the
                               FP64 path always uses one list per atom */
    int max_iter;           /* BiCGSTAB iteration limit before the 100x fallback and
                               CAPAC_ERR_NOT_CONVERGED; 0 = the reference's MAX_ITER, 1000
                               (typedef.h:85, bicg_stab.c:546-570) */
    int wait_polls;         /* persistent solver: polls of a grid barrier before it gives up and the
                               call returns CAPAC_ERR_CUDA (the context stays usable); 0 = 2^24, about
                               a second.  Also settable on a live context (capac_set "wait_polls") */
} capac_options;

void capac_options_default(capac_options *o);

typedef struct capac_ctx capac_ctx;

int capac_create(const capac_desc *d, const capac_options *opt, capac_ctx **out);
int capac_destroy(capac_ctx *ctx);

/* One full force evaluation on the device-resident state, mpi_force semantics
 * (force.c:2097-2320): zero forces/energies/virial, nonbonded pairs, Sutton-Chen
 * density and forces, CPIM RHS, matrix, BiCGSTAB (warm-started from the
 * current induced vector), CPIM forces, external field on permanent charges.
 * potential[0] is left for the caller (sum_potential). */
int capac_force(capac_ctx *ctx);

/* mpi_force with host buffers (drop-in mode): copies positions in, evaluates,
 * copies forces, energies, virial and the CPIM vectors out.  vec_pq is in/out
 * (warm start, as Metal.vec_pq).  Any output pointer may be NULL.
 * Sizes: rx..fz n_atoms, potential 15, virial 9, vec_pq/vec_ext/diag_relay
 * n_mat, inv_sqrt_dens n_metal. */
int capac_mpi_force(capac_ctx *ctx, const double *rx, const double *ry, const double *rz,
                    double *fx, double *fy, double *fz, double *potential, double *virial,
                    double *vec_pq, double *vec_ext, double *diag_relay, double *inv_sqrt_dens);

/* CPIM stages on the device state, for stage-by-stage checks. */
int capac_qsc(capac_ctx *ctx);                          /* mpi_qsc_dens + mpi_qsc_force */
int capac_cpff_vec_ext(capac_ctx *ctx);                 /* mpi_cpff_vec_ext */
int capac_cpff_mat_relay(capac_ctx *ctx, long *nnz);    /* mpi_cpff_mat_relay_COO */
int capac_bicgstab(capac_ctx *ctx, int *iterations);    /* mpi_precon_bicg_stab_COO */
int capac_cpff_force(capac_ctx *ctx);                   /* mpi_cpff_force */

/* y = A x with the CPIM matrix of the last assembly; x and y are host arrays
 * of n_mat doubles in the reference layout (mpi_mat_vec_COO, bicg_stab.c:46-63). */
int capac_cpim_matvec(capac_ctx *ctx, const double *x, double *y);

/* capac_force without the BiCGSTAB solve: every term is evaluated with the
 * induced vector currently held (set with capac_set "vec_pq"). */
int capac_force_given_pq(capac_ctx *ctx);

/* Dense FP64 4x4 CPIM blocks of the metal rows row0 .. row0 + rows - 1
 * against every metal column, from the current positions:
 * out[((i - row0) * n_metal + j) * 16 + 4 * r + c], r and c over
 * (p_x, p_y, p_z, q).  The entries are those mpi_cpff_mat_relay_COO forms
 * (cpff.c:245-436, |e| <= 1e-15 dropped); diagonal blocks are
 * diag(1/polar x3, -1/capac).  For a caller that keeps the matrix on the host,
 * e.g. in the reference's COO form (the drop-in mpi_cpff_mat_relay_COO). */
int capac_cpim_blocks(capac_ctx *ctx, int row0, int rows, double *out);

/* Load the CPIM matrix from the reference's COO form: nnz entries val, row,
 * col in the reference vector layout, as mpi_cpff_mat_relay_COO leaves
 * Metal.vec_val / vec_row_ind / vec_col_ind (cpff.c:205-519).  It replaces the
 * assembled matrix until the next force call or assembly, and capac_bicgstab
 * then solves with it (the drop-in mpi_precon_bicg_stab_COO,
 * bicg_stab.h:58-59).  The matrix is symmetric, so the upper block triangle is
 * read; the diagonal blocks and neutrality couplings are the context's own
 * constants (equal to the reference's).  FP64 contexts with the symmetric
 * matrix layout only (CAPAC_ERR_UNSUPPORTED otherwise). */
int capac_cpim_set_coo(capac_ctx *ctx, long nnz, const double *val, const long *row, const long *col);

/* rattle_1st / rattle_2nd (force.h:85-95, force.c:1907-2090) on host arrays
 * of n_atoms doubles, for a caller that keeps its own integrator.  stage 1:
 * positions rx..rz and velocities vx..vz corrected in place towards the
 * constraint lengths along the old positions ox..oz (before the drift);
 * stage 2: velocities corrected in place, the constraint virial added to
 * virial[9] (ox..oz unused, may be NULL).  dt is the time step; constraints,
 * masses and box are the context's.  CAPAC_ERR_RATTLE with the reference's
 * message when a molecule does not converge. */
int capac_rattle(capac_ctx *ctx, int stage, double dt, double *rx, double *ry, double *rz, const double *ox,
                 const double *oy, const double *oz, double *vx, double *vy, double *vz, double *virial);

/* CPIM solve that allocates no device memory.  No counterpart in the
 * reference: it serves callers that cannot call cudaMalloc -- a host code that
 * hands all device memory to its own pool at start-up and forbids later
 * allocations, or a per-time-step caller for which an allocation (which may
 * synchronise the device) is not acceptable.  Same Jacobi-preconditioned
 * BiCGSTAB as capac_bicgstab, with the same breakdown guard (a zero or
 * non-finite alpha or omega leaves x at its last finite value and restarts
 * from there, up to eight starts) and the same acceptance of 100x the
 * criterion after MAX_ITER iterations (CAPAC_OK, with the reference's
 * "Loosen bicg_stab convergence criteria" note on stderr), on arrays the
 * caller owns (device pointers):
 *   mat   the 4x4-block matrix, mat[(i*16 + 4*row + col)*mat_stride + j] for
 *         block row i and block column j of n_metal metal atoms, rows/cols of a
 *         block ordered (p_x, p_y, p_z, q);
 *   rhs, diag  n_mat = 4*n_metal + n_nps values, reference vector layout;
 *   x     in: warm start, out: solution.
 * np_start/np_end are HOST arrays of metal-local atom ranges.  tol: criterion
 * rTr < tol*bTb (0 = 1e-8).  stream: a cudaStream_t, NULL for the default;
 * the call reads the convergence state back every four iterations and
 * returns when the solve has ended on that stream.  iterations: summed over
 * the starts.
 * Limits: n_mat <= 16384 and n_nps <= 16 (CAPAC_ERR_CAPACITY beyond).  The
 * work space is one static device array of about 1.2 MB that every device
 * loading the library holds until exit; the first call on a device looks up
 * its address (make that first call before any stream capture).  All calls
 * share the work space, so calls that overlap on the GPU race. */
int capac_bicgstab_static(const double *mat, int n_metal, int mat_stride, int n_nps, const int *np_start,
                          const int *np_end, const double *rhs, const double *diag, double *x, double tol,
                          int *iterations, void *stream);

/* MD steps on the device (mpi-main.c:874-1013, file output left out):
 * heating ramp, Nose-Hoover chain (nvt), half kick, drift, RATTLE, force,
 * half kick, RATTLE, kinetic energy, Nose-Hoover chain, COM removal; every
 * n_save steps apply_pbc and get_fmax_rms. */
int capac_md_steps(capac_ctx *ctx, int n_steps);

/* The reference's start-up after the first mpi_force (mpi-main.c:614-655):
 * sum_potential, remove_comm, kinetic_energy, first/ext temperature. */
int capac_md_init(capac_ctx *ctx);

/* Energy minimisation, steepest descent ("em") or conjugate gradient ("cg")
 * as run_type in mdset.txt selects (mpi-main.c:700-865).  capac_em_init
 * (after capac_md_init) sets the direction to the forces; each
 * capac_em_step moves the atoms by s / F_max * em_length, applies RATTLE and
 * zeroes the velocities, evaluates the forces, scales em_length by 1.2 or
 * 0.2 by the sign of the energy change, tests the reference's three
 * convergence criteria and, unless converged, updates the direction
 * (Polak-Ribiere gamma for "cg", 0 for "em"). */
typedef struct capac_em_status {
    int step;         /* steps taken since capac_em_init */
    int converged;    /* F_max < tol, F_rms < tol / 2 and |dE| < tol / 10 */
    double f_max, f_rms, energy, delta_pot, em_length;
} capac_em_status;
int capac_em_init(capac_ctx *ctx);
int capac_em_step(capac_ctx *ctx, capac_em_status *out);

/* Checkpoint of the whole dynamic state (no counterpart in the reference,
 * whose restart is the .gro file with vQ[0] in its title line, file.c:156-160):
 * positions, velocities, forces, energies, virial, the induced vector, the
 * mixed path's warm-start history, the full thermostat chain and step
 * counters.  A loaded state continues the run as if uninterrupted, up to the
 * summation order of the neighbour list, which is rebuilt at load. */
int capac_checkpoint_save(capac_ctx *ctx, const char *path);
int capac_checkpoint_load(capac_ctx *ctx, const char *path);

/* State transfer.  Names for per-atom arrays (n_atoms doubles):
 * rx ry rz vx vy vz fx fy fz.  Others: potential(15) virial(9) vec_pq vec_ext
 * diag_relay (n_mat) inv_sqrt_dens(n_metal) vQ(10) thermo(4: eKsum inst_temp
 * ref_temp ndf) box(6) fmax_rms(2: get_fmax_rms's largest and rms force at
 * the last n_save step); after a gradient call (read only, n_mat each):
 * adjoint_dedx (dE/dx), adjoint_dpsidx (dPsi/dx of the force matching),
 * adjoint_mu, adjoint_nu (the adjoint solutions).  Read-only diagnostics:
 * pair_list(2: 1 when the pair kernel walks the cluster list, cluster count),
 * pair_split(3: 1 when the half-list pair launch is split in two -- the
 * pair terms, then the CPIM term over the clusters next to metal -- as it
 * is when those are under 8% of the clusters; their count; all clusters),
 * potential and virial are settable too (to zero them before a stage call).
 * solver_layout(4: 1 when the mixed path's persistent solver works in the
 * order of its block-Jacobi groups, its tiles assembled in that order; the
 * tiles each of its blocks holds in tensor memory for the whole solve, 0 when
 * all are streamed from HBM each pass; the resident blocks per SM of the
 * group-ordered solver without and with tiles in tensor memory; the CTAs of
 * the cluster that last inverted the coarse matrix, 1 for one block, 0 none),
 * inner_stalls(1: inner solves of the mixed path's refinement that stopped
 * because their (r, r) had not halved in 60 iterations and handed their
 * iterate back to the FP64 refinement),
 * solver_phases(9: mean ns per iteration of the persistent solver's phases
 * when CAPAC_SOLVER_PHASES is set, then the iterations timed).  Set only:
 * wait_polls(1), the option of that name on the live context.  capac_get
 * returns the count written, <0 on error. */
int capac_get(capac_ctx *ctx, const char *name, double *out);
int capac_set(capac_ctx *ctx, const char *name, const double *in);

/* Statistics of the last force call: BiCGSTAB iterations, neighbour-list
 * rebuilds so far, list entries, pairs inside the cut-off.  list_entries,
 * max_neighbors and list_capacity describe the list the pair kernel walks:
 * per cluster of four atoms on the mixed path's cluster list, else per atom. */
typedef struct capac_stats {
    int solver_iterations;
    int solver_outer;           /* refinement sweeps (mixed path) */
    double solver_rel_residual; /* sqrt(rTr/bTb) at exit */
    long list_builds;
    long list_entries;
    long max_neighbors;
    int list_capacity;
    long md_step;
    double solver_initial_rel_residual; /* sqrt(rTr/bTb) of the warm start */
} capac_stats;
int capac_get_stats(capac_ctx *ctx, capac_stats *out);

/* Pair-set fingerprint of the current positions: number of nonbonded pairs
 * j<i inside the cut-off that the reference loop (force.c:1419-1473) visits,
 * and a 64-bit order-independent hash of those (i,j).  from_list = 1 reads
 * the neighbour list, 0 enumerates all N(N-1)/2 pairs on the GPU. */
int capac_pair_fingerprint(capac_ctx *ctx, int from_list, long *count, unsigned long long *hash);

/* Per-phase device times of the last force call in ms, in the reference's
 * time_used slots (mpi-main.c:119-128): 1 QSC density, 2 QSC force,
 * 4 nonbonded, 5 CPIM matrix, 6 CPIM vector, 7 CPIM solve, 8 CPIM force. */
int capac_phase_times(capac_ctx *ctx, double out_ms[15]);

/* Number of kernels this library launched since the context was created. */
long capac_kernel_launches(capac_ctx *ctx);

/* Device time of the MD steps, measured with CUDA events on the library's
 * stream around n_steps of capac_md_steps. */
int capac_time_md_steps(capac_ctx *ctx, int n_steps, double *ms);

/* Per-kernel device times.  While enabled, every launch of the kernels named
 * below is bracketed by CUDA events on the library's stream; capac_profile_get
 * returns the launch count and total milliseconds of one kernel class since
 * the last capac_profile_enable.  Classes: "pair", "spmv", "matrix",
 * "cpim_metal", "cpim_rhs", "qsc", "list_build", "solver_vec", "integrate",
 * "resid" (mixed path FP64 residual), "solve" (persistent solver: one launch
 * per BiCGSTAB solve) and "spmv_effective" (SpMV products that did work, with
 * total_ms 0). */
int capac_profile_enable(capac_ctx *ctx, int on);
int capac_profile_get(capac_ctx *ctx, const char *cls, long *launches, double *total_ms);

/* Metal parameters for fitting (no counterpart in the reference, which reads
 * them once from param.txt: file.c:533-549).  Names: "cpff_capac",
 * "cpff_polar" (a.u.), "cpim_rq", "cpim_rp" (the Gaussian widths in Bohr;
 * each follows its parameter the way the reference derives it,
 * mpi-main.c:315-323, until it is set on its own; setting it to 0 ties it
 * again; "cpim_rq_tied" and "cpim_rp_tied" read 1 while tied), "qsc_eps",
 * "qsc_c", "qsc_a",
 * "qsc_n", "qsc_m" (Sutton-Chen, force.c:385-542; n and m may be real).
 * A change takes effect at the next force call. */
int capac_param_get(capac_ctx *ctx, const char *name, double *value);
int capac_param_set(capac_ctx *ctx, const char *name, double value);

/* Gradients of the state of the last force call (which must have solved the
 * CPIM system, with no change of positions, induced vector or parameters
 * since).  E is the sum of the energy terms potential[1..14] (force.c
 * sum_potential); x the induced vector.  The reference's forces are -dE/dr
 * at fixed x (cpff.c:526-950), and E is not stationary in x at the solution,
 * so the total derivatives below include the response of the CPIM solve,
 * computed with the adjoint system A mu = dE/dx (one extra solve).
 *
 * capac_energy_grad: dE/dtheta for the nine parameters above, in that order
 * (kJ/mol per unit), and dE/dr (kJ/mol/nm, n_atoms each); pass NULL for
 * what is not wanted.  For a system without CPIM dE/dr = -F.
 *
 * capac_force_match_grad: L = sum over atoms and axes of
 * (F - F_target)^2 / (3 n_atoms) for the given target forces (host arrays,
 * n_atoms each), dL/dtheta for the nine parameters and dL/dr (n_atoms each);
 * grad or the position arrays may be NULL.  Second-order adjoint: one extra
 * solve, and Hessian-vector products of every force term recomputed on dual
 * numbers from the neighbour list. */
int capac_energy_grad(capac_ctx *ctx, double grad[9], double *gx, double *gy, double *gz);
int capac_force_match_grad(capac_ctx *ctx, const double *tfx, const double *tfy, const double *tfz,
                           double *loss, double grad[9], double *gx, double *gy, double *gz);

#ifdef __cplusplus
}
#endif

#endif /* CAPACMD_H */
