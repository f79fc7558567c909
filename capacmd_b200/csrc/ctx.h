// Device-resident state of one simulation and the launchers of its kernels.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "capacmd.h"
#include "capac_internal.h"
#include "device.cuh"

namespace capac {

// Scalars of one BiCGSTAB solve, kept in device memory (bicg_stab.c:280-303).
struct SolverScalars {
    double bTb, crit, rho, rho_old, alpha, omega, rTr, skip;
    double res0;     // refinement: FP64 residual norm^2 at the sweep start
    double rr0;      // (r, r) of the warm start
    int iter, done, status, max_iter;
};

// Thermostat and integrator scalars (System, typedef.h:353-401).
struct ThermoState {
    double eksum, inst_temp, ref_temp, first_temp, ext_temp, kT, scale;
    double vQ[kNhc], aQ[kNhc];
    double vcom[4];
    double fmax, frms;
};

// Read-only parameters passed by value to the kernels.
struct DevParams {
    Box box;
    int N, M, n_mat, n_nps, n_types, metal_min;
    int use_vdw, use_coulomb;
    double rc, rc2, list_r2;  // list_r2 = (rc + skin)^2
    double inv_rc12, inv_rc6, w_alpha, w_a2_sqrtpi, w_const, w_erfc_arcut;
    double inv_polar, inv_capac, inv_r_qq, inv_r_pq, inv_r_pp;
    double qsc_eps, qsc_c, qsc_a;
    double qsc_n, qsc_m;  // integers in the reference's input; reals for parameter gradients
    double efield[3];
    // per atom
    const int *type, *mol_id, *mol_type, *atom_in_mol;
    const unsigned char *is_metal;
    const double *charge, *mass, *inv_mass;
    // per molecule type
    const int *mol_atoms, *excl_offset;
    const unsigned char *excl;
    const int *nb_funct;
    const double4 *nb_par;  // (c6, c12, a, b)
    // nanoparticles
    const int *np_start, *np_end;
    const double *np_charge;
    // per type: 1 metal, 0 not (valid when metal_by_type: every atom of a type agrees)
    const unsigned char *type_metal;
    int metal_by_type;
};

// Bonded terms and virtual sites per molecule type (capac_desc bt_*, vs_*).
struct BondedView {
    int n_mols;
    const int *mol_first;
    const int *bt_offset, *bt_count, *bt_kind, *bt_atoms;
    const double *bt_par;
    const int *vs_offset, *vs_count, *vs_atoms;
    const double *vs_par;
    double scale_lj, scale_qq;
};

// Kernel classes for the event-based profiler.
enum KClass {
    K_PAIR = 0, K_SPMV, K_MATRIX, K_CPIM_METAL, K_CPIM_RHS, K_QSC, K_LIST, K_SOLVER_VEC, K_INTEGRATE, K_RESID,
    K_SOLVE,  // persistent solver: a whole BiCGSTAB solve in one launch
    K_NCLASS
};

// Pool of CUDA event pairs bracketing launches while profiling is on.
struct Profiler {
    bool on = false;
    std::vector<cudaEvent_t> ev;  // 2 per slot
    std::vector<int> cls;
    int used = 0;
    long count[K_NCLASS] = {};
    double ms[K_NCLASS] = {};
    long spmv_effective = 0;  // SpMV launches that did work (1 + 2 per iteration per solve)
};

// A captured chunk of solver iterations, replayed with cudaGraphLaunch.
struct SolveGraph {
    const double *b = nullptr;
    double *x = nullptr;
    bool prof = false;                 // captured with event-record nodes
    cudaGraphExec_t exec = nullptr;
    long kernels = 0;                  // kernels per replay
    std::vector<int> cls;              // kernel class of each event pair
    std::vector<cudaEvent_t> ev;       // event pairs recorded by the replay
};

}  // namespace capac

struct capac_ctx {
    capac::DevParams P{};
    capac_consts c{};
    capac_options opt{};
    int N = 0, M = 0, n_mat = 0, n_nps = 0, n_mols = 0, mol_types = 0;
    int ensemble = 0, fix_metal = 0, use_cpff = 0, n_save = 1, n_heating = 0;
    int metal_min = 0;
    double dt = 0.0;
    double dt_over_tau = 0.0;  // Berendsen coupling: dt / tau_T_in_ps
    // energy minimisation (mpi-main.c:700-865): run type, step length, tolerance
    int run_type = 0;
    double em_length = 0.0, em_tol = 0.0;
    double *em_buf = nullptr;     // [6N]: direction s and previous forces, allocated by capac_em_init
    long em_step = 0;
    bool has_cstr = false;
    bool has_bonded = false, has_vsites = false;
    capac::BondedView bview{};
    std::vector<void *> bonded_buffers;  // device arrays behind bview
    cudaStream_t stream = nullptr;
    long launches = 0;
    long md_step = 0;
    long list_builds = 0;
    int device = 0;
    int num_sms = 148;

    // host copies needed on the host side
    std::vector<int> h_np_start, h_np_end;

    // state (SoA, FP64)
    double *rx = nullptr, *ry = nullptr, *rz = nullptr, *vx = nullptr, *vy = nullptr, *vz = nullptr;
    double *fx = nullptr, *fy = nullptr, *fz = nullptr, *ox = nullptr, *oy = nullptr, *oz = nullptr;
    double4 *pos4 = nullptr;  // (x, y, z, q) packed for gathers
    float4 *pos4f = nullptr;  // mixed path: FP32 copy
    // topology
    int *type = nullptr, *mol_id = nullptr, *mol_type = nullptr, *atom_in_mol = nullptr;
    unsigned char *is_metal = nullptr;
    unsigned char *type_metal = nullptr;  // [n_types]
    double *charge = nullptr, *mass = nullptr, *inv_mass = nullptr;
    int *mol_atoms = nullptr, *excl_offset = nullptr;
    unsigned char *excl = nullptr;
    int *nb_funct = nullptr;
    double4 *nb_par = nullptr;
    int *mol_first = nullptr, *mol_last = nullptr, *cstr_off = nullptr, *cstr_cnt = nullptr;
    int *cstr_i = nullptr, *cstr_j = nullptr;
    double *cstr_r = nullptr;
    int *np_start = nullptr, *np_end = nullptr;
    double *np_charge = nullptr;

    // neighbour list
    int cap = 0;             // entries per atom
    uint32_t *nbr = nullptr; // [N * cap]
    int *nnb = nullptr;      // [N]
    double *rx0 = nullptr, *ry0 = nullptr, *rz0 = nullptr;  // positions at the last build
    int ncell[3] = {1, 1, 1};
    double cell_len[3] = {0, 0, 0};
    int n_cells = 1;
    int *cell_key = nullptr, *cell_key_sorted = nullptr, *atom_ids = nullptr, *cell_atoms = nullptr;
    int *cell_start = nullptr;   // [n_cells + 1] first sorted position of each cell
    double4 *spos = nullptr;     // [N] positions in cell order, atom index in w
    void *sort_tmp = nullptr;
    size_t sort_tmp_bytes = 0;
    int *flags = nullptr;      // [0] rebuild needed, [1] list overflow max count, [2] rattle error,
                               // [4] cluster-list overflow max count, [5] cluster extent (float bits),
                               // [7] cluster-pair list overflow max count
    int *h_flags = nullptr;    // pinned mirror
    bool list_valid = false;
    int cell_sub_bits = 0;     // sub-cell Morton bits below the cell index in cell_key

    // cluster-pair list (mixed path): clusters of up to four atoms, consecutive
    // in the sub-cell order of one cell; per cluster the j atoms with a mask of
    // the members each is a list neighbour of (see k_list.cu)
    bool clusters = false;        // the pair kernel runs on the cluster list (decided at each build)
    bool atom_list_full = true;   // atom-list rows exist for every atom (else metal rows only)
    bool need_full_list = false;  // a caller (the gradients) needs every atom-list row
    int cl_cap = 0;               // entries per cluster
    int cl_max = 0;               // cluster slots allocated (N / 4 + cells + 1)
    int cl_cells = 0;             // cell count cl_cell_start was sized for
    int n_clusters = 0;
    int4 *cl_atoms = nullptr;          // [cl_max] member atoms, -1 padding at the end
    int *cl_cell_start = nullptr;      // [cells + 1] first cluster of each cell; [cells] = count
    int *cl_counts = nullptr;          // [cells + 1] scratch: clusters per cell
    uint32_t *cl_nbr = nullptr;        // [cl_max * cl_cap]
    int *cl_nnb = nullptr;             // [cl_max]
    unsigned char *cl_metal = nullptr; // [cl_max] the cluster has a metal neighbour (or, on the
                                       // half list, a metal member)
    bool cl_half = false;              // half list: every pair once, Newton's third law (pair_list 2)
    int *cl_of = nullptr;              // [N] the cluster of each atom (half list)
    int *cl_next = nullptr;            // the cluster pair kernel's work counter (next cluster to take)
    int *cl_sel = nullptr;             // [cl_max] clusters with a metal member or neighbour (any order)
    int *n_cl_sel = nullptr;           // their count (device)

    // the nonbonded pairs run on a second stream, one block per SM, while the
    // CPIM right-hand side, matrix and solve run on `stream` (mixed path on
    // the half cluster list); the CPIM forces on water atoms follow the solve
    bool overlap = false;
    // half cluster list: the pair terms over all clusters, then the
    // water-side CPIM term over the clusters next to metal, in two launches
    // when those clusters are fewer than kPairSplitShare of all (decided at
    // every list build; CAPAC_PAIR_SPLIT=1 or 0 at creation forces it)
    bool pair_split = false;
    int pair_split_force = -1;   // -1 decide, 0 never, 1 always
    int n_sel_host = 0;          // clusters next to metal at the last build
    cudaStream_t stream2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    double *partials2 = nullptr;       // block partials of the overlapped pair launch (partials_cap)
    unsigned async_grid = 0;           // blocks of the overlapped pair launch
    cudaStream_t work_stream = nullptr; // stream of the launches being issued (null: `stream`)

    // i-cluster x j-cluster list (pair_list 4): per cluster the clusters of
    // the same or a higher index with a 4 x 4 mask of the member pairs within
    // the list radius, every pair once (see k_list.cu, k_pair.cu)
    bool cpairs = false;               // the pair kernel runs on the cluster-pair list (decided at each build)
    int cp_cap = 0;                    // entries per cluster
    int cp_max = 0;                    // cluster slots the cluster-pair arrays were sized for
    uint2 *cp_list = nullptr;          // [cl_max * cp_cap] j-cluster, mask | (either has metal) << 16
    int *cp_n = nullptr;               // [cl_max] entries of each cluster
    double4 *cp_cent = nullptr;        // [cl_max] centroid of each cluster (recomputed every step)
    float4 *cp_off = nullptr;          // [4 cl_max] member offsets from the centroid and charge (every step)
    int *cp_ti = nullptr;              // [4 cl_max] member atom | type << 24, -1 for an empty slot
    void *scan_tmp = nullptr;
    size_t scan_tmp_bytes = 0;

    // metal / CPIM
    int Mp = 0;                  // M padded to a multiple of 32
    double *isd = nullptr;       // inv_sqrt_dens [M]
    double *vec_ext = nullptr, *vec_pq = nullptr, *diag = nullptr;  // [n_mat]
    double *mat = nullptr;       // [M * 16 * Mp] 4x4 blocks, plane layout
    float *matf = nullptr;       // mixed path copy
    void *msym = nullptr;        // symmetric packed tiles (float on the mixed path, else double)
    double *sympart = nullptr;   // per-tile partial sums of the symmetric SpMV
    int coop_grid = 0;           // blocks of the persistent solver (0: per-step launches)
    int *g_atoms = nullptr;      // block-Jacobi groups of 32 metal atoms (mixed path inner solver)
    float *dinv = nullptr;       // their inverse diagonal blocks, 128 x 128 each
    // group-ordered persistent solver (mixed path, block-Jacobi): the stored
    // tiles follow the groups' atom order and the solver works in that order
    bool grouped = false;
    bool tmem_tiles = false;     // the grouped solver holds part of its tiles in tensor memory
    int group_grid = 0;          // blocks of the grouped solver's launch (<= coop_grid)
    float tile_l2 = -1.f;        // L2 policy of the persistent solvers' streamed tiles: -1 evict-first (default), 0 none, f > 0 keep f (CAPAC_TILE_L2)
    int inner_stall = 0;         // set during the refinement's inner solves: see GroupArgs::stall
    // two-level inner preconditioner (inner_precond 2, k_coarse.cu)
    bool twolevel = false;
    int cz_nc = 0;               // coarse columns: cz_modes per group and one per nanoparticle
    int cz_modes = 1;            // 1: the group's charge sum; 4: its dipole sums and charge sum
    float *cz_az = nullptr;      // A Z
    float *cz_w = nullptr;       // (A Z) E^-1
    float *cz_einv = nullptr;    // E^-1
    double *cz_aug = nullptr;    // [E | I] workspace of the inversion
    double *cz_zbuf = nullptr;   // Z^T v inside the solver
    int cz_cluster = 0;          // CTAs of the last inversion's cluster (1: one block)
    bool cz_one_block = false;   // invert in one block (CAPAC_COARSE_ONE_BLOCK at creation)
    long inner_stalls = 0;       // inner solves ended that way
    int *slot_np = nullptr;      // [32 nG] nanoparticle of each group slot's atom, -1 none
    int *np_off = nullptr;       // [n_nps + 1] offsets into np_rows
    int *np_rows = nullptr;      // [M] internal charge rows of each nanoparticle's atoms
    double *gvec = nullptr;      // 12 internal vectors of group_rows() doubles
    long precond_age = 0;        // matrix builds since the inverse blocks were computed
    long coarse_age = 0;         // refreshes of the inverse blocks since the coarse part was computed
    // the metal's CPIM parameters (a.u.) and Gaussian widths (Bohr), which the
    // widths follow unless set on their own (k_grad.cu)
    double capac = 0.0, polar = 0.0, rq = 0.0, rp = 0.0;
    bool rq_tied = true, rp_tied = true;  // widths derived from capac / polar
    bool grad_ready = false;              // the state is that of a force call with a solve
    // persistent-solver phase timer (CAPAC_SOLVER_PHASES set at create)
    bool phase_timer = false;
    void *phase_buf = nullptr;
    double phase_ns[8] = {};
    long phase_iters = 0;
    double *gw = nullptr;                 // gradient workspace (k_grad.cu), allocated on first use
    double *coop_bp = nullptr;   // its per-block dot partials
    void *coop_bar = nullptr;    // its grid barrier
    double *bw = nullptr;        // BiCGSTAB work vectors, 11 * n_mat
    float *bwf = nullptr;        // (unused)
    double *rres = nullptr, *dcorr = nullptr;  // mixed path: FP64 residual and correction, n_mat each
    double *xprev = nullptr;     // mixed path: the three solutions before the last (warm-start extrapolation)
    int n_solves = 0;            // completed solves since the history was reset
    capac::SolverScalars *ss = nullptr;
    capac::SolverScalars *h_ss = nullptr;  // pinned
    long nnz = 0;
    int last_iters = 0, last_outer = 0;
    double last_rel_res = 0.0, last_init_res = 0.0;

    // reductions and outputs
    double *partials = nullptr;
    size_t partials_cap = 0;     // doubles
    double *pot = nullptr, *vir = nullptr;  // [15], [9]
    capac::ThermoState *th = nullptr;
    capac::ThermoState *h_th = nullptr;

    // timing
    cudaEvent_t ev[16] = {};
    float phase_ms[15] = {};
    capac::Profiler prof;
    std::vector<capac::SolveGraph> graphs;
    capac::SolveGraph *capturing = nullptr;  // set while a solver chunk is being captured
    bool use_graphs = true;
};

namespace capac {

void cuda_check(cudaError_t e, const char *what);
#define CAPAC_CUDA(call) ::capac::cuda_check((call), #call)

// Kernel launchers (one stream; every launch is counted).
void launch_pack_positions(capac_ctx *c);
// cluster centroids and member offsets (pair_list 4); statics: atoms, types, metal flags too
void launch_cluster_frames(capac_ctx *c, bool statics);
// overlap of the nonbonded pairs with the CPIM solve (half cluster list)
void launch_pair_nonbonded_async(capac_ctx *c);
void launch_pair_join(capac_ctx *c);
void launch_list_maintenance(capac_ctx *c, bool force_rebuild);
// Rebuild the lists with an atom-list row for every atom, now and at every
// later build (the gradient kernels walk all rows).
void ensure_full_atom_list(capac_ctx *c);
void launch_pair_forces(capac_ctx *c, int mode);  // mode: 0 full, 1 CPIM water side only
void launch_qsc(capac_ctx *c);
void launch_cpim_rhs(capac_ctx *c);
void launch_cpim_matrix(capac_ctx *c);
int run_bicgstab(capac_ctx *c);  // returns status
int run_refined_solve(capac_ctx *c);  // mixed path: FP64 refinement around FP32-matrix BiCGSTAB
void launch_cpim_spmv(capac_ctx *c, const double *x, double *y);  // plain y = A x
void launch_cpim_block_rows(capac_ctx *c, int i0, int rows, double *out);  // dense FP64 blocks of some rows
// the symmetric FP64 tiles from a matrix in the reference's COO form (k_cpim_sym.cu)
void sym_tiles_from_coo(capac_ctx *c, long nnz, const double *val, const long *row, const long *col);
// symmetric packed storage (k_cpim_sym.cu)
int sym_tiles(int M);
size_t sym_matrix_elems(int M);
size_t sym_partial_doubles(int M);
void launch_sym_assemble(capac_ctx *c);
int sym_reduce_blocks(const capac_ctx *c);
void launch_sym_spmv(capac_ctx *c, int dot, const double *x, double *y, const double *d1, const double *d2,
                     const SolverScalars *ss);
void launch_sym_spmv_free(capac_ctx *c, const double *x, double *y);  // FP64, blocks from positions
// block-Jacobi preconditioner of the mixed path's inner solves (k_precond.cu)
int precond_groups(int M);
size_t precond_inverse_floats(int M);
std::vector<int> precond_group_atoms(int M, int metal_min, const double *rx, const double *ry, const double *rz);
void launch_block_inverse(capac_ctx *c);
void param_defaults(capac_ctx *c, const capac_desc *d);  // k_grad.cu
void spmv_free(capac_ctx *c, const double *x, double *y);  // FP64 A x with blocks from positions
int bicgstab_core(capac_ctx *c, const double *b, double *x, double tol, double skip);
void launch_force_derivative(capac_ctx *c, const double *wdir, double *dfx, double *dfy, double *dfz, double *isd_v,
                             double *isd_d);  // k_grad_forces.cu
constexpr int W_Y_SLOT = 7, W_V_SLOT = 4;  // BiCGSTAB work-vector slots used as scratch
constexpr double kPairSplitShare = 0.08;  // share of clusters next to metal below which the pair launch is split
// persistent cooperative solver (k_solve_coop.cu)
int coop_grid_size(int device, bool mixed);
size_t coop_barrier_bytes();
size_t coop_partial_doubles(int grid);
int bicgstab_coop(capac_ctx *c, const double *b, double *x, double tol, double skip);
// group-ordered solver (k_solve_coop.cu): internal vector length, blocks
int group_tmem_tiles();
int coarse_columns(int M, int n_nps, int modes);
int coarse_columns_max();  // the most coarse columns the solver holds
size_t coarse_az_floats(int M, int n_nps, int modes);
void launch_coarse_refresh(capac_ctx *c);
size_t group_rows(int M, int n_nps);
int group_grid_size(int device, bool hold);
int group_blocks_per_sm(int device, bool hold);
void launch_cpim_metal_forces(capac_ctx *c);
void launch_external_field(capac_ctx *c);
// per-block partials (src, default c->partials) summed into energy and virial slots
void launch_finalize(capac_ctx *c, int nblocks, int K, const int *slots_pot, const int *slots_vir,
                     const double *src = nullptr);
void launch_pair_fingerprint(capac_ctx *c, int from_list, long *count, unsigned long long *hash);

// integrator
void launch_md_half_kick(capac_ctx *c, bool with_nhc_scale);
void launch_md_drift(capac_ctx *c);
void launch_rattle(capac_ctx *c, int second);
void launch_kinetic(capac_ctx *c);
void launch_nhc(capac_ctx *c);
void launch_berendsen(capac_ctx *c);
void launch_scale_velocities(capac_ctx *c);
void launch_remove_com(capac_ctx *c);
void launch_apply_pbc(capac_ctx *c);
void launch_fmax_rms(capac_ctx *c);
void launch_heating(capac_ctx *c, long step);
void launch_sum_potential(capac_ctx *c);
void launch_build_vsites(capac_ctx *c);   // k_bonded.cu
void launch_bonded(capac_ctx *c);
void launch_vsite_forces(capac_ctx *c);
void launch_em_move(capac_ctx *c);                 // old_r = r; r += s / f_max * em_length
void launch_em_direction(capac_ctx *c, double gamma);  // s = F + gamma s; old F = F
void launch_em_dots(capac_ctx *c);                 // partials of (F,F), (F_old,F), (F_old,F_old)

size_t partials_needed(const capac_ctx *c);

// Profiler hooks: a ProfScope brackets the launches issued in its lifetime.
void prof_begin(capac_ctx *c, int cls);
void prof_end(capac_ctx *c);
void prof_flush(capac_ctx *c);
void prof_graph_replayed(capac_ctx *c, const SolveGraph &g);
struct ProfScope {
    capac_ctx *c;
    ProfScope(capac_ctx *cc, int cls) : c(cc) { prof_begin(c, cls); }
    ~ProfScope() { prof_end(c); }
};

inline unsigned grid_for(long n, int block) { return (unsigned)((n + block - 1) / block); }

inline int solver_max_iter(const capac_ctx *c) { return c->opt.max_iter > 0 ? c->opt.max_iter : kMaxIter; }

}  // namespace capac
