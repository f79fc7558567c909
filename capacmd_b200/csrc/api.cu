// C ABI of the force-and-solve path: context set-up, the mpi_force-equivalent
// orchestration (force.c:2097-2320), the MD loop (mpi-main.c:874-1013) and
// state transfer.  All state lives on one device; one stream orders the work.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "ctx.h"

namespace capac {

namespace {
thread_local std::string g_last_error;

template <class T>
T *dalloc(size_t n)
{
    T *p = nullptr;
    CAPAC_CUDA(cudaMalloc(&p, sizeof(T) * (n > 0 ? n : 1)));
    return p;
}

template <class T>
T *dupload(const T *h, size_t n, cudaStream_t s)
{
    T *p = dalloc<T>(n);
    if (n > 0 && h) CAPAC_CUDA(cudaMemcpyAsync(p, h, sizeof(T) * n, cudaMemcpyHostToDevice, s));
    return p;
}

void check_ctx(capac_ctx *c)
{
    if (!c) throw Error(CAPAC_ERR_INVALID, "null context");
}

void check_flags(capac_ctx *c)
{
    CAPAC_CUDA(cudaMemcpyAsync(c->h_flags, c->flags, sizeof(int) * 4, cudaMemcpyDeviceToHost, c->stream));
    CAPAC_CUDA(cudaStreamSynchronize(c->stream));
    if (c->h_flags[2]) {
        const bool first = c->h_flags[2] & 1;
        CAPAC_CUDA(cudaMemsetAsync(c->flags + 2, 0, sizeof(int), c->stream));
        throw Error(CAPAC_ERR_RATTLE, first ? "RATTLE_1 not converged!" : "RATTLE_2 not converged!");
    }
}

void record(capac_ctx *c, int k) { CAPAC_CUDA(cudaEventRecord(c->ev[k], c->stream)); }

// One mpi_force equivalent on the device state; solve = false keeps the
// induced vector as it is.
void force(capac_ctx *c, bool solve = true)
{
    cudaStream_t s = c->stream;
    c->grad_ready = false;
    record(c, 0);
    launch_build_vsites(c);  // build_vsites before everything (force.c:2124-2129)
    launch_list_maintenance(c, false);
    launch_pack_positions(c);
    CAPAC_CUDA(cudaMemsetAsync(c->fx, 0, sizeof(double) * c->N, s));
    CAPAC_CUDA(cudaMemsetAsync(c->fy, 0, sizeof(double) * c->N, s));
    CAPAC_CUDA(cudaMemsetAsync(c->fz, 0, sizeof(double) * c->N, s));
    CAPAC_CUDA(cudaMemsetAsync(c->pot, 0, sizeof(double) * 15, s));
    CAPAC_CUDA(cudaMemsetAsync(c->vir, 0, sizeof(double) * 9, s));
    record(c, 1);
    const bool cpim = c->M > 0 && c->use_cpff;
    launch_bonded(c);
    if (c->M > 0) launch_qsc(c);
    // the nonbonded pairs (their own stream) meanwhile with the CPIM stages
    const bool ovl = c->overlap && cpim && solve && c->clusters && c->cl_half;
    if (ovl) launch_pair_nonbonded_async(c);
    record(c, 2);
    int st = CAPAC_OK;
    try {
        if (cpim) launch_cpim_rhs(c);
        record(c, 3);
        if (cpim) launch_cpim_matrix(c);
        record(c, 4);
        if (cpim && solve) st = c->opt.precision == CAPAC_PREC_MIXED ? run_refined_solve(c) : run_bicgstab(c);
    } catch (...) {
        if (ovl) cudaStreamWaitEvent(c->stream, c->ev_join, 0);  // nothing left running on stream2
        throw;
    }
    record(c, 5);
    if (ovl)
        launch_pair_join(c);
    else
        launch_pair_forces(c, 0);
    record(c, 6);
    if (cpim) launch_cpim_metal_forces(c);
    launch_external_field(c);
    launch_vsite_forces(c);  // mpi_vsites after all force terms (force.c:2290-2296)
    record(c, 7);
    if (st != CAPAC_OK) {
        char msg[160];
        snprintf(msg, sizeof msg, "Error: bicg_stab not converged. rTr= %e, bTb= %e", c->h_ss->rTr, c->h_ss->bTb);
        throw Error(st, msg);
    }
    c->grad_ready = solve;
}

void md_step(capac_ctx *c)
{
    const long step = ++c->md_step;
    const bool nvt = c->ensemble == CAPAC_NVT;
    launch_heating(c, step);
    if (nvt) launch_nhc(c);
    launch_md_half_kick(c, nvt);
    launch_md_drift(c);
    launch_rattle(c, 0);
    force(c);
    check_flags(c);
    launch_sum_potential(c);
    launch_md_half_kick(c, false);
    launch_rattle(c, 1);
    launch_kinetic(c);
    if (nvt) {
        launch_nhc(c);
        launch_scale_velocities(c);
    } else if (c->ensemble == CAPAC_BERENDSEN) {
        launch_berendsen(c);
        launch_scale_velocities(c);
    }
    launch_remove_com(c);
    launch_kinetic(c);
    if (step % c->n_save == 0) {
        launch_apply_pbc(c);
        launch_fmax_rms(c);
    }
}

double *state_array(capac_ctx *c, const std::string &n, int *count)
{
    const int N = c->N;
    struct E { const char *nm; double *p; int cnt; } tab[] = {
        {"rx", c->rx, N}, {"ry", c->ry, N}, {"rz", c->rz, N}, {"vx", c->vx, N}, {"vy", c->vy, N},
        {"vz", c->vz, N}, {"fx", c->fx, N}, {"fy", c->fy, N}, {"fz", c->fz, N},
        {"potential", c->pot, 15}, {"virial", c->vir, 9},
        {"vec_pq", c->vec_pq, c->M > 0 ? c->n_mat : 0}, {"vec_ext", c->vec_ext, c->M > 0 ? c->n_mat : 0},
        {"diag_relay", c->diag, c->M > 0 ? c->n_mat : 0}, {"inv_sqrt_dens", c->isd, c->M},
        // gradient workspace (k_grad.cu): dE/dx, dPsi/dx, mu, nu of the last gradient call
        {"adjoint_dedx", c->gw, c->gw ? c->n_mat : 0},
        {"adjoint_dpsidx", c->gw ? c->gw + c->n_mat : nullptr, c->gw ? c->n_mat : 0},
        {"adjoint_mu", c->gw ? c->gw + 2 * (size_t)c->n_mat : nullptr, c->gw ? c->n_mat : 0},
        {"adjoint_nu", c->gw ? c->gw + 3 * (size_t)c->n_mat : nullptr, c->gw ? c->n_mat : 0},
    };
    for (auto &e : tab) {
        if (n == e.nm) {
            *count = e.cnt;
            return e.p;
        }
    }
    return nullptr;
}

}  // namespace

void set_last_error(const std::string &msg) { g_last_error = msg; }

constexpr int kProfSlots = 4096;

void prof_flush(capac_ctx *c)
{
    Profiler &p = c->prof;
    if (p.used == 0) return;
    CAPAC_CUDA(cudaStreamSynchronize(c->stream));
    for (int s = 0; s < p.used; ++s) {
        float ms = 0.f;
        CAPAC_CUDA(cudaEventElapsedTime(&ms, p.ev[2 * s], p.ev[2 * s + 1]));
        p.ms[p.cls[s]] += ms;
        p.count[p.cls[s]] += 1;
    }
    p.used = 0;
}

void prof_begin(capac_ctx *c, int cls)
{
    Profiler &p = c->prof;
    if (!p.on) return;
    if (SolveGraph *g = c->capturing) {
        // inside a capture: the replay records a pair of the graph's own events
        cudaEvent_t a, b;
        CAPAC_CUDA(cudaEventCreate(&a));
        CAPAC_CUDA(cudaEventCreate(&b));
        g->ev.push_back(a);
        g->ev.push_back(b);
        g->cls.push_back(cls);
        CAPAC_CUDA(cudaEventRecordWithFlags(a, c->stream, cudaEventRecordExternal));
        return;
    }
    if (p.used == kProfSlots) prof_flush(c);
    p.cls[p.used] = cls;
    CAPAC_CUDA(cudaEventRecord(p.ev[2 * p.used], c->work_stream ? c->work_stream : c->stream));
}

void prof_end(capac_ctx *c)
{
    Profiler &p = c->prof;
    if (!p.on) return;
    if (SolveGraph *g = c->capturing) {
        CAPAC_CUDA(cudaEventRecordWithFlags(g->ev.back(), c->stream, cudaEventRecordExternal));
        return;
    }
    CAPAC_CUDA(cudaEventRecord(p.ev[2 * p.used + 1], c->work_stream ? c->work_stream : c->stream));
    ++p.used;
}

// After a replay of a profiled graph has completed: add its event pairs.
void prof_graph_replayed(capac_ctx *c, const SolveGraph &g)
{
    if (!c->prof.on || !g.prof) return;
    for (size_t k = 0; k < g.cls.size(); ++k) {
        float ms = 0.f;
        CAPAC_CUDA(cudaEventElapsedTime(&ms, g.ev[2 * k], g.ev[2 * k + 1]));
        c->prof.ms[g.cls[k]] += ms;
        c->prof.count[g.cls[k]] += 1;
    }
}

void cuda_check(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw Error(CAPAC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace capac

using namespace capac;

extern "C" {

const char *capac_last_error(void) { return g_last_error.c_str(); }

void capac_options_default(capac_options *o)
{
    if (!o) return;
    memset(o, 0, sizeof *o);
    o->precision = CAPAC_PREC_FP64;
    o->device = 0;
    o->skin = 0.2;
    o->list_every = 0;
    o->max_neighbors = 0;
    o->solver_tol = 0.0;
    o->refine_tol = 1.0e-10;
    o->matrix_layout = 0;
    o->predictor = 3;
    o->solver_kernel = 0;
    o->inner_precond = 3;
    o->pair_list = 0;
}

int capac_create(const capac_desc *d, const capac_options *opt, capac_ctx **out)
{
    return guard([&] {
        if (!d || !out) throw Error(CAPAC_ERR_INVALID, "null argument");
        *out = nullptr;
        if ((d->n_bonded_terms > 0 && !d->bt_offset) || (d->n_vsites_total > 0 && !d->vs_offset))
            throw Error(CAPAC_ERR_INVALID, "bonded terms or virtual sites counted but not described");
        if (d->n_atoms <= 1 || d->n_atoms >= (1 << kIdxBits))
            throw Error(CAPAC_ERR_INVALID, "atom count out of range");
        if (d->n_types <= 0 || d->n_types > 255) throw Error(CAPAC_ERR_INVALID, "type count out of range");
        if (d->r_cut <= 0.0) throw Error(CAPAC_ERR_INVALID, "cut_off_radius must be positive");
        for (int a = 0; a < 3; ++a)
            if (!(d->box[a] > 0.0)) throw Error(CAPAC_ERR_INVALID, "box lengths must be positive");
        for (int k = 0; k < d->n_nps; ++k)
            if (d->n_metal == 0 || d->np_start[k] < d->metal_min || d->np_end[k] > d->metal_max ||
                d->np_start[k] > d->np_end[k])
                throw Error(CAPAC_ERR_INVALID, "START_END_CHG range outside MM_METAL");
        if (d->n_nps > 256) throw Error(CAPAC_ERR_UNSUPPORTED, "more than 256 nanoparticles");
        if (d->ensemble == CAPAC_BERENDSEN && !(d->tau_temp > 0.0))
            throw Error(CAPAC_ERR_INVALID, "tau_T_in_ps must be positive for the Berendsen thermostat");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
            throw Error(CAPAC_ERR_NO_DEVICE, "no CUDA device");
        capac_options o;
        capac_options_default(&o);
        if (opt) o = *opt;
        if (o.skin <= 0.0) o.skin = 0.2;
        if (o.device < 0 || o.device >= ndev) throw Error(CAPAC_ERR_NO_DEVICE, "device ordinal out of range");
        cudaDeviceProp prop;
        CAPAC_CUDA(cudaGetDeviceProperties(&prop, o.device));
        if (prop.major != 10) throw Error(CAPAC_ERR_NO_DEVICE, std::string("needs an sm_100 device, found ") + prop.name);
        CAPAC_CUDA(cudaSetDevice(o.device));

        capac_ctx *c = new capac_ctx();
        try {
            c->opt = o;
            c->device = o.device;
            c->num_sms = prop.multiProcessorCount;
            c->use_graphs = getenv("CAPAC_NO_GRAPHS") == nullptr;
            c->phase_timer = getenv("CAPAC_SOLVER_PHASES") != nullptr;
            derive(d, &c->c);
            c->N = d->n_atoms;
            c->M = d->n_metal;
            c->n_nps = d->n_nps;
            c->n_mat = c->c.n_mat;
            c->n_mols = d->n_mols;
            c->mol_types = d->mol_types;
            c->ensemble = d->ensemble;
            c->fix_metal = d->fix_metal;
            c->use_cpff = d->use_cpff;
            c->n_save = d->n_save > 0 ? d->n_save : 1;
            c->n_heating = d->n_heating;
            c->dt = d->dt;
            if (d->ensemble == CAPAC_BERENDSEN) c->dt_over_tau = d->dt / d->tau_temp;
            c->run_type = d->run_type;
            c->em_length = d->em_length;
            c->em_tol = d->em_tol;
            c->metal_min = d->metal_min;
            c->has_cstr = d->n_cstr_total > 0;
            CAPAC_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
            cudaStream_t s = c->stream;
            for (auto &e : c->ev) CAPAC_CUDA(cudaEventCreate(&e));
            const size_t N = c->N;

            // state
            c->rx = dupload(d->rx, N, s); c->ry = dupload(d->ry, N, s); c->rz = dupload(d->rz, N, s);
            c->vx = dupload(d->vx, N, s); c->vy = dupload(d->vy, N, s); c->vz = dupload(d->vz, N, s);
            c->fx = dalloc<double>(N); c->fy = dalloc<double>(N); c->fz = dalloc<double>(N);
            c->ox = dalloc<double>(N); c->oy = dalloc<double>(N); c->oz = dalloc<double>(N);
            c->rx0 = dalloc<double>(N); c->ry0 = dalloc<double>(N); c->rz0 = dalloc<double>(N);
            c->pos4 = dalloc<double4>(N);

            // topology
            c->type = dupload(d->atom_type, N, s);
            c->mol_id = dupload(d->mol_id, N, s);
            c->mol_type = dupload(d->mol_type, N, s);
            c->atom_in_mol = dupload(d->atom_in_mol, N, s);
            c->is_metal = dupload(d->is_metal, N, s);
            {
                // metal flag per type, when all atoms of a type agree
                std::vector<int> tm(d->n_types, -1);
                bool by_type = true;
                for (int i = 0; i < N && by_type; ++i) {
                    int &f = tm[d->atom_type[i]];
                    const int m = d->is_metal[i] ? 1 : 0;
                    if (f < 0) f = m;
                    else if (f != m) by_type = false;
                }
                std::vector<unsigned char> tmb(d->n_types);
                for (int t = 0; t < d->n_types; ++t) tmb[t] = tm[t] == 1 ? 1 : 0;
                c->type_metal = dupload(tmb.data(), tmb.size(), s);
                c->P.metal_by_type = by_type ? 1 : 0;
            }
            c->charge = dupload(d->charge, N, s);
            c->mass = dupload(d->mass, N, s);
            c->inv_mass = dupload(d->inv_mass, N, s);
            const int T = d->mol_types;
            size_t excl_n = 0;
            for (int m = 0; m < T; ++m) excl_n = std::max(excl_n, (size_t)d->excl_offset[m] + (size_t)d->mol_atoms[m] * d->mol_atoms[m]);
            c->mol_atoms = dupload(d->mol_atoms, T, s);
            c->excl_offset = dupload(d->excl_offset, T, s);
            c->excl = dupload(d->excl, excl_n, s);
            const int NT = d->n_types;
            std::vector<double4> par(NT * NT);
            for (int k = 0; k < NT * NT; ++k) par[k] = make_double4(d->nb_c6[k], d->nb_c12[k], d->nb_a[k], d->nb_b[k]);
            c->nb_funct = dupload(d->nb_funct, (size_t)NT * NT, s);
            c->nb_par = dupload(par.data(), par.size(), s);
            c->mol_first = dupload(d->mol_first, d->n_mols, s);
            // bonded terms and virtual sites per molecule type
            c->has_bonded = d->n_bonded_terms > 0;
            c->has_vsites = d->n_vsites_total > 0;
            if (c->has_bonded || c->has_vsites) {
                const int T = d->mol_types;
                size_t nt = 0, nv = 0;
                for (int m = 0; m < T; ++m) {
                    if (d->bt_offset) nt = std::max(nt, (size_t)(d->bt_offset[m] + d->bt_count[m]));
                    if (d->vs_offset) nv = std::max(nv, (size_t)(d->vs_offset[m] + d->vs_count[m]));
                }
                auto keep = [&](void *p) {
                    c->bonded_buffers.push_back(p);
                    return p;
                };
                const std::vector<int> zeros(T, 0);
                BondedView &B = c->bview;
                B.n_mols = d->n_mols;
                B.mol_first = c->mol_first;
                B.scale_lj = d->scale_lj;
                B.scale_qq = d->scale_qq;
                B.bt_offset = (int *)keep(dupload(d->bt_offset ? d->bt_offset : zeros.data(), T, s));
                B.bt_count = (int *)keep(dupload(d->bt_count ? d->bt_count : zeros.data(), T, s));
                B.bt_kind = (int *)keep(dupload(d->bt_kind, std::max<size_t>(nt, 1), s));
                B.bt_atoms = (int *)keep(dupload(d->bt_atoms, 4 * std::max<size_t>(nt, 1), s));
                B.bt_par = (double *)keep(dupload(d->bt_par, 6 * std::max<size_t>(nt, 1), s));
                B.vs_offset = (int *)keep(dupload(d->vs_offset ? d->vs_offset : zeros.data(), T, s));
                B.vs_count = (int *)keep(dupload(d->vs_count ? d->vs_count : zeros.data(), T, s));
                B.vs_atoms = (int *)keep(dupload(d->vs_atoms, 4 * std::max<size_t>(nv, 1), s));
                B.vs_par = (double *)keep(dupload(d->vs_par, 3 * std::max<size_t>(nv, 1), s));
                CAPAC_CUDA(cudaStreamSynchronize(s));
            }
            c->mol_last = dupload(d->mol_last, d->n_mols, s);
            c->cstr_off = dupload(d->cstr_offset, T, s);
            c->cstr_cnt = dupload(d->cstr_count, T, s);
            size_t ncs = 0;
            for (int m = 0; m < T; ++m) ncs = std::max(ncs, (size_t)d->cstr_offset[m] + d->cstr_count[m]);
            c->cstr_i = dupload(d->cstr_i, ncs, s);
            c->cstr_j = dupload(d->cstr_j, ncs, s);
            c->cstr_r = dupload(d->cstr_r, ncs, s);
            c->h_np_start.assign(d->np_start, d->np_start + d->n_nps);
            c->h_np_end.assign(d->np_end, d->np_end + d->n_nps);
            c->np_start = dupload(d->np_start, d->n_nps, s);
            c->np_end = dupload(d->np_end, d->n_nps, s);
            c->np_charge = dupload(d->np_charge, d->n_nps, s);

            // parameters
            DevParams &P = c->P;
            for (int a = 0; a < 3; ++a) {
                P.box.L[a] = d->box[a];
                P.box.H[a] = d->box[a] * 0.5;
            }
            P.N = c->N;
            P.M = c->M;
            P.n_mat = c->n_mat;
            P.n_nps = c->n_nps;
            P.n_types = NT;
            P.metal_min = c->M > 0 ? d->metal_min : 0;
            P.use_vdw = d->use_vdw;
            P.use_coulomb = d->use_coulomb;
            P.rc = d->r_cut;
            P.rc2 = c->c.r_cut2;
            P.list_r2 = (d->r_cut + o.skin) * (d->r_cut + o.skin);
            P.inv_rc12 = c->c.inv_rc12;
            P.inv_rc6 = c->c.inv_rc6;
            P.w_alpha = d->w_alpha;
            P.w_a2_sqrtpi = c->c.w_a2_sqrtpi;
            P.w_const = c->c.w_const;
            P.w_erfc_arcut = c->c.w_erfc_arcut;
            P.inv_polar = c->c.inv_polar;
            P.inv_capac = c->c.inv_capac;
            P.inv_r_qq = c->c.inv_r_qq;
            P.inv_r_pq = c->c.inv_r_pq;
            P.inv_r_pp = c->c.inv_r_pp;
            P.qsc_eps = d->qsc_eps;
            P.qsc_c = d->qsc_c;
            P.qsc_a = d->qsc_a;
            P.qsc_n = d->qsc_n;
            P.qsc_m = d->qsc_m;
            if (d->n_metal > 0) param_defaults(c, d);
            for (int a = 0; a < 3; ++a) P.efield[a] = d->efield[a];
            P.type = c->type;
            P.mol_id = c->mol_id;
            P.mol_type = c->mol_type;
            P.atom_in_mol = c->atom_in_mol;
            P.is_metal = c->is_metal;
            P.type_metal = c->type_metal;
            P.charge = c->charge;
            P.mass = c->mass;
            P.inv_mass = c->inv_mass;
            P.mol_atoms = c->mol_atoms;
            P.excl_offset = c->excl_offset;
            P.excl = c->excl;
            P.nb_funct = c->nb_funct;
            P.nb_par = c->nb_par;
            P.np_start = c->np_start;
            P.np_end = c->np_end;
            P.np_charge = c->np_charge;

            // neighbour list: capacity from the densest plausible environment
            {
                const double V = d->box[0] * d->box[1] * d->box[2];
                const double rl = d->r_cut + o.skin;
                const double sphere = 4.0 / 3.0 * M_PI * rl * rl * rl;
                double dens = std::max((double)N / V, 60.0);  // at least metallic gold density
                long est = (long)(1.25 * dens * sphere) + 64;
                if (o.max_neighbors > 0) est = o.max_neighbors;
                est = std::min<long>(est, (long)N);
                c->cap = (int)((est + 31) & ~31L);
            }
            c->nbr = dalloc<uint32_t>(N * (size_t)c->cap);
            c->nnb = dalloc<int>(N);
            c->cell_key = dalloc<int>(N);
            c->cell_key_sorted = dalloc<int>(N);
            c->atom_ids = dalloc<int>(N);
            c->cell_atoms = dalloc<int>(N);
            c->flags = dalloc<int>(8);
            CAPAC_CUDA(cudaMemsetAsync(c->flags, 0, sizeof(int) * 8, s));
            CAPAC_CUDA(cudaMallocHost(&c->h_flags, sizeof(int) * 8));

            // metal / CPIM
            if (c->M > 0) {
                const int M = c->M, n = c->n_mat;
                c->Mp = (M + 31) & ~31;
                c->isd = dalloc<double>(M);
                c->vec_ext = dalloc<double>(n);
                c->vec_pq = dalloc<double>(n);
                c->diag = dalloc<double>(n);
                CAPAC_CUDA(cudaMemsetAsync(c->vec_ext, 0, sizeof(double) * n, s));
                CAPAC_CUDA(cudaMemsetAsync(c->vec_pq, 0, sizeof(double) * n, s));
                std::vector<double> diag(n, 1.0);  // mpi-main.c:584-590: 1 until the matrix is built
                for (int i = 0; i < M && c->use_cpff; ++i) {
                    diag[3 * i] = diag[3 * i + 1] = diag[3 * i + 2] = c->c.inv_polar;
                    diag[3 * M + i] = -c->c.inv_capac;
                }
                CAPAC_CUDA(cudaMemcpyAsync(c->diag, diag.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
                CAPAC_CUDA(cudaStreamSynchronize(s));
                if (c->use_cpff) {
                    const bool mixed = o.precision == CAPAC_PREC_MIXED;
                    if (o.matrix_layout == 0) {
                        const size_t ne = sym_matrix_elems(M);
                        c->msym = mixed ? (void *)dalloc<float>(ne) : (void *)dalloc<double>(ne);
                        c->sympart = dalloc<double>(sym_partial_doubles(M));
                        if (o.solver_kernel == 0) c->coop_grid = coop_grid_size(c->device, mixed);
                        if (const char *l2 = getenv("CAPAC_TILE_L2")) c->tile_l2 = (float)atof(l2);
                        if (c->coop_grid > 0) {
                            c->coop_bp = dalloc<double>(coop_partial_doubles(c->coop_grid));
                            c->coop_bar = dalloc<unsigned char>(coop_barrier_bytes());
                            if (mixed && o.inner_precond >= 1 && o.inner_precond <= 3) {
                                const std::vector<int> g =
                                    precond_group_atoms(M, d->metal_min, d->rx, d->ry, d->rz);
                                c->g_atoms = dupload(g.data(), g.size(), s);
                                c->dinv = dalloc<float>(precond_inverse_floats(M));
                                // the group-ordered solver (unless CAPAC_SOLVER_UNGROUPED is set)
                                if (!getenv("CAPAC_SOLVER_UNGROUPED") && group_grid_size(c->device, false) == c->coop_grid) {
                                    std::vector<int> slot_np(g.size(), -1), off(d->n_nps + 1, 0), rows;
                                    for (int k = 0; k < d->n_nps; ++k) {
                                        for (size_t q = 0; q < g.size(); ++q) {
                                            const int atom = g[q] < 0 ? -1 : d->metal_min + g[q];
                                            if (atom >= d->np_start[k] && atom <= d->np_end[k]) {
                                                if (slot_np[q] < 0) slot_np[q] = k;
                                                rows.push_back((int)(4 * q + 3));
                                            }
                                        }
                                        off[k + 1] = (int)rows.size();
                                    }
                                    c->slot_np = dupload(slot_np.data(), slot_np.size(), s);
                                    c->np_off = dupload(off.data(), off.size(), s);
                                    c->np_rows = dupload(rows.data(), rows.size(), s);
                                    const size_t nv = 12 * group_rows(M, d->n_nps);
                                    c->gvec = dalloc<double>(nv);
                                    CAPAC_CUDA(cudaMemsetAsync(c->gvec, 0, sizeof(double) * nv, s));
                                    c->grouped = true;
                                    const int nm = o.inner_precond == 3 ? 4 : 1;
                                    const int nc = coarse_columns(M, d->n_nps, nm);
                                    if (o.inner_precond >= 2 && nc <= coarse_columns_max()) {
                                        c->twolevel = true;
                                        c->cz_modes = nm;
                                        c->cz_one_block = getenv("CAPAC_COARSE_ONE_BLOCK") != nullptr;
                                        c->cz_nc = nc;
                                        c->cz_az = dalloc<float>(coarse_az_floats(M, d->n_nps, nm));
                                        c->cz_w = dalloc<float>(coarse_az_floats(M, d->n_nps, nm));
                                        c->cz_einv = dalloc<float>((size_t)nc * nc);
                                        c->cz_aug = dalloc<double>((size_t)nc * 2 * nc);
                                        c->cz_zbuf = dalloc<double>(nc);
                                    }
                                    // the variant that holds tiles in tensor memory runs one
                                    // block per SM: the default when every tile fits there
                                    // (CAPAC_SOLVER_STREAM streams them all the same,
                                    // CAPAC_SOLVER_TMEM holds part of a larger matrix)
                                    c->group_grid = c->coop_grid;
                                    const int g = group_grid_size(c->device, true);
                                    const long nG = precond_groups(M), ntiles = nG * (nG + 1) / 2;
                                    const bool fits = (long)g * group_tmem_tiles() >= ntiles;
                                    c->tmem_tiles = g > 0 && g <= c->coop_grid &&
                                                    ((fits && !getenv("CAPAC_SOLVER_STREAM")) ||
                                                     getenv("CAPAC_SOLVER_TMEM") != nullptr);
                                    if (c->tmem_tiles) c->group_grid = g;
                                }
                            }
                        }
                    } else if (mixed) {
                        c->matf = dalloc<float>((size_t)M * 16 * c->Mp);
                    } else {
                        c->mat = dalloc<double>((size_t)M * 16 * c->Mp);
                    }
                    if (mixed) {
                        c->rres = dalloc<double>(n);
                        c->dcorr = dalloc<double>(n);
                        c->xprev = dalloc<double>((size_t)3 * n);
                    }
                    c->bw = dalloc<double>((size_t)n * 11);
                    CAPAC_CUDA(cudaMemsetAsync(c->bw, 0, sizeof(double) * n * 11, s));
                }
                c->nnz = 0;
            }
            c->ss = dalloc<SolverScalars>(1);
            CAPAC_CUDA(cudaMemsetAsync(c->ss, 0, sizeof(SolverScalars), s));
            CAPAC_CUDA(cudaMallocHost(&c->h_ss, sizeof(SolverScalars)));
            memset(c->h_ss, 0, sizeof(SolverScalars));

            c->partials_cap = partials_needed(c);
            c->partials = dalloc<double>(c->partials_cap);
            if (const char *ps = getenv("CAPAC_PAIR_SPLIT")) c->pair_split_force = ps[0] == '0' ? 0 : 1;
            if (o.precision == CAPAC_PREC_MIXED && d->n_metal > 0 && d->use_cpff && getenv("CAPAC_OVERLAP")) {
                c->overlap = true;
                CAPAC_CUDA(cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking));
                CAPAC_CUDA(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
                CAPAC_CUDA(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
                c->partials2 = dalloc<double>(c->partials_cap);
                // the solver then runs one block per SM beside the pair kernel's:
                // the variant that holds tiles in tensor memory where it runs
                if (c->grouped) {
                    const int g = group_grid_size(c->device, true);
                    if (g > 0 && g <= c->coop_grid && !getenv("CAPAC_SOLVER_STREAM")) {
                        c->tmem_tiles = true;
                        c->group_grid = g;
                    } else {
                        c->tmem_tiles = false;
                        c->group_grid = std::min(c->coop_grid, c->num_sms);
                    }
                }
            }
            c->pot = dalloc<double>(15);
            c->vir = dalloc<double>(9);
            CAPAC_CUDA(cudaMemsetAsync(c->pot, 0, sizeof(double) * 15, s));
            CAPAC_CUDA(cudaMemsetAsync(c->vir, 0, sizeof(double) * 9, s));
            ThermoState th;
            memset(&th, 0, sizeof th);
            th.ref_temp = d->ref_temp;
            th.ext_temp = d->ref_temp;
            th.kT = c->c.kT;
            th.scale = 1.0;
            th.vQ[0] = d->vq0;
            c->th = dupload(&th, 1, s);
            CAPAC_CUDA(cudaMallocHost(&c->h_th, sizeof(ThermoState)));
            c->h_ss->done = 0;
            CAPAC_CUDA(cudaStreamSynchronize(s));
            *out = c;
        } catch (...) {
            capac_destroy(c);
            throw;
        }
    });
}

int capac_destroy(capac_ctx *c)
{
    if (!c) return CAPAC_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    void *dev[] = {c->rx, c->ry, c->rz, c->vx, c->vy, c->vz, c->fx, c->fy, c->fz, c->ox, c->oy, c->oz,
                   c->rx0, c->ry0, c->rz0, c->pos4, c->pos4f, c->type, c->mol_id, c->mol_type,
                   c->atom_in_mol, c->is_metal, c->type_metal, c->charge, c->mass, c->inv_mass, c->mol_atoms,
                   c->excl_offset, c->excl, c->nb_funct, c->nb_par, c->mol_first, c->mol_last, c->cstr_off,
                   c->cstr_cnt, c->cstr_i, c->cstr_j, c->cstr_r, c->np_start, c->np_end, c->np_charge,
                   c->nbr, c->nnb, c->cell_key, c->cell_key_sorted, c->atom_ids, c->cell_atoms,
                   c->cell_start, c->spos, c->sort_tmp, c->flags, c->cl_atoms, c->cl_cell_start, c->cl_counts,
                   c->cl_nbr, c->cl_nnb, c->cl_metal, c->cl_of, c->cl_next, c->cl_sel, c->n_cl_sel, c->partials2,
                   c->cp_list,
                   c->cp_n, c->cp_cent, c->cp_off, c->cp_ti, c->cz_az, c->cz_w, c->cz_einv, c->cz_aug, c->cz_zbuf, c->scan_tmp, c->isd, c->vec_ext, c->vec_pq,
                   c->diag, c->mat, c->matf, c->msym, c->sympart, c->coop_bp, c->coop_bar, c->g_atoms, c->dinv, c->slot_np, c->np_off, c->np_rows, c->gvec, c->gw, c->em_buf, c->phase_buf, c->rres, c->dcorr, c->xprev, c->bw, c->bwf, c->ss, c->partials, c->pot, c->vir, c->th};
    for (void *p : dev)
        if (p) cudaFree(p);
    for (void *p : c->bonded_buffers)
        if (p) cudaFree(p);
    if (c->h_flags) cudaFreeHost(c->h_flags);
    if (c->h_ss) cudaFreeHost(c->h_ss);
    if (c->h_th) cudaFreeHost(c->h_th);
    for (auto &e : c->ev)
        if (e) cudaEventDestroy(e);
    for (auto &e : c->prof.ev)
        if (e) cudaEventDestroy(e);
    for (auto &g : c->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        for (auto &e : g.ev)
            if (e) cudaEventDestroy(e);
    }
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->stream2) cudaStreamDestroy(c->stream2);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return CAPAC_OK;
}

int capac_force(capac_ctx *c)
{
    return guard([&] {
        check_ctx(c);
        force(c);
        check_flags(c);
    });
}

int capac_mpi_force(capac_ctx *c, const double *rx, const double *ry, const double *rz, double *fx, double *fy,
                    double *fz, double *potential, double *virial, double *vec_pq, double *vec_ext,
                    double *diag_relay, double *inv_sqrt_dens)
{
    return guard([&] {
        check_ctx(c);
        if (!rx || !ry || !rz) throw Error(CAPAC_ERR_INVALID, "positions are required");
        cudaStream_t s = c->stream;
        const size_t nb = sizeof(double) * c->N;
        CAPAC_CUDA(cudaMemcpyAsync(c->rx, rx, nb, cudaMemcpyHostToDevice, s));
        CAPAC_CUDA(cudaMemcpyAsync(c->ry, ry, nb, cudaMemcpyHostToDevice, s));
        CAPAC_CUDA(cudaMemcpyAsync(c->rz, rz, nb, cudaMemcpyHostToDevice, s));
        if (vec_pq && c->M > 0)
            CAPAC_CUDA(cudaMemcpyAsync(c->vec_pq, vec_pq, sizeof(double) * c->n_mat, cudaMemcpyHostToDevice, s));
        force(c);
        if (fx) CAPAC_CUDA(cudaMemcpyAsync(fx, c->fx, nb, cudaMemcpyDeviceToHost, s));
        if (fy) CAPAC_CUDA(cudaMemcpyAsync(fy, c->fy, nb, cudaMemcpyDeviceToHost, s));
        if (fz) CAPAC_CUDA(cudaMemcpyAsync(fz, c->fz, nb, cudaMemcpyDeviceToHost, s));
        if (potential) CAPAC_CUDA(cudaMemcpyAsync(potential, c->pot, sizeof(double) * 15, cudaMemcpyDeviceToHost, s));
        if (virial) CAPAC_CUDA(cudaMemcpyAsync(virial, c->vir, sizeof(double) * 9, cudaMemcpyDeviceToHost, s));
        if (c->M > 0) {
            const size_t mb = sizeof(double) * c->n_mat;
            if (vec_pq) CAPAC_CUDA(cudaMemcpyAsync(vec_pq, c->vec_pq, mb, cudaMemcpyDeviceToHost, s));
            if (vec_ext) CAPAC_CUDA(cudaMemcpyAsync(vec_ext, c->vec_ext, mb, cudaMemcpyDeviceToHost, s));
            if (diag_relay) CAPAC_CUDA(cudaMemcpyAsync(diag_relay, c->diag, mb, cudaMemcpyDeviceToHost, s));
            if (inv_sqrt_dens)
                CAPAC_CUDA(cudaMemcpyAsync(inv_sqrt_dens, c->isd, sizeof(double) * c->M, cudaMemcpyDeviceToHost, s));
        }
        check_flags(c);
    });
}

int capac_force_given_pq(capac_ctx *c)
{
    return guard([&] {
        check_ctx(c);
        force(c, false);
        check_flags(c);
    });
}

int capac_cpim_matvec(capac_ctx *c, const double *x, double *y)
{
    return guard([&] {
        check_ctx(c);
        if (!x || !y) throw Error(CAPAC_ERR_INVALID, "null argument");
        if (c->M > 0 && !c->use_cpff) {  // use_cpff 0: the reference's COO matrix stays empty
            std::fill(y, y + c->n_mat, 0.0);
            return;
        }
        if (c->M == 0 || (!c->mat && !c->matf && !c->msym)) throw Error(CAPAC_ERR_INVALID, "no CPIM matrix in this system");
        double *dx = c->bw + (size_t)W_Y_SLOT * c->n_mat, *dy = c->bw + (size_t)W_V_SLOT * c->n_mat;
        const size_t nb = sizeof(double) * c->n_mat;
        CAPAC_CUDA(cudaMemcpyAsync(dx, x, nb, cudaMemcpyHostToDevice, c->stream));
        launch_cpim_spmv(c, dx, dy);
        CAPAC_CUDA(cudaMemcpyAsync(y, dy, nb, cudaMemcpyDeviceToHost, c->stream));
        CAPAC_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int capac_cpim_blocks(capac_ctx *c, int row0, int rows, double *out)
{
    return guard([&] {
        check_ctx(c);
        if (!out) throw Error(CAPAC_ERR_INVALID, "null argument");
        if (row0 < 0 || rows < 0 || row0 + (long)rows > c->M) throw Error(CAPAC_ERR_INVALID, "rows outside the metal atoms");
        if (rows == 0) return;
        launch_pack_positions(c);
        // chunks of rows through a temporary device buffer of at most 64 MB
        const size_t row_doubles = (size_t)c->M * 16;
        const int chunk = (int)std::max<size_t>(1, std::min<size_t>(rows, (64u << 20) / (8 * row_doubles)));
        double *tmp = nullptr;
        CAPAC_CUDA(cudaMalloc(&tmp, sizeof(double) * row_doubles * chunk));
        try {
            for (int i = 0; i < rows; i += chunk) {
                const int n = std::min(chunk, rows - i);
                launch_cpim_block_rows(c, row0 + i, n, tmp);
                CAPAC_CUDA(cudaMemcpyAsync(out + row_doubles * i, tmp, sizeof(double) * row_doubles * n,
                                           cudaMemcpyDeviceToHost, c->stream));
                CAPAC_CUDA(cudaStreamSynchronize(c->stream));
            }
        } catch (...) {
            cudaFree(tmp);
            throw;
        }
        CAPAC_CUDA(cudaFree(tmp));
    });
}

int capac_cpim_set_coo(capac_ctx *c, long nnz, const double *val, const long *row, const long *col)
{
    return guard([&] {
        check_ctx(c);
        if (nnz < 0 || (nnz > 0 && (!val || !row || !col))) throw Error(CAPAC_ERR_INVALID, "null argument");
        if (!c->msym || c->opt.precision != CAPAC_PREC_FP64)
            throw Error(CAPAC_ERR_UNSUPPORTED, "a COO matrix loads into the FP64 symmetric layout only");
        CAPAC_CUDA(cudaStreamSynchronize(c->stream));
        sym_tiles_from_coo(c, nnz, val, row, col);
        c->grad_ready = false;
    });
}

int capac_rattle(capac_ctx *c, int stage, double dt, double *rx, double *ry, double *rz, const double *ox,
                 const double *oy, const double *oz, double *vx, double *vy, double *vz, double *virial)
{
    return guard([&] {
        check_ctx(c);
        if (stage != 1 && stage != 2) throw Error(CAPAC_ERR_INVALID, "stage must be 1 or 2");
        if (!rx || !ry || !rz || !vx || !vy || !vz || (stage == 1 && (!ox || !oy || !oz)) || (stage == 2 && !virial))
            throw Error(CAPAC_ERR_INVALID, "null argument");
        cudaStream_t s = c->stream;
        const size_t nb = sizeof(double) * c->N;
        double *pos[3] = {rx, ry, rz}, *vel[3] = {vx, vy, vz};
        const double *old[3] = {ox, oy, oz};
        double *dpos[3] = {c->rx, c->ry, c->rz}, *dvel[3] = {c->vx, c->vy, c->vz}, *dold[3] = {c->ox, c->oy, c->oz};
        for (int a = 0; a < 3; ++a) {
            CAPAC_CUDA(cudaMemcpyAsync(dpos[a], pos[a], nb, cudaMemcpyHostToDevice, s));
            CAPAC_CUDA(cudaMemcpyAsync(dvel[a], vel[a], nb, cudaMemcpyHostToDevice, s));
            if (stage == 1) CAPAC_CUDA(cudaMemcpyAsync(dold[a], old[a], nb, cudaMemcpyHostToDevice, s));
        }
        c->list_valid = false;  // the positions came from outside
        c->grad_ready = false;
        const double dt_run = c->dt;
        c->dt = dt;
        if (stage == 2) CAPAC_CUDA(cudaMemsetAsync(c->vir, 0, sizeof(double) * 9, s));
        launch_rattle(c, stage == 2);
        c->dt = dt_run;
        for (int a = 0; a < 3; ++a) {
            if (stage == 1) CAPAC_CUDA(cudaMemcpyAsync(pos[a], dpos[a], nb, cudaMemcpyDeviceToHost, s));
            CAPAC_CUDA(cudaMemcpyAsync(vel[a], dvel[a], nb, cudaMemcpyDeviceToHost, s));
        }
        double w[9] = {0.0};
        if (stage == 2 && c->has_cstr) CAPAC_CUDA(cudaMemcpyAsync(w, c->vir, sizeof w, cudaMemcpyDeviceToHost, s));
        CAPAC_CUDA(cudaStreamSynchronize(s));
        check_flags(c);
        if (stage == 2)
            for (int k = 0; k < 9; ++k) virial[k] += w[k];
    });
}

int capac_qsc(capac_ctx *c)
{
    return guard([&] {
        check_ctx(c);
        launch_pack_positions(c);
        if (c->M > 0) launch_qsc(c);
        CAPAC_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int capac_cpff_vec_ext(capac_ctx *c)
{
    return guard([&] {
        check_ctx(c);
        if (c->M == 0) return;
        launch_list_maintenance(c, false);
        launch_pack_positions(c);
        launch_cpim_rhs(c);
        CAPAC_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int capac_cpff_mat_relay(capac_ctx *c, long *nnz)
{
    return guard([&] {
        check_ctx(c);
        if (c->M == 0 || (!c->mat && !c->matf && !c->msym)) return;
        launch_pack_positions(c);
        launch_cpim_matrix(c);
        CAPAC_CUDA(cudaStreamSynchronize(c->stream));
        // entries the reference's COO form would hold (cpff.c:245-516):
        // 16 per off-diagonal block, 4 per diagonal block, 2 per NP member
        if (nnz) {
            long lam = 0;
            for (int k = 0; k < c->n_nps; ++k) lam += 2L * (c->h_np_end[k] - c->h_np_start[k] + 1);
            *nnz = 16L * c->M * (c->M - 1) + 4L * c->M + lam;
        }
    });
}

int capac_bicgstab(capac_ctx *c, int *iterations)
{
    return guard([&] {
        check_ctx(c);
        if (c->M == 0 || (!c->mat && !c->matf && !c->msym)) return;
        const int st = c->opt.precision == CAPAC_PREC_MIXED ? run_refined_solve(c) : run_bicgstab(c);
        if (iterations) *iterations = c->last_iters;
        if (st != CAPAC_OK) throw Error(st, "Error: bicg_stab not converged.");
    });
}

int capac_cpff_force(capac_ctx *c)
{
    return guard([&] {
        check_ctx(c);
        if (c->M == 0 || !c->use_cpff) return;
        launch_list_maintenance(c, false);
        launch_pack_positions(c);
        launch_pair_forces(c, 1);
        launch_cpim_metal_forces(c);
        CAPAC_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int capac_md_init(capac_ctx *c)
{
    return guard([&] {
        check_ctx(c);
        force(c);
        check_flags(c);
        launch_sum_potential(c);
        launch_remove_com(c);
        launch_kinetic(c);
        CAPAC_CUDA(cudaMemcpyAsync(c->h_th, c->th, sizeof(ThermoState), cudaMemcpyDeviceToHost, c->stream));
        CAPAC_CUDA(cudaStreamSynchronize(c->stream));
        c->h_th->first_temp = c->h_th->inst_temp;
        c->h_th->ext_temp = c->h_th->ref_temp;
        CAPAC_CUDA(cudaMemcpyAsync(c->th, c->h_th, sizeof(ThermoState), cudaMemcpyHostToDevice, c->stream));
        launch_fmax_rms(c);
        CAPAC_CUDA(cudaStreamSynchronize(c->stream));
        c->md_step = 0;
    });
}

int capac_em_init(capac_ctx *c)
{
    return guard([&] {
        check_ctx(c);
        const size_t N = c->N;
        if (!c->em_buf) c->em_buf = dalloc<double>(6 * N);
        // s = F, old F = F (mpi-main.c:716-727); thermostat velocities zero
        CAPAC_CUDA(cudaMemcpyAsync(c->em_buf, c->fx, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
        CAPAC_CUDA(cudaMemcpyAsync(c->em_buf + N, c->fy, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
        CAPAC_CUDA(cudaMemcpyAsync(c->em_buf + 2 * N, c->fz, sizeof(double) * N, cudaMemcpyDeviceToDevice,
                                   c->stream));
        CAPAC_CUDA(cudaMemcpyAsync(c->em_buf + 3 * N, c->em_buf, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice,
                                   c->stream));
        CAPAC_CUDA(cudaMemcpyAsync(c->h_th, c->th, sizeof(ThermoState), cudaMemcpyDeviceToHost, c->stream));
        CAPAC_CUDA(cudaStreamSynchronize(c->stream));
        for (double &v : c->h_th->vQ) v = 0.0;
        CAPAC_CUDA(cudaMemcpyAsync(c->th, c->h_th, sizeof(ThermoState), cudaMemcpyHostToDevice, c->stream));
        CAPAC_CUDA(cudaStreamSynchronize(c->stream));
        c->em_step = 0;
    });
}

int capac_em_step(capac_ctx *c, capac_em_status *out)
{
    return guard([&] {
        check_ctx(c);
        if (!c->em_buf) throw Error(CAPAC_ERR_INVALID, "capac_em_init has not been called");
        cudaStream_t s = c->stream;
        double old_pot = 0.0;
        CAPAC_CUDA(cudaMemcpy(&old_pot, c->pot, sizeof(double), cudaMemcpyDeviceToHost));
        // move along s, constrain, zero the velocities (mpi-main.c:730-763)
        launch_em_move(c);
        launch_rattle(c, 0);
        CAPAC_CUDA(cudaMemsetAsync(c->vx, 0, sizeof(double) * c->N, s));
        CAPAC_CUDA(cudaMemsetAsync(c->vy, 0, sizeof(double) * c->N, s));
        CAPAC_CUDA(cudaMemsetAsync(c->vz, 0, sizeof(double) * c->N, s));
        force(c);
        check_flags(c);
        launch_sum_potential(c);
        launch_fmax_rms(c);
        double pot0 = 0.0;
        CAPAC_CUDA(cudaMemcpyAsync(&pot0, c->pot, sizeof(double), cudaMemcpyDeviceToHost, s));
        CAPAC_CUDA(cudaMemcpyAsync(c->h_th, c->th, sizeof(ThermoState), cudaMemcpyDeviceToHost, s));
        CAPAC_CUDA(cudaStreamSynchronize(s));
        const double fmax = c->h_th->fmax, frms = c->h_th->frms;
        // step length and convergence (mpi-main.c:770-816)
        const double delta = pot0 - old_pot;
        c->em_length *= delta <= 0.0 ? 1.2 : 0.2;
        const bool converged = fmax < c->em_tol && frms < c->em_tol * 0.5 && fabs(delta) < c->em_tol * 0.1;
        ++c->em_step;
        if (!converged) {
            double gamma = 0.0;  // steepest descent
            if (c->run_type == CAPAC_RUN_CG) {
                const unsigned nb = grid_for(c->N, 256);
                launch_em_dots(c);
                std::vector<double> h((size_t)nb * 3);
                CAPAC_CUDA(cudaMemcpyAsync(h.data(), c->partials, sizeof(double) * h.size(), cudaMemcpyDeviceToHost,
                                           s));
                CAPAC_CUDA(cudaStreamSynchronize(s));
                double g22 = 0.0, g12 = 0.0, g11 = 0.0;
                for (unsigned b = 0; b < nb; ++b) {
                    g22 += h[3 * b];
                    g12 += h[3 * b + 1];
                    g11 += h[3 * b + 2];
                }
                gamma = (g22 - g12) / g11;
            }
            launch_em_direction(c, gamma);
            CAPAC_CUDA(cudaStreamSynchronize(s));
        }
        if (out) {
            out->step = (int)c->em_step;
            out->converged = converged ? 1 : 0;
            out->f_max = fmax;
            out->f_rms = frms;
            out->energy = pot0;
            out->delta_pot = delta;
            out->em_length = c->em_length;
        }
    });
}

namespace {

// Checkpoint file: magic, version, sizes, step counters, then the arrays.
constexpr char kCkptMagic[8] = {'C', 'A', 'P', 'A', 'C', 'K', 'P', '1'};
struct CkptHeader {
    char magic[8];
    int version, N, n_mat, has_hist;
    long md_step, em_step;
    int n_solves, pad;
    double em_length;
    double box[3];
};

}  // namespace

namespace {
// Closes a FILE on every way out of a scope.
struct FileGuard {
    FILE *f;
    explicit FileGuard(FILE *ff) : f(ff) {}
    ~FileGuard()
    {
        if (f) fclose(f);
    }
    int close()
    {
        const int r = fclose(f);
        f = nullptr;
        return r;
    }
};
}  // namespace

int capac_checkpoint_save(capac_ctx *c, const char *path)
{
    return guard([&] {
        check_ctx(c);
        if (!path) throw Error(CAPAC_ERR_INVALID, "null path");
        CAPAC_CUDA(cudaStreamSynchronize(c->stream));
        CkptHeader h{};
        memcpy(h.magic, kCkptMagic, 8);
        h.version = 1;
        h.N = c->N;
        h.n_mat = c->M > 0 ? c->n_mat : 0;
        h.has_hist = c->xprev != nullptr;
        h.md_step = c->md_step;
        h.em_step = c->em_step;
        h.n_solves = c->n_solves;
        h.em_length = c->em_length;
        for (int a = 0; a < 3; ++a) h.box[a] = c->P.box.L[a];
        ThermoState th;
        CAPAC_CUDA(cudaMemcpy(&th, c->th, sizeof th, cudaMemcpyDeviceToHost));
        FileGuard fg(fopen(path, "wb"));
        if (!fg.f) throw Error(CAPAC_ERR_IO, std::string("cannot write ") + path);
        std::vector<double> buf;
        auto put = [&](const double *d, size_t n) {
            buf.resize(n);
            if (n) CAPAC_CUDA(cudaMemcpy(buf.data(), d, sizeof(double) * n, cudaMemcpyDeviceToHost));
            if (fwrite(buf.data(), sizeof(double), n, fg.f) != n) throw Error(CAPAC_ERR_IO, "short write");
        };
        if (fwrite(&h, sizeof h, 1, fg.f) != 1 || fwrite(&th, sizeof th, 1, fg.f) != 1)
            throw Error(CAPAC_ERR_IO, "short write");
        const size_t N = c->N;
        for (const double *p : {c->rx, c->ry, c->rz, c->vx, c->vy, c->vz, c->fx, c->fy, c->fz}) put(p, N);
        put(c->pot, 15);
        put(c->vir, 9);
        if (h.n_mat) put(c->vec_pq, h.n_mat);
        if (h.has_hist) put(c->xprev, (size_t)3 * c->n_mat);
        if (fg.close() != 0) throw Error(CAPAC_ERR_IO, "close failed");
    });
}

// The whole file is read and checked before any device state changes: a
// truncated or foreign file leaves the context as it was.
int capac_checkpoint_load(capac_ctx *c, const char *path)
{
    return guard([&] {
        check_ctx(c);
        if (!path) throw Error(CAPAC_ERR_INVALID, "null path");
        CkptHeader h{};
        ThermoState th;
        std::vector<double> data;
        size_t n_hist = 0;
        {
            FileGuard fg(fopen(path, "rb"));
            if (!fg.f) throw Error(CAPAC_ERR_IO, std::string("cannot read ") + path);
            const bool head = fread(&h, sizeof h, 1, fg.f) == 1 && fread(&th, sizeof th, 1, fg.f) == 1;
            if (!head || memcmp(h.magic, kCkptMagic, 8) != 0 || h.version != 1)
                throw Error(CAPAC_ERR_IO, "not a checkpoint of this library");
            if (h.N != c->N || h.n_mat != (c->M > 0 ? c->n_mat : 0) || (h.has_hist && !c->xprev))
                throw Error(CAPAC_ERR_INVALID, "checkpoint is of a different system or precision");
            for (int a = 0; a < 3; ++a)
                if (h.box[a] != c->P.box.L[a]) throw Error(CAPAC_ERR_INVALID, "checkpoint is of a different box");
            n_hist = h.has_hist ? (size_t)3 * c->n_mat : 0;
            const size_t total = 9 * (size_t)c->N + 15 + 9 + (size_t)h.n_mat + n_hist;
            data.resize(total);
            if (fread(data.data(), sizeof(double), total, fg.f) != total)
                throw Error(CAPAC_ERR_IO, "truncated checkpoint");
        }
        // the context's stream may still be using the arrays about to be replaced
        CAPAC_CUDA(cudaStreamSynchronize(c->stream));
        const double *src = data.data();
        auto put = [&](double *d, size_t n) {
            if (n) CAPAC_CUDA(cudaMemcpyAsync(d, src, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
            src += n;
        };
        const size_t N = c->N;
        for (double *p : {c->rx, c->ry, c->rz, c->vx, c->vy, c->vz, c->fx, c->fy, c->fz}) put(p, N);
        put(c->pot, 15);
        put(c->vir, 9);
        if (h.n_mat) put(c->vec_pq, h.n_mat);
        if (n_hist) put(c->xprev, n_hist);
        CAPAC_CUDA(cudaMemcpyAsync(c->th, &th, sizeof th, cudaMemcpyHostToDevice, c->stream));
        CAPAC_CUDA(cudaStreamSynchronize(c->stream));
        c->md_step = h.md_step;
        c->em_step = h.em_step;
        c->em_length = h.em_length;
        c->n_solves = h.has_hist ? h.n_solves : 0;
        c->list_valid = false;   // the list is rebuilt from the restored positions
        c->precond_age = 0;
        c->grad_ready = false;
    });
}

int capac_md_steps(capac_ctx *c, int n)
{
    return guard([&] {
        check_ctx(c);
        if (n < 0) throw Error(CAPAC_ERR_INVALID, "negative step count");
        for (int k = 0; k < n; ++k) md_step(c);
        CAPAC_CUDA(cudaStreamSynchronize(c->stream));
        check_flags(c);
    });
}

int capac_get(capac_ctx *c, const char *name, double *out)
{
    int count = -1;
    const int st = guard([&] {
        check_ctx(c);
        if (!name || !out) throw Error(CAPAC_ERR_INVALID, "null argument");
        std::string n(name);
        CAPAC_CUDA(cudaStreamSynchronize(c->stream));
        int cnt = 0;
        if (double *p = state_array(c, n, &cnt)) {
            if (cnt > 0) CAPAC_CUDA(cudaMemcpy(out, p, sizeof(double) * cnt, cudaMemcpyDeviceToHost));
            count = cnt;
            return;
        }
        if (n == "vQ" || n == "thermo" || n == "fmax_rms") {
            ThermoState th;
            CAPAC_CUDA(cudaMemcpy(&th, c->th, sizeof th, cudaMemcpyDeviceToHost));
            if (n == "vQ") {
                memcpy(out, th.vQ, sizeof th.vQ);
                count = kNhc;
            } else if (n == "thermo") {
                out[0] = th.eksum;
                out[1] = th.inst_temp;
                out[2] = th.ref_temp;
                out[3] = c->c.ndf;
                count = 4;
            } else {
                out[0] = th.fmax;
                out[1] = th.frms;
                count = 2;
            }
            return;
        }
        if (n == "pair_list") {  // 1 on the cluster list, 2 on the cluster-pair list, then the cluster count
            out[0] = c->cpairs ? 2.0 : (c->clusters ? 1.0 : 0.0);
            out[1] = (double)c->n_clusters;
            count = 2;
            return;
        }
        if (n == "pair_split") {  // 1 when the pair launch is split; clusters next to metal; all clusters
            out[0] = c->pair_split ? 1.0 : 0.0;
            out[1] = (double)c->n_sel_host;
            out[2] = (double)c->n_clusters;
            count = 3;
            return;
        }
        if (n == "solver_layout") {  // 1 when the persistent solver runs in the block-Jacobi groups' order;
                                     // its tiles per block held in tensor memory
            out[0] = c->grouped ? 1.0 : 0.0;
            out[1] = c->grouped && c->tmem_tiles ? (double)group_tmem_tiles() : 0.0;
            out[2] = (double)group_blocks_per_sm(c->device, false);
            out[3] = (double)group_blocks_per_sm(c->device, true);
            out[4] = (double)c->cz_cluster;
            count = 5;
            return;
        }
        if (n == "inner_stalls") {  // inner solves of the refinement stopped for lack of progress
            out[0] = (double)c->inner_stalls;
            count = 1;
            return;
        }
        if (n == "solver_phases") {  // mean ns per iteration of each phase, then the iteration count
            for (int k = 0; k < 8; ++k) out[k] = c->phase_iters ? c->phase_ns[k] / c->phase_iters : 0.0;
            out[8] = (double)c->phase_iters;
            count = 9;
            return;
        }
        if (n == "box") {
            for (int a = 0; a < 3; ++a) {
                out[a] = c->P.box.L[a];
                out[3 + a] = c->P.box.H[a];
            }
            count = 6;
            return;
        }
        throw Error(CAPAC_ERR_INVALID, "unknown array " + n);
    });
    return st == CAPAC_OK ? count : st;
}

int capac_set(capac_ctx *c, const char *name, const double *in)
{
    int count = -1;
    const int st = guard([&] {
        check_ctx(c);
        if (!name || !in) throw Error(CAPAC_ERR_INVALID, "null argument");
        std::string n(name);
        CAPAC_CUDA(cudaStreamSynchronize(c->stream));
        if (n == "wait_polls") {  // the persistent solver's grid-barrier poll limit (0: the default)
            if (!(in[0] >= 0.0 && in[0] <= 2147483647.0)) throw Error(CAPAC_ERR_INVALID, "wait_polls out of range");
            c->opt.wait_polls = (int)in[0];
            count = 1;
            return;
        }
        int cnt = 0;
        double *p = state_array(c, n, &cnt);
        if (!p || n == "inv_sqrt_dens" || n == "diag_relay" || n.rfind("adjoint_", 0) == 0)
            throw Error(CAPAC_ERR_INVALID, "array " + n + " cannot be set");
        if (cnt > 0) CAPAC_CUDA(cudaMemcpy(p, in, sizeof(double) * cnt, cudaMemcpyHostToDevice));
        if (n == "rx" || n == "ry" || n == "rz" || n == "vec_pq") c->grad_ready = false;
        if (n == "rx" || n == "ry" || n == "rz") c->list_valid = false;
        if (n == "vec_pq") c->n_solves = 0;  // a new warm start restarts the predictor history
        if (n == "rx" || n == "ry" || n == "rz") c->precond_age = 0;  // new positions: fresh preconditioner
        count = cnt;
    });
    return st == CAPAC_OK ? count : st;
}

int capac_get_stats(capac_ctx *c, capac_stats *out)
{
    return guard([&] {
        check_ctx(c);
        if (!out) throw Error(CAPAC_ERR_INVALID, "null argument");
        memset(out, 0, sizeof *out);
        out->solver_iterations = c->last_iters;
        out->solver_outer = c->last_outer;
        out->solver_rel_residual = c->last_rel_res;
        out->solver_initial_rel_residual = c->last_init_res;
        out->list_builds = c->list_builds;
        out->list_capacity = c->cpairs ? c->cp_cap : (c->clusters ? c->cl_cap : c->cap);
        out->md_step = c->md_step;
        if (c->list_valid) {
            // entries of the list the pair kernel walks: per cluster (atoms, or
            // clusters on the cluster-pair list) or per atom
            const int rows = c->clusters || c->cpairs ? c->n_clusters : c->N;
            std::vector<int> nn(rows);
            CAPAC_CUDA(cudaStreamSynchronize(c->stream));
            CAPAC_CUDA(cudaMemcpy(nn.data(), c->cpairs ? c->cp_n : (c->clusters ? c->cl_nnb : c->nnb),
                                  sizeof(int) * rows, cudaMemcpyDeviceToHost));
            long tot = 0, mx = 0;
            for (int v : nn) {
                tot += v;
                mx = std::max<long>(mx, v);
            }
            out->list_entries = tot;
            out->max_neighbors = mx;
        }
    });
}

int capac_pair_fingerprint(capac_ctx *c, int from_list, long *count, unsigned long long *hash)
{
    return guard([&] {
        check_ctx(c);
        if (!count || !hash) throw Error(CAPAC_ERR_INVALID, "null argument");
        launch_pair_fingerprint(c, from_list, count, hash);
    });
}

int capac_phase_times(capac_ctx *c, double out_ms[15])
{
    return guard([&] {
        check_ctx(c);
        CAPAC_CUDA(cudaStreamSynchronize(c->stream));
        for (int k = 0; k < 15; ++k) out_ms[k] = 0.0;
        auto span = [&](int a, int b) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, c->ev[a], c->ev[b]) != cudaSuccess) return 0.0;
            return (double)ms;
        };
        out_ms[10] = span(0, 1);  // list maintenance and packing
        out_ms[1] = span(1, 2);   // Sutton-Chen density + force
        out_ms[6] = span(2, 3);   // CPIM vector
        out_ms[5] = span(3, 4);   // CPIM matrix
        out_ms[7] = span(4, 5);   // CPIM solve
        out_ms[4] = span(5, 6);   // nonbonded (+ water side of CPIM)
        out_ms[8] = span(6, 7);   // CPIM force, external field
        out_ms[0] = span(0, 7);
    });
}

long capac_kernel_launches(capac_ctx *c) { return c ? c->launches : 0; }

int capac_time_md_steps(capac_ctx *c, int n, double *ms)
{
    return guard([&] {
        check_ctx(c);
        if (!ms || n < 0) throw Error(CAPAC_ERR_INVALID, "bad argument");
        CAPAC_CUDA(cudaEventRecord(c->ev[14], c->stream));
        for (int k = 0; k < n; ++k) md_step(c);
        CAPAC_CUDA(cudaEventRecord(c->ev[15], c->stream));
        CAPAC_CUDA(cudaEventSynchronize(c->ev[15]));
        float t = 0.f;
        CAPAC_CUDA(cudaEventElapsedTime(&t, c->ev[14], c->ev[15]));
        *ms = t;
        check_flags(c);
    });
}

int capac_profile_enable(capac_ctx *c, int on)
{
    return guard([&] {
        check_ctx(c);
        Profiler &p = c->prof;
        if (p.ev.empty()) {
            p.ev.resize(2 * kProfSlots);
            p.cls.resize(kProfSlots);
            for (auto &e : p.ev) CAPAC_CUDA(cudaEventCreate(&e));
        }
        prof_flush(c);
        for (int k = 0; k < K_NCLASS; ++k) {
            p.count[k] = 0;
            p.ms[k] = 0.0;
        }
        p.spmv_effective = 0;
        p.on = on != 0;
    });
}

int capac_profile_get(capac_ctx *c, const char *cls, long *launches, double *total_ms)
{
    return guard([&] {
        check_ctx(c);
        if (!cls || !launches || !total_ms) throw Error(CAPAC_ERR_INVALID, "null argument");
        static const char *names[K_NCLASS] = {"pair", "spmv", "matrix", "cpim_metal", "cpim_rhs",
                                              "qsc", "list_build", "solver_vec", "integrate", "resid", "solve"};
        prof_flush(c);
        if (0 == strcmp(cls, "spmv_effective")) {
            *launches = c->prof.spmv_effective;
            *total_ms = 0.0;
            return;
        }
        for (int k = 0; k < K_NCLASS; ++k) {
            if (0 == strcmp(cls, names[k])) {
                *launches = c->prof.count[k];
                *total_ms = c->prof.ms[k];
                return;
            }
        }
        throw Error(CAPAC_ERR_INVALID, std::string("unknown kernel class ") + cls);
    });
}

}  // extern "C"
