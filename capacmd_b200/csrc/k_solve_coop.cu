// BiCGSTAB for the CPIM system in one persistent, cooperatively launched
// kernel (symmetric packed 4x4-block matrix, FP32 or FP64 entries).
//
// Same algorithm and stopping rules as bicgstab_core (bicg_stab.c:253-573,
// plus the breakdown guard); the host launches one kernel per solve instead of
// about ten small kernels per iteration.  Phases of one iteration, each ended
// by a grid barrier:
//   P  p = r + beta (p - omega v), y = K p
//   T  tile SpMV of y -> partials          R  v = A y, partials of (r0, v)
//   S  alpha; s = r - alpha v, z = K s
//   T  tile SpMV of z -> partials          R  t = A z, Kt, partials of (Kt, z), (Kt, Kt)
//   X  omega; x += alpha y + omega z, r = s - omega t, partials of (r, r), (r0, r)
// Every block reduces the per-block dot partials itself, in one fixed order,
// so all blocks compute bit-identical scalars and take the same branch at
// every test.
//
// The grid barrier is a counter/generation pair in global memory with a
// bounded wait: a block that polls more than 2^24 times sets the error word
// and leaves; every block checks that word after each barrier and returns,
// and the host reports the error.  The launch is cooperative, so either all
// blocks are resident or the launch fails.
#include <cooperative_groups.h>

#include "terms.cuh"

namespace capac {

namespace {

constexpr int kT = 32;
constexpr int kPlanes = 10;
constexpr size_t kTileElems = (size_t)kPlanes * kT * kT;
constexpr int kBlock = 256;
constexpr long kSpinLimit = 1L << 24;

__host__ __device__ __forceinline__ size_t tile_index(int I, int J, int nT)
{
    return (size_t)I * nT - (size_t)I * (I - 1) / 2 + (size_t)(J - I);
}
__device__ __forceinline__ size_t elem_offset(int p, int a, int b)
{
    return ((size_t)p * (kT / 4) + (b >> 2)) * (kT * 4) + (size_t)a * 4 + (b & 3);
}
__device__ __forceinline__ void load4(const float *p, double out[4])
{
    const float4 v = *reinterpret_cast<const float4 *>(p);
    out[0] = v.x; out[1] = v.y; out[2] = v.z; out[3] = v.w;
}
__device__ __forceinline__ void load4(const double *p, double out[4])
{
    const double2 u = *reinterpret_cast<const double2 *>(p);
    const double2 v = *reinterpret_cast<const double2 *>(p + 2);
    out[0] = u.x; out[1] = u.y; out[2] = v.x; out[3] = v.y;
}

}  // namespace

struct CoopBarrier {
    unsigned count;
    unsigned gen;
    int error;
    int pad;
};

struct CoopArgs {
    int M, n, n4, nT, ntiles, n_nps, metal_min, max_iter;
    double inv_polar, inv_capac;
    const int *np_start, *np_end;
    const void *mat;
    double *part;  // nT * nT * 128 tile partials
    double *bp;    // dot partials: 3 sets of 2 doubles per block
    const double *b, *diag;
    double *x;
    double *r0, *r, *p, *v, *s, *t, *y, *z, *K;
    double tol, skip;
    SolverScalars *ss;
    CoopBarrier *bar;
};

namespace {

// Bounded grid barrier; false if any block gave up waiting.
__device__ bool grid_barrier(CoopBarrier *bar)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *gen = &bar->gen;
        const unsigned g = *gen;
        __threadfence();
        const unsigned arrived = atomicAdd(&bar->count, 1u);
        if (arrived == gridDim.x - 1) {
            bar->count = 0;
            __threadfence();
            atomicAdd(&bar->gen, 1u);
        } else {
            long spins = 0;
            while (*gen == g) {
                if (++spins > kSpinLimit) {
                    atomicExch(&bar->error, 1);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        ok = *(volatile int *)&bar->error == 0;
    }
    __syncthreads();
    return ok != 0;
}

// Sum the per-block dot partials in a fixed order; every block gets the same.
__device__ void sum_bp(const double *bp, int nb, double &a, double &b)
{
    __shared__ double sh[64];
    __shared__ double out[2];
    double v[2] = {0.0, 0.0};
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        v[0] += __ldcg(bp + 2 * k);
        v[1] += __ldcg(bp + 2 * k + 1);
    }
    block_sum<2>(v, sh);
    if (threadIdx.x == 0) {
        out[0] = v[0];
        out[1] = v[1];
    }
    __syncthreads();
    a = out[0];
    b = out[1];
    __syncthreads();
}

__device__ void put_bp(double *bp, double a, double b)
{
    __shared__ double sh[64];
    double v[2] = {a, b};
    block_sum<2>(v, sh);
    if (threadIdx.x == 0) {
        bp[2 * blockIdx.x] = v[0];
        bp[2 * blockIdx.x + 1] = v[1];
    }
}

// Tile SpMV of `in` into the tile partials (as k_sym_tiles).
template <typename T>
__device__ void tiles_phase(const CoopArgs &A, const double *in)
{
    __shared__ double xr[kT][4], xc[kT][4];
    __shared__ double rowacc[8][kT][4];
    __shared__ double colacc[kT][4];
    const T *mat = static_cast<const T *>(A.mat);
    const int M = A.M;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
        int I = 0;
        while (tile_index(I + 1, I + 1, A.nT) <= (size_t)t && I + 1 < A.nT) ++I;
        const int J = I + (int)((size_t)t - tile_index(I, I, A.nT));
        {
            const int side = threadIdx.x >> 7, q = threadIdx.x & 127, at = q >> 2, comp = q & 3;
            const int atom = (side ? J : I) * kT + at;
            double val = 0.0;
            if (atom < M) val = __ldcg(in + (comp < 3 ? 3 * atom + comp : 3 * M + atom));
            if (side == 0) xr[at][comp] = val;
            else xc[at][comp] = val;
        }
        __syncthreads();
        const T *tile = mat + (size_t)t * kTileElems;
        const int a = lane;
        double vv[kPlanes][4];
#pragma unroll
        for (int pl = 0; pl < kPlanes; ++pl) load4(tile + elem_offset(pl, a, 4 * w), vv[pl]);
        double ra[4] = {0.0, 0.0, 0.0, 0.0};
        double cb[4][4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int b = 4 * w + k;
            const double Axx = vv[0][k], Axy = vv[1][k], Axz = vv[2][k], Ayy = vv[3][k], Ayz = vv[4][k],
                         Azz = vv[5][k], m0 = vv[6][k], m1 = vv[7][k], m2 = vv[8][k], C = vv[9][k];
            const double xb0 = xc[b][0], xb1 = xc[b][1], xb2 = xc[b][2], xb3 = xc[b][3];
            const double xa0 = xr[a][0], xa1 = xr[a][1], xa2 = xr[a][2], xa3 = xr[a][3];
            ra[0] += Axx * xb0 + Axy * xb1 + Axz * xb2 + m0 * xb3;
            ra[1] += Axy * xb0 + Ayy * xb1 + Ayz * xb2 + m1 * xb3;
            ra[2] += Axz * xb0 + Ayz * xb1 + Azz * xb2 + m2 * xb3;
            ra[3] += -(m0 * xb0 + m1 * xb1 + m2 * xb2) + C * xb3;
            cb[k][0] = Axx * xa0 + Axy * xa1 + Axz * xa2 - m0 * xa3;
            cb[k][1] = Axy * xa0 + Ayy * xa1 + Ayz * xa2 - m1 * xa3;
            cb[k][2] = Axz * xa0 + Ayz * xa1 + Azz * xa2 - m2 * xa3;
            cb[k][3] = m0 * xa0 + m1 * xa1 + m2 * xa2 + C * xa3;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int q = 0; q < 4; ++q) cb[k][q] = warp_sum(cb[k][q]);
#pragma unroll
        for (int q = 0; q < 4; ++q) rowacc[w][a][q] = ra[q];
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int q = 0; q < 4; ++q) colacc[4 * w + k][q] = cb[k][q];
        }
        __syncthreads();
        double *pr = A.part + ((size_t)I * A.nT + J) * (kT * 4);
        double *pc = A.part + ((size_t)J * A.nT + I) * (kT * 4);
        if (threadIdx.x < kT * 4) {
            const int aa = threadIdx.x >> 2, q = threadIdx.x & 3;
            double s = 0.0;
#pragma unroll
            for (int ww = 0; ww < 8; ++ww) s += rowacc[ww][aa][q];
            pr[threadIdx.x] = I == J ? s + colacc[aa][q] : s;
        } else if (I != J) {
            const int q = threadIdx.x - kT * 4;
            pc[q] = colacc[q >> 2][q & 3];
        }
        __syncthreads();
    }
}

// out = A in: sums the tile partials of each row in a fixed order (8 groups
// per output combined by shuffles), adds the diagonal block and the
// neutrality couplings.  Returns this thread's dot contributions:
//   DOT 0: (d1, out)            DOT 1: Kt = K out, (Kt, d1), (Kt, Kt)
template <int DOT>
__device__ void reduce_phase(const CoopArgs &A, const double *in, double *out, const double *d1, double &p0,
                             double &p1)
{
    const int M = A.M;
    const long nwork = (long)A.nT * 128 * 8;
    const long gthreads = (long)gridDim.x * blockDim.x;
    for (long base = 0; base < nwork; base += gthreads) {
        const long id = base + (long)blockIdx.x * blockDim.x + threadIdx.x;
        double s = 0.0;
        const int g = (int)(id & 7), o = (int)((id >> 3) & 127), I = (int)(id >> 10);
        if (id < nwork) {
            const double *src = A.part + (size_t)I * A.nT * (kT * 4) + o;
            for (int Kk = g; Kk < A.nT; Kk += 8) s += __ldcg(src + (size_t)Kk * (kT * 4));
        }
        s += __shfl_xor_sync(0xffffffffu, s, 1);
        s += __shfl_xor_sync(0xffffffffu, s, 2);
        s += __shfl_xor_sync(0xffffffffu, s, 4);
        if (id < nwork && g == 0) {
            const int atom = I * kT + (o >> 2), comp = o & 3;
            if (atom < M) {
                const int row = comp < 3 ? 3 * atom + comp : 3 * M + atom;
                const double xin = __ldcg(in + row);
                if (comp < 3) {
                    s += A.inv_polar * xin;
                } else {
                    s += -A.inv_capac * xin;
                    const int im = A.metal_min + atom;
                    for (int k = 0; k < A.n_nps; ++k)
                        if (im >= A.np_start[k] && im <= A.np_end[k]) s += __ldcg(in + 4 * M + k);
                }
                out[row] = s;
                if (DOT == 0) p0 += __ldcg(d1 + row) * s;
                if (DOT == 1) {
                    const double kt = __ldcg(A.K + row) * s;
                    p0 += kt * __ldcg(d1 + row);
                    p1 += kt * kt;
                }
            }
        }
    }
    // Lagrange rows: sum of the NP's charges of `in`
    for (int k = blockIdx.x; k < A.n_nps; k += gridDim.x) {
        __shared__ double sh[32];
        double acc[1] = {0.0};
        for (int at = A.np_start[k] + threadIdx.x; at <= A.np_end[k]; at += blockDim.x)
            acc[0] += __ldcg(in + 3 * M + (at - A.metal_min));
        block_sum<1>(acc, sh);
        if (threadIdx.x == 0) {
            const int row = 4 * M + k;
            out[row] = acc[0];
            if (DOT == 0) p0 += __ldcg(d1 + row) * acc[0];
            if (DOT == 1) {
                p0 += acc[0] * __ldcg(d1 + row);  // K = 1 on Lagrange rows
                p1 += acc[0] * acc[0];
            }
        }
        __syncthreads();
    }
}

template <typename T>
__global__ void __launch_bounds__(kBlock) k_bicgstab_coop(CoopArgs A)
{
    SolverScalars *ss = A.ss;
    const int n = A.n;
    const long gthreads = (long)gridDim.x * blockDim.x;
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nb = gridDim.x;
    // Separate partial sets per dot kind: a block may write the x/r partials
    // while a slower block still reads the omega partials (no barrier lies
    // between those two phases).
    double *bpV = A.bp, *bpT = A.bp + 2 * nb, *bpX = A.bp + 4 * nb;
    double a1;

    // start: bTb, Ax0, r0 = r = b - A x, p = v = 0, K
    {
        double pb = 0.0;
        for (long k = tid; k < n; k += gthreads) {
            const double bk = A.b[k];
            pb += bk * bk;
            A.K[k] = k < A.n4 ? 1.0 / A.diag[k] : 1.0;
        }
        put_bp(bpX, pb, 0.0);
    }
    if (!grid_barrier(A.bar)) return;
    double bTb;
    sum_bp(bpX, nb, bTb, a1);
    const double crit = bTb * A.tol;
    if (bTb < A.skip) {
        if (tid == 0) {
            ss->bTb = bTb;
            ss->iter = 0;
            ss->done = 1;
            ss->status = 0;
            ss->rTr = 0.0;
            ss->rr0 = 0.0;
        }
        return;
    }
    tiles_phase<T>(A, A.x);
    if (!grid_barrier(A.bar)) return;
    {
        double q0 = 0.0, q1 = 0.0;
        reduce_phase<2>(A, A.x, A.t, nullptr, q0, q1);  // t = A x (no dots)
    }
    if (!grid_barrier(A.bar)) return;
    {
        double pr = 0.0;
        for (long k = tid; k < n; k += gthreads) {
            const double rk = A.b[k] - __ldcg(A.t + k);
            A.r0[k] = rk;
            A.r[k] = rk;
            A.p[k] = 0.0;
            A.v[k] = 0.0;
            pr += rk * rk;
        }
        put_bp(bpX, pr, 0.0);
    }
    if (!grid_barrier(A.bar)) return;
    double rho;
    sum_bp(bpX, nb, rho, a1);
    double rTr = rho, rr0 = rho, rho_old = 1.0, alpha = 1.0, omega = 1.0;
    int iter = 0, status = 0, done = 0;
    if (rho < A.skip) done = 1;  // warm start already converged (bicg_stab.c:368)

    while (!done) {
        // P
        const double beta = (rho / rho_old) * (alpha / omega);
        for (long k = tid; k < n; k += gthreads) {
            const double pk = __ldcg(A.r + k) + beta * (__ldcg(A.p + k) - omega * __ldcg(A.v + k));
            A.p[k] = pk;
            A.y[k] = pk * __ldcg(A.K + k);
        }
        if (!grid_barrier(A.bar)) return;
        tiles_phase<T>(A, A.y);
        if (!grid_barrier(A.bar)) return;
        {
            double q0 = 0.0, q1 = 0.0;
            reduce_phase<0>(A, A.y, A.v, A.r0, q0, q1);
            put_bp(bpV, q0, 0.0);
        }
        if (!grid_barrier(A.bar)) return;
        // S
        double r0v;
        sum_bp(bpV, nb, r0v, a1);
        const double al = rho / r0v;
        if (!isfinite(al)) {
            status = rTr < crit * 100.0 ? 1 : -2;
            break;
        }
        alpha = al;
        for (long k = tid; k < n; k += gthreads) {
            const double sk = __ldcg(A.r + k) - alpha * __ldcg(A.v + k);
            A.s[k] = sk;
            A.z[k] = sk * __ldcg(A.K + k);
        }
        if (!grid_barrier(A.bar)) return;
        tiles_phase<T>(A, A.z);
        if (!grid_barrier(A.bar)) return;
        {
            double q0 = 0.0, q1 = 0.0;
            reduce_phase<1>(A, A.z, A.t, A.z, q0, q1);
            put_bp(bpT, q0, q1);
        }
        if (!grid_barrier(A.bar)) return;
        // X
        double ktz, ktkt;
        sum_bp(bpT, nb, ktz, ktkt);
        const double om = ktz / ktkt;
        if (!isfinite(om) || om == 0.0) {
            status = rTr < crit * 100.0 ? 1 : -2;
            break;
        }
        omega = om;
        {
            double q0 = 0.0, q1 = 0.0;
            for (long k = tid; k < n; k += gthreads) {
                A.x[k] += alpha * __ldcg(A.y + k) + omega * __ldcg(A.z + k);
                const double rk = __ldcg(A.s + k) - omega * __ldcg(A.t + k);
                A.r[k] = rk;
                q0 += rk * rk;
                q1 += __ldcg(A.r0 + k) * rk;
            }
            put_bp(bpX, q0, q1);
        }
        if (!grid_barrier(A.bar)) return;
        double r0r;
        sum_bp(bpX, nb, rTr, r0r);
        rho_old = rho;
        rho = r0r;
        ++iter;
        if (rTr < crit) {
            done = 1;
        } else if (iter > A.max_iter) {
            status = rTr < crit * 100.0 ? 1 : -1;
            done = 1;
        }
    }
    if (tid == 0) {
        ss->bTb = bTb;
        ss->crit = crit;
        ss->rTr = rTr;
        ss->rr0 = rr0;
        ss->iter = iter;
        ss->done = 1;
        ss->status = status;
    }
}

}  // namespace

size_t coop_barrier_bytes() { return sizeof(CoopBarrier); }

// Launch the persistent solver; returns the status as bicgstab_core does.
int bicgstab_coop(capac_ctx *c, const double *b, double *x, double tol, double skip)
{
    const int n = c->n_mat;
    double *bw = c->bw;
    auto W = [&](int k) { return bw + (size_t)k * n; };
    CoopArgs A;
    A.M = c->M;
    A.n = n;
    A.n4 = 4 * c->M;
    A.nT = sym_tiles(c->M);
    A.ntiles = A.nT * (A.nT + 1) / 2;
    A.n_nps = c->n_nps;
    A.metal_min = c->P.metal_min;
    A.max_iter = kMaxIter;
    A.inv_polar = c->P.inv_polar;
    A.inv_capac = c->P.inv_capac;
    A.np_start = c->np_start;
    A.np_end = c->np_end;
    A.mat = c->msym;
    A.part = c->sympart;
    A.bp = c->coop_bp;
    A.b = b;
    A.diag = c->diag;
    A.x = x;
    // work vectors: slots of bw (Ax slot reused for t's start value)
    A.r0 = W(1); A.r = W(2); A.p = W(3); A.v = W(4); A.s = W(5); A.t = W(6); A.y = W(7); A.z = W(8);
    A.K = W(10);
    A.tol = tol;
    A.skip = skip;
    A.ss = c->ss;
    A.bar = reinterpret_cast<CoopBarrier *>(c->coop_bar);
    CAPAC_CUDA(cudaMemsetAsync(c->coop_bar, 0, sizeof(CoopBarrier), c->stream));
    void *args[] = {&A};
    {
        ProfScope ps(c, K_SOLVE);
        if (c->opt.precision == CAPAC_PREC_MIXED)
            CAPAC_CUDA(cudaLaunchCooperativeKernel((const void *)k_bicgstab_coop<float>, dim3(c->coop_grid),
                                                   dim3(kBlock), args, 0, c->stream));
        else
            CAPAC_CUDA(cudaLaunchCooperativeKernel((const void *)k_bicgstab_coop<double>, dim3(c->coop_grid),
                                                   dim3(kBlock), args, 0, c->stream));
    }
    ++c->launches;
    CAPAC_CUDA(cudaMemcpyAsync(c->h_ss, c->ss, sizeof(SolverScalars), cudaMemcpyDeviceToHost, c->stream));
    CoopBarrier hb;
    CAPAC_CUDA(cudaMemcpyAsync(&hb, c->coop_bar, sizeof hb, cudaMemcpyDeviceToHost, c->stream));
    CAPAC_CUDA(cudaStreamSynchronize(c->stream));
    if (hb.error) throw Error(CAPAC_ERR_CUDA, "solver grid barrier timed out");
    if (c->prof.on && c->h_ss->bTb >= skip) c->prof.spmv_effective += 1 + 2L * c->h_ss->iter;
    if (c->h_ss->status < 0) return CAPAC_ERR_NOT_CONVERGED;
    return c->h_ss->status == 1 ? 1 : CAPAC_OK;
}

// Largest co-resident grid for the persistent solver (0 if unsupported).
int coop_grid_size(int device, bool mixed)
{
    int coop = 0;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) != cudaSuccess || !coop) return 0;
    int sms = 0;
    CAPAC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    int per_sm = 0;
    if (mixed)
        CAPAC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bicgstab_coop<float>, kBlock, 0));
    else
        CAPAC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bicgstab_coop<double>, kBlock, 0));
    if (per_sm <= 0) return 0;
    return sms * std::min(per_sm, 2);
}

}  // namespace capac
