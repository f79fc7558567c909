// CPIM BiCGSTAB solve that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host code that hands all device
// memory to its own pool at start-up and forbids later allocations, or a
// per-time-step caller for which an allocation (which may synchronise the
// device) is not acceptable.  This entry point serves them: the caller passes
// the matrix, right-hand side, diagonal and solution vector (all device
// memory it owns), and the solver's own work space lives in one file-scope
// static device array of fixed size, reserved when the library is loaded on
// a device and held by every device that loads the library until exit.
//
// The algorithm is the same Jacobi-preconditioned BiCGSTAB as the context
// solver (bicg_stab.c:253-573): warm start from x, stop when
// rTr < tol * bTb, accept 100x that after MAX_ITER iterations (with the
// reference's note on stderr).  A breakdown (a zero or non-finite alpha or
// omega, which the reference does not guard) leaves x at its last finite value
// and restarts from there with a fresh shadow residual, up to eight starts, as
// the context solver does.
#include <cstdio>
#include <mutex>
#include <string>

#include "ctx.h"

namespace capac {

namespace {

// Largest system the static work space holds: n_mat = 4 * n_metal + n_nps.
constexpr int kStaticMaxN = 16384;
constexpr int kStaticMaxNps = 16;
constexpr int kStaticBlock = 256;
constexpr int kStaticMaxRowBlocks = kStaticMaxN / 4 + kStaticMaxNps;        // SpMV blocks
constexpr int kStaticMaxVecBlocks = (kStaticMaxN + kStaticBlock - 1) / kStaticBlock;

// Layout of the work space, in doubles.
constexpr int kVecs = 9;  // r0 r p v s t y z K
constexpr size_t kOffVec = 0;
constexpr size_t kOffPart = kOffVec + (size_t)kVecs * kStaticMaxN;
constexpr size_t kPartDoubles = 2 * (size_t)(kStaticMaxRowBlocks > kStaticMaxVecBlocks ? kStaticMaxRowBlocks
                                                                                        : kStaticMaxVecBlocks);
constexpr size_t kOffScal = kOffPart + kPartDoubles;
constexpr size_t kScalDoubles = 16;
constexpr size_t kOffNp = kOffScal + kScalDoubles;  // 2 * kStaticMaxNps ints stored in doubles' space
constexpr size_t kScratchDoubles = kOffNp + kStaticMaxNps;  // 16 doubles hold 32 ints

// The solver's work space: about 1.2 MB per device.  Every call shares it and
// it keeps the last call's contents, so calls that overlap on the GPU (on two
// streams, or from two host threads) race; serialise them.
static __device__ __align__(256) double g_solve_scratch[kScratchDoubles];

struct Scal {  // lives at kOffScal
    double bTb, crit, rho, rho_old, alpha, omega, rTr, skip;
    int iter, done, status, pad2;  // status: 0 ok, 1 loosened criterion, -1 failed, -2 breakdown
};
static_assert(sizeof(Scal) <= kScalDoubles * sizeof(double), "scalar block too small");

enum { V_R0 = 0, V_R, V_P, V_V, V_S, V_T, V_Y, V_Z, V_K };

struct Sys {
    const double *mat;
    int M, Mp, n, n_nps;
};

__device__ __forceinline__ Scal *scal(double *ws) { return reinterpret_cast<Scal *>(ws + kOffScal); }
__device__ __forceinline__ const int *np_ranges(const double *ws) { return reinterpret_cast<const int *>(ws + kOffNp); }

__device__ __forceinline__ void sum2(const double *part, int nb, double *sh, double &a, double &b)
{
    double v[2] = {0.0, 0.0};
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        v[0] += part[2 * k];
        v[1] += part[2 * k + 1];
    }
    block_sum<2>(v, sh);
    a = v[0];
    b = v[1];
}

// y = A x; DOT 1: partial (d1, y); DOT 2: Kt = K y, partials (Kt, d1), (Kt, Kt).
template <int DOT>
__global__ void __launch_bounds__(kStaticBlock) ks_spmv(Sys S, double *ws, const double *__restrict__ x,
                                                        double *__restrict__ y, const double *__restrict__ d1,
                                                        const double *__restrict__ K)
{
    __shared__ double sh[32 * 4];
    if (scal(ws)->done) return;
    double *part = ws + kOffPart;
    const int *npr = np_ranges(ws);
    const int M = S.M, b = blockIdx.x;
    if (b < M) {
        const double *row = S.mat + (size_t)b * 16 * S.Mp;
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int j = threadIdx.x; j < M; j += blockDim.x) {
            const double xv[4] = {x[3 * j], x[3 * j + 1], x[3 * j + 2], x[3 * M + j]};
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r] += row[(size_t)(4 * r + c) * S.Mp + j] * xv[c];
        }
        block_sum<4>(acc, sh);
        if (threadIdx.x == 0) {
            for (int k = 0; k < S.n_nps; ++k)
                if (b >= npr[2 * k] && b <= npr[2 * k + 1]) acc[3] += x[4 * M + k];
            const int rows[4] = {3 * b, 3 * b + 1, 3 * b + 2, 3 * M + b};
            double p0 = 0.0, p1 = 0.0;
            for (int r = 0; r < 4; ++r) {
                y[rows[r]] = acc[r];
                if (DOT == 1) p0 += d1[rows[r]] * acc[r];
                if (DOT == 2) {
                    const double kt = K[rows[r]] * acc[r];
                    p0 += kt * d1[rows[r]];
                    p1 += kt * kt;
                }
            }
            part[2 * b] = p0;
            part[2 * b + 1] = p1;
        }
    } else {
        const int k = b - M;
        double acc[1] = {0.0};
        for (int a = npr[2 * k] + threadIdx.x; a <= npr[2 * k + 1]; a += blockDim.x) acc[0] += x[3 * M + a];
        block_sum<1>(acc, sh);
        if (threadIdx.x == 0) {
            const int r = 4 * M + k;
            y[r] = acc[0];
            part[2 * b] = DOT == 0 ? 0.0 : acc[0] * d1[r];
            part[2 * b + 1] = DOT == 2 ? acc[0] * acc[0] : 0.0;
        }
    }
}

__global__ void __launch_bounds__(kStaticBlock) ks_dot_bb(int n, const double *__restrict__ b, double *ws)
{
    __shared__ double sh[64];
    double v[2] = {0.0, 0.0};
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) v[0] = b[k] * b[k];
    block_sum<2>(v, sh);
    if (threadIdx.x == 0) {
        ws[kOffPart + 2 * blockIdx.x] = v[0];
        ws[kOffPart + 2 * blockIdx.x + 1] = 0.0;
    }
}

// bTb, criterion and the reference's zero right-hand-side exit (bicg_stab.c:
// 296-303); `skip` is that exit's threshold: 1e-10 on the first start, only an
// exact zero on a restart after a breakdown.
__global__ void ks_start(int nb, double tol, double skip, double *ws)
{
    __shared__ double sh[64];
    double a, b;
    sum2(ws + kOffPart, nb, sh, a, b);
    if (threadIdx.x == 0) {
        Scal *s = scal(ws);
        s->bTb = a;
        s->crit = a * tol;
        s->rho_old = s->alpha = s->omega = 1.0;
        s->rho = s->rTr = 0.0;
        s->skip = skip;
        s->iter = 0;
        s->status = 0;
        s->done = a < skip ? 1 : 0;
    }
}

// Status of a breakdown: the last residual judged like the MAX_ITER fallback
// (accepted within 100x the criterion), else -2, a restart from the current x.
__device__ __forceinline__ int ks_breakdown_status(const Scal *s) { return s->rTr < s->crit * 100.0 ? 1 : -2; }

// r0 = r = b - A x (A x left in t), p = v = 0, K = 1/diag (1 on Lagrange rows)
__global__ void __launch_bounds__(kStaticBlock) ks_init(int n, int n4, const double *__restrict__ b,
                                                        const double *__restrict__ diag, double *ws)
{
    __shared__ double sh[64];
    if (scal(ws)->done) return;
    double *V = ws + kOffVec;
    double v[2] = {0.0, 0.0};
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) {
        const double r = b[k] - V[V_T * kStaticMaxN + k];
        V[V_R0 * kStaticMaxN + k] = r;
        V[V_R * kStaticMaxN + k] = r;
        V[V_P * kStaticMaxN + k] = 0.0;
        V[V_V * kStaticMaxN + k] = 0.0;
        V[V_K * kStaticMaxN + k] = k < n4 ? 1.0 / diag[k] : 1.0;
        v[0] = r * r;
    }
    block_sum<2>(v, sh);
    if (threadIdx.x == 0) {
        ws[kOffPart + 2 * blockIdx.x] = v[0];
        ws[kOffPart + 2 * blockIdx.x + 1] = 0.0;
    }
}

__global__ void ks_rho0(int nb, double *ws)
{
    __shared__ double sh[64];
    if (scal(ws)->done) return;
    double a, b;
    sum2(ws + kOffPart, nb, sh, a, b);
    if (threadIdx.x == 0) scal(ws)->rho = scal(ws)->rTr = a;  // (r0, r0) = (r, r) at the start
}

__global__ void __launch_bounds__(kStaticBlock) ks_p(int n, double *ws)
{
    Scal *s = scal(ws);
    if (s->done) return;
    if (s->iter == 0 && s->rho < s->skip) {
        if (blockIdx.x == 0 && threadIdx.x == 0) s->done = 1;
        return;
    }
    const double beta = (s->rho / s->rho_old) * (s->alpha / s->omega), om = s->omega;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double *V = ws + kOffVec;
    const double p = V[V_R * kStaticMaxN + k] + beta * (V[V_P * kStaticMaxN + k] - om * V[V_V * kStaticMaxN + k]);
    V[V_P * kStaticMaxN + k] = p;
    V[V_Y * kStaticMaxN + k] = p * V[V_K * kStaticMaxN + k];
}

__global__ void ks_alpha(int nb, double *ws)
{
    __shared__ double sh[64];
    if (scal(ws)->done) return;
    double a, b;
    sum2(ws + kOffPart, nb, sh, a, b);
    if (threadIdx.x == 0) {
        Scal *s = scal(ws);
        const double al = s->rho / a;
        if (isfinite(al)) {
            s->alpha = al;
        } else {  // breakdown: x keeps its last finite value
            s->done = 1;
            s->status = ks_breakdown_status(s);
        }
    }
}

__global__ void __launch_bounds__(kStaticBlock) ks_s(int n, double *ws)
{
    const Scal *s = scal(ws);
    if (s->done) return;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double *V = ws + kOffVec;
    const double v = V[V_R * kStaticMaxN + k] - s->alpha * V[V_V * kStaticMaxN + k];
    V[V_S * kStaticMaxN + k] = v;
    V[V_Z * kStaticMaxN + k] = v * V[V_K * kStaticMaxN + k];
}

__global__ void ks_omega(int nb, double *ws)
{
    __shared__ double sh[64];
    if (scal(ws)->done) return;
    double a, b;
    sum2(ws + kOffPart, nb, sh, a, b);
    if (threadIdx.x == 0) {
        Scal *s = scal(ws);
        const double om = a / b;
        if (isfinite(om) && om != 0.0) {
            s->omega = om;
        } else {  // breakdown before x is touched
            s->done = 1;
            s->status = ks_breakdown_status(s);
        }
    }
}

__global__ void __launch_bounds__(kStaticBlock) ks_x(int n, double *ws, double *__restrict__ x)
{
    __shared__ double sh[64];
    const Scal *s = scal(ws);
    if (s->done) return;
    double *V = ws + kOffVec;
    double v[2] = {0.0, 0.0};
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) {
        x[k] += s->alpha * V[V_Y * kStaticMaxN + k] + s->omega * V[V_Z * kStaticMaxN + k];
        const double r = V[V_S * kStaticMaxN + k] - s->omega * V[V_T * kStaticMaxN + k];
        V[V_R * kStaticMaxN + k] = r;
        v[0] = r * r;
        v[1] = V[V_R0 * kStaticMaxN + k] * r;
    }
    block_sum<2>(v, sh);
    if (threadIdx.x == 0) {
        ws[kOffPart + 2 * blockIdx.x] = v[0];
        ws[kOffPart + 2 * blockIdx.x + 1] = v[1];
    }
}

__global__ void ks_check(int nb, double *ws)
{
    __shared__ double sh[64];
    Scal *s = scal(ws);
    if (s->done) return;
    double rTr, r0r;
    sum2(ws + kOffPart, nb, sh, rTr, r0r);
    if (threadIdx.x == 0) {
        s->rho_old = s->rho;
        s->rho = r0r;
        s->rTr = rTr;
        s->iter += 1;
        if (rTr < s->crit) {
            s->done = 1;
        } else if (s->iter > kMaxIter) {
            s->done = 1;
            s->status = rTr < s->crit * 100.0 ? 1 : -1;
        }
    }
}

// Device address of the work space, looked up once per device.
std::mutex g_addr_mutex;
double *g_addr[64] = {};

double *scratch_address()
{
    int dev = 0;
    CAPAC_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw Error(CAPAC_ERR_INVALID, "device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (!g_addr[dev]) {
        double *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_solve_scratch);
        if (e != cudaSuccess || !p)
            throw Error(CAPAC_ERR_CUDA, std::string("cudaGetSymbolAddress of the solver work space failed: ") +
                                            cudaGetErrorString(e));
        g_addr[dev] = p;
    }
    return g_addr[dev];
}

}  // namespace

}  // namespace capac

using namespace capac;

extern "C" int capac_bicgstab_static(const double *mat, int n_metal, int mat_stride, int n_nps,
                                     const int *np_start, const int *np_end, const double *rhs,
                                     const double *diag, double *x, double tol, int *iterations, void *stream)
{
    return guard([&] {
        if (!mat || !rhs || !diag || !x) throw Error(CAPAC_ERR_INVALID, "null device pointer");
        if (n_metal <= 0) throw Error(CAPAC_ERR_INVALID, "n_metal must be positive");
        if (mat_stride < n_metal) throw Error(CAPAC_ERR_INVALID, "mat_stride smaller than n_metal");
        if (n_nps < 0 || n_nps > kStaticMaxNps)
            throw Error(CAPAC_ERR_CAPACITY, "n_nps above the static solver's limit of " + std::to_string(kStaticMaxNps));
        const long n = 4L * n_metal + n_nps;
        if (n > kStaticMaxN)
            throw Error(CAPAC_ERR_CAPACITY, "system of " + std::to_string(n) +
                                                " unknowns exceeds the static solver's limit of " +
                                                std::to_string(kStaticMaxN) + " (4*n_metal + n_nps)");
        if (n_nps > 0 && (!np_start || !np_end)) throw Error(CAPAC_ERR_INVALID, "null nanoparticle ranges");
        int ranges[2 * kStaticMaxNps] = {0};
        for (int k = 0; k < n_nps; ++k) {
            if (np_start[k] < 0 || np_end[k] >= n_metal || np_start[k] > np_end[k])
                throw Error(CAPAC_ERR_INVALID, "nanoparticle range outside 0..n_metal-1");
            ranges[2 * k] = np_start[k];
            ranges[2 * k + 1] = np_end[k];
        }
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        double *ws = scratch_address();
        CAPAC_CUDA(cudaMemcpyAsync(ws + kOffNp, ranges, sizeof ranges, cudaMemcpyHostToDevice, s));
        const Sys S{mat, n_metal, mat_stride, (int)n, n_nps};
        const int nbv = (int)grid_for(n, kStaticBlock), nbm = n_metal + n_nps;
        double *V = ws + kOffVec;
        auto vec = [&](int k) { return V + (size_t)k * kStaticMaxN; };
        const double crit = tol > 0.0 ? tol : 1.0e-8;
        struct {
            double v[kScalDoubles];
        } host{};
        // One start from the current x: r0 = r = b - A x, then chunks of four
        // iterations until the scalar block says done.
        auto solve_from_x = [&](double skip) {
            // the scalar block must start clean: a previous call leaves its state
            CAPAC_CUDA(cudaMemsetAsync(ws + kOffScal, 0, sizeof(double) * kScalDoubles, s));
            ks_dot_bb<<<nbv, kStaticBlock, 0, s>>>((int)n, rhs, ws);
            ks_start<<<1, kStaticBlock, 0, s>>>(nbv, crit, skip, ws);
            ks_spmv<0><<<nbm, kStaticBlock, 0, s>>>(S, ws, x, vec(V_T), nullptr, nullptr);
            ks_init<<<nbv, kStaticBlock, 0, s>>>((int)n, 4 * n_metal, rhs, diag, ws);
            ks_rho0<<<1, kStaticBlock, 0, s>>>(nbv, ws);
            CAPAC_CUDA(cudaGetLastError());
            const int chunk = 4;
            for (int it = 0; it <= kMaxIter + chunk; it += chunk) {
                for (int q = 0; q < chunk; ++q) {
                    ks_p<<<nbv, kStaticBlock, 0, s>>>((int)n, ws);
                    ks_spmv<1><<<nbm, kStaticBlock, 0, s>>>(S, ws, vec(V_Y), vec(V_V), vec(V_R0), nullptr);
                    ks_alpha<<<1, kStaticBlock, 0, s>>>(nbm, ws);
                    ks_s<<<nbv, kStaticBlock, 0, s>>>((int)n, ws);
                    ks_spmv<2><<<nbm, kStaticBlock, 0, s>>>(S, ws, vec(V_Z), vec(V_T), vec(V_Z), vec(V_K));
                    ks_omega<<<1, kStaticBlock, 0, s>>>(nbm, ws);
                    ks_x<<<nbv, kStaticBlock, 0, s>>>((int)n, ws, x);
                    ks_check<<<1, kStaticBlock, 0, s>>>(nbv, ws);
                }
                CAPAC_CUDA(cudaGetLastError());
                CAPAC_CUDA(cudaMemcpyAsync(host.v, ws + kOffScal, sizeof host.v, cudaMemcpyDeviceToHost, s));
                CAPAC_CUDA(cudaStreamSynchronize(s));
                if (reinterpret_cast<const Scal *>(host.v)->done) break;
            }
            return *reinterpret_cast<const Scal *>(host.v);
        };
        Scal sc = solve_from_x(1.0e-10);
        int iters = sc.iter, starts = 1;
        while (sc.done && sc.status == -2 && starts < 8) {
            sc = solve_from_x(1.0e-300);  // not the reference's first start: only an exact zero exits
            iters += sc.iter;
            ++starts;
        }
        if (iterations) *iterations = iters;
        if (!sc.done || sc.status < 0) {
            char msg[160];
            snprintf(msg, sizeof msg, "Error: bicg_stab not converged. rTr= %e, bTb= %e", sc.rTr, sc.bTb);
            throw Error(CAPAC_ERR_NOT_CONVERGED, msg);
        }
        if (sc.status == 1) fprintf(stderr, "Note: Loosen bicg_stab convergence criteria to 1e-6 for this step.\n");
    });
}
