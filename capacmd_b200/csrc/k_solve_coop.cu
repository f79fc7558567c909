// BiCGSTAB for the CPIM system in one persistent, cooperatively launched
// kernel on the symmetric packed 4x4-block matrix (FP32 or FP64 entries).
//
// Same algorithm and stopping rules as bicgstab_core (bicg_stab.c:253-573,
// with the breakdown guard); the host launches one kernel per solve instead
// of about ten small kernels per iteration.  Two blocks per SM on the FP32
// matrix, one on the FP64 matrix.  Each block owns the tiles t = blockIdx.x
// + k * gridDim.x and streams them from HBM into a two-tile shared-memory
// ring with bulk asynchronous copies (cp.async.bulk + mbarrier); the matrix
// does not change during a solve, so the ring runs on across phases and
// iterations.  A tile takes one block barrier: its row and column sums go
// to one of two accumulator sets while the other set is written out.
//
// An iteration, with a grid barrier after each of its four phases:
//   P  tile pass of y = K p, p = r + beta (p - omega v), r = s - omega t,
//      all formed on the fly; the owner of diagonal tile (I, I) stores r, p
//      and y of block row I and applies the previous iteration's
//      x += alpha y + omega z to it
//   V  v = A y from the tile partials (fixed order), partials of (r0, v)
//   S  alpha; tile pass of z = K s, s = r - alpha v formed on the fly;
//      the diagonal-tile owner stores s and z
//   T  t = A z, Kt, partials of (Kt, z), (Kt, Kt), (r0, s), (r0, t), (s, s),
//      (s, t), (t, t): omega, rho = (r0, s - omega t) and (r, r) follow
//      without a pass of their own
// p and v are double-buffered, since blocks form y from the old p and v
// while others store the new ones.  Every block sums the per-block dot
// partials itself in one fixed order, so all blocks compute bit-identical
// scalars and take the same branch at every test.  (r, r) from the merged
// dots differs from the directly summed one by rounding only; the value
// returned is summed directly from the final residual.
//
// The mixed path with the block-Jacobi preconditioner runs a variant in the
// preconditioner's group order (k_bicgstab_group below): four grid barriers
// per iteration instead of six.
//
// Every wait is bounded.  The grid barrier (one arrival word, see
// grid_barrier) gives up after 2^24 polls (the context's wait_polls option
// when set), a ring-stage wait after 2^20 polls of at most 1 us each; either
// sets the error word and the barrier word's abort bit, the block then waits
// (bounded) for its own copies in flight and returns, the other blocks leave
// their current or next barrier at once, and the host reports the error.  The
// launch is cooperative, so either all blocks are resident or the launch
// fails.  The tiles are copied with an L2 evict-first policy (CAPAC_TILE_L2
// at context creation: 0 none, a fraction f > 0 keeps f of the lines
// evict-last), so the matrix streamed every pass leaves the vectors and
// partial sums of the reduction phases in L2.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "terms.cuh"

namespace capac {

namespace {

constexpr int kT = 32;
constexpr int kPlanes = 10;
constexpr int kTileElems = kPlanes * kT * kT;
constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;
constexpr int kCols = kT / kWarps;  // tile columns per warp
// Tile ring per block: two FP32 tiles (two blocks per SM) or two FP64 tiles
// (one block per SM).
template <typename T>
__host__ __device__ constexpr int ring_tiles_bytes()
{
    return 2 * kTileElems * (int)sizeof(T);
}
// tiles whose inputs a pass gathers at once
template <typename T>
__host__ __device__ constexpr int chunk_tiles()
{
    return 8;
}
constexpr int kGroups = 4;              // partial-sum groups per output row in the reduce phases
constexpr int kBatch = 16;              // partials one thread loads at once in the reduce phases
constexpr long kSpinLimit = 1L << 24;
constexpr long kWaitPolls = 1L << 20;
constexpr unsigned kSuspendNs = 1000;

enum { MODE_X = 0, MODE_P = 1, MODE_S = 2 };

__host__ __device__ __forceinline__ size_t tile_index(int I, int J, int nT)
{
    return (size_t)I * nT - (size_t)I * (I - 1) / 2 + (size_t)(J - I);
}
__device__ __forceinline__ int elem_offset(int p, int a, int b)
{
    return ((p * (kT / 4) + (b >> 2)) * (kT * 4)) + a * 4 + (b & 3);
}
// The kCols consecutive columns of one plane row (kCols = 2 or 4).
template <typename R>
__device__ __forceinline__ void ldsc(const R *p, R (&out)[kCols])
{
#pragma unroll
    for (int k = 0; k < kCols; k += 2) {
        if constexpr (sizeof(R) == 4) {
            const float2 v = *reinterpret_cast<const float2 *>(p + k);
            out[k] = v.x;
            out[k + 1] = v.y;
        } else {
            const double2 v = *reinterpret_cast<const double2 *>(p + k);
            out[k] = v.x;
            out[k + 1] = v.y;
        }
    }
}

// Sums of V values over the 32 lanes of a warp by recursive halving: at
// each step a lane keeps half of its values and adds the partner's copy of
// that half (V/2 + V/4 + ... + 1 exchanges), then plain exchanges for the
// remaining lane bits; V - 1 + 5 - log2 V shuffles instead of 5 V.  Lane l
// returns the sum of value l >> (5 - log2 V).  The order of additions is
// fixed.
template <int V, typename R>
__device__ __forceinline__ R warp_sum_halving(R (&v)[V], int lane)
{
    int m = 16;
#pragma unroll
    for (int half = V / 2; half >= 1; half >>= 1, m >>= 1) {
        const bool upper = (lane & m) != 0;
#pragma unroll
        for (int i = 0; i < half; ++i) {
            const R send = upper ? v[i] : v[i + half];
            const R keep = upper ? v[i + half] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, m);
        }
    }
    R s = v[0];
#pragma unroll
    for (; m >= 1; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m);
    return s;
}

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// One bulk copy global -> this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// The same copy with an L2 eviction-priority policy for the copied lines.
__device__ __forceinline__ void bulk_load_hint(void *dst, const void *src, unsigned bytes, uint64_t *bar,
                                               uint64_t policy)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}
// L2 policy for streamed matrix tiles: frac > 0 keeps that fraction of the
// lines at evict_last priority and marks the rest evict_first; frac < 0
// marks every line evict_first.
__device__ __forceinline__ uint64_t tile_l2_policy(float frac)
{
    uint64_t pol;
    if (frac > 0.f)
        asm volatile("createpolicy.fractional.L2::evict_last.L2::evict_first.b64 %0, %1;" : "=l"(pol) : "f"(frac));
    else
        asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(kSuspendNs)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity)
{
    for (long i = 0; i < kWaitPolls; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Tensor memory (TMEM) as storage for matrix tiles that stay on chip for a
// whole solve.  Allocation and release by one whole warp; a warp reads and
// writes only the 32 lanes of its quadrant (warp rank mod 4).
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// 40 consecutive columns of the thread's lane: one 32-column and one
// 8-column access.
__device__ __forceinline__ void tmem_st40(uint32_t taddr, const float (&v)[40])
{
    const uint32_t *u = reinterpret_cast<const uint32_t *>(v);
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};" ::"r"(taddr),
        "r"(u[0]), "r"(u[1]), "r"(u[2]), "r"(u[3]), "r"(u[4]), "r"(u[5]), "r"(u[6]), "r"(u[7]), "r"(u[8]), "r"(u[9]),
        "r"(u[10]), "r"(u[11]), "r"(u[12]), "r"(u[13]), "r"(u[14]), "r"(u[15]), "r"(u[16]), "r"(u[17]), "r"(u[18]),
        "r"(u[19]), "r"(u[20]), "r"(u[21]), "r"(u[22]), "r"(u[23]), "r"(u[24]), "r"(u[25]), "r"(u[26]), "r"(u[27]),
        "r"(u[28]), "r"(u[29]), "r"(u[30]), "r"(u[31])
        : "memory");
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr + 32),
                 "r"(u[32]), "r"(u[33]), "r"(u[34]), "r"(u[35]), "r"(u[36]), "r"(u[37]), "r"(u[38]), "r"(u[39])
                 : "memory");
}
__device__ __forceinline__ void tmem_ld40(uint32_t taddr, float (&v)[40])
{
    uint32_t *u = reinterpret_cast<uint32_t *>(v);
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7]), "=r"(u[8]),
          "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]), "=r"(u[14]), "=r"(u[15]), "=r"(u[16]),
          "=r"(u[17]), "=r"(u[18]), "=r"(u[19]), "=r"(u[20]), "=r"(u[21]), "=r"(u[22]), "=r"(u[23]), "=r"(u[24]),
          "=r"(u[25]), "=r"(u[26]), "=r"(u[27]), "=r"(u[28]), "=r"(u[29]), "=r"(u[30]), "=r"(u[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(u[32]), "=r"(u[33]), "=r"(u[34]), "=r"(u[35]), "=r"(u[36]), "=r"(u[37]), "=r"(u[38]),
                   "=r"(u[39])
                 : "r"(taddr + 32)
                 : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

}  // namespace

struct CoopSync {
    unsigned count;  // grid-barrier arrivals of the launch; bit 31: a block gave up
    unsigned unused;
    int error;  // 1 grid barrier timed out, 2 ring-stage wait timed out
    int pad;
};

struct CoopArgs {
    int M, n, n4, nT, ntiles, n_nps, metal_min, max_iter;
    long spin_limit;  // polls of a grid barrier before it gives up
    double inv_polar, inv_capac;
    const int *np_start, *np_end;
    const void *mat;
    double *part;  // nT * nT * 128 tile partials
    double *bp;    // dot partials: 2 sets of kBp doubles per block
    const double *b, *diag;
    double *x, *r0, *r, *s, *t, *y, *z, *K;
    double *p[2], *v[2];
    double tol, skip;
    SolverScalars *ss;
    CoopSync *sync;
    // block-Jacobi mode (bj != 0): K is the inverse of the diagonal blocks of
    // nG groups of 32 metal atoms; K r, K v, K t are carried as vectors and
    // y = K p, z = K s follow from them elementwise (see the kernel)
    int bj, nG;
    const int *g_atoms;
    const float *dinv;
    double *Kr, *Kv, *Kt;
    double *yb[2];
    // phase timer (null: off): block 0 records %globaltimer at the end of
    // each phase of the first kPhaseIters iterations, kPhases per iteration
    unsigned long long *ptime;
    float l2_frac;  // L2 policy of the streamed tiles (tile_l2_policy; 0: none)
};

constexpr int kPhases = 8;
constexpr int kPhaseIters = 256;

namespace {

__device__ __forceinline__ void phase_mark(const CoopArgs &A, int iter, int k)
{
    if (A.ptime && blockIdx.x == 0 && threadIdx.x == 0 && iter < kPhaseIters) {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        A.ptime[iter * kPhases + k] = t;
    }
}

// Bounded grid barrier (`limit` polls); false if any block gave up.
//
// count only grows during a launch (zeroed before it): the k-th barrier of
// the launch is complete when it reaches k * gridDim.x, so each block learns
// its target from the value its own arrival returns and then polls the same
// word, with nothing to reset and no second word to read (a block cannot
// arrive at barrier k + 1 before every block has arrived at k).  A block that
// gives up sets the error word and bit 31 of count, which ends every other
// block's wait at once.  Release: this block's writes are ordered before its
// arrival by the fence (after the block barrier); acquire: the polling load,
// then the block barrier orders the block's later reads after it.
constexpr unsigned kBarAbort = 0x80000000u;

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ bool grid_barrier(CoopSync *bar, long limit)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned arrived = atomicAdd(&bar->count, 1u);
        bool good = (arrived & kBarAbort) == 0;
        const unsigned target = ((arrived & ~kBarAbort) / gridDim.x + 1) * gridDim.x;
        long spins = 0;
        while (good) {
            const unsigned cnt = ld_acquire_gpu(&bar->count);
            if (cnt & kBarAbort) {
                good = false;
            } else if (cnt >= target) {
                break;
            } else if (++spins > limit) {
                atomicCAS(&bar->error, 0, 1);
                atomicOr(&bar->count, kBarAbort);
                good = false;
            } else {
                __nanosleep(32);
            }
        }
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// A block that stops early (a ring wait that gave up) ends the other blocks'
// barrier waits.
__device__ __forceinline__ void grid_abort(CoopSync *bar, int code)
{
    atomicCAS(&bar->error, 0, code);
    atomicOr(&bar->count, kBarAbort);
}

// Dot partials: kBp doubles per block.  sum_bp sums them over the blocks
// in one fixed order, so every block gets the same K sums.
constexpr int kBp = 16;
template <int K>
__device__ void sum_bp(const double *bp, int nb, double (&out)[K])
{
    __shared__ double sh[kWarps * kBp];
    __shared__ double res[kBp];
    double v[K];
#pragma unroll
    for (int q = 0; q < K; ++q) v[q] = 0.0;
    // two blocks' partials per thread per round of loads (the grid is at
    // most two blocks per SM, so one round covers it)
    for (int k = threadIdx.x; k < nb; k += 2 * blockDim.x) {
        const int k2 = k + (int)blockDim.x;
        double a[K], b[K];
#pragma unroll
        for (int q = 0; q < K; ++q) {
            a[q] = __ldcg(bp + (size_t)kBp * k + q);
            b[q] = k2 < nb ? __ldcg(bp + (size_t)kBp * k2 + q) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < K; ++q) v[q] += a[q] + b[q];
    }
    block_sum<K>(v, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < K; ++q) res[q] = v[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < K; ++q) out[q] = res[q];
    __syncthreads();
}

template <int K>
__device__ void put_bp(double *bp, double (&v)[K])
{
    __shared__ double sh[kWarps * kBp];
    block_sum<K>(v, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < K; ++q) bp[(size_t)kBp * blockIdx.x + q] = v[q];
}

// Scalars of the current tile pass.
struct PassScalars {
    double beta, omega, alpha;  // MODE_P: beta, and omega, alpha of the previous iteration; MODE_S: alpha
    int cur;    // p[cur], v[cur] are the old p and v (MODE_P); v[cur] is the new v (MODE_S)
    int first;  // MODE_P of the first iteration: r is stored, no update of x is pending
};

// MODE_P, one CPIM row: the residual r = s - omega t of the previous
// iteration (stored r on the first), the new p, and on `store` the row's
// deferred updates: r, and x += alpha y + omega z of the previous iteration
// (y is read before it is overwritten).  Returns the new p.
__device__ __forceinline__ double p_row(const CoopArgs &A, const PassScalars &S, int row, bool store)
{
    const double r = S.first ? __ldcg(A.r + row) : fma(-S.omega, __ldcg(A.t + row), __ldcg(A.s + row));
    const double pn = fma(S.beta, fma(-S.omega, __ldcg(A.v[S.cur] + row), __ldcg(A.p[S.cur] + row)), r);
    if (store) {
        if (!S.first) {
            A.r[row] = r;
            A.x[row] += S.alpha * __ldcg(A.y + row) + S.omega * __ldcg(A.z + row);
        }
        A.p[S.cur ^ 1][row] = pn;
    }
    return pn;
}

// The ring of tiles of one block: Stages = ring bytes / tile bytes slots;
// sequence number q -> slot q % Stages, whose k-th use waits for parity
// k & 1; tile of q = blockIdx.x + (q mod n_my) * gridDim.x.  Every thread
// counts `consumed`; thread 0 alone issues the copies and counts `issued`
// (always consumed + Stages).
template <typename T>
struct Ring {
    static constexpr int Stages = ring_tiles_bytes<T>() / (int)(kTileElems * sizeof(T));
    T *buf;
    uint64_t *bar;  // Stages mbarriers
    long issued, consumed;
    int n_my;       // tiles streamed through the ring
    int first = 0;  // tiles of the block before the streamed ones (held elsewhere)
    bool hint = false;   // copy with the L2 policy `pol`
    uint64_t pol = 0;
    __device__ int tile_of(long q) const { return blockIdx.x + (first + (int)(q % n_my)) * gridDim.x; }
    __device__ T *stage(int st) const { return buf + (size_t)st * kTileElems; }
    __device__ void set_l2(float frac)
    {
        hint = frac != 0.f;
        if (hint) pol = tile_l2_policy(frac);
    }
    __device__ void issue(const T *mat)  // thread 0
    {
        const long q = issued++;
        const int st = (int)(q % Stages);
        const T *src = mat + (size_t)tile_of(q) * kTileElems;
        if (hint)
            bulk_load_hint(stage(st), src, kTileElems * sizeof(T), bar + st, pol);
        else
            bulk_load(stage(st), src, kTileElems * sizeof(T), bar + st);
    }
    // thread 0: bounded wait for every copy still in flight
    __device__ void drain()
    {
        for (long q = consumed; q < issued; ++q) mbar_wait(bar + (q % Stages), (unsigned)((q / Stages) & 1));
        consumed = issued;
    }
};

// Block-Jacobi MODE_P, one row: with K r = z - omega K t (K r itself on the
// first iteration), y = K r + beta (y_old - omega K v); on `store` the row's
// deferred updates: r = s - omega t, K r, and x += alpha y_old + omega z of
// the previous iteration.  Returns the new y.
__device__ __forceinline__ double bj_p_row(const CoopArgs &A, const PassScalars &S, int row, bool store)
{
    const double y_old = __ldcg(A.yb[S.cur] + row);
    const double kr = S.first ? __ldcg(A.Kr + row) : fma(-S.omega, __ldcg(A.Kt + row), __ldcg(A.z + row));
    const double yn = fma(S.beta, fma(-S.omega, __ldcg(A.Kv + row), y_old), kr);
    if (store) {
        if (!S.first) {
            A.r[row] = fma(-S.omega, __ldcg(A.t + row), __ldcg(A.s + row));
            A.Kr[row] = kr;
            A.x[row] += S.alpha * y_old + S.omega * __ldcg(A.z + row);
        }
        A.yb[S.cur ^ 1][row] = yn;
    }
    return yn;
}

// Shared arrays of a tile pass (one copy for all pass kinds).  The pass
// inputs are held in the matrix's type: the products run in FP32 on the
// FP32 matrix, and every sum across columns or tiles is in FP64.
template <typename T>
struct PassSmem {
    T in[chunk_tiles<T>()][2][kT][4];  // pass inputs of the chunk's tiles: block rows I and J
    T rowacc[2][kWarps][kT][4];        // two sets: tile k + 1 fills one while tile k's is written out
    double colacc[2][kT][4];
    int tile_i[chunk_tiles<T>()], tile_j[chunk_tiles<T>()];
};

// Tile pass: partial products of the block's tiles with the pass input.
// The inputs of up to chunk_tiles<T>() tiles are gathered in one batch of
// independent loads before the tiles are processed.  Returns false when a
// ring wait timed out.
template <typename T, int MODE>
__device__ bool tiles_pass(const CoopArgs &A, const PassScalars &S, Ring<T> &ring, PassSmem<T> &sm)
{
    constexpr int Stages = Ring<T>::Stages;
    const int M = A.M;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;

    // the Lagrange rows of the stored vectors (K = 1 there)
    if (MODE != MODE_X && threadIdx.x == 0) {
        for (int k = blockIdx.x; k < A.n_nps; k += gridDim.x) {
            const int row = A.n4 + k;
            if (MODE == MODE_P) {
                if (A.bj) bj_p_row(A, S, row, true);  // K = 1 on the Lagrange rows
                else A.y[row] = p_row(A, S, row, true);
            } else {
                const double sn = fma(-S.alpha, __ldcg(A.v[S.cur] + row), __ldcg(A.r + row));
                A.s[row] = sn;
                A.z[row] = A.bj ? fma(-S.alpha, __ldcg(A.Kv + row), __ldcg(A.Kr + row)) : sn;
            }
        }
    }

    constexpr int kChunk = chunk_tiles<T>();
    for (int c0 = 0; c0 < ring.n_my; c0 += kChunk) {
        const int nc = min(kChunk, ring.n_my - c0);
        if (threadIdx.x < nc) {
            const int t = blockIdx.x + (c0 + threadIdx.x) * gridDim.x;
            int I = 0;
            while (tile_index(I + 1, I + 1, A.nT) <= (size_t)t && I + 1 < A.nT) ++I;
            sm.tile_i[threadIdx.x] = I;
            sm.tile_j[threadIdx.x] = I + (int)((size_t)t - tile_index(I, I, A.nT));
        }
        __syncthreads();
        // gather: element (tile, side, atom, comp) of the chunk's tiles
#pragma unroll 4
        for (int e = threadIdx.x; e < nc * 256; e += kBlock) {
            const int kk = e >> 8, side = (e >> 7) & 1, q4 = e & 127, at = q4 >> 2, comp = q4 & 3;
            const int I = sm.tile_i[kk], J = sm.tile_j[kk];
            const int atom = (side ? J : I) * kT + at;
            double val = 0.0;
            if (atom < M) {
                const int row = comp < 3 ? 3 * atom + comp : 3 * M + atom;
                if (MODE == MODE_X) {
                    val = __ldcg(A.x + row);
                } else if (MODE == MODE_P) {
                    const bool owner = I == J && side == 0;  // the diagonal-tile owner stores block row I
                    if (A.bj) {
                        val = bj_p_row(A, S, row, owner);
                    } else {
                        val = __dmul_rn(__ldcg(A.K + row), p_row(A, S, row, owner));
                        if (owner) A.y[row] = val;
                    }
                } else {
                    const double sn = fma(-S.alpha, __ldcg(A.v[S.cur] + row), __ldcg(A.r + row));
                    val = A.bj ? fma(-S.alpha, __ldcg(A.Kv + row), __ldcg(A.Kr + row))
                               : __dmul_rn(__ldcg(A.K + row), sn);
                    if (I == J && side == 0) {
                        A.s[row] = sn;
                        A.z[row] = val;
                    }
                }
            }
            sm.in[kk][side][at][comp] = (T)val;
        }
        __syncthreads();

        for (int kk = 0; kk < nc; ++kk) {
            const int I = sm.tile_i[kk], J = sm.tile_j[kk];
            const int set = kk & 1;
            const long q = ring.consumed;
            const int st = (int)(q % Stages);
            const unsigned parity = (unsigned)((q / Stages) & 1);
            const bool landed = mbar_wait(ring.bar + st, parity);  // every thread, bounded
            const T *tile = ring.stage(st);
            const T(*xr)[4] = sm.in[kk][0];
            const T(*xc)[4] = sm.in[kk][1];
            // thread (row a = lane, columns b = kCols w ...): row partials of
            // a, column partials of b summed over the warp's 32 rows
            const int a = lane;
            T ra[4] = {0, 0, 0, 0};
            T cb[kCols * 4];
            const T xa0 = xr[a][0], xa1 = xr[a][1], xa2 = xr[a][2], xa3 = xr[a][3];
            if (landed) {
                T vv[kPlanes][kCols];
#pragma unroll
                for (int pl = 0; pl < kPlanes; ++pl) ldsc(tile + elem_offset(pl, a, kCols * w), vv[pl]);
#pragma unroll
                for (int k = 0; k < kCols; ++k) {
                    const int b = kCols * w + k;
                    const T Axx = vv[0][k], Axy = vv[1][k], Axz = vv[2][k], Ayy = vv[3][k], Ayz = vv[4][k],
                            Azz = vv[5][k], m0 = vv[6][k], m1 = vv[7][k], m2 = vv[8][k], C = vv[9][k];
                    const T xb0 = xc[b][0], xb1 = xc[b][1], xb2 = xc[b][2], xb3 = xc[b][3];
                    ra[0] += Axx * xb0 + Axy * xb1 + Axz * xb2 + m0 * xb3;
                    ra[1] += Axy * xb0 + Ayy * xb1 + Ayz * xb2 + m1 * xb3;
                    ra[2] += Axz * xb0 + Ayz * xb1 + Azz * xb2 + m2 * xb3;
                    ra[3] += -(m0 * xb0 + m1 * xb1 + m2 * xb2) + C * xb3;
                    cb[4 * k + 0] = Axx * xa0 + Axy * xa1 + Axz * xa2 - m0 * xa3;
                    cb[4 * k + 1] = Axy * xa0 + Ayy * xa1 + Ayz * xa2 - m1 * xa3;
                    cb[4 * k + 2] = Axz * xa0 + Ayz * xa1 + Azz * xa2 - m2 * xa3;
                    cb[4 * k + 3] = m0 * xa0 + m1 * xa1 + m2 * xa2 + C * xa3;
                }
            } else {
#pragma unroll
                for (int k = 0; k < kCols * 4; ++k) cb[k] = 0;
            }
            // lane l ends with value v = l >> (5 - log2(4 kCols)) (= 4 k + c) summed over the rows
            const T colsum = warp_sum_halving<kCols * 4>(cb, lane);
#pragma unroll
            for (int c = 0; c < 4; ++c) sm.rowacc[set][w][a][c] = ra[c];
            constexpr int kShift = 5 - (kCols == 1 ? 2 : kCols == 2 ? 3 : kCols == 4 ? 4 : 5);
            if ((lane & ((1 << kShift) - 1)) == 0) {
                const int v = lane >> kShift;
                sm.colacc[set][kCols * w + (v >> 2)][v & 3] = (double)colsum;
            }
            // one barrier per tile: the stage is free, this tile's sums are
            // complete, and the previous tile's set has been written out
            if (__syncthreads_or(!landed)) return false;
            ++ring.consumed;  // every thread keeps the same count
            if (threadIdx.x == 0) ring.issue(static_cast<const T *>(A.mat));  // the tile this slot holds next
            double *pr = A.part + ((size_t)I * A.nT + J) * (kT * 4);
            double *pc = A.part + ((size_t)J * A.nT + I) * (kT * 4);
            if (threadIdx.x < kT * 4) {
                const int aa = threadIdx.x >> 2, c = threadIdx.x & 3;
                double s = 0.0;
#pragma unroll
                for (int ww = 0; ww < kWarps; ++ww) s += (double)sm.rowacc[set][ww][aa][c];
                pr[threadIdx.x] = I == J ? s + sm.colacc[set][aa][c] : s;
            } else if (threadIdx.x < 2 * kT * 4 && I != J) {
                const int c = threadIdx.x - kT * 4;
                pc[c] = sm.colacc[set][c >> 2][c & 3];
            }
        }
        __syncthreads();  // rowacc, colacc and the chunk inputs are free again
    }
    return true;
}

enum { RED_START = 0, RED_V = 1, RED_T = 2 };

// The dot contributions of one output row (see reduce_pass).
template <int RED>
__device__ __forceinline__ void reduce_row(const CoopArgs &A, const PassScalars &S, int row, double out, double in,
                                           double Krow, double (&d)[7])
{
    if (RED == RED_START) {
        const double rk = A.b[row] - out;
        A.r0[row] = rk;
        A.r[row] = rk;
        d[0] += rk * rk;
    } else if (RED == RED_V) {
        A.v[S.cur ^ 1][row] = out;
        d[0] += __ldcg(A.r0 + row) * out;
    } else {
        A.t[row] = out;
        const double kt = Krow * out, sr = __ldcg(A.s + row), r0 = __ldcg(A.r0 + row);
        if (!A.bj) {  // block-Jacobi: (K t, z), (K t, K t) come from the preconditioner pass
            d[0] += kt * in;  // (K t, z)
            d[1] += kt * kt;
        }
        d[2] += r0 * sr;
        d[3] += r0 * out;
        d[4] += sr * sr;
        d[5] += sr * out;
        d[6] += out * out;
    }
}

// out = A in from the tile partials (kGroups groups per output, combined by
// shuffles in a fixed order), the diagonal and the neutrality couplings.
// RED_START: r0 = r = b - A x, dot (r, r).  RED_V: v = A y, dot (r0, v).
// RED_T: t = A z and the dots (K t, z), (K t, K t), (r0, s), (r0, t), (s, s),
// (s, t), (t, t), from which omega, the next rho and (r, r) of r = s - omega t
// follow without another pass.  Writes the block's dot partials to bp.
template <int RED>
__device__ void reduce_pass(const CoopArgs &A, const PassScalars &S, double *bp)
{
    const int M = A.M;
    // RED_V in block-Jacobi mode: the tile pass just stored y in yb[cur ^ 1]
    const double *in = RED == RED_START ? A.x : (RED == RED_V ? (A.bj ? A.yb[S.cur ^ 1] : A.y) : A.z);
    double d[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const long nwork = (long)A.nT * 128 * kGroups;
    const long gthreads = (long)gridDim.x * blockDim.x;
    for (long base = 0; base < nwork; base += gthreads) {
        const long id = base + (long)blockIdx.x * blockDim.x + threadIdx.x;
        const int g = (int)(id % kGroups), o = (int)((id / kGroups) & 127), I = (int)(id / (128 * kGroups));
        double s = 0.0;
        if (id < nwork) {
            // kBatch independent loads in flight, summed in a fixed order
            const double *src = A.part + (size_t)I * A.nT * (kT * 4) + o;
            for (int K0 = g; K0 < A.nT; K0 += kBatch * kGroups) {
                double vals[kBatch];
#pragma unroll
                for (int u = 0; u < kBatch; ++u) {
                    const int Kk = K0 + u * kGroups;
                    vals[u] = Kk < A.nT ? __ldcg(src + (size_t)Kk * (kT * 4)) : 0.0;
                }
#pragma unroll
                for (int u = 0; u < kBatch; ++u) s += vals[u];
            }
        }
        s += __shfl_xor_sync(0xffffffffu, s, 1);
        s += __shfl_xor_sync(0xffffffffu, s, 2);
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
                        if (im >= A.np_start[k] && im <= A.np_end[k]) s += __ldcg(in + A.n4 + k);
                }
                reduce_row<RED>(A, S, row, s, xin, RED == RED_T ? __ldcg(A.K + row) : 0.0, d);
            }
        }
    }
    // Lagrange rows: the sum of the nanoparticle's charges of `in`
    for (int k = (int)gridDim.x - 1 - (int)blockIdx.x; k < A.n_nps; k += gridDim.x) {
        __shared__ double sh[32];
        double acc[1] = {0.0};
        for (int at = A.np_start[k] + threadIdx.x; at <= A.np_end[k]; at += blockDim.x)
            acc[0] += __ldcg(in + 3 * M + (at - A.metal_min));
        block_sum<1>(acc, sh);
        if (threadIdx.x == 0) {
            const int row = A.n4 + k;
            reduce_row<RED>(A, S, row, acc[0], __ldcg(in + row), 1.0, d);  // K = 1 on Lagrange rows
        }
        __syncthreads();
    }
    if (RED == RED_T) {
        put_bp<7>(bp, d);
    } else {
        double d1[1] = {d[0]};
        put_bp<1>(bp, d1);
    }
}

// Block-Jacobi application out = K in.  Work item w = (group G, quarter h):
// rows 32 h .. 32 h + 31 of the group's 128; thread (row, part) sums 16 of
// the 128 columns (FP32 inverse entries, FP64 products), the 8 parts of a row
// are combined by shuffles in a fixed order; 4 nG items spread over the grid.
// The Lagrange rows copy (K = 1).  WITH_DOTS: partials of (out, z),
// (out, out), i.e. (K t, z) and (K t, K t).
template <bool WITH_DOTS>
__device__ void prec_pass(const CoopArgs &A, const double *in, double *out, double *bp)
{
    __shared__ double xin[128];
    const int M = A.M, tid = threadIdx.x;
    double d[2] = {0.0, 0.0};
    for (int w = blockIdx.x; w < 4 * A.nG; w += gridDim.x) {
        const int G = w >> 2, h = w & 3;
        if (tid < 128) {
            const int atom = A.g_atoms[G * 32 + (tid >> 2)], comp = tid & 3;
            xin[tid] = atom >= 0 ? __ldcg(in + (comp < 3 ? 3 * atom + comp : 3 * M + atom)) : 0.0;
        }
        __syncthreads();
        const int o = 32 * h + (tid >> 3), part = tid & 7;
        const float *col = A.dinv + (size_t)G * 128 * 128 + (size_t)(16 * part) * 128 + o;
        float m[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) m[c] = __ldg(col + (size_t)c * 128);
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < 16; ++c) acc = fma((double)m[c], xin[16 * part + c], acc);
        acc += __shfl_xor_sync(0xffffffffu, acc, 1);
        acc += __shfl_xor_sync(0xffffffffu, acc, 2);
        acc += __shfl_xor_sync(0xffffffffu, acc, 4);
        const int atom = A.g_atoms[G * 32 + (o >> 2)], comp = o & 3;
        if (part == 0 && atom >= 0) {
            const int row = comp < 3 ? 3 * atom + comp : 3 * M + atom;
            out[row] = acc;
            if (WITH_DOTS) {
                d[0] += acc * __ldcg(A.z + row);
                d[1] += acc * acc;
            }
        }
        __syncthreads();  // xin free again
    }
    if (blockIdx.x == gridDim.x - 1)
        for (int k = tid; k < A.n_nps; k += blockDim.x) {
            const int row = A.n4 + k;
            const double v = __ldcg(in + row);
            out[row] = v;
            if (WITH_DOTS) {
                d[0] += v * __ldcg(A.z + row);
                d[1] += v * v;
            }
        }
    if (WITH_DOTS) put_bp<2>(bp, d);
}

template <typename T>
__host__ __device__ constexpr size_t ring_bytes()
{
    return (size_t)Ring<T>::Stages * kTileElems * sizeof(T);
}

template <typename T>
__global__ void __launch_bounds__(kBlock, sizeof(T) == 4 ? 2 : 1) k_bicgstab_coop(CoopArgs A)
{
    extern __shared__ __align__(128) unsigned char ring_smem[];
    constexpr int Stages = Ring<T>::Stages;
    __shared__ __align__(8) uint64_t ring_bar[Stages];
    PassSmem<T> &psm = *reinterpret_cast<PassSmem<T> *>(ring_smem + ring_bytes<T>());
    SolverScalars *ss = A.ss;
    const int n = A.n;
    const long gthreads = (long)gridDim.x * blockDim.x;
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nb = gridDim.x;
    // bpB holds the 7 dots of the T phase and, in block-Jacobi mode, the 2 of
    // the K t phase behind them, so one summation serves both
    double *bpA = A.bp, *bpB = A.bp + (size_t)kBp * nb;

    Ring<T> ring;
    ring.buf = reinterpret_cast<T *>(ring_smem);
    ring.bar = ring_bar;
    ring.issued = ring.consumed = 0;
    ring.n_my = (int)blockIdx.x < A.ntiles ? (A.ntiles - 1 - (int)blockIdx.x) / nb + 1 : 0;
    if (threadIdx.x == 0) ring.set_l2(A.l2_frac);
    if (threadIdx.x == 0) {
        for (int st = 0; st < Stages; ++st) mbar_init(ring_bar + st, 1);
        fence_mbar_init();
        if (ring.n_my > 0)
            for (int st = 0; st < Stages; ++st) ring.issue(static_cast<const T *>(A.mat));
    }
    __syncthreads();

    PassScalars S{0.0, 0.0, 0.0, 0, 1};
    int iter = 0, status = 0;
    double bTb = 0.0, crit = 0.0, rTr = 0.0, rr0 = 0.0;
    bool ok = true;

    // start: bTb, the count of non-zero entries of x, K, p = v = 0 (first buffers)
    {
        double pb[2] = {0.0, 0.0};
        for (long k = tid; k < n; k += gthreads) {
            const double bk = A.b[k];
            pb[0] += bk * bk;
            pb[1] += A.x[k] != 0.0 ? 1.0 : 0.0;
            A.K[k] = k < A.n4 ? 1.0 / A.diag[k] : 1.0;
            A.p[0][k] = 0.0;  // block-Jacobi: the first y buffer
            A.v[0][k] = 0.0;
            if (A.bj) A.Kv[k] = 0.0;
        }
        put_bp<2>(bpA, pb);
    }
    ok = grid_barrier(A.sync, A.spin_limit);
    bool x_zero = false;
    if (ok) {
        double t2[2];
        sum_bp<2>(bpA, nb, t2);
        bTb = t2[0];
        x_zero = t2[1] == 0.0;  // the same in every block
        crit = bTb * A.tol;
    }
    bool done = !ok || bTb < A.skip;  // zero right-hand side: x stays (bicg_stab.c:303-307)
    if (!done) {
        if (x_zero) {
            // r0 = r = b - A 0 = b: no product pass (the refinement sweeps
            // start their correction from zero); the tile ring is untouched,
            // so the next pass starts on the same tiles
            for (long k = tid; k < n; k += gthreads) {
                const double bk = A.b[k];
                A.r0[k] = bk;
                A.r[k] = bk;
            }
        } else {
            ok = tiles_pass<T, MODE_X>(A, S, ring, psm) && grid_barrier(A.sync, A.spin_limit);
            if (ok) reduce_pass<RED_START>(A, S, bpB);
        }
        ok = ok && grid_barrier(A.sync, A.spin_limit);
        if (ok && A.bj) {  // K r of the start residual; y = K r on the first iteration
            prec_pass<false>(A, A.r, A.Kr, nullptr);
            ok = grid_barrier(A.sync, A.spin_limit);
        }
        done = !ok;
    }
    double rho = 0.0, rho_old = 1.0, alpha = 1.0, omega = 1.0;
    if (!done) {
        if (x_zero) {
            rho = rTr = rr0 = bTb;
        } else {
            double t1[1];
            sum_bp<1>(bpB, nb, t1);
            rho = rTr = rr0 = t1[0];
        }
        if (rho < A.skip) done = true;  // warm start already converged (bicg_stab.c:368)
    }
    bool pending = false;  // x += alpha y + omega z of the last iteration not yet applied
    while (!done) {
        phase_mark(A, iter, 0);
        S.beta = (rho / rho_old) * (alpha / omega);
        S.omega = omega;
        S.alpha = alpha;
        ok = tiles_pass<T, MODE_P>(A, S, ring, psm);
        phase_mark(A, iter, 1);
        ok = ok && grid_barrier(A.sync, A.spin_limit);
        if (!ok) break;
        pending = false;  // the P pass applied the previous iteration's x update
        phase_mark(A, iter, 2);
        S.first = 0;
        reduce_pass<RED_V>(A, S, bpA);
        if (!grid_barrier(A.sync, A.spin_limit)) {
            ok = false;
            break;
        }
        phase_mark(A, iter, 3);
        if (A.bj) {  // K v
            prec_pass<false>(A, A.v[0], A.Kv, nullptr);
            if (!grid_barrier(A.sync, A.spin_limit)) {
                ok = false;
                break;
            }
        }
        phase_mark(A, iter, 4);
        double r0v[1];
        sum_bp<1>(bpA, nb, r0v);
        const double al = rho / r0v[0];
        if (!isfinite(al)) {  // breakdown: x is the start of this iteration
            status = rTr < crit * 100.0 ? 1 : -2;
            break;
        }
        alpha = al;
        S.cur ^= 1;  // v[cur] and p[cur] are now the new ones
        S.alpha = alpha;
        ok = tiles_pass<T, MODE_S>(A, S, ring, psm) && grid_barrier(A.sync, A.spin_limit);
        if (!ok) break;
        phase_mark(A, iter, 5);
        reduce_pass<RED_T>(A, S, bpB);
        if (!grid_barrier(A.sync, A.spin_limit)) {
            ok = false;
            break;
        }
        phase_mark(A, iter, 6);
        if (A.bj) {  // K t with (K t, z), (K t, K t)
            prec_pass<true>(A, A.t, A.Kt, bpB + 7);
            if (!grid_barrier(A.sync, A.spin_limit)) {
                ok = false;
                break;
            }
        }
        phase_mark(A, iter, 7);
        double d[9];
        if (A.bj) {
            sum_bp<9>(bpB, nb, d);
            d[0] = d[7];  // (K t, z), (K t, K t) of the preconditioner pass
            d[1] = d[8];
        } else {
            double d7[7];
            sum_bp<7>(bpB, nb, d7);
            for (int q = 0; q < 7; ++q) d[q] = d7[q];
        }
        const double om = d[0] / d[1];
        if (!isfinite(om) || om == 0.0) {
            status = rTr < crit * 100.0 ? 1 : -2;
            break;
        }
        omega = om;
        // r = s - omega t: (r0, r) and (r, r) from the merged dots
        rho_old = rho;
        rho = fma(-omega, d[3], d[2]);
        rTr = fma(omega * omega, d[6], fma(-2.0 * omega, d[5], d[4]));
        ++iter;
        pending = true;
        if (rTr < crit) {
            done = true;
        } else if (iter > A.max_iter) {
            status = rTr < crit * 100.0 ? 1 : -1;
            done = true;
        }
    }
    if (ok && pending) {  // the last update of x, and (r, r) of the final residual
        double q[1] = {0.0};
        for (long k = tid; k < n; k += gthreads) {
            A.x[k] += alpha * __ldcg((A.bj ? A.yb[S.cur] : A.y) + k) + omega * __ldcg(A.z + k);
            const double rk = __ldcg(A.s + k) - omega * __ldcg(A.t + k);
            A.r[k] = rk;
            q[0] += rk * rk;
        }
        put_bp<1>(bpA, q);
        ok = grid_barrier(A.sync, A.spin_limit);
        if (ok) {
            sum_bp<1>(bpA, nb, q);
            rTr = q[0];
        }
    }
    if (threadIdx.x == 0) {
        if (!ok) grid_abort(A.sync, 2);
        ring.drain();
    }
    if (ok && tid == 0) {
        ss->bTb = bTb;
        ss->crit = crit;
        ss->rTr = rTr;
        ss->rr0 = rr0;
        ss->iter = iter;
        ss->done = 1;
        ss->status = status;
    }
}

template <typename T>
size_t dyn_smem_bytes()
{
    return ring_bytes<T>() + sizeof(PassSmem<T>);
}

// ---------------------------------------------------------------------------
// Group-ordered solver (mixed path, block-Jacobi preconditioner).
//
// The metal atoms are numbered inside the solver by the preconditioner's
// groups (32 atoms each, along a Morton curve): slot a of group G is
// internal atom 32 G + a, and its four unknowns are the contiguous internal
// rows 128 G + 4 a + c (c = 0..2 dipole, 3 charge); the Lagrange rows follow
// at 128 nG + k.  The tiles are assembled in that order (tile (I, J) couples
// groups I and J), so
//   * a tile pass gathers its inputs as two contiguous runs of 128 rows, and
//   * the rows a block reduces from the tile partials are exactly one group,
//     so the same block applies the group's inverse diagonal block at once:
//     the V and T reductions and the preconditioner applications K v, K t
//     become one phase each, four grid barriers per iteration instead of six.
// The right-hand side and the solution stay in the reference layout outside
// the solver: b is gathered into the internal order at the start, x is read
// at the start and written back at the end.
struct GroupArgs {
    int M, nG, ntiles, n_nps, ni, max_iter;
    int stall;                   // > 0: stop (status 1) after this many iterations without halving (r, r)
    int nc;                      // > 0: the two-level operator with nc coarse columns (k_coarse.cu)
    int nm;                      // coarse columns per group: 1 (charge) or 4 (dipole x, y, z, charge)
    const float *w, *einv;       // (A Z) E^-1 and E^-1 of the coarse space
    double *zbuf;                // Z^T of the vector being preconditioned (nc)
    long spin_limit;
    double inv_polar, inv_capac;
    const int *g_atoms;          // [32 nG] metal-local atom of each slot, -1 padding
    const int *slot_np;          // [32 nG] nanoparticle of the slot's atom, -1 none
    const int *np_off, *np_rows; // internal charge rows of each nanoparticle's atoms
    const float *mat;            // tiles of the group order (I <= J)
    double *part;                // nG * nG * 128 tile partials
    double *bp;                  // dot partials, 2 sets of kBp per block
    const double *b;             // right-hand side, reference layout
    double *x;                   // solution, reference layout (in: start, out: result)
    double *xi, *r0, *r, *s, *t, *z, *Kr, *Kv, *Kt, *v, *yb[2];  // internal vectors (ni)
    const float *dinv;           // inverse diagonal blocks, [G][c][o]
    double tol, skip;
    SolverScalars *ss;
    CoopSync *sync;
    unsigned long long *ptime;
    float l2_frac;  // L2 policy of the streamed tiles (tile_l2_policy; 0: none)
};

// Reference row of internal row q (-1 for a padding slot).
__device__ __forceinline__ int g_ref_row(const GroupArgs &A, int q)
{
    const int base = 128 * A.nG;
    if (q >= base) return 4 * A.M + (q - base);
    const int m = A.g_atoms[q >> 2];
    if (m < 0) return -1;
    const int c = q & 3;
    return c < 3 ? 3 * m + c : 3 * A.M + m;
}

__device__ __forceinline__ void g_phase_mark(const GroupArgs &A, int iter, int k)
{
    if (A.ptime && blockIdx.x == 0 && threadIdx.x == 0 && iter < kPhaseIters) {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        A.ptime[iter * kPhases + k] = t;
    }
}

// MODE_P, one internal row (see bj_p_row): y = K r + beta (y_old - omega K v)
// with K r = z - omega K t; on `store` the deferred updates of the row.
__device__ __forceinline__ double g_p_row(const GroupArgs &A, const PassScalars &S, int row, bool store)
{
    const double y_old = __ldcg(A.yb[S.cur] + row);
    const double kr = S.first ? __ldcg(A.Kr + row) : fma(-S.omega, __ldcg(A.Kt + row), __ldcg(A.z + row));
    const double yn = fma(S.beta, fma(-S.omega, __ldcg(A.Kv + row), y_old), kr);
    if (store) {
        if (!S.first) {
            A.r[row] = fma(-S.omega, __ldcg(A.t + row), __ldcg(A.s + row));
            A.Kr[row] = kr;
            A.xi[row] += S.alpha * y_old + S.omega * __ldcg(A.z + row);
        }
        A.yb[S.cur ^ 1][row] = yn;
    }
    return yn;
}

// Tile pass on the group-ordered tiles (tiles_pass with contiguous inputs).
// The block's first n_res tiles are held in tensor memory (tw: this warp's
// address of the first one, kResCols columns apart); the others stream
// through the ring.
// A kernel that allocates tensor memory runs one block per SM, which takes
// all 512 columns.
constexpr int kResTiles = 6;           // tiles per block held in tensor memory
constexpr int kResCols = 2 * kPlanes * kCols;  // columns per tile (two warps share a lane quadrant)
constexpr uint32_t kTmemCols = 512;    // columns allocated per block
static_assert(kResTiles * kResCols <= (int)kTmemCols, "resident tiles exceed the allocation");
template <int MODE>
__device__ bool tiles_pass_g(const GroupArgs &A, const PassScalars &S, Ring<float> &ring, PassSmem<float> &sm,
                             int n_res, uint32_t tw)
{
    constexpr int Stages = Ring<float>::Stages;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nT = A.nG;
    if (MODE != MODE_X && threadIdx.x == 0) {
        for (int k = blockIdx.x; k < A.n_nps; k += gridDim.x) {
            const int row = 128 * nT + k;
            if (MODE == MODE_P) {
                g_p_row(A, S, row, true);
            } else {
                A.s[row] = fma(-S.alpha, __ldcg(A.v + row), __ldcg(A.r + row));
                A.z[row] = fma(-S.alpha, __ldcg(A.Kv + row), __ldcg(A.Kr + row));
            }
        }
    }
    constexpr int kChunk = chunk_tiles<float>();
    const int n_all = n_res + ring.n_my;
    for (int c0 = 0; c0 < n_all; c0 += kChunk) {
        const int nc = min(kChunk, n_all - c0);
        if (threadIdx.x < nc) {
            const int t = blockIdx.x + (c0 + threadIdx.x) * gridDim.x;
            int I = 0;
            while (tile_index(I + 1, I + 1, nT) <= (size_t)t && I + 1 < nT) ++I;
            sm.tile_i[threadIdx.x] = I;
            sm.tile_j[threadIdx.x] = I + (int)((size_t)t - tile_index(I, I, nT));
        }
        __syncthreads();
#pragma unroll 4
        for (int e = threadIdx.x; e < nc * 256; e += kBlock) {
            const int kk = e >> 8, side = (e >> 7) & 1, q4 = e & 127;
            const int I = sm.tile_i[kk], J = sm.tile_j[kk];
            const int row = 128 * (side ? J : I) + q4;
            double val;
            if (MODE == MODE_X) {
                val = __ldcg(A.xi + row);
            } else if (MODE == MODE_P) {
                val = g_p_row(A, S, row, I == J && side == 0);  // the diagonal-tile owner stores group I
            } else {
                val = fma(-S.alpha, __ldcg(A.Kv + row), __ldcg(A.Kr + row));
                if (I == J && side == 0) {
                    A.s[row] = fma(-S.alpha, __ldcg(A.v + row), __ldcg(A.r + row));
                    A.z[row] = val;
                }
            }
            sm.in[kk][side][q4 >> 2][q4 & 3] = (float)val;
        }
        __syncthreads();

        for (int kk = 0; kk < nc; ++kk) {
            const int I = sm.tile_i[kk], J = sm.tile_j[kk];
            const int set = kk & 1;
            const int qi = c0 + kk;
            const bool res = qi < n_res;  // block-uniform
            bool landed = true;
            const float *tile = nullptr;
            if (!res) {
                const long q = ring.consumed;
                const int st = (int)(q % Stages);
                const unsigned parity = (unsigned)((q / Stages) & 1);
                landed = mbar_wait(ring.bar + st, parity);
                tile = ring.stage(st);
            }
            const float(*xr)[4] = sm.in[kk][0];
            const float(*xc)[4] = sm.in[kk][1];
            const int a = lane;
            float ra[4] = {0, 0, 0, 0};
            float cb[kCols * 4];
            const float xa0 = xr[a][0], xa1 = xr[a][1], xa2 = xr[a][2], xa3 = xr[a][3];
            if (landed) {
                float vv[kPlanes][kCols];
                if (res) {
                    tmem_ld40(tw + (uint32_t)(qi * kResCols), reinterpret_cast<float(&)[40]>(vv));
                } else {
#pragma unroll
                    for (int pl = 0; pl < kPlanes; ++pl) ldsc(tile + elem_offset(pl, a, kCols * w), vv[pl]);
                }
#pragma unroll
                for (int k = 0; k < kCols; ++k) {
                    const int bb = kCols * w + k;
                    const float Axx = vv[0][k], Axy = vv[1][k], Axz = vv[2][k], Ayy = vv[3][k], Ayz = vv[4][k],
                                Azz = vv[5][k], m0 = vv[6][k], m1 = vv[7][k], m2 = vv[8][k], C = vv[9][k];
                    const float xb0 = xc[bb][0], xb1 = xc[bb][1], xb2 = xc[bb][2], xb3 = xc[bb][3];
                    ra[0] += Axx * xb0 + Axy * xb1 + Axz * xb2 + m0 * xb3;
                    ra[1] += Axy * xb0 + Ayy * xb1 + Ayz * xb2 + m1 * xb3;
                    ra[2] += Axz * xb0 + Ayz * xb1 + Azz * xb2 + m2 * xb3;
                    ra[3] += -(m0 * xb0 + m1 * xb1 + m2 * xb2) + C * xb3;
                    cb[4 * k + 0] = Axx * xa0 + Axy * xa1 + Axz * xa2 - m0 * xa3;
                    cb[4 * k + 1] = Axy * xa0 + Ayy * xa1 + Ayz * xa2 - m1 * xa3;
                    cb[4 * k + 2] = Axz * xa0 + Ayz * xa1 + Azz * xa2 - m2 * xa3;
                    cb[4 * k + 3] = m0 * xa0 + m1 * xa1 + m2 * xa2 + C * xa3;
                }
            } else {
#pragma unroll
                for (int k = 0; k < kCols * 4; ++k) cb[k] = 0;
            }
            const float colsum = warp_sum_halving<kCols * 4>(cb, lane);
#pragma unroll
            for (int c = 0; c < 4; ++c) sm.rowacc[set][w][a][c] = ra[c];
            constexpr int kShift = 5 - (kCols == 1 ? 2 : kCols == 2 ? 3 : kCols == 4 ? 4 : 5);
            if ((lane & ((1 << kShift) - 1)) == 0) {
                const int vv2 = lane >> kShift;
                sm.colacc[set][kCols * w + (vv2 >> 2)][vv2 & 3] = (double)colsum;
            }
            if (__syncthreads_or(!landed)) return false;
            if (!res) {
                ++ring.consumed;
                if (threadIdx.x == 0) ring.issue(A.mat);
            }
            double *pr = A.part + ((size_t)I * nT + J) * (kT * 4);
            double *pc = A.part + ((size_t)J * nT + I) * (kT * 4);
            if (threadIdx.x < kT * 4) {
                const int aa = threadIdx.x >> 2, c = threadIdx.x & 3;
                double sacc = 0.0;
#pragma unroll
                for (int ww = 0; ww < kWarps; ++ww) sacc += (double)sm.rowacc[set][ww][aa][c];
                pr[threadIdx.x] = I == J ? sacc + sm.colacc[set][aa][c] : sacc;
            } else if (threadIdx.x < 2 * kT * 4 && I != J) {
                const int c = threadIdx.x - kT * 4;
                pc[c] = sm.colacc[set][c >> 2][c & 3];
            }
        }
        __syncthreads();
    }
    return true;
}

// This thread's share of the sum of `in` over the charge rows of
// nanoparticle k (the constraint row's product): the rows' indices and then
// their values loaded kBatch at a time, so a block covers 16 x 256 atoms per
// round of loads.
__device__ __forceinline__ double np_charge_sum(const GroupArgs &A, const double *in, int k)
{
    const int q0 = A.np_off[k], q1 = A.np_off[k + 1];
    double acc = 0.0;
    for (int qb = q0 + (int)threadIdx.x; qb < q1; qb += kBatch * (int)blockDim.x) {
        int rows[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int q = qb + u * (int)blockDim.x;
            rows[u] = q < q1 ? __ldg(A.np_rows + q) : -1;
        }
        double vals[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) vals[u] = rows[u] >= 0 ? __ldcg(in + rows[u]) : 0.0;
#pragma unroll
        for (int u = 0; u < kBatch; ++u) acc += vals[u];
    }
    return acc;
}

// One group's reduction fused with its preconditioner block.  out = A in for
// the group's 128 rows from the nG tile partials of its block row (two
// halves of the threads sum alternate tiles, added in a fixed order), the
// diagonal and the neutrality couplings; then K out with the group's inverse
// block.  RED_START: r0 = r = b - A x (or b when x is zero), K r.
// RED_V: v = A y, K v, dot (r0, v).  RED_T: t = A z, K t, the dots (K t, z),
// (K t, K t), (r0, s), (r0, t), (s, s), (s, t), (t, t).  The Lagrange rows
// (K = 1 there) follow from the sums of the nanoparticles' charges.
template <int RED>
__device__ void reduce_group(const GroupArgs &A, const PassScalars &S, double *bp, bool products)
{
    __shared__ double vrow[128];
    __shared__ double hsum[128];
    const int nG = A.nG, tid = threadIdx.x;
    const double *in = RED == RED_START ? A.xi : (RED == RED_V ? A.yb[S.cur ^ 1] : A.z);
    double d[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int G = blockIdx.x; G < nG; G += gridDim.x) {
        const int o = tid & 127, h = tid >> 7;
        double sum = 0.0;
        if (products) {
            const double *src = A.part + (size_t)G * nG * (kT * 4) + o;
            for (int K0 = h; K0 < nG; K0 += 2 * kBatch) {
                double vals[kBatch];
#pragma unroll
                for (int u = 0; u < kBatch; ++u) {
                    const int Kk = K0 + 2 * u;
                    vals[u] = Kk < nG ? __ldcg(src + (size_t)Kk * (kT * 4)) : 0.0;
                }
#pragma unroll
                for (int u = 0; u < kBatch; ++u) sum += vals[u];
            }
        }
        if (h == 1) hsum[o] = sum;
        __syncthreads();
        if (h == 0) {
            const int row = 128 * G + o;
            sum += hsum[o];
            const double xin = products ? __ldcg(in + row) : 0.0;
            if ((o & 3) < 3) {
                sum += A.inv_polar * xin;
            } else {
                sum += -A.inv_capac * xin;
                const int k = A.slot_np[row >> 2];
                if (products && k >= 0) sum += __ldcg(in + 128 * nG + k);
            }
            double out;
            if (RED == RED_START) {
                const int rr = g_ref_row(A, row);
                const double bk = rr >= 0 ? A.b[rr] : 0.0;
                out = bk - sum;
                A.r0[row] = out;
                A.r[row] = out;
                d[0] += out * out;
            } else if (RED == RED_V) {
                out = sum;
                A.v[row] = out;
                d[0] += __ldcg(A.r0 + row) * out;
            } else {
                out = sum;
                A.t[row] = out;
                const double sr = __ldcg(A.s + row), r0 = __ldcg(A.r0 + row);
                d[2] += r0 * sr;
                d[3] += r0 * out;
                d[4] += sr * sr;
                d[5] += sr * out;
                d[6] += out * out;
            }
            vrow[o] = out;
        }
        __syncthreads();
        // K out: thread (row o2, half) sums 64 of the 128 columns
        {
            const int o2 = tid >> 1, half = tid & 1;
            const float *col = A.dinv + (size_t)G * 128 * 128 + (size_t)(64 * half) * 128 + o2;
            double acc = 0.0;
#pragma unroll 16
            for (int c = 0; c < 64; ++c) acc = fma((double)__ldg(col + (size_t)c * 128), vrow[64 * half + c], acc);
            acc += __shfl_xor_sync(0xffffffffu, acc, 1);
            if (half == 0) {
                const int row = 128 * G + o2;
                if (RED == RED_START) {
                    A.Kr[row] = acc;
                } else if (RED == RED_V) {
                    A.Kv[row] = acc;
                } else {
                    A.Kt[row] = acc;
                    d[0] += acc * __ldcg(A.z + row);
                    d[1] += acc * acc;
                }
            }
        }
        __syncthreads();  // vrow and hsum free again
    }
    // Lagrange rows: the sum of the nanoparticle's charges of `in`
    for (int k = (int)gridDim.x - 1 - (int)blockIdx.x; k < A.n_nps; k += gridDim.x) {
        __shared__ double shl[32];
        double acc[1] = {0.0};
        if (products)
            acc[0] = np_charge_sum(A, in, k);
        block_sum<1>(acc, shl);
        if (tid == 0) {
            const int row = 128 * nG + k;
            const double val = acc[0];
            if (RED == RED_START) {
                const double out = A.b[4 * A.M + k] - val;
                A.r0[row] = out;
                A.r[row] = out;
                A.Kr[row] = out;
                d[0] += out * out;
            } else if (RED == RED_V) {
                A.v[row] = val;
                A.Kv[row] = val;
                d[0] += __ldcg(A.r0 + row) * val;
            } else {
                A.t[row] = val;
                A.Kt[row] = val;
                const double zr = __ldcg(A.z + row), sr = __ldcg(A.s + row), r0 = __ldcg(A.r0 + row);
                d[0] += val * zr;
                d[1] += val * val;
                d[2] += r0 * sr;
                d[3] += r0 * val;
                d[4] += sr * sr;
                d[5] += sr * val;
                d[6] += val * val;
            }
        }
        __syncthreads();
    }
    if (RED == RED_T) {
        put_bp<7>(bp, d);
    } else {
        double d1[1] = {d[0]};
        put_bp<1>(bp, d1);
    }
}

constexpr int kCoarseMax = 384;  // coarse columns the solver's shared buffer holds

// The reductions of reduce_group with the two-level operator of k_coarse.cu
// in place of the block-Jacobi K alone: first every group's rows of `out`
// (v, t or r), the dots that do not involve K out, and the group's four mode
// sums (and the constraint rows) into zbuf; a grid barrier; then in every
// block c = E^-1 zbuf, and for its groups K out = Z c + K (out - (A Z) c)
// with the dots of K out.  Returns false when the grid barrier gave up.
// scratch: 256 + 2 kCoarseMax doubles of shared memory (the pass inputs'
// buffer, idle between passes).
template <int RED>
__device__ bool reduce_group2(const GroupArgs &A, const PassScalars &S, double *bp, bool products, double *scratch,
                              int iter = 0, int mark = -1)
{
    double *vrow = scratch, *hsum = scratch + 128, *cc = scratch + 256, *zs = scratch + 256 + kCoarseMax;
    const int nG = A.nG, nc = A.nc, tid = threadIdx.x;
    const double *in = RED == RED_START ? A.xi : (RED == RED_V ? A.yb[S.cur ^ 1] : A.z);
    double *outv = RED == RED_START ? A.r : (RED == RED_V ? A.v : A.t);
    double *kout = RED == RED_START ? A.Kr : (RED == RED_V ? A.Kv : A.Kt);
    double d[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int G = blockIdx.x; G < nG; G += gridDim.x) {
        const int o = tid & 127, h = tid >> 7;
        double sum = 0.0;
        if (products) {
            const double *src = A.part + (size_t)G * nG * (kT * 4) + o;
            for (int K0 = h; K0 < nG; K0 += 2 * kBatch) {
                double vals[kBatch];
#pragma unroll
                for (int u = 0; u < kBatch; ++u) {
                    const int Kk = K0 + 2 * u;
                    vals[u] = Kk < nG ? __ldcg(src + (size_t)Kk * (kT * 4)) : 0.0;
                }
#pragma unroll
                for (int u = 0; u < kBatch; ++u) sum += vals[u];
            }
        }
        if (h == 1) hsum[o] = sum;
        __syncthreads();
        if (h == 0) {
            const int row = 128 * G + o;
            sum += hsum[o];
            const double xin = products ? __ldcg(in + row) : 0.0;
            if ((o & 3) < 3) {
                sum += A.inv_polar * xin;
            } else {
                sum += -A.inv_capac * xin;
                const int k = A.slot_np[row >> 2];
                if (products && k >= 0) sum += __ldcg(in + 128 * nG + k);
            }
            double out;
            if (RED == RED_START) {
                const int rr = g_ref_row(A, row);
                const double bk = rr >= 0 ? A.b[rr] : 0.0;
                out = bk - sum;
                A.r0[row] = out;
                d[0] += out * out;
            } else if (RED == RED_V) {
                out = sum;
                d[0] += __ldcg(A.r0 + row) * out;
            } else {
                out = sum;
                const double sr = __ldcg(A.s + row), r0 = __ldcg(A.r0 + row);
                d[2] += r0 * sr;
                d[3] += r0 * out;
                d[4] += sr * sr;
                d[5] += sr * out;
                d[6] += out * out;
            }
            outv[row] = out;
            vrow[o] = A.g_atoms[row >> 2] >= 0 ? out : 0.0;
        }
        __syncthreads();
        if (tid < A.nm) {  // the group's mode sums (padding rows hold zero)
            const int c = A.nm == 4 ? tid : 3;
            double zs = 0.0;
            for (int a = 0; a < kT; ++a) zs += vrow[4 * a + c];
            A.zbuf[A.nm * G + tid] = zs;
        }
        __syncthreads();
    }
    for (int k = (int)gridDim.x - 1 - (int)blockIdx.x; k < A.n_nps; k += gridDim.x) {
        __shared__ double shl[32];
        double acc[1] = {0.0};
        if (products)
            acc[0] = np_charge_sum(A, in, k);
        block_sum<1>(acc, shl);
        if (tid == 0) {
            const int row = 128 * nG + k;
            const double val = acc[0];
            double out = val;
            if (RED == RED_START) {
                out = A.b[4 * A.M + k] - val;
                A.r0[row] = out;
                d[0] += out * out;
            } else if (RED == RED_V) {
                d[0] += __ldcg(A.r0 + row) * val;
            } else {
                const double sr = __ldcg(A.s + row), r0 = __ldcg(A.r0 + row);
                d[2] += r0 * sr;
                d[3] += r0 * val;
                d[4] += sr * sr;
                d[5] += sr * val;
                d[6] += val * val;
            }
            outv[row] = out;
            A.zbuf[A.nm * nG + k] = out;
        }
        __syncthreads();
    }
    if (!grid_barrier(A.sync, A.spin_limit)) return false;
    if (mark >= 0) g_phase_mark(A, iter, mark);  // the phase timer splits the two steps

    const int lane = tid & 31, wid = tid >> 5;
    const bool mine = (int)blockIdx.x < nG || (int)gridDim.x - 1 - (int)blockIdx.x < A.n_nps;
    if (mine) {
        for (int j = tid; j < nc; j += blockDim.x) zs[j] = __ldcg(A.zbuf + j);
        __syncthreads();
    }
    for (int G = blockIdx.x; G < nG; G += gridDim.x) {
        const int o = tid & 127, h = tid >> 7;
        // c of the group's own columns: warp m, lanes over the columns of
        // row nm G + m of E^-1
        if (wid < A.nm) {
            const float *er = A.einv + (size_t)(A.nm * G + wid) * nc;
            double s = 0.0;
            for (int j = lane; j < nc; j += 32) s = fma((double)__ldg(er + j), zs[j], s);
#pragma unroll
            for (int m = 16; m > 0; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m);
            if (lane == 0) cc[wid] = s;
        }
        // (A Z c) of the group's rows = W zbuf: two halves of the columns
        const float *wg = A.w + (size_t)G * nc * 128 + o;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int j = h;
        for (; j + 6 < nc; j += 8) {
            s0 = fma((double)__ldg(wg + (size_t)j * 128), zs[j], s0);
            s1 = fma((double)__ldg(wg + (size_t)(j + 2) * 128), zs[j + 2], s1);
            s2 = fma((double)__ldg(wg + (size_t)(j + 4) * 128), zs[j + 4], s2);
            s3 = fma((double)__ldg(wg + (size_t)(j + 6) * 128), zs[j + 6], s3);
        }
        for (; j < nc; j += 2) s0 = fma((double)__ldg(wg + (size_t)j * 128), zs[j], s0);
        const double s = (s0 + s1) + (s2 + s3);
        if (h == 1) hsum[o] = s;
        __syncthreads();
        if (h == 0) {
            const int row = 128 * G + o;
            const bool valid = A.g_atoms[row >> 2] >= 0;
            vrow[o] = valid ? __ldcg(outv + row) - (s + hsum[o]) : 0.0;
        }
        __syncthreads();
        // K w with the group's inverse block, plus Z c
        {
            const int o2 = tid >> 1, half = tid & 1;
            const float *col = A.dinv + (size_t)G * 128 * 128 + (size_t)(64 * half) * 128 + o2;
            double acc = 0.0;
#pragma unroll 16
            for (int c = 0; c < 64; ++c) acc = fma((double)__ldg(col + (size_t)c * 128), vrow[64 * half + c], acc);
            acc += __shfl_xor_sync(0xffffffffu, acc, 1);
            if (half == 0) {
                const int row = 128 * G + o2;
                if (A.g_atoms[row >> 2] >= 0 && (A.nm == 4 || (o2 & 3) == 3)) acc += cc[A.nm == 4 ? (o2 & 3) : 0];
                kout[row] = acc;
                if (RED == RED_T) {
                    d[0] += acc * __ldcg(A.z + row);
                    d[1] += acc * acc;
                }
            }
        }
        __syncthreads();
    }
    for (int k = (int)gridDim.x - 1 - (int)blockIdx.x; k < A.n_nps; k += gridDim.x) {
        // the whole block over the coarse columns, two per thread at most
        __shared__ double shc[2 * kWarps];
        const int row = 128 * nG + k;
        const float *er = A.einv + (size_t)(A.nm * nG + k) * nc;
        const float *wl = A.w + (size_t)nG * nc * 128 + (size_t)k * nc;
        double cw[2] = {0.0, 0.0};
        for (int j = tid; j < nc; j += blockDim.x) {
            cw[0] = fma((double)__ldg(er + j), zs[j], cw[0]);
            cw[1] = fma((double)__ldg(wl + j), zs[j], cw[1]);
        }
        block_sum<2>(cw, shc);
        if (tid == 0) {
            const double kv = __ldcg(outv + row) - cw[1] + cw[0];  // K = 1 on the constraint rows
            kout[row] = kv;
            if (RED == RED_T) {
                d[0] += kv * __ldcg(A.z + row);
                d[1] += kv * kv;
            }
        }
        __syncthreads();
    }
    if (RED == RED_T) {
        put_bp<7>(bp, d);
    } else {
        double d1[1] = {d[0]};
        put_bp<1>(bp, d1);
    }
    return true;
}

// Two blocks of kBlock threads per SM (the variant that holds tiles in
// tensor memory runs one).
template <bool HOLD>
__global__ void __launch_bounds__(kBlock, 2) k_bicgstab_group(GroupArgs A)
{
    extern __shared__ __align__(128) unsigned char ring_smem[];
    constexpr int Stages = Ring<float>::Stages;
    __shared__ __align__(8) uint64_t ring_bar[Stages];
    PassSmem<float> &psm = *reinterpret_cast<PassSmem<float> *>(ring_smem + ring_bytes<float>());
    // the pass inputs' buffer, idle between passes, holds the two-level reductions' scratch
    static_assert(sizeof(psm.in) >= (256 + 2 * kCoarseMax) * sizeof(double), "reduction scratch does not fit");
    double *pscratch = reinterpret_cast<double *>(&psm.in[0][0][0][0]);
    SolverScalars *ss = A.ss;
    const int ni = A.ni;
    const long gthreads = (long)gridDim.x * blockDim.x;
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nb = gridDim.x;
    double *bpA = A.bp, *bpB = A.bp + (size_t)kBp * nb;

    // the block's tiles: the first n_res held in tensor memory for the whole
    // solve (HOLD), the others streamed through the ring
    const int n_all = (int)blockIdx.x < A.ntiles ? (A.ntiles - 1 - (int)blockIdx.x) / nb + 1 : 0;
    const int n_res = HOLD ? min(n_all, kResTiles) : 0;
    Ring<float> ring;
    ring.buf = reinterpret_cast<float *>(ring_smem);
    ring.bar = ring_bar;
    ring.issued = ring.consumed = 0;
    ring.first = n_res;
    ring.n_my = n_all - n_res;
    if (threadIdx.x == 0) ring.set_l2(A.l2_frac);
    if (threadIdx.x == 0) {
        for (int st = 0; st < Stages; ++st) mbar_init(ring_bar + st, 1);
        fence_mbar_init();
        if (ring.n_my > 0)
            for (int st = 0; st < Stages; ++st) ring.issue(A.mat);
    }
    __shared__ uint32_t s_tmem;
    uint32_t tw = 0;  // this warp's tensor-memory address of resident tile 0
    if (n_res > 0) {
        if (threadIdx.x < 32) tmem_alloc(&s_tmem, kTmemCols);
        tmem_fence_before();
        __syncthreads();
        tmem_fence_after();
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        tw = s_tmem + ((uint32_t)(32 * (w % 4)) << 16) + (uint32_t)((w / 4) * kPlanes * kCols);
        for (int s = 0; s < n_res; ++s) {
            const float *tile = A.mat + (size_t)(blockIdx.x + s * nb) * kTileElems;
            float v[40];
#pragma unroll
            for (int pl = 0; pl < kPlanes; ++pl) {
                const float4 q = __ldg(reinterpret_cast<const float4 *>(tile + elem_offset(pl, lane, kCols * w)));
                v[4 * pl] = q.x;
                v[4 * pl + 1] = q.y;
                v[4 * pl + 2] = q.z;
                v[4 * pl + 3] = q.w;
            }
            tmem_st40(tw + (uint32_t)(s * kResCols), v);
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        tmem_fence_before();
    }
    __syncthreads();
    if (n_res > 0) tmem_fence_after();

    PassScalars S{0.0, 0.0, 0.0, 0, 1};
    int iter = 0, status = 0;
    double bTb = 0.0, crit = 0.0, rTr = 0.0, rr0 = 0.0;
    double ref_rTr = 0.0;  // (r, r) when it last halved
    int last_gain = 0;
    bool ok = true;

    // start: bTb, x gathered into the internal order (counting its non-zero
    // entries), the first y buffer and K v zero
    {
        double pb[2] = {0.0, 0.0};
        for (long k = tid; k < ni; k += gthreads) {
            const int rr = g_ref_row(A, (int)k);
            const double bk = rr >= 0 ? A.b[rr] : 0.0;
            const double xk = rr >= 0 ? A.x[rr] : 0.0;
            pb[0] += bk * bk;
            pb[1] += xk != 0.0 ? 1.0 : 0.0;
            A.xi[k] = xk;
            A.yb[0][k] = 0.0;
            A.Kv[k] = 0.0;
        }
        put_bp<2>(bpA, pb);
    }
    ok = grid_barrier(A.sync, A.spin_limit);
    bool x_zero = false;
    if (ok) {
        double t2[2];
        sum_bp<2>(bpA, nb, t2);
        bTb = t2[0];
        x_zero = t2[1] == 0.0;
        crit = bTb * A.tol;
    }
    bool done = !ok || bTb < A.skip;  // zero right-hand side: x stays (bicg_stab.c:303-307)
    if (!done) {
        // r0 = r = b - A x, K r (x zero: no product pass; the ring is
        // untouched, so the next pass starts on the same tiles)
        if (!x_zero) ok = tiles_pass_g<MODE_X>(A, S, ring, psm, n_res, tw) && grid_barrier(A.sync, A.spin_limit);
        if (ok) {
            if (A.nc > 0)
                ok = reduce_group2<RED_START>(A, S, bpB, !x_zero, pscratch);
            else
                reduce_group<RED_START>(A, S, bpB, !x_zero);
        }
        ok = ok && grid_barrier(A.sync, A.spin_limit);
        done = !ok;
    }
    double rho = 0.0, rho_old = 1.0, alpha = 1.0, omega = 1.0;
    if (!done) {
        double t1[1];
        sum_bp<1>(bpB, nb, t1);
        rho = rTr = rr0 = t1[0];
        ref_rTr = rTr;
        if (rho < A.skip) done = true;  // warm start already converged (bicg_stab.c:368)
    }
    bool pending = false;
    while (!done) {
        g_phase_mark(A, iter, 0);
        S.beta = (rho / rho_old) * (alpha / omega);
        S.omega = omega;
        S.alpha = alpha;
        ok = tiles_pass_g<MODE_P>(A, S, ring, psm, n_res, tw);
        g_phase_mark(A, iter, 1);
        ok = ok && grid_barrier(A.sync, A.spin_limit);
        if (!ok) break;
        pending = false;  // the P pass applied the previous iteration's x update
        g_phase_mark(A, iter, 2);
        S.first = 0;
        if (A.nc > 0) {
            if (!reduce_group2<RED_V>(A, S, bpA, true, pscratch, iter, 3)) {
                ok = false;
                break;
            }
        } else {
            reduce_group<RED_V>(A, S, bpA, true);
        }
        if (!grid_barrier(A.sync, A.spin_limit)) {
            ok = false;
            break;
        }
        if (A.nc == 0) g_phase_mark(A, iter, 3);
        g_phase_mark(A, iter, 4);
        double r0v[1];
        sum_bp<1>(bpA, nb, r0v);
        const double al = rho / r0v[0];
        if (!isfinite(al)) {  // breakdown: x is the start of this iteration
            status = rTr < crit * 100.0 ? 1 : -2;
            break;
        }
        alpha = al;
        S.cur ^= 1;
        S.alpha = alpha;
        ok = tiles_pass_g<MODE_S>(A, S, ring, psm, n_res, tw) && grid_barrier(A.sync, A.spin_limit);
        if (!ok) break;
        g_phase_mark(A, iter, 5);
        if (A.nc > 0) {
            if (!reduce_group2<RED_T>(A, S, bpB, true, pscratch, iter, 6)) {
                ok = false;
                break;
            }
        } else {
            reduce_group<RED_T>(A, S, bpB, true);
        }
        if (!grid_barrier(A.sync, A.spin_limit)) {
            ok = false;
            break;
        }
        if (A.nc == 0) g_phase_mark(A, iter, 6);
        g_phase_mark(A, iter, 7);
        double d[7];
        sum_bp<7>(bpB, nb, d);
        const double om = d[0] / d[1];
        if (!isfinite(om) || om == 0.0) {
            status = rTr < crit * 100.0 ? 1 : -2;
            break;
        }
        omega = om;
        rho_old = rho;
        rho = fma(-omega, d[3], d[2]);
        rTr = fma(omega * omega, d[6], fma(-2.0 * omega, d[5], d[4]));
        ++iter;
        pending = true;
        if (rTr < crit) {
            done = true;
        } else if (iter > A.max_iter) {
            status = rTr < crit * 100.0 ? 1 : -1;
            done = true;
        } else if (A.stall > 0) {
            // an inner solve of the refinement that has stopped making
            // progress (FP32 products limit what it can reach) hands its
            // iterate back; the FP64 residual decides what follows
            if (rTr < 0.5 * ref_rTr) {
                ref_rTr = rTr;
                last_gain = iter;
            } else if (iter - last_gain >= A.stall) {
                status = 1;
                done = true;
            }
        }
    }
    if (ok) {
        // the last update of x, (r, r) of the final residual, x back to the
        // reference layout
        double q[1] = {0.0};
        for (long k = tid; k < ni; k += gthreads) {
            double xk = A.xi[k];
            if (pending) {
                xk += alpha * __ldcg(A.yb[S.cur] + k) + omega * __ldcg(A.z + k);
                const double rk = __ldcg(A.s + k) - omega * __ldcg(A.t + k);
                A.r[k] = rk;
                q[0] += rk * rk;
            }
            const int rr = g_ref_row(A, (int)k);
            if (rr >= 0) A.x[rr] = xk;
        }
        if (pending) {
            put_bp<1>(bpA, q);
            ok = grid_barrier(A.sync, A.spin_limit);
            if (ok) {
                sum_bp<1>(bpA, nb, q);
                rTr = q[0];
            }
        }
    }
    if (threadIdx.x == 0) {
        if (!ok) grid_abort(A.sync, 2);
        ring.drain();
    }
    if (n_res > 0) {  // every path comes here: the block's tensor memory is released
        tmem_fence_before();
        __syncthreads();
        tmem_fence_after();
        if (threadIdx.x < 32) tmem_dealloc(s_tmem, kTmemCols);
    }
    if (ok && tid == 0) {
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

size_t coop_barrier_bytes() { return sizeof(CoopSync); }
size_t coop_partial_doubles(int grid) { return (size_t)2 * kBp * grid; }

int finish_coop(capac_ctx *c, const unsigned long long *ptime, double skip);
int bicgstab_group(capac_ctx *c, const double *b, double *x, double tol, double skip);

// Launch the persistent solver; returns the status as bicgstab_core does.
int bicgstab_coop(capac_ctx *c, const double *b, double *x, double tol, double skip)
{
    if (c->grouped) return bicgstab_group(c, b, x, tol, skip);
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
    A.max_iter = solver_max_iter(c);
    A.spin_limit = c->opt.wait_polls > 0 ? c->opt.wait_polls : kSpinLimit;
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
    // work vectors in the slots of bw; the second p and v buffers take the
    // slots the per-step solver uses for A x0 and K t
    A.r0 = W(1); A.r = W(2); A.p[0] = W(3); A.v[0] = W(4); A.s = W(5); A.t = W(6); A.y = W(7); A.z = W(8);
    A.v[1] = W(9); A.K = W(10); A.p[1] = W(0);
    A.bj = c->dinv != nullptr;
    A.nG = c->dinv ? precond_groups(c->M) : 0;
    A.g_atoms = c->g_atoms;
    A.dinv = c->dinv;
    A.Kr = A.Kv = A.Kt = nullptr;
    A.yb[0] = A.yb[1] = nullptr;
    if (A.bj) {
        // y double-buffered in the p slots; one v buffer; K v, K t, K r in
        // the second v slot, the K slot (K is not read) and slot 0
        A.yb[0] = W(3);
        A.yb[1] = W(7);
        A.y = W(7);
        A.v[1] = A.v[0];
        A.Kv = W(9);
        A.Kt = W(10);
        A.Kr = W(0);
    }
    A.tol = tol;
    A.skip = skip;
    A.ss = c->ss;
    A.sync = reinterpret_cast<CoopSync *>(c->coop_bar);
    A.l2_frac = c->tile_l2;
    A.ptime = nullptr;
    if (c->phase_timer) {
        if (!c->phase_buf) CAPAC_CUDA(cudaMalloc(&c->phase_buf, sizeof(unsigned long long) * kPhases * kPhaseIters));
        A.ptime = static_cast<unsigned long long *>(c->phase_buf);
    }
    CAPAC_CUDA(cudaMemsetAsync(c->coop_bar, 0, sizeof(CoopSync), c->stream));
    void *args[] = {&A};
    const bool mixed = c->opt.precision == CAPAC_PREC_MIXED;
    {
        ProfScope ps(c, K_SOLVE);
        if (mixed)
            CAPAC_CUDA(cudaLaunchCooperativeKernel((const void *)k_bicgstab_coop<float>, dim3(c->coop_grid),
                                                   dim3(kBlock), args, dyn_smem_bytes<float>(), c->stream));
        else
            CAPAC_CUDA(cudaLaunchCooperativeKernel((const void *)k_bicgstab_coop<double>, dim3(c->coop_grid),
                                                   dim3(kBlock), args, dyn_smem_bytes<double>(), c->stream));
    }
    ++c->launches;
    return finish_coop(c, A.ptime, skip);
}

// After a persistent launch: the error word, the phase timer, the status.
int finish_coop(capac_ctx *c, const unsigned long long *ptime, double skip)
{
    CAPAC_CUDA(cudaMemcpyAsync(c->h_ss, c->ss, sizeof(SolverScalars), cudaMemcpyDeviceToHost, c->stream));
    CoopSync hs;
    CAPAC_CUDA(cudaMemcpyAsync(&hs, c->coop_bar, sizeof hs, cudaMemcpyDeviceToHost, c->stream));
    CAPAC_CUDA(cudaStreamSynchronize(c->stream));
    if (hs.error) throw Error(CAPAC_ERR_CUDA, "persistent solver: a bounded wait timed out");
    if (ptime && c->h_ss->iter > 1) {
        // phase k of an iteration ends at mark k + 1 (the last at the next iteration's mark 0)
        const int it = std::min(c->h_ss->iter, kPhaseIters);
        std::vector<unsigned long long> t((size_t)kPhases * it);
        CAPAC_CUDA(cudaMemcpy(t.data(), ptime, sizeof(unsigned long long) * t.size(), cudaMemcpyDeviceToHost));
        for (int i = 0; i + 1 < it; ++i) {
            for (int k = 0; k < kPhases; ++k) {
                const unsigned long long a = t[(size_t)i * kPhases + k];
                const unsigned long long b = k + 1 < kPhases ? t[(size_t)i * kPhases + k + 1] : t[(size_t)(i + 1) * kPhases];
                c->phase_ns[k] += (double)(b - a);
            }
            ++c->phase_iters;
        }
    }
    if (c->prof.on && c->h_ss->bTb >= skip) c->prof.spmv_effective += 1 + 2L * c->h_ss->iter;
    if (c->h_ss->status < 0) return CAPAC_ERR_NOT_CONVERGED;
    return c->h_ss->status == 1 ? 1 : CAPAC_OK;
}

// The group-ordered persistent solver (mixed path, block-Jacobi).
int bicgstab_group(capac_ctx *c, const double *b, double *x, double tol, double skip)
{
    GroupArgs A;
    const int nG = precond_groups(c->M);
    A.M = c->M;
    A.nG = nG;
    A.ntiles = nG * (nG + 1) / 2;
    A.n_nps = c->n_nps;
    A.ni = (int)group_rows(c->M, c->n_nps);
    A.max_iter = solver_max_iter(c);
    A.stall = c->inner_stall;
    A.nc = c->twolevel ? c->cz_nc : 0;
    A.nm = c->cz_modes;
    A.w = c->cz_w;
    A.einv = c->cz_einv;
    A.zbuf = c->cz_zbuf;
    A.spin_limit = c->opt.wait_polls > 0 ? c->opt.wait_polls : kSpinLimit;
    A.inv_polar = c->P.inv_polar;
    A.inv_capac = c->P.inv_capac;
    A.g_atoms = c->g_atoms;
    A.slot_np = c->slot_np;
    A.np_off = c->np_off;
    A.np_rows = c->np_rows;
    A.mat = static_cast<const float *>(c->msym);
    A.part = c->sympart;
    A.bp = c->coop_bp;
    A.b = b;
    A.x = x;
    auto V = [&](int k) { return c->gvec + (size_t)k * A.ni; };
    A.xi = V(0); A.r0 = V(1); A.r = V(2); A.s = V(3); A.t = V(4); A.z = V(5);
    A.Kr = V(6); A.Kv = V(7); A.Kt = V(8); A.v = V(9); A.yb[0] = V(10); A.yb[1] = V(11);
    A.dinv = c->dinv;
    A.tol = tol;
    A.skip = skip;
    A.ss = c->ss;
    A.sync = reinterpret_cast<CoopSync *>(c->coop_bar);
    A.l2_frac = c->tile_l2;
    A.ptime = nullptr;
    if (c->phase_timer) {
        if (!c->phase_buf) CAPAC_CUDA(cudaMalloc(&c->phase_buf, sizeof(unsigned long long) * kPhases * kPhaseIters));
        A.ptime = static_cast<unsigned long long *>(c->phase_buf);
    }
    CAPAC_CUDA(cudaMemsetAsync(c->coop_bar, 0, sizeof(CoopSync), c->stream));
    void *args[] = {&A};
    {
        ProfScope ps(c, K_SOLVE);
        const void *kern = c->tmem_tiles ? (const void *)k_bicgstab_group<true> : (const void *)k_bicgstab_group<false>;
        CAPAC_CUDA(cudaLaunchCooperativeKernel(kern, dim3(c->group_grid), dim3(kBlock), args,
                                               dyn_smem_bytes<float>(), c->stream));
    }
    ++c->launches;
    return finish_coop(c, A.ptime, skip);
}

int group_tmem_tiles() { return kResTiles; }
int coarse_columns_max() { return kCoarseMax; }
size_t group_rows(int M, int n_nps) { return (size_t)128 * precond_groups(M) + n_nps; }

// Blocks of the group-ordered solver: two per SM when they fit, 0 if the
// device cannot run it.
int group_blocks_per_sm(int device, bool hold)
{
    const void *kern = hold ? (const void *)k_bicgstab_group<true> : (const void *)k_bicgstab_group<false>;
    const size_t dyn = dyn_smem_bytes<float>();
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlock, dyn) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return per_sm;
}

int group_grid_size(int device, bool hold)
{
    int coop = 0;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) != cudaSuccess || !coop) return 0;
    int sms = 0;
    CAPAC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int per_sm = group_blocks_per_sm(device, hold);
    // the variant that holds tiles allocates all of an SM's tensor memory:
    // it runs only where no second block can share the SM
    if (hold) return per_sm == 1 ? sms : 0;
    return per_sm < 1 ? 0 : sms * std::min(per_sm, 2);
}

// Blocks of the persistent solver (two per SM for the FP32 matrix, one for
// the FP64 matrix), 0 if the device cannot run
// it (no cooperative launch, or the ring does not fit in shared memory).
int coop_grid_size(int device, bool mixed)
{
    int coop = 0;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) != cudaSuccess || !coop) return 0;
    int sms = 0;
    CAPAC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const void *fn = mixed ? (const void *)k_bicgstab_coop<float> : (const void *)k_bicgstab_coop<double>;
    const size_t dyn = mixed ? dyn_smem_bytes<float>() : dyn_smem_bytes<double>();
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, dyn) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        return 0;
    }
    return sms * std::min(per_sm, mixed ? 2 : 1);
}

}  // namespace capac
