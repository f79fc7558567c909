// Two-level preconditioner of the mixed path's inner solves (inner_precond 2, 3).
//
// The block-Jacobi inverse K of the 32-atom groups leaves the smooth error
// modes of the CPIM system (a group's total charge and total dipole against
// the others', the nanoparticles' constraint rows) to the Krylov iteration.
// The coarse space Z holds, per group g, the indicator of its atoms' charge
// rows (inner_precond 2) or four columns, the indicators of their x, y, z
// dipole rows and of their charge rows (3), and one column per nanoparticle
// constraint row; E = Z^T A Z (nc = nm nG + n_NP, nm = 1 or 4).  The inner
// solves use the multiplicative two-level operator
//     K2 v = Z c + K (v - A Z c),   c = E^-1 Z^T v,
// a fixed linear operator as long as Z, A Z and E^-1 are (they are refreshed
// with the block inverses, every 10 matrix builds), so BiCGSTAB's recurrences
// hold; only the FP64 refinement residual defines the answer.  A Z comes from
// the stored FP32 tiles in the groups' order: row sums of each tile's planes
// for the rows of its first block row, column sums for the second (the
// matrix is symmetric: the 4x4 block of atoms (b, a) is the transpose of that
// of (a, b)), the diagonal terms 1/polar and -1/capac, and the constraint
// couplings.  E sums A Z over each group's rows; E^-1 by Gauss-Jordan with
// partial pivoting in FP64 in one block.
//
// W = (A Z) E^-1, in the layout of A Z, is what the solver reads.
// Layout (group g's columns at nm g ..): az[(g * nc + j) * 128 + r] for internal row 128 g + r (column
// j contiguous over the group's rows), then az[128 nG nc + k * nc + j] for
// constraint row k; einv[j * nc + i] = (E^-1)[i][j] (E is symmetric).
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>

#include "ctx.h"

namespace capac {

namespace {

constexpr int kT = 32;
constexpr int kPlanes = 10;
constexpr int kTileElems = kPlanes * kT * kT;
constexpr int kRows = 4 * kT;  // internal rows of a group
constexpr int kInvThreads = 1024;
constexpr int kMaxCoarse = 384;  // coarse columns the inversion handles (2 kMaxCoarse <= kInvThreads)

__host__ __device__ __forceinline__ size_t tile_index(int I, int J, int nT)
{
    return (size_t)I * nT - (size_t)I * (I - 1) / 2 + (size_t)(J - I);
}
__device__ __forceinline__ int elem_offset(int p, int a, int b)
{
    return ((p * (kT / 4) + (b >> 2)) * (kT * 4)) + a * 4 + (b & 3);
}

// Sum over a set of atom pairs of the 4x4 block's entry (row mode c, column
// mode d) from per-plane sums s[p]: planes 0-5 the symmetric dipole block
// (xx xy xz yy yz zz), 6-8 the dipole-charge column m, 9 charge-charge; the
// charge row of the block is (-m, C).
__device__ __forceinline__ float block_entry(const float (&s)[kPlanes], int c, int d)
{
    if (c < 3 && d < 3) {
        const int lo = min(c, d), hi = max(c, d);
        const int p = lo == 0 ? hi : (lo == 1 ? 2 + hi : 5);
        return s[p];
    }
    if (c < 3) return s[6 + c];
    if (d < 3) return -s[6 + d];
    return s[9];
}

// One block per tile (I, J), I <= J: the A Z entries of the rows of group I
// in the columns of group J and, for I < J, of the rows of J in the columns
// of I; for I = J the strict upper tile gives both halves, plus the diagonal.
__global__ void __launch_bounds__(256) k_coarse_az(const float *__restrict__ mat, int nG, int nc, int nm,
                                                   const int *__restrict__ g_atoms, double inv_polar,
                                                   double inv_capac, float *__restrict__ az)
{
    __shared__ float rs[kPlanes][kT], cs[kPlanes][kT];
    const size_t t = blockIdx.x;
    int I = 0;
    while (tile_index(I + 1, I + 1, nG) <= t && I + 1 < nG) ++I;
    const int J = I + (int)(t - tile_index(I, I, nG));
    const float *tile = mat + t * kTileElems;
    for (int q = threadIdx.x; q < 2 * kPlanes * kT; q += blockDim.x) {
        const int col = q >= kPlanes * kT, p = (q % (kPlanes * kT)) / kT, i = q % kT;
        float s = 0.f;
        for (int k = 0; k < kT; ++k) s += col ? tile[elem_offset(p, k, i)] : tile[elem_offset(p, i, k)];
        (col ? cs : rs)[p][i] = s;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < kRows * nm; q += blockDim.x) {
        const int r = q / nm, m = q % nm, d = nm == 4 ? m : 3, a = r >> 2, c = r & 3;
        float sr[kPlanes], sc[kPlanes];
#pragma unroll
        for (int p = 0; p < kPlanes; ++p) {
            sr[p] = rs[p][a];
            sc[p] = cs[p][a];
        }
        // rows of I, column (J, d): sum over b in J of block (a, b)[c][d]
        float v = block_entry(sr, c, d);
        if (I == J) {
            v += block_entry(sc, d, c);  // the pairs b < a, stored as (b, a)
            if (c == d && g_atoms[(size_t)I * kT + a] >= 0) v += (float)(c < 3 ? inv_polar : -inv_capac);
        }
        az[((size_t)I * nc + nm * J + m) * kRows + r] = v;
        if (I != J) {
            // rows of J (atom a of J here), column (I, d): sum over the atoms
            // of I of block (i, a)^T[c][d] = block (i, a)[d][c]
            az[((size_t)J * nc + nm * I + m) * kRows + r] = block_entry(sc, d, c);
        }
    }
}

// The constraint columns and rows of A Z: charge row of an atom of NP k in
// column 4 nG + k; constraint row k in the charge column of each group with
// the count of that group's atoms in NP k.
__global__ void k_coarse_az_np(int nG, int nc, int nm, int n_nps, const int *__restrict__ slot_np,
                               float *__restrict__ az)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t base = (size_t)nG * nc * kRows;
    if (q < nG * kRows) {
        const int g = q / kRows, r = q % kRows, a = r >> 2, c = r & 3;
        const int k = slot_np[(size_t)g * kT + a];
        for (int j = 0; j < n_nps; ++j)
            az[((size_t)g * nc + nm * nG + j) * kRows + r] = (c == 3 && k == j) ? 1.f : 0.f;
    }
    if (q < n_nps * nc) {
        const int k = q / nc, j = q % nc;
        float v = 0.f;
        if (j < nm * nG && (nm == 1 || (j & 3) == 3)) {  // a group's charge column
            const int g = j / nm;
            for (int a = 0; a < kT; ++a) v += slot_np[(size_t)g * kT + a] == k ? 1.f : 0.f;
        }
        az[base + (size_t)k * nc + j] = v;
    }
}

// E = Z^T (A Z) into the left half of the augmented [E | I] (FP64, nc x 2 nc).
__global__ void k_coarse_e(int nG, int nc, int nm, const int *__restrict__ g_atoms, const float *__restrict__ az,
                           double *__restrict__ aug)
{
    const int i = blockIdx.x;
    for (int j = threadIdx.x; j < 2 * nc; j += blockDim.x) {
        double v = 0.0;
        if (j < nc) {
            if (i < nm * nG) {
                const int g = i / nm, c = nm == 4 ? (i & 3) : 3;
                const float *col = az + ((size_t)g * nc + j) * kRows;
                for (int a = 0; a < kT; ++a)
                    if (g_atoms[(size_t)g * kT + a] >= 0) v += (double)col[4 * a + c];
            } else {
                v = (double)az[(size_t)nG * nc * kRows + (size_t)(i - nm * nG) * nc + j];
            }
        } else {
            v = (j - nc == i) ? 1.0 : 0.0;
        }
        aug[(size_t)i * 2 * nc + j] = v;
    }
}

// Gauss-Jordan with partial pivoting on [E | I] in global memory, one block;
// E^-1 (FP32) to einv, or zeros (the coarse correction then vanishes and K2
// is the block-Jacobi K) when a pivot falls below 1e-13 of the largest entry.
__global__ void __launch_bounds__(kInvThreads) k_coarse_invert(int nc, double *__restrict__ aug,
                                                                float *__restrict__ einv, int *bad_out)
{
    __shared__ double wv[kInvThreads / 32];
    __shared__ int wi[kInvThreads / 32];
    __shared__ int piv, bad;
    __shared__ double amax;
    __shared__ double fcol[kMaxCoarse];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, w2 = 2 * nc;
    if (tid == 0) bad = 0;
    {
        double m = 0.0;
        for (int q = tid; q < nc * nc; q += blockDim.x) m = fmax(m, fabs(aug[(size_t)(q / nc) * w2 + q % nc]));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) wv[wid] = m;
        __syncthreads();
        if (tid == 0) {
            double mm = 0.0;
            for (int w = 0; w < kInvThreads / 32; ++w) mm = fmax(mm, wv[w]);
            amax = mm;
        }
        __syncthreads();
    }
    const double tiny = 1e-13 * amax;
    for (int k = 0; k < nc; ++k) {
        double v = -1.0;
        int vi = nc;
        for (int i = k + tid; i < nc; i += blockDim.x) {
            const double x = fabs(aug[(size_t)i * w2 + k]);
            if (x > v) {
                v = x;
                vi = i;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double v2 = __shfl_xor_sync(0xffffffffu, v, o);
            const int i2 = __shfl_xor_sync(0xffffffffu, vi, o);
            if (v2 > v || (v2 == v && i2 < vi)) {
                v = v2;
                vi = i2;
            }
        }
        if (lane == 0) {
            wv[wid] = v;
            wi[wid] = vi;
        }
        __syncthreads();
        if (tid == 0) {
            double bv = -1.0;
            int bi = nc;
            for (int w = 0; w < kInvThreads / 32; ++w)
                if (wv[w] > bv || (wv[w] == bv && wi[w] < bi)) {
                    bv = wv[w];
                    bi = wi[w];
                }
            piv = bi;
            if (!(bv > tiny) || bi >= nc) bad = 1;
        }
        __syncthreads();
        if (bad) break;
        const int p = piv;
        if (p != k)
            for (int j = tid; j < w2; j += blockDim.x) {
                const double tmp = aug[(size_t)k * w2 + j];
                aug[(size_t)k * w2 + j] = aug[(size_t)p * w2 + j];
                aug[(size_t)p * w2 + j] = tmp;
            }
        __syncthreads();
        const double inv = 1.0 / aug[(size_t)k * w2 + k];
        for (int i = tid; i < nc; i += blockDim.x) fcol[i] = i == k ? 0.0 : aug[(size_t)i * w2 + k];
        __syncthreads();
        for (int j = tid; j < w2; j += blockDim.x) aug[(size_t)k * w2 + j] *= inv;
        __syncthreads();
        // eliminate column k from every other row: thread j owns column j
        // (the factors of column k were saved in fcol before any change)
        if (tid < w2 && tid != k) {
            const double rk = aug[(size_t)k * w2 + tid];
            double *colj = aug + tid;
#pragma unroll 4
            for (int i = 0; i < nc; ++i)
                if (i != k) colj[(size_t)i * w2] = fma(-fcol[i], rk, colj[(size_t)i * w2]);
        }
        __syncthreads();
        for (int i = tid; i < nc; i += blockDim.x)
            if (i != k) aug[(size_t)i * w2 + k] = 0.0;
        __syncthreads();
    }
    // E is symmetric, so E^-1 is: write it column-major, which is row-major
    for (int q = tid; q < nc * nc; q += blockDim.x) {
        const int i = q / nc, j = q % nc;
        einv[(size_t)j * nc + i] = bad ? 0.f : (float)aug[(size_t)i * w2 + nc + j];
    }
    if (tid == 0) *bad_out = bad;
}

// The same inversion by a thread-block cluster: CTA q of the cluster holds
// rows q rp .. q rp + rp - 1 of [E | I] (FP64) in its shared memory, and the
// CTAs exchange the pivot candidates, the swapped rows and the pivot row
// through distributed shared memory with a cluster barrier around each
// exchange.  Every CTA takes the same branches (the pivot and the singular
// case are decided from the same gathered candidates), so every cluster
// barrier is reached by all of them.
__global__ void __launch_bounds__(kInvThreads) k_coarse_invert_cluster(int nc, const double *__restrict__ aug,
                                                                        float *__restrict__ einv, int *bad_out)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank(), ncta = (int)cl.num_blocks();
    extern __shared__ __align__(16) double csm[];
    __shared__ double wv[kInvThreads / 32];
    __shared__ int wi[kInvThreads / 32];
    __shared__ double cand_v, amax_l;
    __shared__ int cand_i, piv_s, bad_s;
    __shared__ double fcol[kMaxCoarse];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, w2 = 2 * nc;
    const int rp = (nc + ncta - 1) / ncta, r0 = rank * rp, r1 = min(nc, r0 + rp), nr = max(0, r1 - r0);
    double *rows = csm;          // nr x w2
    double *prow = csm + (size_t)rp * w2;
    double *trow = prow + w2;
    for (int q = tid; q < nr * w2; q += blockDim.x) rows[q] = aug[(size_t)(r0 + q / w2) * w2 + q % w2];
    // the largest |E| entry, over the cluster
    {
        double m = 0.0;
        for (int q = tid; q < nr * nc; q += blockDim.x) m = fmax(m, fabs(rows[(size_t)(q / nc) * w2 + q % nc]));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) wv[wid] = m;
        __syncthreads();
        if (tid == 0) {
            double mm = 0.0;
            for (int w = 0; w < kInvThreads / 32; ++w) mm = fmax(mm, wv[w]);
            amax_l = mm;
            bad_s = 0;
        }
    }
    cl.sync();
    double tiny = 0.0;
    for (int q = 0; q < ncta; ++q) tiny = fmax(tiny, *cl.map_shared_rank(&amax_l, q));
    tiny *= 1e-13;
    int bad = 0;
    for (int k = 0; k < nc; ++k) {
        // this CTA's candidate: largest |a[i][k]|, i >= k, lowest i on ties
        double v = -1.0;
        int vi = nc;
        for (int i = max(k, r0) + tid; i < r1; i += blockDim.x) {
            const double x = fabs(rows[(size_t)(i - r0) * w2 + k]);
            if (x > v) {
                v = x;
                vi = i;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double v2 = __shfl_xor_sync(0xffffffffu, v, o);
            const int i2 = __shfl_xor_sync(0xffffffffu, vi, o);
            if (v2 > v || (v2 == v && i2 < vi)) {
                v = v2;
                vi = i2;
            }
        }
        if (lane == 0) {
            wv[wid] = v;
            wi[wid] = vi;
        }
        __syncthreads();
        if (tid == 0) {
            double bv = -1.0;
            int bi = nc;
            for (int w = 0; w < kInvThreads / 32; ++w)
                if (wv[w] > bv || (wv[w] == bv && wi[w] < bi)) {
                    bv = wv[w];
                    bi = wi[w];
                }
            cand_v = bv;
            cand_i = bi;
        }
        cl.sync();
        if (tid == 0) {
            double bv = -1.0;
            int bi = nc;
            for (int q = 0; q < ncta; ++q) {
                const double x = *cl.map_shared_rank(&cand_v, q);
                const int xi = *cl.map_shared_rank(&cand_i, q);
                if (x > bv || (x == bv && xi < bi)) {
                    bv = x;
                    bi = xi;
                }
            }
            piv_s = bi;
            bad_s = !(bv > tiny) || bi >= nc;
        }
        __syncthreads();
        if (bad_s) {
            bad = 1;
            break;
        }
        const int p = piv_s, ok = k / rp, op = p / rp;
        if (p != k) {
            if (ok == op) {
                if (rank == ok)
                    for (int j = tid; j < w2; j += blockDim.x) {
                        const double t = rows[(size_t)(k - r0) * w2 + j];
                        rows[(size_t)(k - r0) * w2 + j] = rows[(size_t)(p - r0) * w2 + j];
                        rows[(size_t)(p - r0) * w2 + j] = t;
                    }
                cl.sync();
            } else {
                if (rank == ok)
                    for (int j = tid; j < w2; j += blockDim.x) trow[j] = rows[(size_t)(k - r0) * w2 + j];
                if (rank == op)
                    for (int j = tid; j < w2; j += blockDim.x) trow[j] = rows[(size_t)(p - r0) * w2 + j];
                cl.sync();
                if (rank == ok) {
                    const double *src = cl.map_shared_rank(trow, op);
                    for (int j = tid; j < w2; j += blockDim.x) rows[(size_t)(k - r0) * w2 + j] = src[j];
                }
                if (rank == op) {
                    const double *src = cl.map_shared_rank(trow, ok);
                    for (int j = tid; j < w2; j += blockDim.x) rows[(size_t)(p - r0) * w2 + j] = src[j];
                }
                cl.sync();
            }
        }
        if (rank == ok) {
            const double inv = 1.0 / rows[(size_t)(k - r0) * w2 + k];
            __syncthreads();
            for (int j = tid; j < w2; j += blockDim.x) rows[(size_t)(k - r0) * w2 + j] *= inv;
        }
        cl.sync();
        {
            const double *src = cl.map_shared_rank(csm, ok) + (size_t)(k - ok * rp) * w2;
            for (int j = tid; j < w2; j += blockDim.x) prow[j] = src[j];
        }
        for (int i = r0 + tid; i < r1; i += blockDim.x) fcol[i - r0] = i == k ? 0.0 : rows[(size_t)(i - r0) * w2 + k];
        __syncthreads();
        for (int q = tid; q < nr * w2; q += blockDim.x) {
            const int il = q / w2, j = q % w2;
            if (r0 + il == k) continue;
            rows[q] = j == k ? 0.0 : fma(-fcol[il], prow[j], rows[q]);
        }
        __syncthreads();
    }
    for (int q = tid; q < nr * nc; q += blockDim.x) {
        const int il = q / nc, j = q % nc;
        einv[(size_t)j * nc + r0 + il] = bad ? 0.f : (float)rows[(size_t)il * w2 + nc + j];
    }
    if (rank == 0 && tid == 0) *bad_out = bad;
    cl.sync();  // no CTA leaves while another may still read its shared memory
}

// W = (A Z) E^-1 in the layout of A Z, so that the solver forms A Z c as
// W (Z^T v) with no product by E^-1 of its own: block (g, 32 columns of W),
// thread r one internal row of group g (the constraint rows: g = nG), the
// 32 columns of E^-1 staged per chunk of k in shared memory.
__global__ void __launch_bounds__(128) k_coarse_w(int nG, int nc, int n_nps, const float *__restrict__ az,
                                                  const float *__restrict__ einv, float *__restrict__ w)
{
    __shared__ float es[32][33];
    const int g = blockIdx.x, j0 = blockIdx.y * 32, r = threadIdx.x;
    const size_t lam = (size_t)nG * nc * kRows;
    const bool rows_ok = g < nG || r < n_nps;
    float acc[32];
#pragma unroll
    for (int q = 0; q < 32; ++q) acc[q] = 0.f;
    for (int k0 = 0; k0 < nc; k0 += 32) {
        __syncthreads();
        for (int q = threadIdx.x; q < 32 * 32; q += blockDim.x) {
            const int kk = q >> 5, jj = q & 31;
            es[kk][jj] = (k0 + kk < nc && j0 + jj < nc) ? einv[(size_t)(k0 + kk) * nc + j0 + jj] : 0.f;
        }
        __syncthreads();
        if (rows_ok) {
            const int kn = min(32, nc - k0);
            for (int kk = 0; kk < kn; ++kk) {
                const float a = g < nG ? az[((size_t)g * nc + k0 + kk) * kRows + r] : az[lam + (size_t)r * nc + k0 + kk];
#pragma unroll
                for (int q = 0; q < 32; ++q) acc[q] = fmaf(a, es[kk][q], acc[q]);
            }
        }
    }
    if (!rows_ok) return;
    for (int q = 0; q < 32 && j0 + q < nc; ++q) {
        if (g < nG)
            w[((size_t)g * nc + j0 + q) * kRows + r] = acc[q];
        else
            w[lam + (size_t)r * nc + j0 + q] = acc[q];
    }
}

}  // namespace

int coarse_columns(int M, int n_nps, int nm) { return nm * precond_groups(M) + n_nps; }
static_assert(2 * kMaxCoarse <= kInvThreads, "one thread per column of [E | I]");

size_t coarse_az_floats(int M, int n_nps, int nm)
{
    const int nG = precond_groups(M), nc = coarse_columns(M, n_nps, nm);
    return (size_t)nG * nc * kRows + (size_t)n_nps * nc;
}

// E^-1 by a cluster of 8 (or 16) CTAs when its rows fit their shared memory
// and such a cluster can be resident, else by one block.
void launch_coarse_invert(capac_ctx *c, int nc)
{
    const int w2 = 2 * nc;
    for (int ncta : {8, 16}) {
        const int rp = (nc + ncta - 1) / ncta;
        const size_t smem = (size_t)(rp + 2) * w2 * sizeof(double);
        if (smem > 200 * 1024) continue;
        if (cudaFuncSetAttribute(k_coarse_invert_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
                cudaSuccess ||
            (ncta > 8 &&
             cudaFuncSetAttribute(k_coarse_invert_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                 cudaSuccess)) {
            cudaGetLastError();
            continue;
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(ncta);
        cfg.blockDim = dim3(kInvThreads);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = c->stream;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = ncta;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, k_coarse_invert_cluster, &cfg) != cudaSuccess || clusters < 1) {
            cudaGetLastError();
            continue;
        }
        CAPAC_CUDA(cudaLaunchKernelEx(&cfg, k_coarse_invert_cluster, nc, (const double *)c->cz_aug, c->cz_einv,
                                      c->flags + 6));
        c->cz_cluster = ncta;
        return;
    }
    c->cz_cluster = 1;
    k_coarse_invert<<<1, kInvThreads, 0, c->stream>>>(nc, c->cz_aug, c->cz_einv, c->flags + 6);
}

void launch_coarse_refresh(capac_ctx *c)
{
    const int nG = precond_groups(c->M), nm = c->cz_modes, nc = coarse_columns(c->M, c->n_nps, nm);
    const int ntiles = nG * (nG + 1) / 2;
    cudaStream_t s = c->stream;
    ProfScope ps(c, K_MATRIX);
    k_coarse_az<<<ntiles, 256, 0, s>>>(static_cast<const float *>(c->msym), nG, nc, nm, c->g_atoms,
                                       c->P.inv_polar, c->P.inv_capac, c->cz_az);
    const int nq = std::max(nG * kRows, c->n_nps * nc);
    k_coarse_az_np<<<grid_for(nq, 256), 256, 0, s>>>(nG, nc, nm, c->n_nps, c->slot_np, c->cz_az);
    k_coarse_e<<<nc, 256, 0, s>>>(nG, nc, nm, c->g_atoms, c->cz_az, c->cz_aug);
    if (c->cz_one_block) {
        c->cz_cluster = 1;
        k_coarse_invert<<<1, kInvThreads, 0, s>>>(nc, c->cz_aug, c->cz_einv, c->flags + 6);
    } else {
        launch_coarse_invert(c, nc);
    }
    k_coarse_w<<<dim3(nG + (c->n_nps > 0 ? 1 : 0), (nc + 31) / 32), kRows, 0, s>>>(nG, nc, c->n_nps, c->cz_az,
                                                                                    c->cz_einv, c->cz_w);
    c->launches += 5;
}

}  // namespace capac
