// Block-Jacobi preconditioner for the mixed path's inner BiCGSTAB.
//
// The reference preconditions BiCGSTAB with the matrix diagonal (Jacobi,
// bicg_stab.c:328-347); the FP64 path keeps that.  On the mixed path the
// inner solves only have to reduce the residual of an FP64 refinement
// sweep, so they may use a stronger preconditioner without changing the
// answer, which the FP64 residual defines.  The metal atoms are cut into
// groups of 32 along a Morton (Z-order) curve of their initial positions, so
// a group is a compact piece of the cluster; each group's 128 x 128 diagonal
// block of the CPIM matrix (its dipole-dipole, dipole-charge and
// charge-charge couplings plus the diagonal 1/polar, -1/capac) is inverted in
// FP64 and stored in FP32.  Applying the inverse couples the unknowns of
// neighbouring atoms that the diagonal alone leaves apart; on the 9.3k-atom
// system it cuts the iterations to a relative residual of 1e-10 from 117 to
// about 50.  The neutrality rows keep a unit preconditioner.  The inverse
// blocks are refreshed every 10 matrix builds (and after positions are set
// from outside): in MD the atoms move little between refreshes, and a
// slightly stale preconditioner changes only the inner iteration count.
//
// Layout: g_atoms[G * 32 + a] = metal index (0-based, -1 for padding) of slot
// a of group G; local row o = 4 a + c (c = 0..2 dipole, 3 charge);
// dinv[G][c][o] = (D_G^-1)[o][c] (column-major, so the threads of a warp
// reading one column for their rows are coalesced).
#include <algorithm>
#include <cstdint>
#include <vector>

#include "terms.cuh"

namespace capac {

namespace {

constexpr int kG = 32;             // atoms per group
constexpr int kN = 4 * kG;         // rows per block
constexpr int kInvThreads = 256;

// In-place Gauss-Jordan inversion with partial pivoting of the group's
// block, FP64 in shared memory; one block per group.  A pivot below
// 1e-13 of the block's largest entry falls back to the Jacobi inverse for
// this group (never observed; it keeps a degenerate block harmless).
__global__ void __launch_bounds__(kInvThreads) k_block_inverse(DevParams P, const double4 *__restrict__ pos4,
                                                               const int *__restrict__ g_atoms, float *__restrict__ dinv)
{
    extern __shared__ double Dm[];  // kN * kN, row-major
    __shared__ int piv[kN];
    __shared__ double fcol[kN];
    __shared__ double wv[kInvThreads / 32];
    __shared__ int wi[kInvThreads / 32];
    __shared__ int bad;
    __shared__ double amax;
    const int G = blockIdx.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int *atoms = g_atoms + (size_t)G * kG;
    if (tid == 0) bad = 0;

    // the block: diagonal terms and cpim_block for every ordered pair of the group
    for (int q = tid; q < kG * kG; q += blockDim.x) {
        const int a = q / kG, b = q % kG;
        const int ia = atoms[a], ib = atoms[b];
        double e[16];
        if (ia < 0 || ib < 0) {
#pragma unroll
            for (int k = 0; k < 16; ++k) e[k] = 0.0;
            if (a == b)
#pragma unroll
                for (int k = 0; k < 4; ++k) e[5 * k] = 1.0;  // padding slot: identity
        } else {
            cpim_block(P, pos4[P.metal_min + ia], pos4[P.metal_min + ib], a == b, e);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) Dm[(4 * a + r) * kN + 4 * b + cc] = e[4 * r + cc];
    }
    __syncthreads();
    {
        double m = 0.0;
        for (int q = tid; q < kN * kN; q += blockDim.x) m = fmax(m, fabs(Dm[q]));
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

    for (int k = 0; k < kN; ++k) {
        // pivot: largest |D[i][k]|, i >= k (lowest i on ties)
        double v = -1.0;
        int vi = kN;
        if (tid >= k && tid < kN) {
            v = fabs(Dm[tid * kN + k]);
            vi = tid;
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
            int bi = kN;
            for (int w = 0; w < kInvThreads / 32; ++w)
                if (wv[w] > bv || (wv[w] == bv && wi[w] < bi)) {
                    bv = wv[w];
                    bi = wi[w];
                }
            piv[k] = bi;
            if (!(bv > tiny) || bi >= kN) bad = 1;
        }
        __syncthreads();
        if (bad) break;
        const int p = piv[k];
        if (p != k)
            for (int j = tid; j < kN; j += blockDim.x) {
                const double t = Dm[k * kN + j];
                Dm[k * kN + j] = Dm[p * kN + j];
                Dm[p * kN + j] = t;
            }
        __syncthreads();
        const double inv = 1.0 / Dm[k * kN + k];
        for (int i = tid; i < kN; i += blockDim.x) fcol[i] = i == k ? 0.0 : Dm[i * kN + k];
        __syncthreads();
        for (int j = tid; j < kN; j += blockDim.x) Dm[k * kN + j] = (j == k ? 1.0 : Dm[k * kN + j]) * inv;
        __syncthreads();
        for (int q = tid; q < kN * kN; q += blockDim.x) {
            const int i = q / kN, j = q % kN;
            if (i == k) continue;
            const double base = j == k ? 0.0 : Dm[q];
            Dm[q] = fma(-fcol[i], Dm[k * kN + j], base);
        }
        __syncthreads();
    }
    if (!bad) {
        // undo the row interchanges as column interchanges, last first
        for (int k = kN - 1; k >= 0; --k) {
            const int p = piv[k];
            if (p != k)
                for (int i = tid; i < kN; i += blockDim.x) {
                    const double t = Dm[i * kN + k];
                    Dm[i * kN + k] = Dm[i * kN + p];
                    Dm[i * kN + p] = t;
                }
            __syncthreads();
        }
    }
    float *out = dinv + (size_t)G * kN * kN;
    for (int q = tid; q < kN * kN; q += blockDim.x) {
        const int c = q / kN, o = q % kN;  // out[c][o] = inverse[o][c]
        float val;
        if (!bad) {
            val = (float)Dm[o * kN + c];
        } else {  // Jacobi for this group
            const int a = o >> 2, comp = o & 3;
            const double d = atoms[a] < 0 ? 1.0 : (comp < 3 ? P.inv_polar : -P.inv_capac);
            val = c == o ? (float)(1.0 / d) : 0.0f;
        }
        out[q] = val;
    }
}

// Interleave the low 21 bits of v with two zero bits after each (Morton key).
uint64_t spread3(uint64_t v)
{
    uint64_t out = 0;
    for (int b = 0; b < 21; ++b) out |= ((v >> b) & 1ull) << (3 * b);
    return out;
}

}  // namespace

int precond_groups(int M) { return (M + kG - 1) / kG; }
size_t precond_inverse_floats(int M) { return (size_t)precond_groups(M) * kN * kN; }

// Groups of 32 metal atoms along the Morton curve of the positions given
// (metal_min .. metal_min + M - 1), as g_atoms above.
std::vector<int> precond_group_atoms(int M, int metal_min, const double *rx, const double *ry, const double *rz)
{
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    const double *r[3] = {rx, ry, rz};
    for (int i = 0; i < M; ++i)
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], r[a][metal_min + i]);
            hi[a] = std::max(hi[a], r[a][metal_min + i]);
        }
    double span = 0.0;
    for (int a = 0; a < 3; ++a) span = std::max(span, hi[a] - lo[a]);
    if (span <= 0.0) span = 1.0;
    std::vector<std::pair<uint64_t, int>> key(M);
    for (int i = 0; i < M; ++i) {
        uint64_t k = 0;
        for (int a = 0; a < 3; ++a) {
            const uint64_t q = (uint64_t)std::min(1048575.0, (r[a][metal_min + i] - lo[a]) / span * 1048575.0);
            k |= spread3(q) << a;
        }
        key[i] = {k, i};
    }
    std::stable_sort(key.begin(), key.end(), [](const auto &x, const auto &y) { return x.first < y.first; });
    const int nG = precond_groups(M);
    std::vector<int> g((size_t)nG * kG, -1);
    for (int i = 0; i < M; ++i) g[i] = key[i].second;
    return g;
}

void launch_block_inverse(capac_ctx *c)
{
    const int nG = precond_groups(c->M);
    const size_t smem = sizeof(double) * kN * kN;
    CAPAC_CUDA(cudaFuncSetAttribute(k_block_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ProfScope ps(c, K_MATRIX);
    k_block_inverse<<<nG, kInvThreads, smem, c->stream>>>(c->P, c->pos4, c->g_atoms, c->dinv);
    ++c->launches;
}

}  // namespace capac
