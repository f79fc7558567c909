// CPIM matrix in symmetric packed 4x4-block form and its SpMV.
//
// The CPIM matrix is symmetric (cpff.c:245-436): for metal atoms i, j with
// r = r_j - r_i the ordered block is
//     B_ij = [ A   m  ]      A = -(c1 (3 r r^T - r^2 I) - c2 r r^T)  (symmetric 3x3)
//            [ -m^T C ]      m = c3 r,   C = -erf(r/R_qq)/r
// and B_ji = [ A  -m ; m^T C ].  So one unordered pair needs 10 numbers
// (A: 6, m: 3, C: 1) instead of 32 for the two ordered blocks.  Diagonal
// blocks are diag(1/polar x3, -1/capac) and are applied analytically; the
// neutrality rows and columns as in the plane SpMV.
//
// Storage: tiles of 32 x 32 atoms over the upper triangle (I <= J), 10 planes
// per tile, each plane laid out [b/4][a][b%4] (a = row atom in the tile, b =
// column atom) so a warp reading one plane for a fixed column quad is
// coalesced.  Entries for a >= b of diagonal tiles and for padded atoms are 0.
// At M = 2057 the FP32 form is 85.8 MB and stays in the 126 MB L2 across the
// SpMVs of one solve.
//
// SpMV: one block per tile computes, for its 32 rows, sum_b B_ab x_b and, for
// its 32 columns, sum_a B_ba x_a; the two partial vectors go to
// part[I][J] and part[J][I] (summed together on diagonal tiles).  A second
// kernel adds the nT partials of each block row in a fixed order, applies the
// diagonal and neutrality terms, and writes y with the solver's dot products.
#include <vector>

#include "terms.cuh"

namespace capac {

namespace {

constexpr int kT = 32;        // atoms per tile edge
constexpr int kPlanes = 10;   // A_xx A_xy A_xz A_yy A_yz A_zz m_x m_y m_z C
constexpr size_t kTileElems = (size_t)kPlanes * kT * kT;

__host__ __device__ __forceinline__ size_t tile_index(int I, int J, int nT)
{
    // row-major upper triangle including the diagonal
    return (size_t)I * nT - (size_t)I * (I - 1) / 2 + (size_t)(J - I);
}

__host__ __device__ __forceinline__ size_t elem_offset(int p, int a, int b)
{
    return ((size_t)p * (kT / 4) + (b >> 2)) * (kT * 4) + (size_t)a * 4 + (b & 3);
}

__device__ __forceinline__ void load4(const float *p, double out[4])
{
    const float4 v = *reinterpret_cast<const float4 *>(p);
    out[0] = v.x;
    out[1] = v.y;
    out[2] = v.z;
    out[3] = v.w;
}
__device__ __forceinline__ void load4(const double *p, double out[4])
{
    const double2 u = *reinterpret_cast<const double2 *>(p);
    const double2 v = *reinterpret_cast<const double2 *>(p + 2);
    out[0] = u.x;
    out[1] = u.y;
    out[2] = v.x;
    out[3] = v.y;
}

// Assembly: one block per tile, 256 threads, 4 pairs each.
template <typename T>
// slots: null for the metal atoms in index order, else the atom of each
// tile slot (-1 for padding): the group order of the grouped solver.
__global__ void __launch_bounds__(256) k_sym_assemble(DevParams P, const double4 *__restrict__ pos4, int nT,
                                                      const int *__restrict__ slots, T *__restrict__ mat)
{
    // decode the tile from the linear index
    const size_t t = blockIdx.x;
    int I = 0;
    while (tile_index(I + 1, I + 1, nT) <= t && I + 1 < nT) ++I;
    const int J = I + (int)(t - tile_index(I, I, nT));
    T *tile = mat + t * kTileElems;
    for (int q = threadIdx.x; q < kT * kT; q += blockDim.x) {
        const int a = q & (kT - 1), b = q >> 5;
        int i = I * kT + a, j = J * kT + b;
        if (slots) {
            i = slots[i];
            j = slots[j];
        } else {
            i = i < P.M ? i : -1;
            j = j < P.M ? j : -1;
        }
        double v[kPlanes];
#pragma unroll
        for (int p = 0; p < kPlanes; ++p) v[p] = 0.0;
        if (i >= 0 && j >= 0 && (I != J || a < b)) {
            double e[16];
            cpim_block(P, pos4[P.metal_min + i], pos4[P.metal_min + j], false, e);
            v[0] = e[0]; v[1] = e[1]; v[2] = e[2]; v[3] = e[5]; v[4] = e[6]; v[5] = e[10];
            v[6] = e[3]; v[7] = e[7]; v[8] = e[11];
            v[9] = e[15];
        }
#pragma unroll
        for (int p = 0; p < kPlanes; ++p) tile[elem_offset(p, a, b)] = (T)v[p];
    }
}

// Tile SpMV: thread (a = lane, b quad = warp) handles rows a, columns 4 w..4 w+3.
template <typename T>
__global__ void __launch_bounds__(256) k_sym_tiles(int M, int nT, const T *__restrict__ mat,
                                                   const double *__restrict__ x, double *__restrict__ part,
                                                   const SolverScalars *ss)
{
    __shared__ double xr[kT][4], xc[kT][4];
    __shared__ double rowacc[8][kT][4];
    if (ss && ss->done) return;
    const size_t t = blockIdx.x;
    int I = 0;
    while (tile_index(I + 1, I + 1, nT) <= t && I + 1 < nT) ++I;
    const int J = I + (int)(t - tile_index(I, I, nT));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x < kT) {
        const int i = I * kT + threadIdx.x;
        const bool in = i < M;
        xr[threadIdx.x][0] = in ? x[3 * i] : 0.0;
        xr[threadIdx.x][1] = in ? x[3 * i + 1] : 0.0;
        xr[threadIdx.x][2] = in ? x[3 * i + 2] : 0.0;
        xr[threadIdx.x][3] = in ? x[3 * M + i] : 0.0;
    } else if (threadIdx.x < 2 * kT) {
        const int b = threadIdx.x - kT, j = J * kT + b;
        const bool in = j < M;
        xc[b][0] = in ? x[3 * j] : 0.0;
        xc[b][1] = in ? x[3 * j + 1] : 0.0;
        xc[b][2] = in ? x[3 * j + 2] : 0.0;
        xc[b][3] = in ? x[3 * M + j] : 0.0;
    }
    __syncthreads();
    const T *tile = mat + t * kTileElems;
    const int a = lane;
    // the four columns 4w..4w+3 of every plane: one 4-wide load per plane
    double vv[kPlanes][4];
#pragma unroll
    for (int p = 0; p < kPlanes; ++p) load4(tile + elem_offset(p, a, 4 * w), vv[p]);
    double ra[4] = {0.0, 0.0, 0.0, 0.0};  // row a partial
    double cb[4][4];                       // column partials for b = 4w + k
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int b = 4 * w + k;
        double v[kPlanes];
#pragma unroll
        for (int p = 0; p < kPlanes; ++p) v[p] = vv[p][k];
        const double A[3][3] = {{v[0], v[1], v[2]}, {v[1], v[3], v[4]}, {v[2], v[4], v[5]}};
        const double m[3] = {v[6], v[7], v[8]};
        const double C = v[9];
        // row a:  y_a^p += A x_b^p + m x_b^q ;  y_a^q += -m.x_b^p + C x_b^q
#pragma unroll
        for (int r = 0; r < 3; ++r) ra[r] += A[r][0] * xc[b][0] + A[r][1] * xc[b][1] + A[r][2] * xc[b][2] + m[r] * xc[b][3];
        ra[3] += -(m[0] * xc[b][0] + m[1] * xc[b][1] + m[2] * xc[b][2]) + C * xc[b][3];
        // column b (block B_ba = [A -m; m^T C]):  y_b^p += A x_a^p - m x_a^q ; y_b^q += m.x_a^p + C x_a^q
#pragma unroll
        for (int r = 0; r < 3; ++r)
            cb[k][r] = A[r][0] * xr[a][0] + A[r][1] * xr[a][1] + A[r][2] * xr[a][2] - m[r] * xr[a][3];
        cb[k][3] = m[0] * xr[a][0] + m[1] * xr[a][1] + m[2] * xr[a][2] + C * xr[a][3];
    }
    // column sums over the 32 rows (lanes) of this warp
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int r = 0; r < 4; ++r) cb[k][r] = warp_sum(cb[k][r]);
    // row sums over the 8 warps
#pragma unroll
    for (int r = 0; r < 4; ++r) rowacc[w][a][r] = ra[r];
    __syncthreads();
    double *pr = part + ((size_t)I * nT + J) * (kT * 4);  // rows of block I from tile (I, J)
    double *pc = part + ((size_t)J * nT + I) * (kT * 4);  // rows of block J from tile (I, J)
    if (I != J) {
        if (threadIdx.x < kT * 4) {
            const int aa = threadIdx.x >> 2, r = threadIdx.x & 3;
            double s = 0.0;
#pragma unroll
            for (int ww = 0; ww < 8; ++ww) s += rowacc[ww][aa][r];
            pr[aa * 4 + r] = s;
        }
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int r = 0; r < 4; ++r) pc[(4 * w + k) * 4 + r] = cb[k][r];
        }
    } else {
        // diagonal tile: row and column partials land on the same atoms
        __shared__ double colacc[kT][4];
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int r = 0; r < 4; ++r) colacc[4 * w + k][r] = cb[k][r];
        }
        __syncthreads();
        if (threadIdx.x < kT * 4) {
            const int aa = threadIdx.x >> 2, r = threadIdx.x & 3;
            double s = 0.0;
#pragma unroll
            for (int ww = 0; ww < 8; ++ww) s += rowacc[ww][aa][r];
            pr[aa * 4 + r] = s + colacc[aa][r];
        }
    }
}

// Matrix-free tile product in FP64 (the mixed path's residual): the same
// partials as k_sym_tiles with every unordered pair's block recomputed from
// the positions by cpim_block, so each pair is evaluated once, not twice as in
// the row-wise matrix-free product.  Thread (a = lane, b = 4 w + k).
__global__ void __launch_bounds__(256) k_sym_free_tiles(DevParams P, const double4 *__restrict__ pos4, int nT,
                                                        const double *__restrict__ x, double *__restrict__ part)
{
    __shared__ double xr[kT][4], xc[kT][4];
    __shared__ double4 pr4[kT], pc4[kT];
    __shared__ double rowacc[8][kT][4];
    __shared__ double colacc[kT][4];
    const int M = P.M;
    const size_t t = blockIdx.x;
    int I = 0;
    while (tile_index(I + 1, I + 1, nT) <= t && I + 1 < nT) ++I;
    const int J = I + (int)(t - tile_index(I, I, nT));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x < 2 * kT) {
        const int side = threadIdx.x >> 5, at = threadIdx.x & 31;
        const int i = (side ? J : I) * kT + at;
        const bool in = i < M;
        double *xv = side ? xc[at] : xr[at];
        xv[0] = in ? x[3 * i] : 0.0;
        xv[1] = in ? x[3 * i + 1] : 0.0;
        xv[2] = in ? x[3 * i + 2] : 0.0;
        xv[3] = in ? x[3 * M + i] : 0.0;
        const double4 p = in ? pos4[P.metal_min + i] : make_double4(0, 0, 0, 0);
        if (side) pc4[at] = p;
        else pr4[at] = p;
    }
    __syncthreads();
    const int a = lane, i = I * kT + a;
    double ra[4] = {0.0, 0.0, 0.0, 0.0};
    double cb[4][4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int b = 4 * w + k, j = J * kT + b;
#pragma unroll
        for (int c = 0; c < 4; ++c) cb[k][c] = 0.0;
        if (i < M && j < M && (I != J || a < b)) {
            double e[16];
            cpim_block(P, pr4[a], pc4[b], false, e);
            const double A[3][3] = {{e[0], e[1], e[2]}, {e[4], e[5], e[6]}, {e[8], e[9], e[10]}};
            const double m[3] = {e[3], e[7], e[11]};
            const double C = e[15];
#pragma unroll
            for (int r = 0; r < 3; ++r)
                ra[r] += A[r][0] * xc[b][0] + A[r][1] * xc[b][1] + A[r][2] * xc[b][2] + m[r] * xc[b][3];
            ra[3] += -(m[0] * xc[b][0] + m[1] * xc[b][1] + m[2] * xc[b][2]) + C * xc[b][3];
#pragma unroll
            for (int r = 0; r < 3; ++r)
                cb[k][r] = A[r][0] * xr[a][0] + A[r][1] * xr[a][1] + A[r][2] * xr[a][2] - m[r] * xr[a][3];
            cb[k][3] = m[0] * xr[a][0] + m[1] * xr[a][1] + m[2] * xr[a][2] + C * xr[a][3];
        }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int c = 0; c < 4; ++c) cb[k][c] = warp_sum(cb[k][c]);
#pragma unroll
    for (int c = 0; c < 4; ++c) rowacc[w][a][c] = ra[c];
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int c = 0; c < 4; ++c) colacc[4 * w + k][c] = cb[k][c];
    }
    __syncthreads();
    double *pr = part + ((size_t)I * nT + J) * (kT * 4);
    double *pc = part + ((size_t)J * nT + I) * (kT * 4);
    if (threadIdx.x < kT * 4) {
        const int aa = threadIdx.x >> 2, c = threadIdx.x & 3;
        double s = 0.0;
#pragma unroll
        for (int ww = 0; ww < 8; ++ww) s += rowacc[ww][aa][c];
        pr[threadIdx.x] = I == J ? s + colacc[aa][c] : s;
    } else if (I != J) {
        const int q = threadIdx.x - kT * 4;
        pc[q] = colacc[q >> 2][q & 3];
    }
}

// y = sum of partials + diagonal + neutrality terms; dot epilogue as k_spmv.
// 512 threads per block row: four groups each add every fourth partial
// (coalesced 1 KB rows), then the groups are added in a fixed order.
constexpr int kReduceGroups = 4;
template <int DOT>
__global__ void __launch_bounds__(128 * kReduceGroups) k_sym_reduce(DevParams P, int nT,
                                                                    const double *__restrict__ part,
                                                                    const double *__restrict__ x,
                                                                    double *__restrict__ y,
                                                                    const double *__restrict__ d1,
                                                                    const double *__restrict__ d2,
                                                                    double *__restrict__ partials,
                                                                    const SolverScalars *ss)
{
    __shared__ double sh[64];
    __shared__ double grp[kReduceGroups][128];
    if (ss && ss->done) return;
    const int M = P.M;
    const int I = blockIdx.x;
    double p0 = 0.0, p1 = 0.0;
    if (I < nT) {
        const int o = threadIdx.x & 127, g = threadIdx.x >> 7;
        {
            double s = 0.0;
            const double *base = part + (size_t)I * nT * (kT * 4) + o;
#pragma unroll 4
            for (int K = g; K < nT; K += kReduceGroups) s += base[(size_t)K * (kT * 4)];
            grp[g][o] = s;
        }
        __syncthreads();
        // thread (a, r): a = atom in tile, r = component
        const int a = threadIdx.x >> 2, r = threadIdx.x & 3;
        const int i = I * kT + a;
        if (threadIdx.x < 128 && i < M) {
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < kReduceGroups; ++q) s += grp[q][threadIdx.x];
            const int row = r < 3 ? 3 * i + r : 3 * M + i;
            if (r < 3) {
                s += P.inv_polar * x[row];
            } else {
                s += -P.inv_capac * x[row];
                const int im = P.metal_min + i;
                for (int k = 0; k < P.n_nps; ++k)
                    if (im >= P.np_start[k] && im <= P.np_end[k]) s += x[4 * M + k];
            }
            y[row] = s;
            if (DOT == 1) p0 = d1[row] * s;
            if (DOT == 2) {
                const double kt = d2[row] * s;
                p0 = kt * d1[row];
                p1 = kt * kt;
            }
        }
    } else {
        const int k = I - nT;
        double acc[1] = {0.0};
        for (int a = P.np_start[k] + threadIdx.x; a <= P.np_end[k]; a += blockDim.x) acc[0] += x[3 * M + (a - P.metal_min)];
        block_sum<1>(acc, sh);
        if (threadIdx.x == 0) {
            const int row = 4 * M + k;
            y[row] = acc[0];
            if (DOT == 1) p0 = d1[row] * acc[0];
            if (DOT == 2) {
                p0 = acc[0] * d1[row];
                p1 = acc[0] * acc[0];
            }
        }
        __syncthreads();
    }
    if (DOT != 0) {
        double v[2] = {p0, p1};
        block_sum<2>(v, sh);
        if (threadIdx.x == 0) {
            partials[2 * blockIdx.x] = v[0];
            partials[2 * blockIdx.x + 1] = v[1];
        }
    }
}

}  // namespace

int sym_tiles(int M) { return (M + kT - 1) / kT; }
size_t sym_matrix_elems(int M)
{
    const size_t nT = sym_tiles(M);
    return nT * (nT + 1) / 2 * kTileElems;
}
size_t sym_partial_doubles(int M)
{
    const size_t nT = sym_tiles(M);
    return nT * nT * kT * 4;
}

void launch_sym_assemble(capac_ctx *c)
{
    const int nT = sym_tiles(c->M);
    const unsigned tiles = (unsigned)(nT * (nT + 1) / 2);
    ProfScope ps(c, K_MATRIX);
    if (c->opt.precision == CAPAC_PREC_MIXED)
        k_sym_assemble<float><<<tiles, 256, 0, c->stream>>>(c->P, c->pos4, nT, c->grouped ? c->g_atoms : nullptr,
                                                             static_cast<float *>(c->msym));
    else
        k_sym_assemble<double><<<tiles, 256, 0, c->stream>>>(c->P, c->pos4, nT, nullptr,
                                                              static_cast<double *>(c->msym));
    ++c->launches;
}

// The FP64 tiles from the reference's COO matrix (mpi_cpff_mat_relay_COO,
// cpff.c:205-519; row and column indices in the reference vector layout).
// The matrix is symmetric and its diagonal blocks and neutrality couplings
// are the fixed constants the tile SpMV applies itself, so only the
// off-diagonal metal-metal entries of the upper block triangle are stored:
// for atoms i < j the six dipole-dipole entries with row comp <= column comp,
// the three dipole (row) - charge (column) entries and the charge-charge one.
// Entries absent from the COO (dropped by the reference) are zero.
void sym_tiles_from_coo(capac_ctx *c, long nnz, const double *val, const long *row, const long *col)
{
    const int M = c->M, nT = sym_tiles(M);
    std::vector<double> host(sym_matrix_elems(M), 0.0);
    static const int plane[4][4] = {{0, 1, 2, 6}, {-1, 3, 4, 7}, {-1, -1, 5, 8}, {-1, -1, -1, 9}};
    for (long k = 0; k < nnz; ++k) {
        const long r = row[k], q = col[k];
        if (r < 0 || q < 0 || r >= 4L * M || q >= 4L * M) continue;  // neutrality rows and columns
        const int i = r < 3L * M ? (int)(r / 3) : (int)(r - 3L * M), a = r < 3L * M ? (int)(r % 3) : 3;
        const int j = q < 3L * M ? (int)(q / 3) : (int)(q - 3L * M), b = q < 3L * M ? (int)(q % 3) : 3;
        if (i >= j) continue;  // the diagonal blocks and the lower triangle
        const int p = plane[a][b];
        if (p < 0) continue;   // the symmetric half of a block
        const int I = i / kT, J = j / kT;
        host[tile_index(I, J, nT) * kTileElems + elem_offset(p, i % kT, j % kT)] = val[k];
    }
    CAPAC_CUDA(cudaMemcpy(c->msym, host.data(), sizeof(double) * host.size(), cudaMemcpyHostToDevice));
}

// Number of blocks whose dot partials the reduction writes (for the solver).
int sym_reduce_blocks(const capac_ctx *c) { return sym_tiles(c->M) + c->n_nps; }

void launch_sym_spmv(capac_ctx *c, int dot, const double *x, double *y, const double *d1, const double *d2,
                     const SolverScalars *ss)
{
    const int nT = sym_tiles(c->M);
    const unsigned tiles = (unsigned)(nT * (nT + 1) / 2);
    ProfScope ps(c, K_SPMV);
    if (c->opt.precision == CAPAC_PREC_MIXED)
        k_sym_tiles<float><<<tiles, 256, 0, c->stream>>>(c->M, nT, static_cast<const float *>(c->msym), x, c->sympart,
                                                          ss);
    else
        k_sym_tiles<double><<<tiles, 256, 0, c->stream>>>(c->M, nT, static_cast<const double *>(c->msym), x,
                                                           c->sympart, ss);
    const unsigned nb = (unsigned)(nT + c->n_nps);
    if (dot == 1)
        k_sym_reduce<1><<<nb, 128 * kReduceGroups, 0, c->stream>>>(c->P, nT, c->sympart, x, y, d1, d2, c->partials, ss);
    else if (dot == 2)
        k_sym_reduce<2><<<nb, 128 * kReduceGroups, 0, c->stream>>>(c->P, nT, c->sympart, x, y, d1, d2, c->partials, ss);
    else
        k_sym_reduce<0><<<nb, 128 * kReduceGroups, 0, c->stream>>>(c->P, nT, c->sympart, x, y, d1, d2, c->partials, ss);
    c->launches += 2;
}

void launch_sym_spmv_free(capac_ctx *c, const double *x, double *y)
{
    const int nT = sym_tiles(c->M);
    const unsigned tiles = (unsigned)(nT * (nT + 1) / 2);
    ProfScope ps(c, K_RESID);
    k_sym_free_tiles<<<tiles, 256, 0, c->stream>>>(c->P, c->pos4, nT, x, c->sympart);
    k_sym_reduce<0><<<(unsigned)(nT + c->n_nps), 128 * kReduceGroups, 0, c->stream>>>(
        c->P, nT, c->sympart, x, y, nullptr, nullptr, c->partials, nullptr);
    c->launches += 2;
}

}  // namespace capac
