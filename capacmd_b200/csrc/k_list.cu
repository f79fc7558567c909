// Cell list and Verlet neighbour list.
//
// The reference has no neighbour structure: mpi_nonb_pair (force.c:1419-1473)
// visits every j < i and keeps a pair when it is not excluded and
// dist_2(pbc_12(r_j - r_i)) < rCut^2.  Here atoms are binned into cells of edge
// >= (rc + skin) / 2 (wrapped coordinates) and sorted by cell, with a
// cell-ordered copy of the positions; each atom's full list holds every
// non-excluded j within rc + skin under the same pbc_12 metric on the
// unwrapped coordinates.  A warp scans the 5 x 5 cells around its atom in x
// and y, each as one contiguous run of five z cells of the sorted copy
// (coalesced loads), tests the distance first and the exclusions only for
// the survivors.  The pair kernel re-applies the exact FP64 cut-off
// every step, so the set of interacting pairs equals the reference's as long
// as no atom has moved more than skin/2 since the build; a displacement check
// every step triggers the rebuild.
//
// The atom order within a cell comes from a stable radix sort on the cell key,
// so lists (and hence force summation order) are identical run to run.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>

#include "ctx.h"

namespace capac {

namespace {

__device__ __forceinline__ int cell_coord(double x, double L, double inv_len, int n)
{
    double w = x - L * floor(x / L);
    int c = (int)(w * inv_len);
    return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

struct Grid {
    int n[3];
    double inv_len[3];
};

__global__ void k_cell_keys(int N, const double *__restrict__ rx, const double *__restrict__ ry,
                            const double *__restrict__ rz, Box box, Grid g, int *key, int *ids)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int cx = cell_coord(rx[i], box.L[0], g.inv_len[0], g.n[0]);
    const int cy = cell_coord(ry[i], box.L[1], g.inv_len[1], g.n[1]);
    const int cz = cell_coord(rz[i], box.L[2], g.inv_len[2], g.n[2]);
    key[i] = (cx * g.n[1] + cy) * g.n[2] + cz;
    ids[i] = i;
}

// start[c] = first sorted position with key >= c, for c = 0 .. n_cells
// (empty cells included), so the atoms of cells a..b are start[a] ..
// start[b + 1] - 1.
__global__ void k_cell_starts(int N, int n_cells, const int *__restrict__ key, int *start)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > N) return;
    const int prev = p > 0 ? key[p - 1] : -1;
    const int cur = p < N ? key[p] : n_cells;
    for (int c = prev + 1; c <= cur; ++c) start[c] = p;
}

// Positions in cell order, with the atom index in w.
__global__ void k_sorted_positions(int N, const int *__restrict__ ids, const double *__restrict__ rx,
                                   const double *__restrict__ ry, const double *__restrict__ rz, double4 *spos)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    const int j = ids[p];
    spos[p] = make_double4(rx[j], ry[j], rz[j], (double)j);
}

__device__ __forceinline__ bool excluded(const DevParams &P, int i, int j)
{
    if (P.mol_id[i] != P.mol_id[j]) return false;
    const int m = P.mol_type[i], na = P.mol_atoms[m];
    return P.excl[P.excl_offset[m] + P.atom_in_mol[i] * na + P.atom_in_mol[j]] != 0;
}

// The k-th cell along one axis around cell c: c-2 .. c+2 (periodic) when
// the axis has at least five cells, else the axis has one cell.
__device__ __forceinline__ int axis_count(int n) { return n < 5 ? 1 : 5; }
__device__ __forceinline__ int axis_cell(int c, int n, int k) { return n < 5 ? 0 : (c + k - 2 + n) % n; }

// One warp per atom i.
__global__ void __launch_bounds__(256) k_build_list(DevParams P, Grid g, const double *__restrict__ rx,
                                                    const double *__restrict__ ry,
                                                    const double *__restrict__ rz,
                                                    const double4 *__restrict__ spos,
                                                    const int *__restrict__ cell_start, int cap,
                                                    uint32_t *__restrict__ nbr, int *__restrict__ nnb,
                                                    double *rx0, double *ry0, double *rz0, int *flags)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= P.N) return;
    const double xi = rx[i], yi = ry[i], zi = rz[i];
    const int c0[3] = {cell_coord(xi, P.box.L[0], g.inv_len[0], g.n[0]),
                       cell_coord(yi, P.box.L[1], g.inv_len[1], g.n[1]),
                       cell_coord(zi, P.box.L[2], g.inv_len[2], g.n[2])};
    const int nxs = axis_count(g.n[0]), nys = axis_count(g.n[1]);
    // the z window as one or two runs of consecutive cells
    const int nz = g.n[2];
    int za[2], zb[2], nzr;
    if (nz < 5) {
        za[0] = 0; zb[0] = nz - 1; nzr = 1;
    } else {
        const int lo = c0[2] - 2, hi = c0[2] + 2;
        if (lo < 0) {
            za[0] = lo + nz; zb[0] = nz - 1; za[1] = 0; zb[1] = hi; nzr = 2;
        } else if (hi >= nz) {
            za[0] = lo; zb[0] = nz - 1; za[1] = 0; zb[1] = hi - nz; nzr = 2;
        } else {
            za[0] = lo; zb[0] = hi; nzr = 1;
        }
    }
    const unsigned lt_mask = (1u << lane) - 1u;
    uint32_t *row = nbr + (size_t)i * cap;
    int count = 0;
    for (int ix = 0; ix < nxs; ++ix) {
        for (int iy = 0; iy < nys; ++iy) {
            const int col = (axis_cell(c0[0], g.n[0], ix) * g.n[1] + axis_cell(c0[1], g.n[1], iy)) * nz;
            for (int r = 0; r < nzr; ++r) {
                const int s = cell_start[col + (r ? za[1] : za[0])], e = cell_start[col + (r ? zb[1] : zb[0]) + 1];
                for (int base = s; base < e; base += 32) {
                    const int p = base + lane;
                    bool ok = false;
                    int j = 0;
                    if (p < e) {
                        const double4 q = spos[p];
                        j = (int)q.w;
                        double dx = q.x - xi, dy = q.y - yi, dz = q.z - zi;
                        image(dx, dy, dz, P.box);
                        ok = j != i && norm2_exact(dx, dy, dz) < P.list_r2;
                        if (ok) ok = !excluded(P, i, j);
                    }
                    const unsigned ballot = __ballot_sync(0xffffffffu, ok);
                    const int pos = count + __popc(ballot & lt_mask);
                    if (ok && pos < cap) row[pos] = pack_nb(j, P.type[j]);
                    count += __popc(ballot);
                }
            }
        }
    }
    if (lane == 0) {
        nnb[i] = count < cap ? count : cap;
        if (count > cap) atomicMax(&flags[1], count);
        rx0[i] = xi;
        ry0[i] = yi;
        rz0[i] = zi;
    }
}

__global__ void k_displacement(int N, Box box, double half_skin2, const double *__restrict__ rx,
                               const double *__restrict__ ry, const double *__restrict__ rz,
                               const double *__restrict__ rx0, const double *__restrict__ ry0,
                               const double *__restrict__ rz0, int *flags)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double dx = wrap1(rx[i] - rx0[i], box.L[0]);
    const double dy = wrap1(ry[i] - ry0[i], box.L[1]);
    const double dz = wrap1(rz[i] - rz0[i], box.L[2]);
    if (dx * dx + dy * dy + dz * dz > half_skin2) flags[0] = 1;
}

// Pair-set fingerprint over the list: the j < i entries inside the cut-off.
__global__ void k_fingerprint_list(DevParams P, const double *__restrict__ rx, const double *__restrict__ ry,
                                   const double *__restrict__ rz, const uint32_t *__restrict__ nbr,
                                   const int *__restrict__ nnb, int cap, unsigned long long *out)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= P.N) return;
    unsigned long long cnt = 0, h = 0;
    const double xi = rx[i], yi = ry[i], zi = rz[i];
    for (int k = lane; k < nnb[i]; k += 32) {
        const int j = nb_index(nbr[(size_t)i * cap + k]);
        if (j >= i) continue;
        double dx = rx[j] - xi, dy = ry[j] - yi, dz = rz[j] - zi;
        image(dx, dy, dz, P.box);
        if (norm2_exact(dx, dy, dz) < P.rc2) {
            ++cnt;
            h += mix64(((uint64_t)(uint32_t)i << 32) | (uint32_t)j);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        h += __shfl_xor_sync(0xffffffffu, h, o);
    }
    if (lane == 0 && cnt) {
        atomicAdd(&out[0], cnt);
        atomicAdd(&out[1], h);
    }
}

// Pair-set fingerprint by enumerating all j < i, as the reference loop does.
__global__ void k_fingerprint_all(DevParams P, const double *__restrict__ rx, const double *__restrict__ ry,
                                  const double *__restrict__ rz, unsigned long long *out)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= P.N) return;
    unsigned long long cnt = 0, h = 0;
    const double xi = rx[i], yi = ry[i], zi = rz[i];
    for (int j = lane; j < i; j += 32) {
        if (excluded(P, i, j)) continue;
        double dx = rx[j] - xi, dy = ry[j] - yi, dz = rz[j] - zi;
        image(dx, dy, dz, P.box);
        if (norm2_exact(dx, dy, dz) < P.rc2) {
            ++cnt;
            h += mix64(((uint64_t)(uint32_t)i << 32) | (uint32_t)j);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        h += __shfl_xor_sync(0xffffffffu, h, o);
    }
    if (lane == 0 && cnt) {
        atomicAdd(&out[0], cnt);
        atomicAdd(&out[1], h);
    }
}

__global__ void k_pack(int N, const double *__restrict__ rx, const double *__restrict__ ry,
                       const double *__restrict__ rz, const double *__restrict__ q, double4 *pos4,
                       float4 *pos4f)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double4 p = make_double4(rx[i], ry[i], rz[i], q[i]);
    pos4[i] = p;
    if (pos4f) pos4f[i] = make_float4((float)p.x, (float)p.y, (float)p.z, (float)p.w);
}

Grid make_grid(const capac_ctx *c)
{
    Grid g;
    const double len = 0.5 * (c->P.rc + c->opt.skin);
    for (int a = 0; a < 3; ++a) {
        int n = (int)floor(c->P.box.L[a] / len);
        if (n < 5) n = 1;
        g.n[a] = n;
        g.inv_len[a] = n / c->P.box.L[a];
    }
    return g;
}

void build_list(capac_ctx *c)
{
    const int N = c->N;
    const Grid g = make_grid(c);
    const int n_cells = g.n[0] * g.n[1] * g.n[2];
    if (n_cells != c->n_cells || !c->cell_start) {
        cudaFree(c->cell_start);
        c->cell_start = nullptr;
        CAPAC_CUDA(cudaMalloc(&c->cell_start, sizeof(int) * (n_cells + 1)));
        c->n_cells = n_cells;
    }
    if (!c->spos) CAPAC_CUDA(cudaMalloc(&c->spos, sizeof(double4) * N));
    for (int a = 0; a < 3; ++a) c->ncell[a] = g.n[a];
    cudaStream_t s = c->stream;
    k_cell_keys<<<grid_for(N, 256), 256, 0, s>>>(N, c->rx, c->ry, c->rz, c->P.box, g, c->cell_key, c->atom_ids);
    ++c->launches;
    int end_bit = 1;
    while ((1 << end_bit) < n_cells) ++end_bit;
    size_t need = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, need, c->cell_key, c->cell_key_sorted, c->atom_ids,
                                    c->cell_atoms, N, 0, end_bit, s);
    if (need > c->sort_tmp_bytes) {
        cudaFree(c->sort_tmp);
        CAPAC_CUDA(cudaMalloc(&c->sort_tmp, need));
        c->sort_tmp_bytes = need;
    }
    CAPAC_CUDA(cub::DeviceRadixSort::SortPairs(c->sort_tmp, need, c->cell_key, c->cell_key_sorted,
                                               c->atom_ids, c->cell_atoms, N, 0, end_bit, s));
    k_cell_starts<<<grid_for(N + 1, 256), 256, 0, s>>>(N, n_cells, c->cell_key_sorted, c->cell_start);
    k_sorted_positions<<<grid_for(N, 256), 256, 0, s>>>(N, c->cell_atoms, c->rx, c->ry, c->rz, c->spos);
    c->launches += 2;
    for (int attempt = 0; attempt < 4; ++attempt) {
        CAPAC_CUDA(cudaMemsetAsync(c->flags + 1, 0, sizeof(int), s));
        {
            ProfScope ps(c, K_LIST);
            k_build_list<<<grid_for((long)N * 32, 256), 256, 0, s>>>(
                c->P, g, c->rx, c->ry, c->rz, c->spos, c->cell_start, c->cap, c->nbr, c->nnb, c->rx0,
                c->ry0, c->rz0, c->flags);
        }
        ++c->launches;
        CAPAC_CUDA(cudaMemcpyAsync(c->h_flags, c->flags, sizeof(int) * 4, cudaMemcpyDeviceToHost, s));
        CAPAC_CUDA(cudaStreamSynchronize(s));
        const int need_cap = c->h_flags[1];
        if (need_cap <= c->cap) break;
        // grow the per-atom capacity and rebuild
        int new_cap = (int)std::min<long>((long)(need_cap * 1.25) + 32, 1L << 20);
        new_cap = (new_cap + 31) & ~31;
        cudaFree(c->nbr);
        c->nbr = nullptr;
        CAPAC_CUDA(cudaMalloc(&c->nbr, sizeof(uint32_t) * (size_t)N * new_cap));
        c->cap = new_cap;
        if (attempt == 3) throw Error(CAPAC_ERR_CAPACITY, "neighbour list capacity could not be met");
    }
    c->list_valid = true;
    ++c->list_builds;
}

}  // namespace

void launch_pack_positions(capac_ctx *c)
{
    k_pack<<<grid_for(c->N, 256), 256, 0, c->stream>>>(c->N, c->rx, c->ry, c->rz, c->charge, c->pos4,
                                                       c->pos4f);
    ++c->launches;
}

void launch_list_maintenance(capac_ctx *c, bool force_rebuild)
{
    if (!c->list_valid || force_rebuild) {
        build_list(c);
        return;
    }
    const double hs = 0.5 * c->opt.skin;
    CAPAC_CUDA(cudaMemsetAsync(c->flags, 0, sizeof(int), c->stream));
    k_displacement<<<grid_for(c->N, 256), 256, 0, c->stream>>>(c->N, c->P.box, hs * hs, c->rx, c->ry, c->rz,
                                                               c->rx0, c->ry0, c->rz0, c->flags);
    ++c->launches;
    CAPAC_CUDA(cudaMemcpyAsync(c->h_flags, c->flags, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CAPAC_CUDA(cudaStreamSynchronize(c->stream));
    if (c->h_flags[0]) build_list(c);
}

void launch_pair_fingerprint(capac_ctx *c, int from_list, long *count, unsigned long long *hash)
{
    unsigned long long *d = reinterpret_cast<unsigned long long *>(c->partials);
    CAPAC_CUDA(cudaMemsetAsync(d, 0, 2 * sizeof(unsigned long long), c->stream));
    if (from_list) {
        launch_list_maintenance(c, false);
        k_fingerprint_list<<<grid_for((long)c->N * 32, 256), 256, 0, c->stream>>>(
            c->P, c->rx, c->ry, c->rz, c->nbr, c->nnb, c->cap, d);
    } else {
        k_fingerprint_all<<<grid_for((long)c->N * 32, 256), 256, 0, c->stream>>>(c->P, c->rx, c->ry, c->rz, d);
    }
    ++c->launches;
    unsigned long long h[2];
    CAPAC_CUDA(cudaMemcpyAsync(h, d, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    CAPAC_CUDA(cudaStreamSynchronize(c->stream));
    *count = (long)h[0];
    *hash = h[1];
}

}  // namespace capac
