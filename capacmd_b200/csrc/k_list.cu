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
// so lists (and hence force summation order) are identical run to run.  The
// key carries, below the cell index, a Morton code of the atom's position on
// an 8 x 8 x 8 grid inside its cell, so consecutive atoms of a cell are
// close together.
//
// Mixed path, cluster list: the atoms of each cell are cut, in that order,
// into clusters of up to four.  Per cluster a warp scans the same 5 x 5 x 5
// cell window; a candidate j within rc + skin + (cluster radius) of the
// cluster's centroid is tested against each member k in FP32 (j's FP64
// minimum image from the centroid, rounded, minus the member's offset) with
// the list radius widened by 1e-5 relative, far beyond the rounding, and
// against the exclusions, and kept with the mask of the members that pass.
// Each member's entries are thus a superset of its atom-list row; the pair
// kernel's per-step cut-off decides the pair set, which the pair-set
// fingerprint checks against the reference.  The pair kernel rounds j's minimum-image
// difference from the centroid and the members' offsets from it to FP32; the
// composite is the pair's minimum image whenever rc + (largest member offset
// at the build) + skin < half the shortest box edge, which each build checks,
// falling back to the atom list otherwise.  Metal atoms keep atom-list rows
// (the CPIM kernels walk them); the gradients ask for every atom's row.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>

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

// Cell coordinate and, in sub, the position inside the cell on a grid of
// 2^sub_per cells per axis.
__device__ __forceinline__ int cell_coord_sub(double x, double L, double inv_len, int n, int sub_per, int &sub)
{
    const double u = (x - L * floor(x / L)) * inv_len;
    int c = (int)u;
    c = c < 0 ? 0 : (c >= n ? n - 1 : c);
    const int ns = 1 << sub_per;
    int s = (int)((u - c) * ns);
    sub = s < 0 ? 0 : (s >= ns ? ns - 1 : s);
    return c;
}

__global__ void k_cell_keys(int N, const double *__restrict__ rx, const double *__restrict__ ry,
                            const double *__restrict__ rz, Box box, Grid g, int sub_bits, int *key, int *ids)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int per = sub_bits / 3;
    int sx, sy, sz;
    const int cx = cell_coord_sub(rx[i], box.L[0], g.inv_len[0], g.n[0], per, sx);
    const int cy = cell_coord_sub(ry[i], box.L[1], g.inv_len[1], g.n[1], per, sy);
    const int cz = cell_coord_sub(rz[i], box.L[2], g.inv_len[2], g.n[2], per, sz);
    int sub = 0;
    for (int b = 0; b < per; ++b)
        sub |= (((sx >> b) & 1) << (3 * b + 2)) | (((sy >> b) & 1) << (3 * b + 1)) | (((sz >> b) & 1) << (3 * b));
    key[i] = (((cx * g.n[1] + cy) * g.n[2] + cz) << sub_bits) | sub;
    ids[i] = i;
}

// start[c] = first sorted position with key >= c, for c = 0 .. n_cells
// (empty cells included), so the atoms of cells a..b are start[a] ..
// start[b + 1] - 1.
__global__ void k_cell_starts(int N, int n_cells, int sub_bits, const int *__restrict__ key, int *start)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > N) return;
    const int prev = p > 0 ? key[p - 1] >> sub_bits : -1;
    const int cur = p < N ? key[p] >> sub_bits : n_cells;
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

// The z window c-2 .. c+2 as one or two runs of consecutive cells.
struct ZRuns {
    int a[2], b[2], n;
};
__device__ __forceinline__ ZRuns z_runs(int cz, int nz)
{
    ZRuns z;
    if (nz < 5) {
        z.a[0] = 0; z.b[0] = nz - 1; z.n = 1;
    } else {
        const int lo = cz - 2, hi = cz + 2;
        if (lo < 0) {
            z.a[0] = lo + nz; z.b[0] = nz - 1; z.a[1] = 0; z.b[1] = hi; z.n = 2;
        } else if (hi >= nz) {
            z.a[0] = lo; z.b[0] = nz - 1; z.a[1] = 0; z.b[1] = hi - nz; z.n = 2;
        } else {
            z.a[0] = lo; z.b[0] = hi; z.n = 1;
        }
    }
    return z;
}

// One warp per atom i, for the rows i0 .. i0 + rows - 1.
__global__ void __launch_bounds__(256) k_build_list(DevParams P, Grid g, int i0, int rows,
                                                    const double *__restrict__ rx,
                                                    const double *__restrict__ ry,
                                                    const double *__restrict__ rz,
                                                    const double4 *__restrict__ spos,
                                                    const int *__restrict__ cell_start, int cap,
                                                    uint32_t *__restrict__ nbr, int *__restrict__ nnb,
                                                    double *rx0, double *ry0, double *rz0, int *flags)
{
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= rows) return;
    const int i = i0 + w;
    const double xi = rx[i], yi = ry[i], zi = rz[i];
    const int c0[3] = {cell_coord(xi, P.box.L[0], g.inv_len[0], g.n[0]),
                       cell_coord(yi, P.box.L[1], g.inv_len[1], g.n[1]),
                       cell_coord(zi, P.box.L[2], g.inv_len[2], g.n[2])};
    const int nxs = axis_count(g.n[0]), nys = axis_count(g.n[1]);
    const int nz = g.n[2];
    const ZRuns zr = z_runs(c0[2], nz);
    const unsigned lt_mask = (1u << lane) - 1u;
    uint32_t *row = nbr + (size_t)i * cap;
    int count = 0;
    for (int ix = 0; ix < nxs; ++ix) {
        for (int iy = 0; iy < nys; ++iy) {
            const int col = (axis_cell(c0[0], g.n[0], ix) * g.n[1] + axis_cell(c0[1], g.n[1], iy)) * nz;
            for (int r = 0; r < zr.n; ++r) {
                const int s = cell_start[col + zr.a[r]], e = cell_start[col + zr.b[r] + 1];
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

// ------------------------------------------------------------ clusters

// Clusters per cell, ceil(atoms / 4); counts[n_cells] = 0 so that the
// exclusive scan's last element is the total.
__global__ void k_cluster_counts(int n_cells, const int *__restrict__ cell_start, int *counts)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > n_cells) return;
    counts[c] = c < n_cells ? (cell_start[c + 1] - cell_start[c] + 3) / 4 : 0;
}

struct InvBox {
    double L[3], inv[3];
};

// Member offsets from the centroid of a cluster (minimum image from the
// first member); returns the number of members.
__device__ __forceinline__ int cluster_offsets(const int m[4], const double *__restrict__ rx,
                                               const double *__restrict__ ry, const double *__restrict__ rz,
                                               const InvBox &B, double o[4][3], double c[3])
{
    const double *r[3] = {rx, ry, rz};
    int nk = 0;
    double s[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (m[k] < 0) break;
        ++nk;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            o[k][a] = min_image(r[a][m[k]] - r[a][m[0]], B.L[a], B.inv[a]);
            s[a] += o[k][a];
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double mean = s[a] / nk;
        c[a] = r[a][m[0]] + mean;
        for (int k = 0; k < nk; ++k) o[k][a] -= mean;
    }
    return nk;
}

// The clusters of one cell (a thread per cell), and in flags[5] the largest
// component of a member's offset from its cluster's centroid (float bits,
// rounded up).
// cl_of (half list, else null): the cluster of each atom.
__global__ void k_make_clusters(int n_cells, const int *__restrict__ cell_start, const int *__restrict__ cl_start,
                                const int *__restrict__ cell_atoms, const double *__restrict__ rx,
                                const double *__restrict__ ry, const double *__restrict__ rz, InvBox B,
                                int4 *cl_atoms, int *cl_of, int *flags)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells) return;
    const int s = cell_start[c], e = cell_start[c + 1];
    int cl = cl_start[c];
    double emax = 0.0;
    for (int p = s; p < e; p += 4, ++cl) {
        int m[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) m[t] = p + t < e ? cell_atoms[p + t] : -1;
        cl_atoms[cl] = make_int4(m[0], m[1], m[2], m[3]);
        if (cl_of)
            for (int t = 0; t < 4; ++t)
                if (m[t] >= 0) cl_of[m[t]] = cl;
        double o[4][3], cc[3];
        const int nk = cluster_offsets(m, rx, ry, rz, B, o, cc);
        for (int k = 0; k < nk; ++k)
            for (int a = 0; a < 3; ++a) emax = fmax(emax, fabs(o[k][a]));
    }
    if (emax > 0.0) atomicMax(&flags[5], __float_as_int(__double2float_ru(emax)));
}

// One warp per cluster: the cluster list (see the file comment).
__global__ void __launch_bounds__(256) k_build_cluster_list(DevParams P, Grid g, InvBox B,
                                                            const double *__restrict__ rx,
                                                            const double *__restrict__ ry,
                                                            const double *__restrict__ rz,
                                                            const double4 *__restrict__ spos,
                                                            const int *__restrict__ cell_start,
                                                            const int4 *__restrict__ cl_atoms,
                                                            const int *__restrict__ n_cl, int cap,
                                                            uint32_t *__restrict__ nbr, int *__restrict__ nnb,
                                                            unsigned char *__restrict__ cl_metal, double *rx0,
                                                            double *ry0, double *rz0, int *flags,
                                                            const int *__restrict__ cl_of,
                                                            const int *__restrict__ cl_cell_start)
{
    // cl_of (half list): a pair is listed once, by the lower-numbered cluster
    // of its two atoms, and inside one cluster by the earlier member; cells
    // whose clusters all precede this one are skipped
    const int cl = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (cl >= *n_cl) return;
    const int4 A = cl_atoms[cl];
    const int m[4] = {A.x, A.y, A.z, A.w};
    double o[4][3], cc[3];
    const int nk = cluster_offsets(m, rx, ry, rz, B, o, cc);
    double xm[4], ym[4], zm[4], R2 = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int a = k < nk ? m[k] : m[0];
        xm[k] = rx[a];
        ym[k] = ry[a];
        zm[k] = rz[a];
        if (k < nk) R2 = fmax(R2, o[k][0] * o[k][0] + o[k][1] * o[k][1] + o[k][2] * o[k][2]);
    }
    // prefilter radius, widened by a relative 1e-12 against rounding
    const double pre = (sqrt(P.list_r2) + sqrt(R2)) * (1.0 + 1e-12);
    const double pre2 = pre * pre;
    // FP32 member test: the list radius widened by 1e-5 relative; the
    // members' offsets from the centroid (selected by member, in registers)
    const float lr2f = (float)(P.list_r2 * (1.0 + 1e-5));
    const float ofx0 = (float)o[0][0], ofy0 = (float)o[0][1], ofz0 = (float)o[0][2];
    const float ofx1 = nk > 1 ? (float)o[1][0] : 0.f, ofy1 = nk > 1 ? (float)o[1][1] : 0.f,
                ofz1 = nk > 1 ? (float)o[1][2] : 0.f;
    const float ofx2 = nk > 2 ? (float)o[2][0] : 0.f, ofy2 = nk > 2 ? (float)o[2][1] : 0.f,
                ofz2 = nk > 2 ? (float)o[2][2] : 0.f;
    const float ofx3 = nk > 3 ? (float)o[3][0] : 0.f, ofy3 = nk > 3 ? (float)o[3][1] : 0.f,
                ofz3 = nk > 3 ? (float)o[3][2] : 0.f;
    // all members are in the cell of the first one (the cells were assigned
    // from the same positions)
    const int c0[3] = {cell_coord(xm[0], P.box.L[0], g.inv_len[0], g.n[0]),
                       cell_coord(ym[0], P.box.L[1], g.inv_len[1], g.n[1]),
                       cell_coord(zm[0], P.box.L[2], g.inv_len[2], g.n[2])};
    const int nxs = axis_count(g.n[0]), nys = axis_count(g.n[1]);
    const int nz = g.n[2];
    const ZRuns zr = z_runs(c0[2], nz);
    const unsigned lt_mask = (1u << lane) - 1u;
    uint32_t *row = nbr + (size_t)cl * cap;
    int count = 0;
    bool metal = false;
    for (int ix = 0; ix < nxs; ++ix) {
        for (int iy = 0; iy < nys; ++iy) {
            const int col = (axis_cell(c0[0], g.n[0], ix) * g.n[1] + axis_cell(c0[1], g.n[1], iy)) * nz;
            for (int r = 0; r < zr.n; ++r) {
                int za = zr.a[r];
                if (cl_of)
                    while (za <= zr.b[r] && cl_cell_start[col + za + 1] <= cl) ++za;
                const int s = cell_start[col + za], e = cell_start[col + zr.b[r] + 1];
                for (int base = s; base < e; base += 32) {
                    const int p = base + lane;
                    unsigned mask = 0;
                    int j = 0;
                    const double4 q = p < e ? spos[p] : make_double4(0.0, 0.0, 0.0, 0.0);
                    const int cj = p < e && cl_of ? cl_of[(int)q.w] : cl + 1;
                    if (p < e && cj >= cl) {
                        j = (int)q.w;
                        // on the half list, members before j's own position when j is one
                        const int jpos = cj != cl ? 4 : (j == m[0] ? 0 : j == m[1] ? 1 : j == m[2] ? 2 : 3);
                        const double ex = min_image(q.x - cc[0], B.L[0], B.inv[0]);
                        const double ey = min_image(q.y - cc[1], B.L[1], B.inv[1]);
                        const double ez = min_image(q.z - cc[2], B.L[2], B.inv[2]);
                        if (ex * ex + ey * ey + ez * ez < pre2) {
#pragma unroll
                            for (int k = 0; k < 4; ++k) {
                                if (k >= nk || j == m[k] || k >= jpos) continue;
                                const float ox = k == 0 ? ofx0 : k == 1 ? ofx1 : k == 2 ? ofx2 : ofx3;
                                const float oy = k == 0 ? ofy0 : k == 1 ? ofy1 : k == 2 ? ofy2 : ofy3;
                                const float oz = k == 0 ? ofz0 : k == 1 ? ofz1 : k == 2 ? ofz2 : ofz3;
                                const float sx = (float)ex - ox, sy = (float)ey - oy, sz = (float)ez - oz;
                                if (fmaf(sz, sz, fmaf(sy, sy, sx * sx)) < lr2f && !excluded(P, m[k], j))
                                    mask |= 1u << k;
                            }
                        }
                    }
                    const bool ok = mask != 0;
                    const unsigned ballot = __ballot_sync(0xffffffffu, ok);
                    const int pos = count + __popc(ballot & lt_mask);
                    if (ok) {
                        if (pos < cap) row[pos] = pack_cl(j, mask, P.type[j]);
                        metal |= P.is_metal[j] != 0;
                    }
                    count += __popc(ballot);
                }
            }
        }
    }
    if (cl_of)  // the half list: a metal member takes water neighbours' CPIM terms too
        for (int k = 0; k < nk; ++k) metal |= P.is_metal[m[k]] != 0;
    metal = __any_sync(0xffffffffu, metal);
    if (lane == 0) {
        nnb[cl] = count < cap ? count : cap;
        if (count > cap) atomicMax(&flags[4], count);
        cl_metal[cl] = metal ? 1 : 0;
    }
    if (lane < nk) {
        rx0[m[lane]] = lane == 0 ? xm[0] : lane == 1 ? xm[1] : lane == 2 ? xm[2] : xm[3];
        ry0[m[lane]] = lane == 0 ? ym[0] : lane == 1 ? ym[1] : lane == 2 ? ym[2] : ym[3];
        rz0[m[lane]] = lane == 0 ? zm[0] : lane == 1 ? zm[1] : lane == 2 ? zm[2] : zm[3];
    }
}

// Pair-set fingerprint over the cluster list: per member i the j < i
// entries of its mask inside the cut-off.
// On the half list each listed pair counts once, oriented as the reference
// orients it (the larger index is i, r = r_j - r_i).
__global__ void k_fingerprint_clusters(DevParams P, const double *__restrict__ rx, const double *__restrict__ ry,
                                       const double *__restrict__ rz, const int4 *__restrict__ cl_atoms,
                                       const int *__restrict__ n_cl, const uint32_t *__restrict__ nbr,
                                       const int *__restrict__ nnb, int cap, int half, unsigned long long *out)
{
    const int cl = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (cl >= *n_cl) return;
    const int4 A = cl_atoms[cl];
    const int m[4] = {A.x, A.y, A.z, A.w};
    unsigned long long cnt = 0, h = 0;
    for (int k = lane; k < nnb[cl]; k += 32) {
        const uint32_t e = nbr[(size_t)cl * cap + k];
        const int j = (int)(e & kClIdxMask);
        const unsigned mask = (e >> kClMaskShift) & 15u;
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            if (!((mask >> t) & 1u)) continue;
            int i = m[t], jj = j;
            if (half && jj > i) {
                i = j;
                jj = m[t];
            }
            if (jj >= i) continue;
            double dx = rx[jj] - rx[i], dy = ry[jj] - ry[i], dz = rz[jj] - rz[i];
            image(dx, dy, dz, P.box);
            if (norm2_exact(dx, dy, dz) < P.rc2) {
                ++cnt;
                h += mix64(((uint64_t)(uint32_t)i << 32) | (uint32_t)jj);
            }
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

// The clusters with a metal member or a metal list neighbour (cl_metal), in
// any order: the CPIM pass over the water side visits only these.
__global__ void k_select_metal_clusters(const int *__restrict__ n_cl, const unsigned char *__restrict__ cl_metal,
                                        int *__restrict__ sel, int *__restrict__ n_sel)
{
    const int ncl = *n_cl;
    for (int cl = blockIdx.x * blockDim.x + threadIdx.x; cl < ncl; cl += gridDim.x * blockDim.x)
        if (cl_metal[cl]) sel[atomicAdd(n_sel, 1)] = cl;
}

// ------------------------------------------------------------ cluster pairs
//
// pair_list 4: the clusters above, paired.  Before each pair launch
// k_cluster_frames writes every cluster's centroid (FP64: the first member
// plus the mean of the members' minimum images from it) and its members'
// offsets from the centroid (FP32) with their charges; at a build also each
// member's atom and type.  The list of cluster I holds every cluster J >= I
// of the 5 x 5 x 5 cell window with at least one member pair (a in I, b in
// J; for J = I only b after a) that is not excluded and lies within the list
// radius (widened by 1e-5 relative) in FP32, measured as the FP64 minimum
// image of the centroid difference, rounded once, plus the two offsets: a
// 16-bit mask, bit 4 k + m for member k of I with member m of J.  The pair
// kernel applies the cut-off to the masked pairs every step.  That composite
// difference is the pair's minimum image while rc + 2 (largest offset
// component) < half the shortest box edge; offsets grow by at most the skin
// between builds, so each build checks rc + skin + 2 (largest offset at the
// build + skin) < half the edge and otherwise falls back to the cluster list.

// Centroids and member offsets of every cluster; with `statics` also the
// member atoms and types and whether the cluster has a metal member.
__global__ void k_cluster_frames(int ncl, const int4 *__restrict__ cl_atoms, const double *__restrict__ rx,
                                 const double *__restrict__ ry, const double *__restrict__ rz,
                                 const double *__restrict__ charge, InvBox B, double4 *__restrict__ cent,
                                 float4 *__restrict__ off, int statics, const int *__restrict__ type,
                                 const unsigned char *__restrict__ is_metal, int *__restrict__ ti,
                                 unsigned char *__restrict__ cl_metal)
{
    const int cl = blockIdx.x * blockDim.x + threadIdx.x;
    if (cl >= ncl) return;
    const int4 A = cl_atoms[cl];
    const int m[4] = {A.x, A.y, A.z, A.w};
    double o[4][3], cc[3];
    const int nk = cluster_offsets(m, rx, ry, rz, B, o, cc);
    cent[cl] = make_double4(cc[0], cc[1], cc[2], 0.0);
    bool metal = false;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const bool in = k < nk;
        off[4 * cl + k] = in ? make_float4((float)o[k][0], (float)o[k][1], (float)o[k][2], (float)charge[m[k]])
                             : make_float4(0.f, 0.f, 0.f, 0.f);
        if (statics) {
            ti[4 * cl + k] = in ? (m[k] | (type[m[k]] << kCpTypeShift)) : -1;
            metal |= in && is_metal[m[k]] != 0;
        }
    }
    if (statics) cl_metal[cl] = metal ? 1 : 0;
}

// One warp per cluster I: its cluster-pair list (see above).  Lanes take the
// window's clusters J >= I in turn; each computes the 16 member distances.
__global__ void __launch_bounds__(256) k_build_cpair_list(DevParams P, Grid g, InvBox B, int ncl,
                                                          const double4 *__restrict__ cent,
                                                          const float4 *__restrict__ off,
                                                          const int *__restrict__ ti,
                                                          const unsigned char *__restrict__ cl_metal,
                                                          const int *__restrict__ cl_cell_start, int cap,
                                                          uint2 *__restrict__ list, int *__restrict__ cnt,
                                                          int *flags, const double *__restrict__ rx,
                                                          const double *__restrict__ ry,
                                                          const double *__restrict__ rz, double *rx0, double *ry0,
                                                          double *rz0)
{
    const int ic = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (ic >= ncl) return;
    const double4 ci = cent[ic];
    float oix[4], oiy[4], oiz[4];
    int ai[4];
    float Ri = 0.f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float4 o = off[4 * ic + k];
        const int t = ti[4 * ic + k];
        ai[k] = t < 0 ? -1 : (t & kCpIdxMask);
        oix[k] = o.x;
        oiy[k] = o.y;
        oiz[k] = o.z;
        if (t >= 0) Ri = fmaxf(Ri, sqrtf(o.x * o.x + o.y * o.y + o.z * o.z));
    }
    const bool metal_i = cl_metal[ic] != 0;
    const double rl = sqrt(P.list_r2);
    const float lr2f = (float)(P.list_r2 * (1.0 + 1e-5));
    const int a0 = ai[0];
    const int c0[3] = {cell_coord(rx[a0], P.box.L[0], g.inv_len[0], g.n[0]),
                       cell_coord(ry[a0], P.box.L[1], g.inv_len[1], g.n[1]),
                       cell_coord(rz[a0], P.box.L[2], g.inv_len[2], g.n[2])};
    const int nxs = axis_count(g.n[0]), nys = axis_count(g.n[1]);
    const int nz = g.n[2];
    const ZRuns zr = z_runs(c0[2], nz);
    const unsigned lt_mask = (1u << lane) - 1u;
    uint2 *row = list + (size_t)ic * cap;
    int count = 0;
    for (int ix = 0; ix < nxs; ++ix) {
        for (int iy = 0; iy < nys; ++iy) {
            const int col = (axis_cell(c0[0], g.n[0], ix) * g.n[1] + axis_cell(c0[1], g.n[1], iy)) * nz;
            for (int r = 0; r < zr.n; ++r) {
                const int s = max(cl_cell_start[col + zr.a[r]], ic), e = cl_cell_start[col + zr.b[r] + 1];
                for (int base = s; base < e; base += 32) {
                    const int jc = base + lane;
                    unsigned mask = 0;
                    if (jc < e) {
                        const double4 cj = cent[jc];
                        const double dx = min_image(cj.x - ci.x, B.L[0], B.inv[0]);
                        const double dy = min_image(cj.y - ci.y, B.L[1], B.inv[1]);
                        const double dz = min_image(cj.z - ci.z, B.L[2], B.inv[2]);
                        float ojx[4], ojy[4], ojz[4];
                        int aj[4];
                        float Rj = 0.f;
#pragma unroll
                        for (int m = 0; m < 4; ++m) {
                            const float4 o = off[4 * jc + m];
                            const int t = ti[4 * jc + m];
                            aj[m] = t < 0 ? -1 : (t & kCpIdxMask);
                            ojx[m] = o.x;
                            ojy[m] = o.y;
                            ojz[m] = o.z;
                            if (t >= 0) Rj = fmaxf(Rj, sqrtf(o.x * o.x + o.y * o.y + o.z * o.z));
                        }
                        // centroid prefilter, widened against rounding
                        const double pre = (rl + (double)Ri + (double)Rj) * (1.0 + 1e-6);
                        if (dx * dx + dy * dy + dz * dz < pre * pre) {
                            const float fx = (float)dx, fy = (float)dy, fz = (float)dz;
#pragma unroll
                            for (int k = 0; k < 4; ++k) {
#pragma unroll
                                for (int m = 0; m < 4; ++m) {
                                    if (ai[k] < 0 || aj[m] < 0 || (jc == ic && m <= k)) continue;
                                    const float sx = fx + (ojx[m] - oix[k]), sy = fy + (ojy[m] - oiy[k]),
                                                sz = fz + (ojz[m] - oiz[k]);
                                    if (fmaf(sz, sz, fmaf(sy, sy, sx * sx)) < lr2f && !excluded(P, ai[k], aj[m]))
                                        mask |= 1u << (4 * k + m);
                                }
                            }
                        }
                    }
                    const bool ok = mask != 0;
                    const unsigned ballot = __ballot_sync(0xffffffffu, ok);
                    const int pos = count + __popc(ballot & lt_mask);
                    if (ok && pos < cap)
                        row[pos] = make_uint2((uint32_t)jc, mask | ((metal_i || cl_metal[jc] != 0) ? kCpMetalBit : 0u));
                    count += __popc(ballot);
                }
            }
        }
    }
    if (lane == 0) {
        cnt[ic] = count < cap ? count : cap;
        if (count > cap) atomicMax(&flags[7], count);
    }
    if (lane < 4 && ai[lane] >= 0) {  // displacement reference of the members
        const int a = ai[lane];
        rx0[a] = rx[a];
        ry0[a] = ry[a];
        rz0[a] = rz[a];
    }
}

// Pair-set fingerprint over the cluster-pair list: every masked member pair
// inside the cut-off, oriented as the reference orients it.
__global__ void k_fingerprint_cpairs(DevParams P, const double *__restrict__ rx, const double *__restrict__ ry,
                                     const double *__restrict__ rz, int ncl, const int *__restrict__ ti,
                                     const uint2 *__restrict__ list, const int *__restrict__ cnt, int cap,
                                     unsigned long long *out)
{
    const int ic = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (ic >= ncl) return;
    unsigned long long n = 0, h = 0;
    for (int q = lane; q < cnt[ic]; q += 32) {
        const uint2 e = list[(size_t)ic * cap + q];
        const int jc = (int)e.x;
        for (int b = 0; b < 16; ++b) {
            if (!((e.y >> b) & 1u)) continue;
            const int a = ti[4 * ic + (b >> 2)] & kCpIdxMask, c = ti[4 * jc + (b & 3)] & kCpIdxMask;
            const int i = max(a, c), j = min(a, c);
            double dx = rx[j] - rx[i], dy = ry[j] - ry[i], dz = rz[j] - rz[i];
            image(dx, dy, dz, P.box);
            if (norm2_exact(dx, dy, dz) < P.rc2) {
                ++n;
                h += mix64(((uint64_t)(uint32_t)i << 32) | (uint32_t)j);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n += __shfl_xor_sync(0xffffffffu, n, o);
        h += __shfl_xor_sync(0xffffffffu, h, o);
    }
    if (lane == 0 && n) {
        atomicAdd(&out[0], n);
        atomicAdd(&out[1], h);
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

// Sub-cell Morton bits below the cell index: three per axis, as many as fit
// a non-negative int key (at most 9).
int sub_cell_bits(int n_cells)
{
    int b = 1;
    while ((1L << b) < n_cells) ++b;
    return std::max(0, std::min(9, (31 - b) / 3 * 3));
}

InvBox inv_box(const capac_ctx *c)
{
    InvBox B;
    for (int a = 0; a < 3; ++a) {
        B.L[a] = c->P.box.L[a];
        B.inv[a] = 1.0 / c->P.box.L[a];
    }
    return B;
}

bool cluster_list_allowed(const capac_ctx *c)
{
    return c->opt.precision == CAPAC_PREC_MIXED && c->opt.pair_list != 1 &&
           c->N < (1 << kClIdxBits) &&
           c->P.n_types <= kClMaxTypes;
}

// Cluster slots and the first per-cluster capacity, from the densest
// plausible environment of a cluster (radius rc + skin + 0.5 nm).
void ensure_cluster_buffers(capac_ctx *c, int n_cells)
{
    const int N = c->N;
    if (n_cells != c->cl_cells) {
        cudaFree(c->cl_cell_start);
        cudaFree(c->cl_counts);
        c->cl_cell_start = c->cl_counts = nullptr;
        CAPAC_CUDA(cudaMalloc(&c->cl_cell_start, sizeof(int) * (n_cells + 1)));
        CAPAC_CUDA(cudaMalloc(&c->cl_counts, sizeof(int) * (n_cells + 1)));
        c->cl_cells = n_cells;
    }
    const int need = N / 4 + n_cells + 1;
    if (need > c->cl_max || !c->cl_nbr) {
        if (c->cl_cap == 0) {
            const double V = c->P.box.L[0] * c->P.box.L[1] * c->P.box.L[2];
            const double rl = c->P.rc + c->opt.skin + 0.5;
            const double dens = std::max((double)N / V, 60.0);
            long est = (long)(1.25 * dens * 4.0 / 3.0 * M_PI * rl * rl * rl) + 64;
            est = std::min<long>(est, (long)N);
            c->cl_cap = (int)((est + 31) & ~31L);
        }
        cudaFree(c->cl_atoms);
        cudaFree(c->cl_nbr);
        cudaFree(c->cl_nnb);
        cudaFree(c->cl_metal);
        cudaFree(c->cl_sel);
        c->cl_atoms = nullptr;
        c->cl_nbr = nullptr;
        c->cl_nnb = nullptr;
        c->cl_metal = nullptr;
        c->cl_sel = nullptr;
        CAPAC_CUDA(cudaMalloc(&c->cl_atoms, sizeof(int4) * need));
        CAPAC_CUDA(cudaMalloc(&c->cl_nbr, sizeof(uint32_t) * (size_t)need * c->cl_cap));
        CAPAC_CUDA(cudaMalloc(&c->cl_nnb, sizeof(int) * need));
        CAPAC_CUDA(cudaMalloc(&c->cl_metal, need));
        CAPAC_CUDA(cudaMalloc(&c->cl_sel, sizeof(int) * need));
        c->cl_max = need;
    }
    c->cl_half = c->opt.pair_list != 3;  // 0 (default) and 2: every pair once; 3: the full cluster list
    if (c->cl_half && !c->cl_of) CAPAC_CUDA(cudaMalloc(&c->cl_of, sizeof(int) * N));
    if (!c->cl_next) CAPAC_CUDA(cudaMalloc(&c->cl_next, sizeof(int)));
    if (!c->n_cl_sel) CAPAC_CUDA(cudaMalloc(&c->n_cl_sel, sizeof(int)));
}

// Clusters of the sorted cells; returns false when the largest member offset
// breaks the minimum-image condition (see the file comment).
bool make_clusters(capac_ctx *c, int n_cells)
{
    cudaStream_t s = c->stream;
    ensure_cluster_buffers(c, n_cells);
    k_cluster_counts<<<grid_for(n_cells + 1, 256), 256, 0, s>>>(n_cells, c->cell_start, c->cl_counts);
    size_t need = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, need, c->cl_counts, c->cl_cell_start, n_cells + 1, s);
    if (need > c->scan_tmp_bytes) {
        cudaFree(c->scan_tmp);
        c->scan_tmp = nullptr;
        CAPAC_CUDA(cudaMalloc(&c->scan_tmp, need));
        c->scan_tmp_bytes = need;
    }
    CAPAC_CUDA(cub::DeviceScan::ExclusiveSum(c->scan_tmp, need, c->cl_counts, c->cl_cell_start, n_cells + 1, s));
    CAPAC_CUDA(cudaMemsetAsync(c->flags + 5, 0, sizeof(int), s));
    k_make_clusters<<<grid_for(n_cells, 128), 128, 0, s>>>(n_cells, c->cell_start, c->cl_cell_start, c->cell_atoms,
                                                           c->rx, c->ry, c->rz, inv_box(c), c->cl_atoms,
                                                           c->cl_half ? c->cl_of : nullptr, c->flags);
    c->launches += 3;
    CAPAC_CUDA(cudaMemcpyAsync(c->h_flags + 6, c->cl_cell_start + n_cells, sizeof(int), cudaMemcpyDeviceToHost, s));
    CAPAC_CUDA(cudaMemcpyAsync(c->h_flags + 5, c->flags + 5, sizeof(int), cudaMemcpyDeviceToHost, s));
    CAPAC_CUDA(cudaStreamSynchronize(s));
    c->n_clusters = c->h_flags[6];
    float ext;
    memcpy(&ext, &c->h_flags[5], sizeof ext);
    const double half = 0.5 * std::min(c->P.box.L[0], std::min(c->P.box.L[1], c->P.box.L[2]));
    return c->P.rc + (double)ext + c->opt.skin < half;
}

void build_cluster_list(capac_ctx *c, const Grid &g, int n_cells)
{
    cudaStream_t s = c->stream;
    const int *n_cl = c->cl_cell_start + n_cells;
    for (int attempt = 0; attempt < 4; ++attempt) {
        CAPAC_CUDA(cudaMemsetAsync(c->flags + 4, 0, sizeof(int), s));
        {
            ProfScope ps(c, K_LIST);
            k_build_cluster_list<<<grid_for((long)c->n_clusters * 32, 256), 256, 0, s>>>(
                c->P, g, inv_box(c), c->rx, c->ry, c->rz, c->spos, c->cell_start, c->cl_atoms, n_cl, c->cl_cap,
                c->cl_nbr, c->cl_nnb, c->cl_metal, c->rx0, c->ry0, c->rz0, c->flags,
                c->cl_half ? c->cl_of : nullptr, c->cl_cell_start);
        }
        ++c->launches;
        CAPAC_CUDA(cudaMemcpyAsync(c->h_flags + 4, c->flags + 4, sizeof(int), cudaMemcpyDeviceToHost, s));
        CAPAC_CUDA(cudaStreamSynchronize(s));
        const int need_cap = c->h_flags[4];
        if (need_cap <= c->cl_cap) {
            CAPAC_CUDA(cudaMemsetAsync(c->n_cl_sel, 0, sizeof(int), s));
            k_select_metal_clusters<<<grid_for(c->n_clusters, 256), 256, 0, s>>>(n_cl, c->cl_metal, c->cl_sel,
                                                                                  c->n_cl_sel);
            ++c->launches;
            // the pair launch is split when few clusters are next to metal:
            // the second launch costs about as much per cluster it visits
            // as the CPIM branches save per cluster of the first (measured:
            // faster with 5% of the clusters next to metal, slower with 20%)
            CAPAC_CUDA(cudaMemcpyAsync(c->h_flags + 7, c->n_cl_sel, sizeof(int), cudaMemcpyDeviceToHost, s));
            CAPAC_CUDA(cudaStreamSynchronize(s));
            c->n_sel_host = c->h_flags[7];
            c->pair_split = c->pair_split_force >= 0 ? c->pair_split_force == 1
                                                     : c->n_sel_host < kPairSplitShare * c->n_clusters;
            return;
        }
        if (attempt == 3) throw Error(CAPAC_ERR_CAPACITY, "cluster list capacity could not be met");
        int new_cap = (int)std::min<long>((long)(need_cap * 1.25) + 32, 1L << 20);
        new_cap = (new_cap + 31) & ~31;
        cudaFree(c->cl_nbr);
        c->cl_nbr = nullptr;
        CAPAC_CUDA(cudaMalloc(&c->cl_nbr, sizeof(uint32_t) * (size_t)c->cl_max * new_cap));
        c->cl_cap = new_cap;
    }
}

// Cluster-pair arrays for the current cluster slots; the first per-cluster
// capacity from the densest plausible environment (radius rc + skin + 0.6 nm,
// clusters of four, each pair once).
void ensure_cpair_buffers(capac_ctx *c)
{
    if (c->cp_max != c->cl_max || !c->cp_cent) {
        cudaFree(c->cp_cent);
        cudaFree(c->cp_off);
        cudaFree(c->cp_ti);
        cudaFree(c->cp_n);
        cudaFree(c->cp_list);
        c->cp_cent = nullptr;
        c->cp_off = nullptr;
        c->cp_ti = nullptr;
        c->cp_n = nullptr;
        c->cp_list = nullptr;
        if (c->cp_cap == 0) {
            const double V = c->P.box.L[0] * c->P.box.L[1] * c->P.box.L[2];
            const double rl = c->P.rc + c->opt.skin + 0.6;
            const double dens = std::max((double)c->N / V, 60.0);
            long est = (long)(1.3 * dens * 4.0 / 3.0 * M_PI * rl * rl * rl / 8.0) + 64;
            est = std::min<long>(est, (long)c->cl_max);
            c->cp_cap = (int)((est + 31) & ~31L);
        }
        CAPAC_CUDA(cudaMalloc(&c->cp_cent, sizeof(double4) * c->cl_max));
        CAPAC_CUDA(cudaMalloc(&c->cp_off, sizeof(float4) * 4 * (size_t)c->cl_max));
        CAPAC_CUDA(cudaMalloc(&c->cp_ti, sizeof(int) * 4 * (size_t)c->cl_max));
        CAPAC_CUDA(cudaMalloc(&c->cp_n, sizeof(int) * c->cl_max));
        CAPAC_CUDA(cudaMalloc(&c->cp_list, sizeof(uint2) * (size_t)c->cl_max * c->cp_cap));
        c->cp_max = c->cl_max;
    }
}

// The cluster-pair list is usable while the composite minimum image holds
// (see the comment above k_cluster_frames); ext is the largest member offset
// component of the clusters just made.
bool cpair_list_allowed(const capac_ctx *c, double ext)
{
    const double half = 0.5 * std::min(c->P.box.L[0], std::min(c->P.box.L[1], c->P.box.L[2]));
    return c->opt.pair_list == 4 && c->P.rc + c->opt.skin + 2.0 * (ext + c->opt.skin) < half;
}

void build_cpair_list(capac_ctx *c, const Grid &g)
{
    cudaStream_t s = c->stream;
    ensure_cpair_buffers(c);
    launch_cluster_frames(c, true);
    const int *cs = c->cl_cell_start;
    for (int attempt = 0; attempt < 4; ++attempt) {
        CAPAC_CUDA(cudaMemsetAsync(c->flags + 7, 0, sizeof(int), s));
        {
            ProfScope ps(c, K_LIST);
            k_build_cpair_list<<<grid_for((long)c->n_clusters * 32, 256), 256, 0, s>>>(
                c->P, g, inv_box(c), c->n_clusters, c->cp_cent, c->cp_off, c->cp_ti, c->cl_metal, cs, c->cp_cap,
                c->cp_list, c->cp_n, c->flags, c->rx, c->ry, c->rz, c->rx0, c->ry0, c->rz0);
        }
        ++c->launches;
        CAPAC_CUDA(cudaMemcpyAsync(c->h_flags + 7, c->flags + 7, sizeof(int), cudaMemcpyDeviceToHost, s));
        CAPAC_CUDA(cudaStreamSynchronize(s));
        const int need_cap = c->h_flags[7];
        if (need_cap <= c->cp_cap) return;
        if (attempt == 3) throw Error(CAPAC_ERR_CAPACITY, "cluster-pair list capacity could not be met");
        int new_cap = (int)std::min<long>((long)(need_cap * 1.25) + 32, 1L << 20);
        new_cap = (new_cap + 31) & ~31;
        cudaFree(c->cp_list);
        c->cp_list = nullptr;
        CAPAC_CUDA(cudaMalloc(&c->cp_list, sizeof(uint2) * (size_t)c->cl_max * new_cap));
        c->cp_cap = new_cap;
    }
}

// Atom-list rows i0 .. i0 + rows - 1, growing the per-atom capacity as needed.
void build_atom_rows(capac_ctx *c, const Grid &g, int i0, int rows)
{
    const int N = c->N;
    cudaStream_t s = c->stream;
    for (int attempt = 0; attempt < 4; ++attempt) {
        CAPAC_CUDA(cudaMemsetAsync(c->flags + 1, 0, sizeof(int), s));
        {
            ProfScope ps(c, K_LIST);
            k_build_list<<<grid_for((long)rows * 32, 256), 256, 0, s>>>(
                c->P, g, i0, rows, c->rx, c->ry, c->rz, c->spos, c->cell_start, c->cap, c->nbr, c->nnb, c->rx0,
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
    const int sub_bits = sub_cell_bits(n_cells);
    c->cell_sub_bits = sub_bits;
    cudaStream_t s = c->stream;
    k_cell_keys<<<grid_for(N, 256), 256, 0, s>>>(N, c->rx, c->ry, c->rz, c->P.box, g, sub_bits, c->cell_key,
                                                 c->atom_ids);
    ++c->launches;
    int end_bit = 1;
    while ((1 << end_bit) < n_cells) ++end_bit;
    end_bit += sub_bits;
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
    k_cell_starts<<<grid_for(N + 1, 256), 256, 0, s>>>(N, n_cells, sub_bits, c->cell_key_sorted, c->cell_start);
    k_sorted_positions<<<grid_for(N, 256), 256, 0, s>>>(N, c->cell_atoms, c->rx, c->ry, c->rz, c->spos);
    c->launches += 2;

    bool use_cl = cluster_list_allowed(c) && make_clusters(c, n_cells);
    float ext = 0.f;
    memcpy(&ext, &c->h_flags[5], sizeof ext);  // written by make_clusters
    const bool use_cp = use_cl && cpair_list_allowed(c, (double)ext);
    if (use_cp)
        build_cpair_list(c, g);
    else if (use_cl)
        build_cluster_list(c, g, n_cells);
    // atom-list rows: every atom on the atom path or when asked for, else
    // the metal atoms (the CPIM kernels walk their rows)
    if (!use_cl || c->need_full_list)
        build_atom_rows(c, g, 0, N);
    else if (c->M > 0)
        build_atom_rows(c, g, c->metal_min, c->M);
    c->clusters = use_cl && !use_cp;
    c->cpairs = use_cp;
    c->atom_list_full = !use_cl || c->need_full_list;
    c->list_valid = true;
    ++c->list_builds;
}

}  // namespace

void launch_cluster_frames(capac_ctx *c, bool statics)
{
    k_cluster_frames<<<grid_for(c->n_clusters, 128), 128, 0, c->stream>>>(
        c->n_clusters, c->cl_atoms, c->rx, c->ry, c->rz, c->charge, inv_box(c), c->cp_cent, c->cp_off,
        statics ? 1 : 0, c->type, c->is_metal, c->cp_ti, c->cl_metal);
    ++c->launches;
}

void launch_pack_positions(capac_ctx *c)
{
    k_pack<<<grid_for(c->N, 256), 256, 0, c->stream>>>(c->N, c->rx, c->ry, c->rz, c->charge, c->pos4,
                                                       c->pos4f);
    ++c->launches;
}

void ensure_full_atom_list(capac_ctx *c)
{
    c->need_full_list = true;
    if (!c->list_valid || !c->atom_list_full) build_list(c);
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
        if (c->cpairs)
            k_fingerprint_cpairs<<<grid_for((long)c->n_clusters * 32, 256), 256, 0, c->stream>>>(
                c->P, c->rx, c->ry, c->rz, c->n_clusters, c->cp_ti, c->cp_list, c->cp_n, c->cp_cap, d);
        else if (c->clusters)
            k_fingerprint_clusters<<<grid_for((long)c->n_clusters * 32, 256), 256, 0, c->stream>>>(
                c->P, c->rx, c->ry, c->rz, c->cl_atoms, c->cl_cell_start + c->n_cells, c->cl_nbr, c->cl_nnb,
                c->cl_cap, c->cl_half ? 1 : 0, d);
        else
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
