// Device-side helpers shared by the kernels of the force-and-solve path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace capac {

// Physical constants of the reference (typedef.h:44-93, cpff.c:72-75, 758-759).
constexpr double kFQQ = 138.935457696552;
constexpr double kNm2Bohr = 18.8972612456506;
constexpr double kBoltz = 0.00831446214546895;
constexpr double kInvSqrtPi = 0.564189583547756;
constexpr double kThreshold = 1.0e-15;
constexpr double kConvE = 2.01552955019358e-05;
constexpr double kConvV = 3.80879884583368e-04;
constexpr double kFqqAu2 = 49614.7526045429;
constexpr double kFqqAu1 = 2625.49964037578;
constexpr int kMaxIter = 1000;
constexpr int kNhc = 10;

// Rectangular box: edge lengths and half lengths (System.box[6], mpi-main.c:536-538).
struct Box {
    double L[3];
    double H[3];
};

// pbc_12 (force.c:111-121): a single conditional shift per axis.
__device__ __forceinline__ void image(double &x, double &y, double &z, const Box &b)
{
    if (x < -b.H[0]) x += b.L[0]; else if (x > b.H[0]) x -= b.L[0];
    if (y < -b.H[1]) y += b.L[1]; else if (y > b.H[1]) y -= b.L[1];
    if (z < -b.H[2]) z += b.L[2]; else if (z > b.H[2]) z -= b.L[2];
}

// dist_2 (force.c:41-44) with the reference's rounding: (x*x + y*y) + z*z,
// no fused multiply-add, so cut-off decisions match the CPU bit for bit.
__device__ __forceinline__ double norm2_exact(double x, double y, double z)
{
    return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

// pbc (force.c:104-109): one conditional shift by the full box length.
__device__ __forceinline__ double wrap1(double dx, double L)
{
    if (dx < -0.5 * L) dx += L; else if (dx > 0.5 * L) dx -= L;
    return dx;
}

__device__ __forceinline__ double keep_entry(double e) { return fabs(e) > kThreshold ? e : 0.0; }

// Deterministic warp sum (fixed butterfly order).
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sumf(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum K values over the block (blockDim.x a multiple of 32, at most 1024) in
// a fixed order; thread 0 receives the totals in v[].  `sh` needs 32*K doubles.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double *sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) sh[wid * K + k] = v[k];
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = lane < nw ? sh[lane * K + k] : 0.0;
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
    }
    __syncthreads();
}

// Write a block's K partial sums to partials[blockIdx.x*K + k].
template <int K>
__device__ __forceinline__ void block_partials(double (&v)[K], double *sh, double *partials)
{
    block_sum<K>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) partials[(size_t)blockIdx.x * K + k] = v[k];
    }
}

// splitmix64 finaliser, used for order-independent pair-set hashes.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x)
{
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

// Neighbour-list entries carry the atom index in the low 24 bits and the
// atom type in the high 8 bits, so the pair kernel needs no type gather.
constexpr int kIdxBits = 24;
constexpr uint32_t kIdxMask = (1u << kIdxBits) - 1u;
__host__ __device__ __forceinline__ uint32_t pack_nb(int j, int t) { return (uint32_t)j | ((uint32_t)t << kIdxBits); }
__host__ __device__ __forceinline__ int nb_index(uint32_t e) { return (int)(e & kIdxMask); }
__host__ __device__ __forceinline__ int nb_type(uint32_t e) { return (int)(e >> kIdxBits); }

// Cluster-list entries: the j atom in the low 22 bits, in bits 22-25 the mask
// of the cluster members j is a list neighbour of, the j type in bits 26-31.
// In the pair kernel's queue bits 22-23 carry the member instead of the mask.
constexpr int kClIdxBits = 22, kClMaskShift = 22, kClTypeShift = 26;
constexpr uint32_t kClIdxMask = (1u << kClIdxBits) - 1u;
constexpr int kClMaxTypes = 64;
// cluster-pair list: a member slot holds atom | type << kCpTypeShift; an
// entry's second word the 16-bit member-pair mask and kCpMetalBit
constexpr int kCpTypeShift = 24;
constexpr int kCpIdxMask = (1 << kCpTypeShift) - 1;
constexpr uint32_t kCpMetalBit = 1u << 16;
__host__ __device__ __forceinline__ uint32_t pack_cl(int j, unsigned mask, int t)
{
    return (uint32_t)j | (mask << kClMaskShift) | ((uint32_t)t << kClTypeShift);
}

// Minimum image by rounding (any number of box lengths apart).
__device__ __forceinline__ double min_image(double d, double L, double inv_L) { return d - L * rint(d * inv_L); }

}  // namespace capac
