// Root cube and octant keys.
//
// Root cube: bounding box of the bodies, centre = box middle, half-width =
// half the largest extent (1 if that is <= 0) -- src/gravity/step.h:69-100.
// Octant key: the path the reference's insertion takes for a body, i.e. at
// every level the octant (x>cx) + 2(y>cy) + 4(z>cz) against the cell centre,
// then the child centre = centre +/- half of the half-width
// (src/gravity/octree.h:49-64).  Computing the descent with the same FP64
// operations makes the key's leading digits equal the reference tree path
// bit for bit, so a tree built from sorted keys has the reference topology.
//
// Memory bound: 24 B of positions read + 12 B of key/index written per body.
#include "box.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace nb {

namespace {

// One system: grid-wide reduction; the last block to finish folds the block
// partials and writes the cube, then re-arms the ticket for the next launch.
__global__ void __launch_bounds__(kBoxThreads)
root_cube_kernel(const double* __restrict__ x, const double* __restrict__ y,
                 const double* __restrict__ z, int64_t n, double* __restrict__ partial,
                 unsigned int* ticket, double4* cube) {
    double lo[3] = {1e30, 1e30, 1e30}, hi[3] = {-1e30, -1e30, -1e30};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double px = x[i], py = y[i], pz = z[i];
        lo[0] = fmin(lo[0], px); hi[0] = fmax(hi[0], px);
        lo[1] = fmin(lo[1], py); hi[1] = fmax(hi[1], py);
        lo[2] = fmin(lo[2], pz); hi[2] = fmax(hi[2], pz);
    }
    block_minmax3(lo, hi);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        for (int a = 0; a < 3; ++a) { partial[6 * blockIdx.x + a] = lo[a]; partial[6 * blockIdx.x + 3 + a] = hi[a]; }
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double l2[3] = {1e30, 1e30, 1e30}, h2[3] = {-1e30, -1e30, -1e30};
    for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x)
        for (int a = 0; a < 3; ++a) {
            l2[a] = fmin(l2[a], __ldcg(partial + 6 * b + a));
            h2[a] = fmax(h2[a], __ldcg(partial + 6 * b + 3 + a));
        }
    block_minmax3(l2, h2);
    if (threadIdx.x == 0) {
        *cube = cube_from_box(l2, h2);
        *ticket = 0u;
    }
}

// Many systems: one block per system.
__global__ void __launch_bounds__(kBoxThreads)
system_cubes_kernel(const double* __restrict__ x, const double* __restrict__ y,
                    const double* __restrict__ z, const int64_t* __restrict__ offsets,
                    int nsys, double4* cube) {
    for (int s = blockIdx.x; s < nsys; s += gridDim.x) {
        double lo[3] = {1e30, 1e30, 1e30}, hi[3] = {-1e30, -1e30, -1e30};
        for (int64_t i = offsets[s] + threadIdx.x; i < offsets[s + 1]; i += blockDim.x) {
            const double px = x[i], py = y[i], pz = z[i];
            lo[0] = fmin(lo[0], px); hi[0] = fmax(hi[0], px);
            lo[1] = fmin(lo[1], py); hi[1] = fmax(hi[1], py);
            lo[2] = fmin(lo[2], pz); hi[2] = fmax(hi[2], pz);
        }
        block_minmax3(lo, hi);
        if (threadIdx.x == 0) cube[s] = cube_from_box(lo, hi);
        __syncthreads();
    }
}

// Bodies per thread (two: more independent descents in flight per thread;
// 16.7 M-body halo 2.00 -> 1.96 ms build less sort).
#ifndef NB_KEYS_PER_THREAD
#define NB_KEYS_PER_THREAD 2
#endif
__global__ void __launch_bounds__(256)
keys_kernel(const double* __restrict__ x, const double* __restrict__ y,
            const double* __restrict__ z, const int32_t* __restrict__ sysid, int64_t n,
            const double4* __restrict__ cubes, int base, int levels,
            uint64_t* __restrict__ keys, uint32_t* __restrict__ idx) {
    const int64_t i0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) * NB_KEYS_PER_THREAD;
#pragma unroll
    for (int u = 0; u < NB_KEYS_PER_THREAD; ++u) {
        const int64_t i = i0 + u;
        if (i >= n) return;
        const int s = sysid ? sysid[i] : 0;
        const double4 c = cubes[s];
        const double px = x[i], py = y[i], pz = z[i];
        double cx = c.x, cy = c.y, cz = c.z, h = c.w;
        uint64_t key = base < 64 ? (static_cast<uint64_t>(s) << base) : 0ull;
        for (int l = 1; l <= levels; ++l) {
            const bool bx = px > cx, by = py > cy, bz = pz > cz;
            const uint64_t oct = static_cast<uint64_t>(bx) | (static_cast<uint64_t>(by) << 1) |
                                 (static_cast<uint64_t>(bz) << 2);
            key |= oct << (base - 3 * l);
            const double hs = h * 0.5;
            cx = cx + (bx ? hs : -hs);
            cy = cy + (by ? hs : -hs);
            cz = cz + (bz ? hs : -hs);
            h = hs;
        }
        keys[i] = key;
        idx[i] = static_cast<uint32_t>(i);
    }
}

}  // namespace

cudaError_t launch_root_cubes(const Bodies& b, int64_t n, const Systems& sys, const int64_t* d_offsets,
                              double* partial, int partial_blocks, unsigned int* ticket,
                              cudaStream_t st) {
    if (sys.n == 1) {
        int blocks = static_cast<int>((n + kBoxThreads - 1) / kBoxThreads);
        if (blocks > partial_blocks) blocks = partial_blocks;
        if (blocks < 1) blocks = 1;
        root_cube_kernel<<<blocks, kBoxThreads, 0, st>>>(b.x, b.y, b.z, n, partial, ticket, sys.cube);
        count_launches(1);
    } else {
        int blocks = sys.n < 4096 ? sys.n : 4096;
        system_cubes_kernel<<<blocks, kBoxThreads, 0, st>>>(b.x, b.y, b.z, d_offsets, sys.n, sys.cube);
        count_launches(1);
    }
    return cudaGetLastError();
}

cudaError_t launch_keys(const Bodies& b, const int32_t* sysid, int64_t n, const Systems& sys,
                        uint64_t* keys, uint32_t* idx, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int blocks = static_cast<int>((n + 256 * NB_KEYS_PER_THREAD - 1) / (256 * NB_KEYS_PER_THREAD));
    keys_kernel<<<blocks, 256, 0, st>>>(b.x, b.y, b.z, sys.n > 1 ? sysid : nullptr, n, sys.cube,
                                        sys.base, sys.levels, keys, idx);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace nb
