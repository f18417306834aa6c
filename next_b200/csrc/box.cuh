// Block-wide bounding boxes of bodies and the root cube built from one
// (shared by the root-cube kernel and the fused kick-drift that also boxes
// the drifted positions).  Root cube: centre = box middle, half-width = half
// the largest extent (1 if that is <= 0) -- src/gravity/step.h:69-100.
#pragma once

namespace nb {

constexpr int kBoxThreads = 256;

__device__ __forceinline__ void warp_minmax(double& lo, double& hi) {
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
}

// Block-wide min/max of 3 axes; result valid in thread 0.
__device__ __forceinline__ void block_minmax3(double lo[3], double hi[3]) {
    __shared__ double s_lo[3][kBoxThreads / 32], s_hi[3][kBoxThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int a = 0; a < 3; ++a) {
        warp_minmax(lo[a], hi[a]);
        if (lane == 0) { s_lo[a][w] = lo[a]; s_hi[a][w] = hi[a]; }
    }
    __syncthreads();
    if (w == 0) {
        for (int a = 0; a < 3; ++a) {
            double l = lane < kBoxThreads / 32 ? s_lo[a][lane] : 1e30;
            double h = lane < kBoxThreads / 32 ? s_hi[a][lane] : -1e30;
            warp_minmax(l, h);
            lo[a] = l; hi[a] = h;
        }
    }
}

__device__ __forceinline__ double4 cube_from_box(const double lo[3], const double hi[3]) {
    double4 c;
    c.x = (lo[0] + hi[0]) * 0.5;
    c.y = (lo[1] + hi[1]) * 0.5;
    c.z = (lo[2] + hi[2]) * 0.5;
    double half = fmax(fmax(hi[0] - lo[0], hi[1] - lo[1]), hi[2] - lo[2]) * 0.5;
    if (half <= 0.0) half = 1.0;
    c.w = half;
    return c;
}

}  // namespace nb
