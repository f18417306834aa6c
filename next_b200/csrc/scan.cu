// Device-wide exclusive prefix sum in three launches (tile sums, one-block
// scan of the tile sums, tile scans + carry).  The element count may live in
// device memory (count_dev), so a launch sized for a capacity works on a
// count that an earlier kernel produced without a host round trip.  The
// total is written to out[n] and, if total_dev is given, to *total_dev.
#include "common.cuh"
#include "kernels.cuh"

namespace nb {

namespace {

#ifndef NB_SCAN_VEC
#define NB_SCAN_VEC 1
#endif
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename T>
__device__ T block_exclusive_scan(T v, T* total) {
    __shared__ T warp_sums[kScanThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const T u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) warp_sums[w] = inc;
    __syncthreads();
    if (w == 0) {
        T s = lane < kScanThreads / 32 ? warp_sums[lane] : T(0);
        for (int o = 1; o < 32; o <<= 1) {
            const T u = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += u;
        }
        if (lane < kScanThreads / 32) warp_sums[lane] = s;
    }
    __syncthreads();
    const T before = w > 0 ? warp_sums[w - 1] : T(0);
    *total = warp_sums[kScanThreads / 32 - 1];
    __syncthreads();
    return before + inc - v;
}

template <typename T>
__device__ __forceinline__ int64_t scan_count(int64_t n, const int64_t* count_dev) {
    // A device count larger than the capacity the launch was sized for is an
    // overflow the caller reports; never index past the capacity.
    if (!count_dev) return n;
    const int64_t c = *count_dev;
    return c < 0 ? 0 : (c > n ? n : c);
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads)
tile_sums_kernel(const T* __restrict__ in, int64_t n, const int64_t* count_dev, T* __restrict__ sums) {
    const int64_t cnt = scan_count<T>(n, count_dev);
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile;
    if (base >= cnt) return;
    T s = 0;
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + k * kScanThreads + threadIdx.x;
        if (i < cnt) s += in[i];
    }
    T total;
    block_exclusive_scan<T>(s, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads)
scan_sums_kernel(T* sums, int64_t n, const int64_t* count_dev) {
    const int64_t cnt = scan_count<T>(n, count_dev);
    const int64_t tiles = (cnt + kScanTile - 1) / kScanTile;
    T carry = 0;
    for (int64_t b = 0; b < tiles; b += kScanThreads) {
        const int64_t i = b + threadIdx.x;
        const T v = i < tiles ? sums[i] : T(0);
        T total;
        const T ex = block_exclusive_scan<T>(v, &total);
        if (i < tiles) sums[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) sums[tiles] = carry;   // prefix of the one-past-the-end tile
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads)
tile_scan_kernel(const T* __restrict__ in, T* __restrict__ out, int64_t n, const int64_t* count_dev,
                 const T* __restrict__ sums, int64_t* total_dev) {
    const int64_t cnt = scan_count<T>(n, count_dev);
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile;
    if (base > cnt) return;
    // blocked layout: thread t owns items base + t*kScanItems .. +kScanItems,
    // moved as 16-byte vectors when all of them lie below the count
    constexpr int kVec = kScanItems * static_cast<int>(sizeof(T)) / 16;
    const int64_t first = base + static_cast<int64_t>(threadIdx.x) * kScanItems;
    const bool whole = NB_SCAN_VEC && first + kScanItems <= cnt;
    T v[kScanItems];
    T s = 0;
    if (whole) {
        const uint4* src = reinterpret_cast<const uint4*>(in + first);
#pragma unroll
        for (int q = 0; q < kVec; ++q) reinterpret_cast<uint4*>(v)[q] = src[q];
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) s += v[k];
    } else {
        for (int k = 0; k < kScanItems; ++k) {
            const int64_t i = first + k;
            v[k] = i < cnt ? in[i] : T(0);
            s += v[k];
        }
    }
    T total;
    T run = block_exclusive_scan<T>(s, &total) + sums[blockIdx.x];
    if (whole) {
        T o[kScanItems];
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) { o[k] = run; run += v[k]; }
        uint4* dst = reinterpret_cast<uint4*>(out + first);
#pragma unroll
        for (int q = 0; q < kVec; ++q) dst[q] = reinterpret_cast<const uint4*>(o)[q];
    } else {                                        // also the owner of out[cnt]
        for (int k = 0; k < kScanItems; ++k) {
            const int64_t i = first + k;
            if (i < cnt) out[i] = run;
            if (i == cnt) {
                out[i] = run;
                if (total_dev) *total_dev = static_cast<int64_t>(run);
            }
            run += v[k];
        }
    }
}

}  // namespace

template <typename T>
cudaError_t exclusive_scan(const T* in, T* out, int64_t n_cap, const int64_t* count_dev, T* tile_sums,
                           int64_t* total_dev, cudaStream_t st) {
    const int64_t tiles = n_cap / kScanTile + 1;   // the +1 tile writes out[n]
    tile_sums_kernel<T><<<static_cast<unsigned>(tiles), kScanThreads, 0, st>>>(in, n_cap, count_dev, tile_sums);
    scan_sums_kernel<T><<<1, kScanThreads, 0, st>>>(tile_sums, n_cap, count_dev);
    tile_scan_kernel<T><<<static_cast<unsigned>(tiles), kScanThreads, 0, st>>>(in, out, n_cap, count_dev,
                                                                                tile_sums, total_dev);
    count_launches(3);
    return cudaGetLastError();
}

int64_t scan_tile_sums_needed(int64_t n_cap) { return n_cap / kScanTile + 2; }

template cudaError_t exclusive_scan<int32_t>(const int32_t*, int32_t*, int64_t, const int64_t*, int32_t*,
                                             int64_t*, cudaStream_t);
template cudaError_t exclusive_scan<int64_t>(const int64_t*, int64_t*, int64_t, const int64_t*, int64_t*,
                                             int64_t*, cudaStream_t);

}  // namespace nb
