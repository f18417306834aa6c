// next_sort_pairs_noalloc: the radix sort for callers that cannot allocate
// device memory.
//
// Some callers hand this library only device buffers they already own and
// must not let it allocate more: host codes that carve each GPU's memory into
// a fixed budget or run their own pool allocator, and steps that cannot
// afford cudaMalloc/cudaFree, which may synchronise the whole device in the
// middle of a pipelined time step.  For them this entry point sorts pairs
// between caller-owned device buffers and takes every byte of scratch --
// the ping-pong half of the LSD passes, the digit histograms, the tile
// tickets, the look-back status words and the error word -- from the
// fixed-size array below.
//
// The array is a file-scope __device__ variable, so every GPU that loads this
// part of the library reserves it (about 14.2 MiB) until the process exits.
// Host code must not use the array's name as a device address: the first
// call on each device, with that device current, looks the address up with
// cudaGetSymbolAddress and keeps it.  All calls share the one array, so the
// scratch that must start at zero is cleared on every call, and calls whose
// work overlaps on the GPU (other streams, other host threads) race on it.
#include <mutex>

#include "common.cuh"
#include "kernels.cuh"

namespace nb {
namespace {

constexpr int64_t kMaxPairs = NEXT_SORT_NOALLOC_MAX_PAIRS;
constexpr size_t kAltKeysBytes = sizeof(uint64_t) * kMaxPairs;
constexpr size_t kAltValsBytes = sizeof(uint32_t) * kMaxPairs;
constexpr size_t kErrBytes = 256;
constexpr size_t kWordsBytes = sizeof(uint32_t) * sort_scratch_words_for(kMaxPairs);
constexpr size_t kScratchBytes = kAltKeysBytes + kAltValsBytes + kErrBytes + kWordsBytes;

static_assert(kAltKeysBytes % 256 == 0 && kAltValsBytes % 256 == 0, "sub-buffers stay 256-byte aligned");

static __device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_addr[kMaxDevices] = {};

// Once per device, with that device current: the array's device address and
// the onesweep kernel's shared-memory attribute.
int device_scratch(unsigned char** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return NEXT_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return NEXT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_sort_scratch) != cudaSuccess || p == nullptr) return NEXT_ERR_CUDA;
        if (sort_prepare() != cudaSuccess) return NEXT_ERR_CUDA;
        g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_addr[dev];
    return NEXT_OK;
}

}  // namespace
}  // namespace nb

extern "C" int next_sort_pairs_noalloc(const uint64_t* d_keys_in, const uint32_t* d_vals_in, uint64_t* d_keys_out,
                                       uint32_t* d_vals_out, int64_t n, int key_bits, void* stream) {
    using namespace nb;
    if (n < 0 || n > kMaxPairs || key_bits < 1 || key_bits > 64) return NEXT_ERR_INVALID_ARGUMENT;
    if (n == 0) return NEXT_OK;
    if (!d_keys_in || !d_vals_in || !d_keys_out || !d_vals_out) return NEXT_ERR_INVALID_ARGUMENT;
    if (static_cast<const void*>(d_keys_in) == static_cast<const void*>(d_keys_out) ||
        static_cast<const void*>(d_vals_in) == static_cast<const void*>(d_vals_out))
        return NEXT_ERR_INVALID_ARGUMENT;
    unsigned char* base = nullptr;
    int rc = device_scratch(&base);
    if (rc) return rc;
    uint64_t* alt_keys = reinterpret_cast<uint64_t*>(base);
    uint32_t* alt_vals = reinterpret_cast<uint32_t*>(base + kAltKeysBytes);
    int* err = reinterpret_cast<int*>(base + kAltKeysBytes + kAltValsBytes);
    uint32_t* words = reinterpret_cast<uint32_t*>(base + kAltKeysBytes + kAltValsBytes + kErrBytes);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(err, 0, sizeof(int), st) != cudaSuccess) return NEXT_ERR_CUDA;
    if (radix_sort_pairs_to(d_keys_in, d_vals_in, d_keys_out, d_vals_out, alt_keys, alt_vals, n, key_bits, words, err,
                            st) != cudaSuccess)
        return NEXT_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return NEXT_ERR_CUDA;
    int bits = 0;
    if (cudaMemcpy(&bits, err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return NEXT_ERR_CUDA;
    return bits ? NEXT_ERR_DEVICE : NEXT_OK;
}
