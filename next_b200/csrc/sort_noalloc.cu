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
// part of the library reserves it (14,844,192 bytes, 14.16 MiB) until the
// process exits.  Host code must not use the array's name as a device
// address: the first call in each CUDA context (normally once per device, in
// its primary context) looks the address up with cudaGetSymbolAddress, with
// that context current, and keeps it for that context.  A context made later
// -- after cudaDeviceReset, or one the caller creates with the driver API --
// gets its own look-up, because the array's address belongs to the context
// that loaded the module.  All calls share the one array, so the scratch
// that must start at zero is cleared on every call, and calls whose work
// overlaps on the GPU (other streams, other host threads) race on it.
#include <cuda.h>

#include <mutex>
#include <vector>

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
static_assert(kScratchBytes == 14844192, "the size the header states");

static __device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

// Driver entry points that identify the current context, resolved through
// the runtime so the library does not link libcuda itself.
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

struct ContextScratch {
    unsigned long long ctx_id;
    unsigned char* addr;
};

std::mutex g_setup_mutex;
std::vector<ContextScratch> g_scratch;   // one entry per context that has called
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;
bool g_entry_points_resolved = false;

// The unique id of the current context (0 if the driver cannot tell, in
// which case nothing is cached and every call looks the address up again).
unsigned long long current_context_id() {
    if (!g_entry_points_resolved) {
        g_entry_points_resolved = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_id = reinterpret_cast<CtxGetIdFn>(f);
    }
    if (!g_ctx_current || !g_ctx_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (g_ctx_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
    if (g_ctx_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Set-up, once per context, with that context current: the array's device
// address and the onesweep kernel's shared-memory attribute.
int context_scratch(unsigned char** out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    unsigned long long id = current_context_id();
    if (id != 0)
        for (const ContextScratch& c : g_scratch)
            if (c.ctx_id == id) { *out = c.addr; return NEXT_OK; }
    // no context yet, or a new one: the look-up makes the current device's
    // primary context current if no context is
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_sort_scratch) != cudaSuccess || p == nullptr) return NEXT_ERR_CUDA;
    if (sort_prepare() != cudaSuccess) return NEXT_ERR_CUDA;
    if (id == 0) id = current_context_id();
    if (id != 0) g_scratch.push_back({id, static_cast<unsigned char*>(p)});
    *out = static_cast<unsigned char*>(p);
    return NEXT_OK;
}

bool overlaps(const void* a, size_t abytes, const void* b, size_t bbytes) {
    const uintptr_t a0 = reinterpret_cast<uintptr_t>(a), b0 = reinterpret_cast<uintptr_t>(b);
    return a0 < b0 + bbytes && b0 < a0 + abytes;
}

}  // namespace
}  // namespace nb

extern "C" int next_sort_pairs_noalloc(const uint64_t* d_keys_in, const uint32_t* d_vals_in, uint64_t* d_keys_out,
                                       uint32_t* d_vals_out, int64_t n, int key_bits, void* stream) {
    using namespace nb;
    if (n < 0 || n > kMaxPairs || key_bits < 1 || key_bits > 64) return NEXT_ERR_INVALID_ARGUMENT;
    if (n == 0) return NEXT_OK;
    if (!d_keys_in || !d_vals_in || !d_keys_out || !d_vals_out) return NEXT_ERR_INVALID_ARGUMENT;
    // no output may share a byte with an input or with the other output
    const size_t kb = sizeof(uint64_t) * static_cast<size_t>(n), vb = sizeof(uint32_t) * static_cast<size_t>(n);
    if (overlaps(d_keys_out, kb, d_keys_in, kb) || overlaps(d_keys_out, kb, d_vals_in, vb) ||
        overlaps(d_vals_out, vb, d_keys_in, kb) || overlaps(d_vals_out, vb, d_vals_in, vb) ||
        overlaps(d_keys_out, kb, d_vals_out, vb))
        return NEXT_ERR_INVALID_ARGUMENT;
    unsigned char* base = nullptr;
    int rc = context_scratch(&base);
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
    // the error word is read back in stream order: no wait on other streams
    int bits = 0;
    if (cudaMemcpyAsync(&bits, err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return NEXT_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return NEXT_ERR_CUDA;
    return bits ? NEXT_ERR_DEVICE : NEXT_OK;
}
