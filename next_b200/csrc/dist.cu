// NCCL access for the sharded (multi-GPU) step.
//
// The library talks to NCCL through dlopen("libnccl.so.2") so that it shares
// whatever NCCL the host process already loaded (for instance the copy a
// Python framework ships) instead of linking a second one; only the stable
// C entry points below are used.  Types and enums come from nccl.h.
#include <dlfcn.h>
#include <nccl.h>

#include <mutex>
#include <string>

#include "dist.cuh"

namespace nb {
namespace {

struct NcclApi {
    bool ok = false;
    std::string why;
    ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*all_gather)(const void*, void*, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    const char* (*error_string)(ncclResult_t) = nullptr;
};

NcclApi& api() {
    static NcclApi a;
    static std::once_flag once;
    std::call_once(once, [] {
        void* lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!lib) {
            a.why = std::string("cannot load libnccl.so.2: ") + dlerror();
            return;
        }
        a.get_unique_id = reinterpret_cast<decltype(a.get_unique_id)>(dlsym(lib, "ncclGetUniqueId"));
        a.comm_init_rank = reinterpret_cast<decltype(a.comm_init_rank)>(dlsym(lib, "ncclCommInitRank"));
        a.all_gather = reinterpret_cast<decltype(a.all_gather)>(dlsym(lib, "ncclAllGather"));
        a.comm_destroy = reinterpret_cast<decltype(a.comm_destroy)>(dlsym(lib, "ncclCommDestroy"));
        a.error_string = reinterpret_cast<decltype(a.error_string)>(dlsym(lib, "ncclGetErrorString"));
        a.ok = a.get_unique_id && a.comm_init_rank && a.all_gather && a.comm_destroy && a.error_string;
        if (!a.ok) a.why = "libnccl.so.2 lacks an expected entry point";
    });
    return a;
}

std::string describe(ncclResult_t r) {
    NcclApi& a = api();
    return a.error_string ? a.error_string(r) : "NCCL error " + std::to_string(static_cast<int>(r));
}

}  // namespace

bool nccl_unique_id(unsigned char out[128], std::string* why) {
    NcclApi& a = api();
    if (!a.ok) { *why = a.why; return false; }
    ncclUniqueId id;
    const ncclResult_t r = a.get_unique_id(&id);
    if (r != ncclSuccess) { *why = "ncclGetUniqueId: " + describe(r); return false; }
    static_assert(sizeof(id.internal) == 128, "ncclUniqueId is 128 bytes");
    for (int i = 0; i < 128; ++i) out[i] = static_cast<unsigned char>(id.internal[i]);
    return true;
}

bool nccl_comm_init(void** comm, int rank, int world, const unsigned char id_bytes[128], std::string* why) {
    NcclApi& a = api();
    if (!a.ok) { *why = a.why; return false; }
    ncclUniqueId id;
    for (int i = 0; i < 128; ++i) id.internal[i] = static_cast<char>(id_bytes[i]);
    ncclComm_t c = nullptr;
    const ncclResult_t r = a.comm_init_rank(&c, world, id, rank);
    if (r != ncclSuccess) { *why = "ncclCommInitRank: " + describe(r); return false; }
    *comm = c;
    return true;
}

// In-place all-gather of `count` doubles per rank: rank r's share sits at
// buf + r*count on every rank.
bool nccl_allgather_inplace(void* comm, double* buf, size_t count, int rank, cudaStream_t st, std::string* why) {
    NcclApi& a = api();
    const ncclResult_t r = a.all_gather(buf + static_cast<size_t>(rank) * count, buf, count, ncclFloat64,
                                        static_cast<ncclComm_t>(comm), st);
    if (r != ncclSuccess) { *why = "ncclAllGather: " + describe(r); return false; }
    return true;
}

void nccl_comm_destroy(void* comm) {
    if (comm && api().ok) api().comm_destroy(static_cast<ncclComm_t>(comm));
}

}  // namespace nb
