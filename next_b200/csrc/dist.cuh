// NCCL entry points used by the sharded step (see dist.cu).
#pragma once
#include <cuda_runtime.h>

#include <string>

namespace nb {

bool nccl_unique_id(unsigned char out[128], std::string* why);
bool nccl_comm_init(void** comm, int rank, int world, const unsigned char id[128], std::string* why);
bool nccl_allgather_inplace(void* comm, double* buf, size_t count, int rank, cudaStream_t st, std::string* why);
void nccl_comm_destroy(void* comm);

}  // namespace nb
