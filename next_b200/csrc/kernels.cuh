// Launch wrappers of the library's kernels (host side, namespace nb).
#pragma once

#include "common.cuh"

namespace nb {

// Host-side count of kernels launched (the library's own kernels only).
void count_launches(int k);
int64_t launches_so_far();

// keys.cu
cudaError_t launch_root_cubes(const Bodies& b, int64_t n, const Systems& sys, const int64_t* d_offsets,
                              double* partial, int partial_blocks, unsigned int* ticket, cudaStream_t st);
cudaError_t launch_keys(const Bodies& b, const int32_t* sysid, int64_t n, const Systems& sys, uint64_t* keys,
                        uint32_t* idx, cudaStream_t st);

// sort.cu
#ifndef NB_SORT_ITEMS
#define NB_SORT_ITEMS 15
#endif
constexpr int64_t kSortTile = 256 * NB_SORT_ITEMS;   // pairs per onesweep tile (threads x items)
constexpr int64_t sort_scratch_words_for(int64_t n) {
    return 2 * 8 * 256 + 8 + 8 * ((n + kSortTile - 1) / kSortTile) * 256;
}
size_t sort_scratch_words(int64_t n);
size_t sort_smem_bytes();
cudaError_t sort_prepare();
cudaError_t radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* alt_keys, uint32_t* alt_vals, int64_t n,
                             int key_bits, uint32_t* scratch, int* err, bool* in_alt, cudaStream_t st);
cudaError_t radix_sort_pairs_to(const uint64_t* keys_in, const uint32_t* vals_in, uint64_t* keys_out,
                                uint32_t* vals_out, uint64_t* alt_keys, uint32_t* alt_vals, int64_t n, int key_bits,
                                uint32_t* scratch, int* err, cudaStream_t st);

// scan.cu
template <typename T>
cudaError_t exclusive_scan(const T* in, T* out, int64_t n_cap, const int64_t* count_dev, T* tile_sums,
                           int64_t* total_dev, cudaStream_t st);
int64_t scan_tile_sums_needed(int64_t n_cap);

// tree.cu
cudaError_t build_tree(const uint64_t* keys, int64_t n, const Bodies& bd, const int32_t* sysid, const Systems& sys,
                       const int64_t* d_offsets, const Params& P, Tree& t, void* scan_tmp, int* err,
                       cudaStream_t st);

// walk_plain.cu
cudaError_t launch_walk_plain(const Bodies& bd, const int32_t* sysid, int64_t n, const Tree& t, const Params& P,
                              bool multi_system, unsigned long long* stats, int* err, cudaStream_t st);
int direct_slices(int64_t n, int64_t k);
// in: k sizes, k masses, k distances; out: k softening lengths (reference law)
cudaError_t launch_softening_eval(const double* in, int64_t k, double* out, cudaStream_t st);
cudaError_t launch_direct(const Bodies& bd, int64_t n, const int64_t* targets, int64_t k, double eps, double G,
                          double* partial, int slices, double* out, cudaStream_t st);

// walk_group.cu: the warp-per-group walk, FP32-mixed or FP64 arithmetic
size_t walk_group_smem(bool fp64, int warps, int stack_cap);
cudaError_t launch_walk_group(const Bodies& bd, int64_t nbodies, const Tree& t, const Params& P, bool potential,
                              bool fp64, int warps, int stack_cap, unsigned int* queue, unsigned long long* stats,
                              int* err, int sm_count, cudaStream_t st);

// integrate.cu
cudaError_t launch_gather_bodies(const Bodies& src, const Bodies& dst, const uint32_t* idx, int64_t n, uint32_t* inv,
                                 int* err, cudaStream_t st);
cudaError_t launch_kick_drift(const Bodies& b, int64_t n, const double* dts, const int* err, cudaStream_t st);
// kick-drift that also writes the root cube of the drifted bodies (one system)
cudaError_t launch_kick_drift_box(const Bodies& b, int64_t n, const double* dts, const int* err, double* partial,
                                  int partial_blocks, unsigned int* ticket, double4* cube, cudaStream_t st);
cudaError_t launch_kick(const Bodies& b, int64_t n, const double* dts, const int* err, cudaStream_t st,
                        unsigned int* done = nullptr);
int reduce_blocks(int64_t n);
cudaError_t launch_adaptive_dt(const Bodies& b, int64_t n, double base_dt, double* partial, unsigned int* ticket,
                               double* out, cudaStream_t st);
cudaError_t launch_diagnostics(const Bodies& b, int64_t n, bool have_pot, double* partial, unsigned int* ticket,
                               double* out, cudaStream_t st);
cudaError_t launch_check_upload(const double* stage, const int* stype, const Bodies& b, const uint32_t* inv, int64_t n,
                                bool compare, int* flags, cudaStream_t st);
cudaError_t launch_load_velocities(const double* stage, const Bodies& b, const uint32_t* inv, int64_t n,
                                   cudaStream_t st);
cudaError_t launch_load_all(const double* stage, const int* stype, const Bodies& b, uint32_t* inv, int64_t n,
                            cudaStream_t st);
// flags[0] = 1 unless in (7 lanes x n, caller order) and type equal prev_out's
// 6 lanes, prev_in's mass lane and prev_type bit for bit (and are finite)
cudaError_t launch_same_as_last(const double* in, const int* type, const double* prev_out, const double* prev_in,
                                const int* prev_type, int64_t n, int* flags, cudaStream_t st);
// gathers `count` (<= kMaxGatherLanes) lanes, given as host-side pointers to device arrays
constexpr int kMaxGatherLanes = 8;
cudaError_t launch_gather_out(const double* const* lanes, int count, const uint32_t* inv, int64_t n, double* out,
                              cudaStream_t st);
cudaError_t launch_ids_to_positions(const int64_t* ids, const uint32_t* inv, int64_t k, int64_t* pos,
                                    cudaStream_t st);
cudaError_t launch_set_dt(double* dts, double dt, cudaStream_t st);
cudaError_t launch_fma_peak(float* out, int blocks, int iters, cudaStream_t st);

}  // namespace nb
