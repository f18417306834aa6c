// Shared definitions of the B200 gravity library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/next_gpu.h"

namespace nb {

constexpr int kMaxLevel = 21;        // 63-bit keys: 21 levels of 3 bits, bit 63 unused
constexpr int kWarp = 32;

// Device error word bits (mirrors NEXT_DEVERR_* in next_gpu.h).
constexpr int kErrTree = NEXT_DEVERR_TREE_OVERFLOW;
constexpr int kErrStack = NEXT_DEVERR_WALK_STACK;
constexpr int kErrSort = NEXT_DEVERR_SORT_TIMEOUT;
constexpr int kErrList = NEXT_DEVERR_LIST_OVERFLOW;
constexpr int kErrIndex = NEXT_DEVERR_BAD_INDEX;
constexpr int kErrAbort = kErrTree | kErrStack | kErrIndex;   // the step's results are invalid

// Bodies in working order (sorted by key after each build).  FP64 SoA.
struct Bodies {
    double *x, *y, *z, *vx, *vy, *vz, *m;
    double *ax, *ay, *az, *pot;
    int* type;
    uint32_t* id;        // caller's index of the body at this position
};

// Per-system geometry: root cube and body range.
struct Systems {
    int n;               // number of systems
    int base;            // key >> base = system number (63 for one system)
    int levels;          // octant levels per key (base / 3)
    const int64_t* offsets;   // n + 1
    double4* cube;       // cx, cy, cz, half
};

// Tree in sibling-contiguous layout.  Nodes 0..nsys-1 are the system roots;
// the children of every internal node are stored consecutively in octant
// order.  Internal nodes also have a depth-first "internal id" q used by the
// build.
// nint_kernel's depth report when leaf_cap + 1 bodies share a cell at the
// last key level (a leaf over capacity: the keys need more levels)
constexpr unsigned kDepthOverfull = 64;

struct Tree {
    // capacities
    int64_t cap_int, cap_node, cap_group;
    // per sorted position
    int8_t* dlev;          // shared-prefix level with the previous key (-1 at a root)
    int32_t* nint;         // internal cells starting here -> exclusive scan in place
    // per internal id q
    int32_t* int_start;
    int8_t* int_level;
    int32_t* int_bounds;   // 9 per q: child c spans [b[c], b[c+1])
    int64_t* int_packed;   // nchild | ngroups << 32 -> exclusive scan in place
    int32_t* int_node;     // node id of q
    int32_t* counter;      // upward-pass arrivals (self-resetting)
    int4* climb;           // node id, first child, child count | level << 8, start position
    // per node
    int2* link;            // internal: (first child, nchild); leaf: (first body, -count)
    int32_t* parent;       // internal id of the parent (-1 for a root)
    int8_t* level;
    double4* com;          // FP64 centre of mass and mass
    double* quad64;        // 8 per node: Qxx Qyy Qzz Qxy Qxz Qyz half-width rcrit
    float4* box;           // FP32 COM and rcrit^2 (mixed walk traversal)
    float4* quad32;        // 2 per node: -G (Qxx Qyy Qzz Qxy) (Qxz Qyz), G m, 0
    // walk groups
    int4* groups;          // (first body, count, root node, 0)
    int32_t* ready;        // upward pass: internal ids whose children are all leaves
    // device scalars: [0] internal count, [1] node count, [2] group count,
    // [3] deepest leaf level, [4] ready-list length
    int64_t* counts;
};

struct Params {
    int physics;           // NEXT_PHYSICS_*
    double theta, eps, G;
    int leaf_cap, group_cap, quad;
    // bodies (working positions) whose forces this device computes; the
    // whole range on one device, one share of it per rank when sharded
    int64_t own_lo = 0, own_hi = INT64_MAX;
};

// Key layout: the system number sits in bits [base, 63), the octant digit of
// level l (1-based) in bits [base - 3l, base - 3l + 3).  One system: base = 63
// and 21 levels; S systems: base = 63 - ceil(log2 S), levels = base / 3.
__device__ __forceinline__ int key_digit(uint64_t key, int level, int base) {
    return static_cast<int>((key >> (base - 3 * level)) & 7u);
}

// Shared-prefix level of two keys: -1 if they belong to different systems,
// else the number of leading octant digits they share (levels when equal).
__device__ __forceinline__ int shared_levels(uint64_t a, uint64_t b, int base, int levels) {
    const uint64_t d = a ^ b;
    if (d == 0) return levels;
    if (base < 64 && (d >> base) != 0) return -1;
    const int lz = __clzll(static_cast<long long>(d)) - (64 - base);
    const int l = lz / 3;
    return l < levels ? l : levels;
}

__device__ __forceinline__ void raise_error(int* err, int bits) { atomicOr(err, bits); }

}  // namespace nb

#define NB_CUDA_OK(expr) ((expr) == cudaSuccess)
