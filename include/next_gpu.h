/*
 * next_gpu.h -- C ABI of the B200 (sm_100a) gravity library libnext_b200.so.
 *
 * The library replaces NEXT's gravity hot path: the per-step tree build and
 * walk inside Step() (src/gravity/step.h:25-204), the octree and its moments
 * (src/gravity/octree.h:25-128), the force walk bhAccel (octree.h:133-179),
 * the softening law (src/dt/softening.h:21-35) and computeAdaptiveDt
 * (src/dt/adaptive.h:23-52).  The reference has no FFI of its own; its
 * boundary is the header-only C++ call Step(ParticleSystem&, real dt) made by
 * src/begrun.cpp:97-98.  These entry points are what that call binds to:
 * next_b200/host/gravity/step.h re-provides Step() and computeAdaptiveDt()
 * with the reference's signatures on top of them.
 *
 * Conventions
 *  - Every call returns an int status (NEXT_OK = 0).  next_last_error()
 *    gives a one-line message for the last failure on a handle.
 *  - All pointers are HOST pointers with plain sizes; device memory is
 *    owned by the handle.  Arrays are the reference's SoA lanes
 *    (src/struct/particle.h:22-31): x y z vx vy vz m as double, type as int.
 *  - Bodies keep the caller's index order at the boundary: index i in an
 *    upload is index i in every download / force query.
 *  - One handle per host thread; calls on a handle are ordered on the
 *    handle's CUDA stream.  Only the calls that return host data block.
 */
#ifndef NEXT_GPU_H
#define NEXT_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define NEXT_OK 0
#define NEXT_ERR_INVALID_ARGUMENT 1 /* bad size, NULL array, non-finite input, m < 0 */
#define NEXT_ERR_CUDA 2             /* a CUDA runtime call failed */
#define NEXT_ERR_OUT_OF_MEMORY 3
#define NEXT_ERR_NO_BODIES 4        /* step/force call before any upload */
#define NEXT_ERR_DEVICE 5           /* a kernel raised its error word (see next_stats.device_error) */

/* bits of the device error word (next_stats.device_error) */
#define NEXT_DEVERR_TREE_OVERFLOW 0x1   /* node/internal/group capacity exceeded */
#define NEXT_DEVERR_WALK_STACK 0x2      /* walk stack capacity exceeded */
#define NEXT_DEVERR_SORT_TIMEOUT 0x4    /* radix-sort look-back wait gave up */
#define NEXT_DEVERR_LIST_OVERFLOW 0x8   /* interaction-list capacity exceeded */
#define NEXT_DEVERR_BAD_INDEX 0x10      /* an index check failed (tree, sort or reorder); results invalid */

/* ---- physics and precision modes ------------------------------------- */
/* NEXT_PHYSICS_REFERENCE: the reference's semantics, reproduced exactly --
 *   one body per leaf, opening test half_width/dist < theta measured to the
 *   COM (octree.h:153), adaptive softening (softening.h:21-35, octree.h:145-148),
 *   the reference's quadrupole (octree.h:114-126, 163-172), G fixed at 1.
 * NEXT_PHYSICS_ACCURATE: Plummer softening eps, full-width opening test
 *   |COM - x| >= 2*half_width/theta + |COM - centre|, traceless quadrupole
 *   with parallel-axis terms and the correct sign, leaf buckets of leaf_cap. */
#define NEXT_PHYSICS_REFERENCE 0
#define NEXT_PHYSICS_ACCURATE 1

/* NEXT_PRECISION_FP64: plain FP64 walk, one thread per body, depth-first in
 *   the reference's child order; two tree builds per step as in step.h.
 * NEXT_PRECISION_MIXED: FP32 interactions in a warp-per-group walk with
 *   shared-memory interaction lists and compensated accumulation; FP64 for
 *   positions, velocities, kick/drift, tree moments and diagnostics.
 *   Requires NEXT_PHYSICS_ACCURATE.
 * NEXT_PRECISION_FP64_GROUP: the same warp-per-group walk as MIXED -- same
 *   leaf buckets, groups, interaction lists, force reuse and graph replays --
 *   with every interaction in FP64.  It differs from MIXED in precision only.
 *   Requires NEXT_PHYSICS_ACCURATE. */
#define NEXT_PRECISION_FP64 0
#define NEXT_PRECISION_MIXED 1
#define NEXT_PRECISION_FP64_GROUP 2

typedef struct next_params {
    int physics;        /* NEXT_PHYSICS_* */
    int precision;      /* NEXT_PRECISION_* */
    double theta;       /* opening angle (reference: 0.5, step.h:32) */
    double eps;         /* Plummer softening length (accurate mode) */
    double G;           /* gravitational constant (reference mode forces 1) */
    int leaf_cap;       /* bodies per leaf before a cell splits (reference mode forces 1) */
    int group_cap;      /* bodies per walk group, <= 32 (group walk: MIXED, FP64_GROUP) */
    int quadrupole;     /* 1: monopole + quadrupole; 0: monopole only (accurate mode) */
    int reuse_forces;   /* 1: the first half-kick reuses a(x_n) from the previous step */
    int walk_warps;     /* warps per block of the group walk (1..4) */
    int walk_stack;     /* per-warp traversal stack entries of the group walk */
    int device;         /* CUDA device ordinal */
} next_params;

typedef struct next_stats {
    int64_t n_bodies;
    int64_t n_systems;
    int64_t n_nodes;         /* tree nodes of the last build */
    int64_t n_internal;
    int64_t n_groups;        /* walk groups of the last build (mixed) */
    int64_t pp_interactions; /* body-body interactions since next_reset_timers */
    int64_t pc_interactions; /* body-cell interactions since next_reset_timers */
    int64_t max_stack;       /* deepest walk stack seen since next_reset_timers (mixed) */
    int32_t device_error;    /* NEXT_DEVERR_* bits */
    int32_t steps;           /* steps timed since next_reset_timers */
    double ms_step;          /* summed device time of timed steps (CUDA events) */
    double ms_build;         /* ... of which keys + sort + reorder + tree + moments */
    double ms_walk;          /* ... of which force walk */
    double ms_sort;          /* ... of which radix sort */
    double ms_other;         /* ... kick/drift and the rest */
    int64_t walk_launches;   /* walks timed */
    int32_t key_levels;      /* octant levels in the keys of the last build (21 = full depth) */
    int32_t recoveries;      /* graph-replayed steps (next_steps) that overflowed a capacity and were
                                finished by re-running their force phase and closing kick */
} next_stats;

typedef struct next_handle next_handle;

/* Fill *p with defaults for a physics/precision pair. */
int next_params_default(next_params* p, int physics, int precision);

int next_create(const next_params* p, next_handle** out);
void next_destroy(next_handle* h);
const char* next_last_error(const next_handle* h);
const char* next_status_string(int status);

/* Upload one system (replaces src/io/load_particle.hpp:100-116's result
 * being handed to Step).  type may be NULL (all type 0).  If the positions
 * and masses equal the ones the handle already holds, forces cached by the
 * previous step stay valid. */
int next_upload(next_handle* h, int64_t n, const double* x, const double* y, const double* z,
                const double* vx, const double* vy, const double* vz, const double* m,
                const int* type);

/* Upload n_systems independent systems at once: system s owns bodies
 * offsets[s] .. offsets[s+1]-1 (offsets has n_systems+1 entries).  Each
 * system gets its own root cube, tree and walk; no force acts between
 * systems.  Segmented keys carry the system number above the octant digits. */
int next_upload_systems(next_handle* h, int64_t n_systems, const int64_t* offsets,
                        const double* x, const double* y, const double* z,
                        const double* vx, const double* vy, const double* vz,
                        const double* m, const int* type);

/* Copy the state back in the caller's order.  Any pointer may be NULL. */
int next_download(next_handle* h, double* x, double* y, double* z,
                  double* vx, double* vy, double* vz);

/* One KDK leapfrog step (step.h:111-189): v += a dt/2, x += v dt, forces at
 * the new positions, v += a dt/2. */
int next_step(next_handle* h, double dt);

/* nsteps steps of fixed dt; with mixed precision each step is one replay of a
 * captured CUDA graph.  The device error word is read every 64 replays and at
 * the end; a replay that overflowed a capacity (tree, walk stack) is finished
 * as next_step would finish it -- capacity grown, force phase and closing kick
 * re-run -- and the steps after it are taken again, so the result equals the
 * same steps taken one by one (next_stats.recoveries counts such replays). */
int next_steps(next_handle* h, double dt, int nsteps);

/* The reference's Step(ParticleSystem&, dt) on host arrays (src/gravity/
 * step.h:25): upload x..vz, m and type (type may be NULL), one KDK step, and
 * the new positions and velocities written back into x..vz in place.  The
 * same as next_upload + next_step + next_download, but faster:
 *  - the positions are copied back while the force phase runs;
 *  - when the previous call on this handle was next_step_host with the same
 *    n and nothing changed the held state since, the step starts on the held
 *    state while the inputs upload, and the inputs are then compared bit for
 *    bit with what that call returned (masses and types with what it was
 *    given).  If they differ, the step is taken again from the inputs.
 * Either way the result is the step of the inputs.  Returns after every copy
 * into the caller's arrays has finished.  Inputs that are rejected
 * (NEXT_ERR_INVALID_ARGUMENT: non-finite values, negative masses) leave
 * x..vz as the caller passed them and the held state as it was. */
int next_step_host(next_handle* h, double dt, int64_t n, double* x, double* y, double* z,
                   double* vx, double* vy, double* vz, const double* m, const int* type);

/* Forces at the current positions (the quantity bhAccel accumulates,
 * octree.h:133), in the caller's order.  pot may be NULL; it is filled only
 * in accurate mode. */
int next_accel(next_handle* h, double* ax, double* ay, double* az, double* pot);

/* computeAdaptiveDt (src/dt/adaptive.h:23-52) as a device reduction. */
int next_adaptive_dt(next_handle* h, double base_dt, double* dt_out);

/* FP64 direct summation with Plummer softening eps (and G) of the handle for
 * the k bodies idx[0..k) (caller's indices).  pot may be NULL. */
int next_direct_accel(next_handle* h, int64_t k, const int64_t* idx,
                      double* ax, double* ay, double* az, double* pot);

/* FP64 diagnostics: out[0] kinetic energy, out[1] potential energy (from the
 * walk; accurate mode), out[2..4] momentum, out[5..7] angular momentum. */
int next_diagnostics(next_handle* h, double* out8);

int next_stats_get(next_handle* h, next_stats* s);
int next_set_timing(next_handle* h, int on);
int next_reset_timers(next_handle* h);
int next_sync(next_handle* h);

/* Octant keys (the reference's insertion path, octree.h:49-64, 21 levels of
 * 3 bits from bit 62 down) of the uploaded bodies in the caller's order, and
 * the root cube (cx, cy, cz, half-width) of step.h:69-100. */
int next_debug_keys(next_handle* h, uint64_t* keys, double* cube4);

/* Test support: the device's reference softening law nextSoftening
 * (src/dt/softening.h:21-35), as the reference-physics walk evaluates it, on
 * k (size, mass, dist) triples. */
int next_debug_softening(int device, int64_t k, const double* size, const double* mass, const double* dist,
                         double* out);

/* Test support: sets the tree's capacity to cap_internal internal cells and
 * from then on grows it only when a build overflows it (not ahead of need),
 * so that tests can make a graph-replayed step overflow. */
int next_debug_fix_tree_capacity(next_handle* h, int64_t cap_internal);

/* Stable key order of the last build: perm[p] = caller's index of the p-th
 * body in key order. */
int next_debug_order(next_handle* h, int64_t* perm);

/* Build the tree at the current positions and export it depth-first
 * (children in octant order, the order bhAccel visits them) as 16 doubles
 * per node: level, m, com x y z, half-width, Qxx Qyy Qzz Qxy Qxz Qyz, leaf,
 * body index (one-body leaf, else -1), 0, body count.  *n_rows = node count. */
int next_debug_tree(next_handle* h, double* rows, int64_t cap, int64_t* n_rows);

/* Stable LSD radix sort of (key, value) pairs on the device, the sort the
 * tree build uses: n pairs in, sorted pairs out (host arrays), ordered by the
 * low key_bits bits of the keys (higher bits are carried through unchanged).
 * NEXT_ERR_DEVICE if the sort raised its device error word. */
int next_sort_pairs(next_handle* h, int64_t n, const uint64_t* keys_in, const uint32_t* vals_in,
                    uint64_t* keys_out, uint32_t* vals_out, int key_bits);

/* Allocation-free variant of next_sort_pairs, for callers that own all device
 * memory themselves (a fixed per-GPU budget, their own pool allocator) or
 * cannot afford the device-wide synchronisation cudaMalloc/cudaFree may cause
 * mid-step.  It has no counterpart in the reference, which sorts nothing.
 *
 * Sorts n (key, value) pairs from caller-owned DEVICE buffers d_keys_in /
 * d_vals_in into caller-owned DEVICE buffers d_keys_out / d_vals_out, stably
 * by the low key_bits bits of the keys (higher bits take no part in the
 * order and are carried through unchanged).  The inputs are left untouched;
 * no output may overlap an input or the other output (checked byte range by
 * byte range: NEXT_ERR_INVALID_ARGUMENT).  It allocates nothing: all scratch
 * comes from one static device array sized for NEXT_SORT_NOALLOC_MAX_PAIRS
 * pairs (14,844,192 bytes = 14.16 MiB, reserved on every GPU that loads the
 * library until the process exits); larger n is rejected with
 * NEXT_ERR_INVALID_ARGUMENT.  The first call in each CUDA context (normally
 * once per device) looks up that array's address and sets the sort kernel's
 * shared-memory limit, so make that first call before any stream capture.
 * Work is queued on `stream` (a cudaStream_t; NULL = default stream) of the
 * current device; the call reads the sort's error word back on that stream
 * and returns after the stream has finished (NEXT_ERR_DEVICE if the sort
 * raised an error).  Every call reuses the same array, so calls whose GPU
 * work overlaps race: serialise them. */
#define NEXT_SORT_NOALLOC_MAX_PAIRS 1048576
int next_sort_pairs_noalloc(const uint64_t* d_keys_in, const uint32_t* d_vals_in, uint64_t* d_keys_out,
                            uint32_t* d_vals_out, int64_t n, int key_bits, void* stream);

/* Sustained FP32 FMA throughput of the device (TFLOP/s), by a chain-of-FMA
 * kernel; the denominator of the walk's roofline. */
int next_fp32_peak(int device, double* tflops, double* sm_mhz_hint);

/* Write a buffer larger than L2 on the handle's stream (untimed helper for
 * benchmarks that flush L2 between steps). */
int next_flush_l2(next_handle* h);

/* Autotuner (mixed precision): times the force phase (tree build + walk) on
 * the uploaded bodies for leaf_cap x group_cap x walk_warps candidates, sizes
 * walk_stack at 1.5x the deepest stack seen, and keeps the fastest setting in
 * the handle.  Positions and velocities are not changed.  No counterpart in
 * the reference (its tree has one body per leaf and no walk groups). */
typedef struct next_tune_result {
    int leaf_cap, group_cap, walk_warps, walk_stack;
    double ms_force_phase;   /* device time of the chosen setting's force phase */
    int candidates;          /* settings timed */
} next_tune_result;
int next_autotune(next_handle* h, next_tune_result* out);

/* The handle's current parameters (after autotuning or capacity growth). */
int next_get_params(const next_handle* h, next_params* p);

/* Sharding one system over several GPUs (one process and one handle per
 * GPU).  Every rank uploads the same bodies and keeps all of them; each builds
 * the full tree (identical on every rank), walks only its share of the bodies
 * (working positions [rank*c, (rank+1)*c), c = ceil(n/world)), and the forces
 * are completed with in-place NCCL all-gathers over NVLink (24 B per body per
 * force phase), so kick and drift stay bit-identical on all ranks.  This
 * replaces the reference's replicated-data MPI decomposition
 * (src/gravity/step.h:36-65, 125-188: slice [rank*N/size, (rank+1)*N/size),
 * MPI_Allreduce of the box, MPI_Iallgatherv of v and x).
 *   next_dist_unique_id: rank 0 makes the 128-byte NCCL id; the caller sends
 *     it to the other ranks (e.g. over its own process group).
 *   next_dist_attach: joins the communicator (blocks until all ranks join).
 *     With id128 == NULL no communicator is made and the handle computes only
 *     its own share (one-device emulation of a rank, for tests).  world = 1
 *     with an id makes a one-rank communicator: every force phase still runs
 *     its all-gathers (trivially), which exercises the NCCL path on one GPU.
 * NCCL is loaded at run time (libnccl.so.2). */
int next_dist_unique_id(unsigned char* id128);
int next_dist_attach(next_handle* h, int rank, int world, const unsigned char* id128);

/* Page-locked host memory for body arrays, so uploads and downloads run at
 * full PCIe/C2C bandwidth.  Free with next_host_free. */
void* next_host_alloc(int64_t bytes);
void next_host_free(void* p);

/* Kernels this library has launched in this process (graph replays count
 * every kernel node of the graph). */
int64_t next_kernel_launches(void);

#ifdef __cplusplus
}
#endif

#endif /* NEXT_GPU_H */
