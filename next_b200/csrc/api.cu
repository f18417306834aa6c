// Host runtime and C ABI of libnext_b200.so (see include/next_gpu.h).
//
// A handle owns one CUDA stream and all device memory of one simulation:
// two ping-pong copies of the body SoA (working order = key order of the
// last build), keys, sort scratch, the tree, and small scalars.  A KDK step
// (src/gravity/step.h:111-189) is
//     [forces at x_n]        -- skipped when reuse_forces and still valid
//     kick + drift           -- v += a dt/2 ; x += v dt
//     forces at x_{n+1}      -- root cubes, keys, sort, reorder, tree, walk
//     kick                   -- v += a dt/2
// A tree/stack capacity overflow raises a device error bit; every later
// kernel of the step then does nothing but permute bodies, so the host grows
// the capacity and re-runs only the force phase and the closing kick.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "common.cuh"
#include "dist.cuh"
#include "kernels.cuh"

using namespace nb;

#include <atomic>

namespace nb {
static std::atomic<int64_t> g_launches{0};
void count_launches(int k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
int64_t launches_so_far() { return g_launches.load(std::memory_order_relaxed); }
}  // namespace nb

namespace {

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    return cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * count);
}

template <typename T>
void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

struct BodyBuf {
    Bodies b{};
    void alloc_all(int64_t n, cudaError_t& e) {
        auto A = [&](auto** p, size_t c) { if (e == cudaSuccess) e = dalloc(p, c); };
        A(&b.x, n); A(&b.y, n); A(&b.z, n); A(&b.vx, n); A(&b.vy, n); A(&b.vz, n); A(&b.m, n);
        A(&b.type, n); A(&b.id, n);
    }
    void free_all() {
        dfree(b.x); dfree(b.y); dfree(b.z); dfree(b.vx); dfree(b.vy); dfree(b.vz); dfree(b.m);
        dfree(b.type); dfree(b.id);
    }
};

constexpr int kReduceMax = 1024;

}  // namespace

struct next_handle {
    next_params prm{};
    Params P{};
    int device = 0;
    int sm_count = 148;
    cudaStream_t st = nullptr;
    std::string last_error;

    // bodies
    int64_t n = 0, cap_n = 0;
    int nsys = 0;
    std::vector<int64_t> offsets_h;
    Systems sys{};
    BodyBuf buf[2];
    int cur = 0;                      // buf[cur] holds the working state
    double *ax = nullptr, *ay = nullptr, *az = nullptr, *pot = nullptr;
    uint64_t *keys = nullptr, *keys_alt = nullptr;
    uint32_t *idx = nullptr, *idx_alt = nullptr;
    uint32_t* inv = nullptr;
    int32_t* sysid = nullptr;
    int64_t* d_offsets = nullptr;
    double4* cubes = nullptr;
    uint32_t* sort_scratch = nullptr;
    size_t sort_words = 0;
    double* stage = nullptr;          // 7 x n staging lanes (upload) / up to 10 x n (download)
    cudaStream_t st_out = nullptr;    // host copies that overlap the force phase (next_step_host)
    cudaEvent_t ev_out = nullptr;
    // next_step_host's uploads and exports in caller order, two sets used by
    // turns: a call's inputs are checked against the previous call's set
    double* io_in[2] = {nullptr, nullptr};    // 7 x n: x y z vx vy vz m as uploaded
    int* io_type[2] = {nullptr, nullptr};
    double* io_out[2] = {nullptr, nullptr};   // 6 x n: x y z vx vy vz as returned
    int64_t io_n = 0;
    int io_cur = 0;                           // the set of the last completed call
    bool io_ready = false;                    // the held state is what that call returned
    cudaStream_t st_in = nullptr;             // the upload of a speculative call
    cudaEvent_t ev_in_pos = nullptr;          // ... its positions have landed
    cudaEvent_t ev_in_vel = nullptr;          // ... its velocities have landed
    int* io_flag = nullptr;
    int* stype = nullptr;

    // tree
    Tree t{};
    void* scan_tmp = nullptr;
    int64_t scan_tmp_elems = 0;

    // small device scalars
    int* err = nullptr;
    unsigned long long* stats = nullptr;   // pp, pc, max stack, spare
    unsigned int* queue = nullptr;
    unsigned int* tickets = nullptr;       // 0: cubes, 1: dt, 2: diagnostics
    double* partial = nullptr;             // kReduceMax * 8
    double* dts = nullptr;                 // dt, dt/2
    double* dt_out = nullptr;              // adaptive dt, half
    double* diag = nullptr;                // 8
    int* changed = nullptr;
    float* fma_out = nullptr;
    unsigned int* done = nullptr;          // closing kicks completed by graph replays (next_steps)

    // pinned host scalars
    double* h_dts = nullptr;
    int* h_err = nullptr;
    int* h_flags = nullptr;                // upload check: changed, non-finite, negative mass
    int64_t* h_counts = nullptr;           // internal, nodes, groups
    unsigned long long* h_stats = nullptr;
    unsigned int* h_done = nullptr;

    // direct summation scratch
    int64_t* d_targets = nullptr;
    int64_t* d_targetpos = nullptr;
    double* d_direct_partial = nullptr;
    double* d_direct_out = nullptr;
    int64_t direct_cap = 0;
    int direct_slice_cap = 0;

    // L2 flush buffer
    void* flush = nullptr;
    size_t flush_bytes = 0;

    // state
    bool have_bodies = false;
    bool forces_valid = false;
    // octant levels held in the keys: the full 21 by default; the FP32-mixed
    // walk of accurate physics trims them to at least the measured tree depth
    // + 2, filling whole sort digits, once per uploaded state (fewer FP64 key
    // levels, fewer sort passes)
    int sys_bits = 0;                 // bits of the system number above the octant digits
    int key_bits = 63;                // sorted key bits
    bool depth_decided = false;
    bool cube_fresh = false;          // the last kick-drift wrote the root cube (one system)
    int64_t builds = 0;               // tree builds enqueued
    int64_t depth_seen = 0;           // the build whose depth report was last acted on
    bool pot_valid = false;
    bool sorted_in_alt = false;
    int64_t recoveries = 0;           // graph replays that overflowed and were finished eagerly
    bool fixed_tree_cap = false;      // test support: grow the tree only on overflow

    // sharding over ranks: every rank holds all bodies, computes the forces of
    // its share [rank*chunk, (rank+1)*chunk) and all-gathers the rest
    int world = 1, rank = 0;
    void* comm = nullptr;

    // graphs: one captured KDK step per buffer parity
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int64_t graph_kernels[2] = {0, 0};
    // next_step_host: force phase + closing kick per buffer parity (its
    // kick-drift and position export run eagerly in front of the replay)
    cudaGraphExec_t fgraph[2] = {nullptr, nullptr};
    int64_t fgraph_kernels[2] = {0, 0};
    // events recorded inside each graph (build start, after keys, after sort,
    // after build, after walk) so a timed replay reports its stages
    std::vector<cudaEvent_t> graph_ev[2];
    std::vector<cudaEvent_t> cap_events;
    bool capturing = false;

    // timing
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::vector<std::vector<int>> ev_steps;   // per timed step: event indices
    double acc_step = 0, acc_build = 0, acc_walk = 0, acc_sort = 0, acc_other = 0;
    int64_t timed_steps = 0, timed_walks = 0;

    Bodies cur_bodies() const {
        Bodies b = buf[cur].b;
        b.ax = ax; b.ay = ay; b.az = az; b.pot = pot;
        return b;
    }
};

namespace {

int fail(next_handle* h, int code, const std::string& msg) {
    if (h) h->last_error = msg;
    return code;
}

int cuda_fail(next_handle* h, cudaError_t e, const char* where) {
    return fail(h, e == cudaErrorMemoryAllocation ? NEXT_ERR_OUT_OF_MEMORY : NEXT_ERR_CUDA,
                std::string(where) + ": " + cudaGetErrorString(e));
}

#define NB_TRY(expr, where)                                   \
    do {                                                      \
        cudaError_t e__ = (expr);                             \
        if (e__ != cudaSuccess) return cuda_fail(h, e__, where); \
    } while (0)

void free_tree(next_handle* h) {
    Tree& t = h->t;
    dfree(t.dlev); dfree(t.nint); dfree(t.int_start); dfree(t.int_level); dfree(t.int_bounds);
    dfree(t.int_packed); dfree(t.int_node); dfree(t.counter); dfree(t.climb); dfree(t.ready); dfree(t.link); dfree(t.parent); dfree(t.level);
    dfree(t.com); dfree(t.quad64); dfree(t.box); dfree(t.quad32); dfree(t.groups);
    dfree(h->scan_tmp);
    t.cap_int = t.cap_node = t.cap_group = 0;
}

void drop_graphs(next_handle* h) {
    for (int p = 0; p < 2; ++p) {
        if (h->graph[p]) { cudaGraphExecDestroy(h->graph[p]); h->graph[p] = nullptr; }
        if (h->fgraph[p]) { cudaGraphExecDestroy(h->fgraph[p]); h->fgraph[p] = nullptr; }
        for (cudaEvent_t ev : h->graph_ev[p]) cudaEventDestroy(ev);
        h->graph_ev[p].clear();
    }
}

int alloc_tree(next_handle* h, int64_t cap_int) {
    drop_graphs(h);
    free_tree(h);
    Tree& t = h->t;
    const int64_t n = h->cap_n;
    t.cap_int = cap_int;
    t.cap_node = std::min<int64_t>(8 * cap_int, cap_int + n) + h->nsys + 64;
    t.cap_group = n + h->nsys + 64;
    cudaError_t e = cudaSuccess;
    auto A = [&](auto** p, size_t c) { if (e == cudaSuccess) e = dalloc(p, c); };
    A(&t.dlev, n + 1); A(&t.nint, n + 1);
    A(&t.int_start, cap_int); A(&t.int_level, cap_int); A(&t.int_bounds, 9 * cap_int);
    A(&t.int_packed, cap_int + 1); A(&t.int_node, cap_int); A(&t.counter, cap_int); A(&t.climb, cap_int);
    A(&t.ready, cap_int);
    A(&t.link, t.cap_node); A(&t.parent, t.cap_node); A(&t.level, t.cap_node);
    A(&t.com, t.cap_node); A(&t.quad64, 8 * t.cap_node);
    if (h->P.physics == NEXT_PHYSICS_ACCURATE) { A(&t.box, t.cap_node); A(&t.quad32, 2 * t.cap_node); }
    A(&t.groups, t.cap_group);
    h->scan_tmp_elems = scan_tile_sums_needed(std::max<int64_t>(n + 1, cap_int + 1));
    int64_t* st64 = nullptr;
    A(&st64, h->scan_tmp_elems);
    h->scan_tmp = st64;
    if (e != cudaSuccess) return cuda_fail(h, e, "tree allocation");
    NB_TRY(cudaMemsetAsync(t.counter, 0, sizeof(int32_t) * cap_int, h->st), "tree counters");
    NB_TRY(cudaMemsetAsync(t.link, 0, sizeof(int2) * t.cap_node, h->st), "tree links");
    return NEXT_OK;
}

int64_t initial_cap_int(const next_handle* h) {
    const int leaf = h->P.physics == NEXT_PHYSICS_REFERENCE ? 1 : std::max(1, h->P.leaf_cap);
    return h->cap_n / leaf + h->cap_n / (4 * leaf) + 1024;
}

// This rank's share of the bodies (working positions) for the force walk.
void set_share(next_handle* h) {
    if (h->world <= 1) {
        h->P.own_lo = 0;
        h->P.own_hi = INT64_MAX;
        return;
    }
    const int64_t chunk = (h->n + h->world - 1) / h->world;
    h->P.own_lo = std::min<int64_t>(h->n, h->rank * chunk);
    h->P.own_hi = std::min<int64_t>(h->n, h->P.own_lo + chunk);
}

void free_bodies(next_handle* h) {
    drop_graphs(h);
    for (auto& b : h->buf) b.free_all();
    dfree(h->ax); dfree(h->ay); dfree(h->az); dfree(h->pot);
    dfree(h->keys); dfree(h->keys_alt); dfree(h->idx); dfree(h->idx_alt); dfree(h->inv);
    dfree(h->sysid); dfree(h->d_offsets); dfree(h->cubes); dfree(h->sort_scratch);
    dfree(h->stage); dfree(h->stype);
    free_tree(h);
    h->cap_n = 0;
}

int alloc_bodies(next_handle* h, int64_t n) {
    free_bodies(h);
    h->cap_n = n;
    cudaError_t e = cudaSuccess;
    h->buf[0].alloc_all(n, e);
    h->buf[1].alloc_all(n, e);
    auto A = [&](auto** p, size_t c) { if (e == cudaSuccess) e = dalloc(p, c); };
    const int64_t padded = ((n + h->world - 1) / h->world) * h->world;   // world equal shares
    A(&h->ax, padded); A(&h->ay, padded); A(&h->az, padded); A(&h->pot, padded);
    A(&h->keys, n); A(&h->keys_alt, n); A(&h->idx, n); A(&h->idx_alt, n); A(&h->inv, n);
    A(&h->sysid, n); A(&h->d_offsets, h->nsys + 1); A(&h->cubes, h->nsys);
    h->sort_words = sort_scratch_words(n);
    A(&h->sort_scratch, h->sort_words);
    A(&h->stage, 10 * n); A(&h->stype, n);
    if (e != cudaSuccess) return cuda_fail(h, e, "body allocation");
    return alloc_tree(h, initial_cap_int(h));
}


// ---- the force phase -------------------------------------------------------

int record(next_handle* h, std::vector<int>* evs) {
    if (!evs) return NEXT_OK;
    if (h->capturing) {
        // inside a capture: a dedicated event becomes an event-record node of
        // the graph (External, so replays really record it)
        cudaEvent_t ev;
        NB_TRY(cudaEventCreate(&ev), "event create");
        NB_TRY(cudaEventRecordWithFlags(ev, h->st, cudaEventRecordExternal), "event record");
        h->cap_events.push_back(ev);
        return NEXT_OK;
    }
    if (h->ev_used >= h->ev_pool.size()) {
        cudaEvent_t ev;
        NB_TRY(cudaEventCreate(&ev), "event create");
        h->ev_pool.push_back(ev);
    }
    NB_TRY(cudaEventRecord(h->ev_pool[h->ev_used], h->st), "event record");
    evs->push_back(static_cast<int>(h->ev_used++));
    return NEXT_OK;
}

// Root cubes, keys, sort, reorder, tree, moments (no walk).
int build(next_handle* h, std::vector<int>* evs) {
    const int64_t n = h->n;
    Bodies src = h->cur_bodies();
    int rc0 = record(h, evs);
    if (rc0) return rc0;
    ++h->builds;
    if (!h->cube_fresh)
        NB_TRY(launch_root_cubes(src, n, h->sys, h->d_offsets, h->partial, kReduceMax, h->tickets + 0, h->st),
               "root cube");
    h->cube_fresh = false;
    NB_TRY(launch_keys(src, h->sysid, n, h->sys, h->keys, h->idx, h->st), "keys");
    rc0 = record(h, evs);
    if (rc0) return rc0;
    bool in_alt = false;
    NB_TRY(radix_sort_pairs(h->keys, h->idx, h->keys_alt, h->idx_alt, n, h->key_bits, h->sort_scratch, h->err, &in_alt,
                            h->st),
           "radix sort");
    h->sorted_in_alt = in_alt;
    int rc = record(h, evs);
    if (rc) return rc;
    const uint64_t* skeys = in_alt ? h->keys_alt : h->keys;
    const uint32_t* sidx = in_alt ? h->idx_alt : h->idx;
    const int other = 1 - h->cur;
    Bodies dst = h->buf[other].b;
    NB_TRY(launch_gather_bodies(h->buf[h->cur].b, dst, sidx, n, h->inv, h->err, h->st), "reorder");
    h->cur = other;
    Bodies bd = h->cur_bodies();
    NB_TRY(build_tree(skeys, n, bd, h->sysid, h->sys, h->d_offsets, h->P, h->t, h->scan_tmp, h->err, h->st),
           "tree build");
    h->forces_valid = false;
    return record(h, evs);
}

// The warp-per-group walk (FP32-mixed or FP64 arithmetic) with its leaf
// buckets, trimmed keys, force reuse, graph replays and autotuner.
bool group_walk(const next_handle* h) {
    return h->prm.precision == NEXT_PRECISION_MIXED || h->prm.precision == NEXT_PRECISION_FP64_GROUP;
}

int walk(next_handle* h, bool potential) {
    Bodies bd = h->cur_bodies();
    if (group_walk(h)) {
        NB_TRY(launch_walk_group(bd, h->n, h->t, h->P, potential, h->prm.precision == NEXT_PRECISION_FP64_GROUP,
                                 h->prm.walk_warps, h->prm.walk_stack, h->queue, h->stats, h->err, h->sm_count, h->st),
               "group walk");
    } else {
        NB_TRY(launch_walk_plain(bd, h->sysid, h->n, h->t, h->P, h->nsys > 1, h->stats, h->err, h->st), "plain walk");
    }
    return NEXT_OK;
}

int exchange_forces(next_handle* h, bool potential) {
    if (!h->comm) return NEXT_OK;   // one rank with a communicator still runs the (trivial) all-gather
    const size_t chunk = static_cast<size_t>((h->n + h->world - 1) / h->world);
    double* lanes[4] = {h->ax, h->ay, h->az, h->pot};
    std::string why;
    for (int c = 0; c < (potential ? 4 : 3); ++c)
        if (!nccl_allgather_inplace(h->comm, lanes[c], chunk, h->rank, h->st, &why))
            return fail(h, NEXT_ERR_CUDA, why);
    count_launches(potential ? 4 : 3);
    return NEXT_OK;
}

int forces(next_handle* h, bool potential, std::vector<int>* evs) {
    int rc = build(h, evs);
    if (rc) return rc;
    rc = walk(h, potential);
    if (rc) return rc;
    rc = exchange_forces(h, potential);
    if (rc) return rc;
    h->forces_valid = true;
    h->pot_valid = potential;
    return record(h, evs);
}

// Octant levels of the keys (and the key layout that goes with them): the
// full depth keeps the upload layout (system number from bit 63 - sys_bits
// down), a trimmed depth packs the digits at the bottom.
void set_key_levels(next_handle* h, int levels) {
    Systems& S = h->sys;
    const int full = std::min(kMaxLevel, (63 - h->sys_bits) / 3);
    levels = std::max(1, std::min(levels, full));
    const int base = levels == full ? 63 - h->sys_bits : 3 * levels;
    if (S.levels != levels || S.base != base) drop_graphs(h);
    S.levels = levels;
    S.base = base;
    h->key_bits = base + h->sys_bits;
}

#ifndef NB_KEY_MARGIN
#define NB_KEY_MARGIN 2
#endif
// Key levels kept once the tree depth is known: at least two below the
// deepest leaf level, and as many more as fill the 8-bit sort digits those
// need (whole passes either way, so the extra levels cost nothing): 1 M-body
// uniform sphere 10 levels (4 passes), 16.7 M-body halo 18 (7 passes).
int trimmed_levels(const next_handle* h, int64_t deepest) {
    const int need = h->sys_bits + 3 * (static_cast<int>(deepest) + NB_KEY_MARGIN);
    const int bits = 8 * ((need + 7) / 8);
    return (bits - h->sys_bits) / 3;
}

bool adaptive_depth(const next_handle* h) {
    return group_walk(h) && h->P.physics == NEXT_PHYSICS_ACCURATE;
}

int read_device_error(next_handle* h, int* bits) {
    NB_TRY(cudaMemcpyAsync(h->h_err, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->st), "error word");
    NB_TRY(cudaMemcpyAsync(h->h_counts, h->t.counts, sizeof(int64_t) * 4, cudaMemcpyDeviceToHost, h->st), "counts");
    NB_TRY(cudaMemcpyAsync(h->h_stats, h->stats, sizeof(unsigned long long) * 4, cudaMemcpyDeviceToHost, h->st), "stats");
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    *bits = *h->h_err;
    // the first build after an upload measured the tree depth: later builds
    // keep three levels of margin below it.  A tree that outgrows them gets
    // leaves of more than leaf_cap bodies at the last level (still exact,
    // slower): seen here, the keys get three more levels.
    const int64_t deepest = h->h_counts[3];
    if (h->depth_seen == h->builds) return NEXT_OK;   // no build since the last look
    h->depth_seen = h->builds;
    if (*bits == 0 && deepest > 0 && adaptive_depth(h)) {
        if (!h->depth_decided) {
            const int keep = trimmed_levels(h, deepest);
            if (keep < h->sys.levels) set_key_levels(h, keep);
        } else if (deepest >= kDepthOverfull) {
            set_key_levels(h, h->sys.levels + 3);
        }
    }
    if (*bits == 0 && deepest > 0) h->depth_decided = true;
    return NEXT_OK;
}

// Grow what overflowed, clear the error word.  Returns NEXT_OK if the step
// can be retried.
int recover(next_handle* h, int bits) {
    if (bits & (kErrSort | kErrList | kErrIndex))
        return fail(h, NEXT_ERR_DEVICE, "device error word " + std::to_string(bits) +
                                            " (sort look-back timeout or failed index check)");
    if (bits & kErrTree) {
        const int64_t need = std::max<int64_t>(h->h_counts[0] + h->h_counts[0] / 2 + 1024, 2 * h->t.cap_int);
        int rc = alloc_tree(h, need);
        if (rc) return rc;
    }
    if (bits & kErrStack) {
        if (h->prm.walk_stack >= (1 << 14)) return fail(h, NEXT_ERR_DEVICE, "walk stack capacity limit reached");
        h->prm.walk_stack *= 2;
        drop_graphs(h);
    }
    NB_TRY(cudaMemsetAsync(h->err, 0, sizeof(int), h->st), "error reset");
    return NEXT_OK;
}

// Force phase with overflow recovery (synchronous).
int forces_checked(next_handle* h, bool potential) {
    for (int attempt = 0; attempt < 8; ++attempt) {
        int rc = forces(h, potential, nullptr);
        if (rc) return rc;
        int bits = 0;
        rc = read_device_error(h, &bits);
        if (rc) return rc;
        if (bits == 0) return NEXT_OK;
        rc = recover(h, bits);
        if (rc) return rc;
    }
    return fail(h, NEXT_ERR_DEVICE, "force phase kept overflowing");
}

int set_dt(next_handle* h, double dt) {
    NB_TRY(launch_set_dt(h->dts, dt, h->st), "dt upload");
    return NEXT_OK;
}

// The opening half-kick and the drift; with one system the same pass boxes
// the new positions, and the next build takes that root cube.
cudaError_t kick_drift_step(next_handle* h, const Bodies& bd) {
    if (h->sys.n != 1) return launch_kick_drift(bd, h->n, h->dts, h->err, h->st);
    const cudaError_t e = launch_kick_drift_box(bd, h->n, h->dts, h->err, h->partial, kReduceMax, h->tickets + 0,
                                                h->sys.cube, h->st);
    h->cube_fresh = e == cudaSuccess;
    return e;
}

// One eager step.  With evs, events bracket the stages for timing.
int step_once(next_handle* h, bool sync_checked) {
    const bool reuse = h->prm.reuse_forces && h->forces_valid;
    std::vector<int> evs;
    std::vector<int>* E = h->timing ? &evs : nullptr;
    int rc = record(h, E);
    if (rc) return rc;
    if (!reuse) {
        rc = sync_checked ? forces_checked(h, false) : forces(h, false, nullptr);
        if (rc) return rc;
    }
    Bodies bd = h->cur_bodies();
    NB_TRY(kick_drift_step(h, bd), "kick-drift");
    rc = forces(h, false, E);
    if (rc) return rc;
    bd = h->cur_bodies();
    NB_TRY(launch_kick(bd, h->n, h->dts, h->err, h->st), "kick");
    rc = record(h, E);
    if (rc) return rc;
    if (E) h->ev_steps.push_back(evs);
    if (!sync_checked) return NEXT_OK;
    int bits = 0;
    rc = read_device_error(h, &bits);
    if (rc) return rc;
    if (bits == 0) return NEXT_OK;
    // the kick-drift ran; redo the force phase and the closing kick
    rc = recover(h, bits);
    if (rc) return rc;
    rc = forces_checked(h, false);
    if (rc) return rc;
    bd = h->cur_bodies();
    NB_TRY(launch_kick(bd, h->n, h->dts, h->err, h->st), "kick");
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    return NEXT_OK;
}

// Capture kick-drift + force phase + kick for the current buffer parity
// (with_kick_drift), or only the force phase + kick into the next_step_host
// graph of that parity.
int capture_graph(next_handle* h, bool with_kick_drift) {
    const int parity = h->cur;
    cudaGraphExec_t* slot = with_kick_drift ? &h->graph[parity] : &h->fgraph[parity];
    if (*slot) return NEXT_OK;
    const bool saved_timing = h->timing;
    h->timing = false;
    const int saved_cur = h->cur;
    cudaGraph_t g = nullptr;
    const int64_t launches_before = launches_so_far();
    const int64_t builds_before = h->builds;   // capturing runs nothing
    NB_TRY(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeRelaxed), "begin capture");
    int rc = NEXT_OK;
    Bodies bd = h->cur_bodies();
    h->capturing = true;
    h->cap_events.clear();
    // stage-timing events only in the next_steps graph
    std::vector<int> unused;
    cudaError_t e = with_kick_drift ? kick_drift_step(h, bd) : cudaSuccess;
    if (e == cudaSuccess) rc = forces(h, false, with_kick_drift ? &unused : nullptr);
    h->capturing = false;
    if (with_kick_drift) h->graph_ev[parity] = h->cap_events;
    h->cap_events.clear();
    if (e == cudaSuccess && rc == NEXT_OK) {
        bd = h->cur_bodies();
        e = launch_kick(bd, h->n, h->dts, h->err, h->st, with_kick_drift ? h->done : nullptr);
    }
    h->builds = builds_before;
    cudaError_t e2 = cudaStreamEndCapture(h->st, &g);
    const int64_t captured = launches_so_far() - launches_before;
    count_launches(static_cast<int>(-captured));   // captured, not launched
    (with_kick_drift ? h->graph_kernels : h->fgraph_kernels)[parity] = captured;
    h->cur = saved_cur;
    h->timing = saved_timing;
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) { if (g) cudaGraphDestroy(g); return cuda_fail(h, e, "capture"); }
    if (e2 != cudaSuccess) return cuda_fail(h, e2, "end capture");
    e = cudaGraphInstantiate(slot, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(h, e, "graph instantiate");
    return NEXT_OK;
}

int check_ready(next_handle* h) {
    if (!h) return NEXT_ERR_INVALID_ARGUMENT;
    if (!h->have_bodies) return fail(h, NEXT_ERR_NO_BODIES, "no bodies uploaded");
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return cuda_fail(h, e, "set device");
    return NEXT_OK;
}

int resolve_timers(next_handle* h) {
    if (h->ev_steps.empty()) return NEXT_OK;
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    for (const auto& ev : h->ev_steps) {
        if (ev.size() != 7) continue;
        auto el = [&](int a, int b) {
            float v = 0.f;
            cudaEventElapsedTime(&v, h->ev_pool[ev[a]], h->ev_pool[ev[b]]);
            return static_cast<double>(v);
        };
        const double step = el(0, 6), build = el(1, 4), walkms = el(4, 5), sortms = el(2, 3);
        h->acc_step += step;
        h->acc_build += build;
        h->acc_walk += walkms;
        h->acc_sort += sortms;
        h->acc_other += step - build - walkms;
        h->timed_steps += 1;
        h->timed_walks += 1;
    }
    h->ev_steps.clear();
    h->ev_used = 0;
    return NEXT_OK;
}

// One timed graph replay: step = the events around the launch; stages from
// the events recorded inside the graph.
int add_graph_timing(next_handle* h, int parity, const std::vector<int>& evs) {
    const std::vector<cudaEvent_t>& g = h->graph_ev[parity];
    if (evs.size() != 2 || g.size() != 5) return NEXT_OK;
    bool ok = true;
    auto el = [&ok](cudaEvent_t a, cudaEvent_t b) {
        float v = 0.f;
        if (cudaEventElapsedTime(&v, a, b) != cudaSuccess) ok = false;
        return static_cast<double>(v);
    };
    const double step = el(h->ev_pool[evs[0]], h->ev_pool[evs[1]]);
    const double build = el(g[0], g[3]), walkms = el(g[3], g[4]), sortms = el(g[1], g[2]);
    if (!ok) {
        cudaGetLastError();   // do not let a timing failure surface as a later launch error
        return fail(h, NEXT_ERR_CUDA, "stage timing of a graph replay failed");
    }
    h->acc_step += step;
    h->acc_build += build;
    h->acc_walk += walkms;
    h->acc_sort += sortms;
    h->acc_other += step - build - walkms;
    h->timed_steps += 1;
    h->timed_walks += 1;
    h->ev_used = 0;
    return NEXT_OK;
}

// Grow capacities that the last build came close to (before a graph capture).
int grow_if_tight(next_handle* h) {
    const int64_t internal = h->h_counts[0], nodes = h->h_counts[1];
    if (!h->fixed_tree_cap && (4 * internal > 3 * h->t.cap_int || 4 * nodes > 3 * h->t.cap_node)) {
        int rc = alloc_tree(h, std::max<int64_t>(2 * internal + 1024, h->t.cap_int));
        if (rc) return rc;
        h->forces_valid = false;
    }
    if (group_walk(h) && 4 * static_cast<int64_t>(h->h_stats[2]) > 3 * h->prm.walk_stack &&
        h->prm.walk_stack < (1 << 14)) {
        h->prm.walk_stack *= 2;
        drop_graphs(h);
    }
    return NEXT_OK;
}

}  // namespace

// ============================================================================
extern "C" {

const char* next_status_string(int s) {
    switch (s) {
        case NEXT_OK: return "ok";
        case NEXT_ERR_INVALID_ARGUMENT: return "invalid argument";
        case NEXT_ERR_CUDA: return "CUDA error";
        case NEXT_ERR_OUT_OF_MEMORY: return "out of device memory";
        case NEXT_ERR_NO_BODIES: return "no bodies uploaded";
        case NEXT_ERR_DEVICE: return "device error";
        default: return "unknown status";
    }
}

const char* next_last_error(const next_handle* h) { return h ? h->last_error.c_str() : "null handle"; }

int next_params_default(next_params* p, int physics, int precision) {
    if (!p) return NEXT_ERR_INVALID_ARGUMENT;
    std::memset(p, 0, sizeof(*p));
    p->physics = physics;
    p->precision = precision;
    p->theta = 0.5;
    p->eps = physics == NEXT_PHYSICS_REFERENCE ? 0.0 : 0.01;
    p->G = 1.0;
    const bool grouped = precision == NEXT_PRECISION_MIXED || precision == NEXT_PRECISION_FP64_GROUP;
    p->leaf_cap = physics == NEXT_PHYSICS_REFERENCE ? 1 : (grouped ? 16 : 1);
    p->group_cap = 32;
    p->quadrupole = 1;
    p->reuse_forces = grouped ? 1 : 0;
    p->walk_warps = 4;
    p->walk_stack = 1024;
    p->device = 0;
    return NEXT_OK;
}

int next_create(const next_params* p, next_handle** out) {
    if (!p || !out) return NEXT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    const bool grouped = p->precision == NEXT_PRECISION_MIXED || p->precision == NEXT_PRECISION_FP64_GROUP;
    if ((p->physics != NEXT_PHYSICS_REFERENCE && p->physics != NEXT_PHYSICS_ACCURATE) ||
        (p->precision != NEXT_PRECISION_FP64 && !grouped) ||
        (grouped && p->physics != NEXT_PHYSICS_ACCURATE) || !(p->theta > 0.0) ||
        !(p->eps >= 0.0) || !std::isfinite(p->eps) || !std::isfinite(p->G) || p->leaf_cap < 1 || p->leaf_cap > 64 ||
        p->group_cap < 1 || p->group_cap > 32 || p->walk_warps < 1 || p->walk_warps > 4 || p->walk_stack < 64 ||
        p->walk_stack > (1 << 14) ||
        (grouped && p->leaf_cap > p->group_cap))
        return NEXT_ERR_INVALID_ARGUMENT;
    next_handle* h = new (std::nothrow) next_handle();
    if (!h) return NEXT_ERR_OUT_OF_MEMORY;
    h->prm = *p;
    h->P.physics = p->physics;
    h->P.theta = p->theta;
    h->P.eps = p->physics == NEXT_PHYSICS_REFERENCE ? 0.0 : p->eps;
    h->P.G = p->physics == NEXT_PHYSICS_REFERENCE ? 1.0 : p->G;
    h->P.leaf_cap = p->physics == NEXT_PHYSICS_REFERENCE ? 1 : p->leaf_cap;
    h->P.group_cap = p->group_cap;
    h->P.quad = p->quadrupole ? 1 : 0;
    h->device = p->device;
    auto bail = [&](cudaError_t e, const char* w) {
        int rc = cuda_fail(h, e, w);
        next_destroy(h);
        return rc;
    };
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return bail(e, "set device");
    e = cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, h->device);
    if (e != cudaSuccess) return bail(e, "device attribute");
    e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(e, "stream");
    e = sort_prepare();
    if (e != cudaSuccess) return bail(e, "sort setup");
    auto A = [&](auto** q, size_t c) { if (e == cudaSuccess) e = dalloc(q, c); };
    A(&h->err, 1); A(&h->stats, 4); A(&h->queue, 1); A(&h->tickets, 4); A(&h->partial, kReduceMax * 8);
    A(&h->dts, 2); A(&h->dt_out, 2); A(&h->diag, 8); A(&h->changed, 4); A(&h->fma_out, 1);
    A(&h->t.counts, 6); A(&h->done, 1);
    if (e != cudaSuccess) return bail(e, "scalars");
    e = cudaMemset(h->err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(h->tickets, 0, sizeof(unsigned int) * 4);
    if (e == cudaSuccess) e = cudaMemset(h->stats, 0, sizeof(unsigned long long) * 4);
    if (e == cudaSuccess) e = cudaMemset(h->t.counts, 0, sizeof(int64_t) * 6);
    if (e == cudaSuccess) e = cudaMemset(h->done, 0, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&h->h_dts), sizeof(double) * 2, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&h->h_err), sizeof(int) * 2, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&h->h_flags), sizeof(int) * 4, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&h->h_counts), sizeof(int64_t) * 4, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&h->h_stats), sizeof(unsigned long long) * 4, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&h->h_done), sizeof(unsigned int), cudaHostAllocDefault);
    if (e != cudaSuccess) return bail(e, "pinned scalars");
    *out = h;
    return NEXT_OK;
}

void next_destroy(next_handle* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->st) cudaStreamSynchronize(h->st);
    if (h->st_in) cudaStreamSynchronize(h->st_in);
    for (int k = 0; k < 2; ++k) { dfree(h->io_in[k]); dfree(h->io_type[k]); dfree(h->io_out[k]); }
    dfree(h->io_flag);
    if (h->ev_in_pos) cudaEventDestroy(h->ev_in_pos);
    if (h->ev_in_vel) cudaEventDestroy(h->ev_in_vel);
    if (h->st_in) cudaStreamDestroy(h->st_in);
    drop_graphs(h);
    nccl_comm_destroy(h->comm);
    h->comm = nullptr;
    free_bodies(h);
    dfree(h->err); dfree(h->stats); dfree(h->queue); dfree(h->tickets); dfree(h->partial);
    dfree(h->dts); dfree(h->dt_out); dfree(h->diag); dfree(h->changed); dfree(h->fma_out); dfree(h->t.counts);
    dfree(h->done);
    dfree(h->d_targets); dfree(h->d_targetpos); dfree(h->d_direct_partial); dfree(h->d_direct_out);
    if (h->flush) cudaFree(h->flush);
    for (auto ev : h->ev_pool) cudaEventDestroy(ev);
    if (h->h_dts) cudaFreeHost(h->h_dts);
    if (h->h_err) cudaFreeHost(h->h_err);
    if (h->h_flags) cudaFreeHost(h->h_flags);
    if (h->h_counts) cudaFreeHost(h->h_counts);
    if (h->h_stats) cudaFreeHost(h->h_stats);
    if (h->h_done) cudaFreeHost(h->h_done);
    if (h->ev_out) cudaEventDestroy(h->ev_out);
    if (h->st_out) cudaStreamDestroy(h->st_out);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
}

// The upload behind next_upload_systems, staged through `stage_override`
// (7 x n doubles) and `stype_override` (n ints), or the handle's staging area.
static int upload_staged(next_handle* h, int64_t n_systems, const int64_t* offsets, const double* x, const double* y,
                  const double* z, const double* vx, const double* vy, const double* vz, const double* m,
                  const int* type, double* stage_override, int* stype_override) {
    if (n_systems < 1 || n_systems > (1 << 20) || !offsets)
        return fail(h, NEXT_ERR_INVALID_ARGUMENT, "n_systems must be in [1, 2^20] with offsets");
    if (offsets[0] != 0) return fail(h, NEXT_ERR_INVALID_ARGUMENT, "offsets[0] must be 0");
    for (int64_t s = 0; s < n_systems; ++s)
        if (offsets[s + 1] < offsets[s]) return fail(h, NEXT_ERR_INVALID_ARGUMENT, "offsets must not decrease");
    const int64_t n = offsets[n_systems];
    if (n < 1 || n >= (int64_t(1) << 30))
        return fail(h, NEXT_ERR_INVALID_ARGUMENT, "body count must be in [1, 2^30)");
    if (!x || !y || !z || !vx || !vy || !vz || !m) return fail(h, NEXT_ERR_INVALID_ARGUMENT, "NULL body array");
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return cuda_fail(h, e, "set device");
    const bool same_layout = h->have_bodies && h->n == n && h->nsys == n_systems &&
                             std::equal(offsets, offsets + n_systems + 1, h->offsets_h.begin());
    if (!same_layout) {
        h->have_bodies = false;
        h->forces_valid = false;
        h->nsys = static_cast<int>(n_systems);
        h->offsets_h.assign(offsets, offsets + n_systems + 1);
        int rc = alloc_bodies(h, n);
        if (rc) return rc;
        h->n = n;
        Systems& S = h->sys;
        S.n = h->nsys;
        int bits = 0;
        while (h->nsys > 1 && (int64_t(1) << bits) < n_systems) ++bits;
        h->sys_bits = bits;
        S.levels = 0;
        set_key_levels(h, kMaxLevel);
        h->depth_decided = false;
        S.offsets = h->d_offsets;
        S.cube = h->cubes;
        set_share(h);
        NB_TRY(cudaMemcpyAsync(h->d_offsets, offsets, sizeof(int64_t) * (n_systems + 1), cudaMemcpyHostToDevice, h->st),
               "offsets");
        std::vector<int32_t> sid(n);
        for (int64_t s = 0; s < n_systems; ++s)
            for (int64_t i = offsets[s]; i < offsets[s + 1]; ++i) sid[i] = static_cast<int32_t>(s);
        NB_TRY(cudaMemcpyAsync(h->sysid, sid.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, h->st), "system ids");
        NB_TRY(cudaStreamSynchronize(h->st), "sync");
    }
    h->cube_fresh = false;
    double* stage = stage_override ? stage_override : h->stage;
    int* stype = stype_override ? stype_override : h->stype;
    const double* lanes[7] = {x, y, z, vx, vy, vz, m};
    for (int c = 0; c < 7; ++c)
        NB_TRY(cudaMemcpyAsync(stage + c * n, lanes[c], sizeof(double) * n, cudaMemcpyHostToDevice, h->st), "upload");
    if (type) {
        NB_TRY(cudaMemcpyAsync(stype, type, sizeof(int) * n, cudaMemcpyHostToDevice, h->st), "upload types");
    } else {
        NB_TRY(cudaMemsetAsync(stype, 0, sizeof(int) * n, h->st), "types");
    }
    // validate on the device (finite values, m >= 0) and, for the same layout,
    // find out whether positions/masses/types changed; the held bodies are
    // only touched once the staged data passed
    Bodies b = h->cur_bodies();
    NB_TRY(cudaMemsetAsync(h->changed, 0, sizeof(int) * 3, h->st), "upload flags");
    NB_TRY(launch_check_upload(stage, stype, b, h->inv, n, same_layout, h->changed, h->st), "upload check");
    NB_TRY(cudaMemcpyAsync(h->h_flags, h->changed, sizeof(int) * 3, cudaMemcpyDeviceToHost, h->st), "upload flags");
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    if (h->h_flags[1]) return fail(h, NEXT_ERR_INVALID_ARGUMENT, "non-finite body data");
    if (h->h_flags[2]) return fail(h, NEXT_ERR_INVALID_ARGUMENT, "negative mass");
    if (same_layout && h->h_flags[0] == 0) {
        NB_TRY(launch_load_velocities(stage, b, h->inv, n, h->st), "velocities");
        return NEXT_OK;   // same positions: tree order and cached forces stay valid
    }
    NB_TRY(launch_load_all(stage, stype, b, h->inv, n, h->st), "load");
    h->forces_valid = false;
    h->have_bodies = true;
    set_key_levels(h, kMaxLevel);     // new positions: measure the depth again
    h->depth_decided = false;
    return NEXT_OK;
}

int next_upload_systems(next_handle* h, int64_t n_systems, const int64_t* offsets, const double* x, const double* y,
                        const double* z, const double* vx, const double* vy, const double* vz, const double* m,
                        const int* type) {
    if (!h) return NEXT_ERR_INVALID_ARGUMENT;
    h->io_ready = false;
    return upload_staged(h, n_systems, offsets, x, y, z, vx, vy, vz, m, type, nullptr, nullptr);
}

int next_upload(next_handle* h, int64_t n, const double* x, const double* y, const double* z, const double* vx,
                const double* vy, const double* vz, const double* m, const int* type) {
    const int64_t offs[2] = {0, n};
    return next_upload_systems(h, 1, offs, x, y, z, vx, vy, vz, m, type);
}

int next_download(next_handle* h, double* x, double* y, double* z, double* vx, double* vy, double* vz) {
    int rc = check_ready(h);
    if (rc) return rc;
    const Bodies b = h->cur_bodies();
    const double* src[6] = {b.x, b.y, b.z, b.vx, b.vy, b.vz};
    double* dst[6] = {x, y, z, vx, vy, vz};
    const double* lanes[6];
    double* outs[6];
    int cnt = 0;
    for (int c = 0; c < 6; ++c)
        if (dst[c]) { lanes[cnt] = src[c]; outs[cnt] = dst[c]; ++cnt; }
    if (cnt == 0) return NEXT_OK;
    NB_TRY(launch_gather_out(lanes, cnt, h->inv, h->n, h->stage, h->st), "gather out");
    for (int c = 0; c < cnt; ++c)
        NB_TRY(cudaMemcpyAsync(outs[c], h->stage + c * h->n, sizeof(double) * h->n, cudaMemcpyDeviceToHost, h->st),
               "download");
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    return NEXT_OK;
}

int next_step(next_handle* h, double dt) {
    int rc = check_ready(h);
    if (rc) return rc;
    h->io_ready = false;
    if (!std::isfinite(dt)) return fail(h, NEXT_ERR_INVALID_ARGUMENT, "dt must be finite");
    rc = set_dt(h, dt);
    if (rc) return rc;
    return step_once(h, !h->timing);
}

// Gather lanes of the working state into caller order at `out` (device) and
// queue their device -> host copies on stream cs.
static int export_lanes(next_handle* h, const double* const* src, double* const* dst, int cnt, double* out,
                        cudaStream_t cs) {
    NB_TRY(launch_gather_out(src, cnt, h->inv, h->n, out, h->st), "gather out");
    if (cs != h->st) {
        NB_TRY(cudaEventRecord(h->ev_out, h->st), "export event");
        NB_TRY(cudaStreamWaitEvent(cs, h->ev_out, 0), "export wait");
    }
    for (int c = 0; c < cnt; ++c)
        NB_TRY(cudaMemcpyAsync(dst[c], out + static_cast<int64_t>(c) * h->n, sizeof(double) * h->n,
                               cudaMemcpyDeviceToHost, cs), "download");
    return NEXT_OK;
}

// Streams, events and the two caller-order buffer sets of next_step_host.
static int ensure_host_io(next_handle* h, int64_t n) {
    if (!h->st_out) {
        NB_TRY(cudaStreamCreateWithFlags(&h->st_out, cudaStreamNonBlocking), "export stream");
        NB_TRY(cudaStreamCreateWithFlags(&h->st_in, cudaStreamNonBlocking), "upload stream");
        NB_TRY(cudaEventCreateWithFlags(&h->ev_out, cudaEventDisableTiming), "export event");
        NB_TRY(cudaEventCreateWithFlags(&h->ev_in_pos, cudaEventDisableTiming), "upload event");
        NB_TRY(cudaEventCreateWithFlags(&h->ev_in_vel, cudaEventDisableTiming), "upload event");
        NB_TRY(cudaMalloc(reinterpret_cast<void**>(&h->io_flag), sizeof(int)), "io flag");
    }
    if (h->io_n == n) return NEXT_OK;
    for (int k = 0; k < 2; ++k) { dfree(h->io_in[k]); dfree(h->io_type[k]); dfree(h->io_out[k]); }
    h->io_n = 0;
    h->io_ready = false;
    cudaError_t e = cudaSuccess;
    auto A = [&](auto** q, size_t c) { if (e == cudaSuccess) e = dalloc(q, c); };
    for (int k = 0; k < 2; ++k) { A(&h->io_in[k], 7 * n); A(&h->io_type[k], n); A(&h->io_out[k], 6 * n); }
    if (e != cudaSuccess) return cuda_fail(h, e, "step_host buffers");
    h->io_n = n;
    return NEXT_OK;
}

// One step on the held state, positions copied out on st_out as soon as the
// drift has made them final (if pos_now), velocities after the closing kick;
// both gathered into caller order at `out` (6 x n) on the way.  With
// pos_now false the positions are only gathered, and copied by the caller.
static int step_and_export(next_handle* h, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                           double* out, bool pos_now, bool* pos_pending) {
    const bool use_graph = group_walk(h) && h->prm.reuse_forces;
    int rc = NEXT_OK;
    if (use_graph && !h->fgraph[h->cur] && h->forces_valid) {
        rc = grow_if_tight(h);   // before a capture, as next_steps does
        if (rc) return rc;
    }
    if (!(h->prm.reuse_forces && h->forces_valid)) {
        rc = forces_checked(h, false);
        if (rc) return rc;
    }
    Bodies bd = h->cur_bodies();
    NB_TRY(kick_drift_step(h, bd), "kick-drift");
    // the positions are final: their copies out run beside the force phase
    // (the gather into caller order precedes the re-sort in stream order)
    const double* pos[3] = {bd.x, bd.y, bd.z};
    double* pos_out[3] = {x, y, z};
    if (pos_now) {
        rc = export_lanes(h, pos, pos_out, 3, out, h->st_out);
    } else {
        NB_TRY(launch_gather_out(pos, 3, h->inv, h->n, out, h->st), "gather out");
        NB_TRY(cudaEventRecord(h->ev_out, h->st), "export event");
        *pos_pending = true;
    }
    if (rc == NEXT_OK && use_graph) {
        rc = capture_graph(h, false);
        if (rc == NEXT_OK) {
            const int parity = h->cur;
            const cudaError_t e = cudaGraphLaunch(h->fgraph[parity], h->st);
            if (e != cudaSuccess) {
                rc = cuda_fail(h, e, "graph launch");
            } else {
                ++h->builds;              // the replay's build
                count_launches(static_cast<int>(h->fgraph_kernels[parity]));
                h->cur = 1 - h->cur;
                h->cube_fresh = false;    // consumed by the replay's build
                h->forces_valid = true;
                h->pot_valid = false;
            }
        }
    } else if (rc == NEXT_OK) {
        rc = forces(h, false, nullptr);
        if (rc == NEXT_OK) {
            bd = h->cur_bodies();
            const cudaError_t e = launch_kick(bd, h->n, h->dts, h->err, h->st);
            if (e != cudaSuccess) rc = cuda_fail(h, e, "kick");
        }
    }
    return rc;
}

// After the force phase: recover from an overflow (redo the force phase and
// the closing kick) and export the velocities.
static int finish_and_export_velocities(next_handle* h, double* vx, double* vy, double* vz, double* out,
                                        cudaEvent_t after = nullptr) {
    int bits = 0;
    int rc = read_device_error(h, &bits);
    if (rc) return rc;
    if (bits) {
        // the kick-drift ran and the positions are out; redo the force phase and the closing kick
        rc = recover(h, bits);
        if (rc) return rc;
        rc = forces_checked(h, false);
        if (rc) return rc;
        NB_TRY(launch_kick(h->cur_bodies(), h->n, h->dts, h->err, h->st), "kick");
    }
    // copies into the caller's velocity arrays wait for `after` (their upload)
    if (after) NB_TRY(cudaStreamWaitEvent(h->st, after, 0), "upload wait");
    const Bodies bd = h->cur_bodies();
    const double* vel[3] = {bd.vx, bd.vy, bd.vz};
    double* vel_out[3] = {vx, vy, vz};
    return export_lanes(h, vel, vel_out, 3, out + 3 * h->n, h->st);
}

int next_step_host(next_handle* h, double dt, int64_t n, double* x, double* y, double* z, double* vx, double* vy,
                   double* vz, const double* m, const int* type) {
    if (!h) return NEXT_ERR_INVALID_ARGUMENT;
    if (!std::isfinite(dt)) return fail(h, NEXT_ERR_INVALID_ARGUMENT, "dt must be finite");
    if (n < 1 || n >= (int64_t(1) << 30) || !x || !y || !z || !vx || !vy || !vz || !m)
        return fail(h, NEXT_ERR_INVALID_ARGUMENT, "bad body arrays");
    NB_TRY(cudaSetDevice(h->device), "set device");
    int rc = ensure_host_io(h, n);
    if (rc) return rc;
    // Speculation: the previous call returned the state the device still
    // holds, and a caller whose arrays are its state passes that back.  The
    // step then starts at once on the held state while the upload lands, and
    // the upload is compared bit for bit with what the previous call
    // returned.  If it differs, the held state is replaced by the upload and
    // the step re-run, so the result is always the step of the inputs.
    const bool spec = h->io_ready && h->have_bodies && h->n == n && h->nsys == 1;
    const int k = spec ? 1 - h->io_cur : h->io_cur;
    double* out = h->io_out[k];
    double* xs[3] = {x, y, z};
    h->io_ready = false;
    if (!spec) {
        const int64_t offs[2] = {0, n};
        rc = upload_staged(h, 1, offs, x, y, z, vx, vy, vz, m, type, h->io_in[k], h->io_type[k]);
        if (rc) return rc;
        rc = set_dt(h, dt);
        if (rc) return rc;
        bool pending = false;
        rc = step_and_export(h, x, y, z, vx, vy, vz, out, true, &pending);
        const cudaError_t es = cudaStreamSynchronize(h->st_out);   // no copy into the caller's arrays outlives the call
        if (rc) return rc;
        if (es != cudaSuccess) return cuda_fail(h, es, "position copies");
        rc = finish_and_export_velocities(h, vx, vy, vz, out);
        const cudaError_t ev = cudaStreamSynchronize(h->st);
        if (rc) return rc;
        if (ev != cudaSuccess) return cuda_fail(h, ev, "sync");
        h->io_cur = k;
        h->io_ready = true;
        return NEXT_OK;
    }
    // The step on the held state goes on st first: it runs while the host
    // queues the upload, which for pageable caller arrays blocks the host
    // until they are staged.  Its results go into the caller's arrays as soon
    // as they are final and those arrays have been uploaded (positions beside
    // the force phase, velocities after the closing kick), before the check
    // has its verdict: the check's kernel may have to wait for the walk's
    // resident blocks to finish.  If the verdict is "changed", the step is
    // taken again from the upload and its results overwrite these; if the
    // upload is invalid, the caller's arrays get the upload back.
    rc = set_dt(h, dt);
    if (rc) return rc;
    bool pending = false;
    rc = step_and_export(h, x, y, z, vx, vy, vz, out, false, &pending);
    if (rc) {
        NB_TRY(cudaStreamSynchronize(h->st), "sync");
        return rc;
    }
    // the upload and its check, on st_in
    const int p = h->io_cur;
    double* in = h->io_in[k];
    const double* lanes[7] = {x, y, z, vx, vy, vz, m};
    for (int c = 0; c < 7; ++c) {
        NB_TRY(cudaMemcpyAsync(in + c * n, lanes[c], sizeof(double) * n, cudaMemcpyHostToDevice, h->st_in), "upload");
        if (c == 2) NB_TRY(cudaEventRecord(h->ev_in_pos, h->st_in), "upload event");
        if (c == 5) NB_TRY(cudaEventRecord(h->ev_in_vel, h->st_in), "upload event");
    }
    if (type) {
        NB_TRY(cudaMemcpyAsync(h->io_type[k], type, sizeof(int) * n, cudaMemcpyHostToDevice, h->st_in), "upload types");
    } else {
        NB_TRY(cudaMemsetAsync(h->io_type[k], 0, sizeof(int) * n, h->st_in), "types");
    }
    NB_TRY(cudaMemsetAsync(h->io_flag, 0, sizeof(int), h->st_in), "io flag");
    NB_TRY(launch_same_as_last(in, h->io_type[k], h->io_out[p], h->io_in[p], h->io_type[p], n, h->io_flag, h->st_in),
           "upload check");
    NB_TRY(cudaMemcpyAsync(h->h_flags + 3, h->io_flag, sizeof(int), cudaMemcpyDeviceToHost, h->st_in), "io flag");
    NB_TRY(cudaStreamWaitEvent(h->st_out, h->ev_out, 0), "export wait");
    NB_TRY(cudaStreamWaitEvent(h->st_out, h->ev_in_pos, 0), "upload wait");
    for (int c = 0; c < 3; ++c)
        NB_TRY(cudaMemcpyAsync(xs[c], out + static_cast<int64_t>(c) * n, sizeof(double) * n, cudaMemcpyDeviceToHost,
                               h->st_out), "download");
    rc = finish_and_export_velocities(h, vx, vy, vz, out, h->ev_in_vel);
    const cudaError_t ei = cudaStreamSynchronize(h->st_in);
    const cudaError_t eo = cudaStreamSynchronize(h->st_out);
    const cudaError_t es = cudaStreamSynchronize(h->st);
    if (rc) return rc;
    if (ei != cudaSuccess) return cuda_fail(h, ei, "upload");
    if (eo != cudaSuccess) return cuda_fail(h, eo, "position copies");
    if (es != cudaSuccess) return cuda_fail(h, es, "sync");
    if (h->h_flags[3] == 0) {
        h->io_cur = k;
        h->io_ready = true;
        return NEXT_OK;
    }
    // The inputs differ from the state the step started from.  Drop the
    // speculative step: validate the upload and load it (the held state is
    // restored from the previous call's set if the upload is invalid), then
    // take the step again.
    {
        int bits = 0;
        rc = read_device_error(h, &bits);
        if (rc) return rc;
        if (bits) NB_TRY(cudaMemsetAsync(h->err, 0, sizeof(int), h->st), "error reset");
    }
    Bodies b = h->cur_bodies();
    NB_TRY(cudaMemsetAsync(h->changed, 0, sizeof(int) * 3, h->st), "upload flags");
    NB_TRY(launch_check_upload(in, h->io_type[k], b, h->inv, n, false, h->changed, h->st), "upload check");
    NB_TRY(cudaMemcpyAsync(h->h_flags, h->changed, sizeof(int) * 3, cudaMemcpyDeviceToHost, h->st), "upload flags");
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    const bool invalid = h->h_flags[1] || h->h_flags[2];
    if (invalid) {
        // back to the state the previous call returned
        for (int c = 0; c < 6; ++c)
            NB_TRY(cudaMemcpyAsync(h->stage + c * n, h->io_out[p] + c * n, sizeof(double) * n,
                                   cudaMemcpyDeviceToDevice, h->st), "restore");
        NB_TRY(cudaMemcpyAsync(h->stage + 6 * n, h->io_in[p] + 6 * n, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                               h->st), "restore");
        NB_TRY(launch_load_all(h->stage, h->io_type[p], b, h->inv, n, h->st), "restore");
    } else {
        NB_TRY(launch_load_all(in, h->io_type[k], b, h->inv, n, h->st), "load");
    }
    h->forces_valid = false;
    h->cube_fresh = false;
    set_key_levels(h, kMaxLevel);
    h->depth_decided = false;
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    if (invalid) {
        // the caller's arrays get their inputs back
        for (int c = 0; c < 6; ++c)
            NB_TRY(cudaMemcpyAsync(c < 3 ? xs[c] : (c == 3 ? vx : c == 4 ? vy : vz), in + static_cast<int64_t>(c) * n,
                                   sizeof(double) * n, cudaMemcpyDeviceToHost, h->st), "restore");
        NB_TRY(cudaStreamSynchronize(h->st), "sync");
        h->io_ready = true;       // the held state is again what the previous call returned
        return fail(h, NEXT_ERR_INVALID_ARGUMENT, h->h_flags[1] ? "non-finite body data" : "negative mass");
    }
    rc = step_and_export(h, x, y, z, vx, vy, vz, out, true, &pending);
    const cudaError_t es2 = cudaStreamSynchronize(h->st_out);
    if (rc) return rc;
    if (es2 != cudaSuccess) return cuda_fail(h, es2, "position copies");
    rc = finish_and_export_velocities(h, vx, vy, vz, out);
    const cudaError_t ev = cudaStreamSynchronize(h->st);
    if (rc) return rc;
    if (ev != cudaSuccess) return cuda_fail(h, ev, "sync");
    h->io_cur = k;
    h->io_ready = true;
    return NEXT_OK;
}

int next_steps(next_handle* h, double dt, int nsteps) {
    int rc = check_ready(h);
    if (rc) return rc;
    h->io_ready = false;
    if (!std::isfinite(dt) || nsteps < 0) return fail(h, NEXT_ERR_INVALID_ARGUMENT, "bad dt or step count");
    rc = set_dt(h, dt);
    if (rc) return rc;
    const bool use_graph = group_walk(h) && h->prm.reuse_forces;
    int done = 0;            // steps completed
    int base = 0;            // `done` when the device's count of completed replays was last zeroed
    int since_check = 0;     // replays launched since the error word was last read
    if (use_graph) NB_TRY(cudaMemsetAsync(h->done, 0, sizeof(unsigned int), h->st), "replay count");
    // Reads the error word of the replays launched since the last look.  A
    // replay that overflowed a capacity stopped after its kick-drift (every
    // later kernel of it, and of the replays after it, skipped its work but
    // the harmless body permutation), so the state is that step's drifted
    // positions: grow what overflowed, redo its force phase and closing kick
    // eagerly -- as step_once does -- and continue from the step after it.
    auto check = [&]() -> int {
        if (since_check == 0) return NEXT_OK;
        since_check = 0;
        NB_TRY(cudaMemcpyAsync(h->h_done, h->done, sizeof(unsigned int), cudaMemcpyDeviceToHost, h->st),
               "replay count");
        int bits = 0;
        int r = read_device_error(h, &bits);
        if (r) return r;
        if (bits == 0) return grow_if_tight(h);
        const int completed = static_cast<int>(*h->h_done);
        r = recover(h, bits);
        if (r) return r;
        r = forces_checked(h, false);
        if (r) return r;
        NB_TRY(launch_kick(h->cur_bodies(), h->n, h->dts, h->err, h->st), "kick");
        h->forces_valid = true;
        ++h->recoveries;
        done = base + completed + 1;
        base = done;
        NB_TRY(cudaMemsetAsync(h->done, 0, sizeof(unsigned int), h->st), "replay count");
        NB_TRY(cudaStreamSynchronize(h->st), "sync");
        return NEXT_OK;
    };
    while (done < nsteps) {
        if (!use_graph || !h->forces_valid) {
            rc = check();
            if (rc) return rc;
            if (done >= nsteps) break;
            rc = step_once(h, !h->timing);
            if (rc) return rc;
            ++done;
            base = done;
            NB_TRY(cudaMemsetAsync(h->done, 0, sizeof(unsigned int), h->st), "replay count");
            continue;
        }
        // replay the captured step; buffers alternate, so keep one graph per parity
        if (!h->graph[h->cur]) {
            rc = check();
            if (rc) return rc;
            if (done >= nsteps) break;
            if (since_check == 0) {
                int bits = 0;
                rc = read_device_error(h, &bits);
                if (rc) return rc;
                rc = grow_if_tight(h);
                if (rc) return rc;
            }
            if (!h->forces_valid) continue;
        }
        rc = capture_graph(h, true);
        if (rc) return rc;
        const int parity = h->cur;
        std::vector<int> evs;
        if (h->timing) {
            rc = resolve_timers(h);   // eager steps timed earlier keep their pool events until read
            if (rc) return rc;
            rc = record(h, &evs);
            if (rc) return rc;
        }
        NB_TRY(cudaGraphLaunch(h->graph[parity], h->st), "graph launch");
        ++h->builds;                       // the replay's build
        count_launches(static_cast<int>(h->graph_kernels[parity]));
        if (h->timing) {
            // stage times of this replay: its in-graph events are overwritten by the next one
            rc = record(h, &evs);
            if (rc) return rc;
            NB_TRY(cudaStreamSynchronize(h->st), "sync");
            rc = add_graph_timing(h, parity, evs);
            if (rc) return rc;
        }
        h->cur = 1 - h->cur;
        ++done;
        ++since_check;
        if (done == nsteps || since_check >= 64) {
            rc = check();
            if (rc) return rc;
        }
    }
    rc = check();
    if (rc) return rc;
    h->forces_valid = true;
    return NEXT_OK;
}

int next_accel(next_handle* h, double* ax, double* ay, double* az, double* pot) {
    int rc = check_ready(h);
    if (rc) return rc;
    const bool want_pot = pot && h->P.physics == NEXT_PHYSICS_ACCURATE;
    if (!h->forces_valid || (want_pot && !h->pot_valid)) {
        rc = forces_checked(h, want_pot);
        if (rc) return rc;
    }
    const double* lanes[4] = {h->ax, h->ay, h->az, h->pot};
    double* outs[4] = {ax, ay, az, pot};
    const int cnt = want_pot ? 4 : 3;
    NB_TRY(launch_gather_out(lanes, cnt, h->inv, h->n, h->stage, h->st), "gather out");
    for (int c = 0; c < cnt; ++c)
        if (outs[c])
            NB_TRY(cudaMemcpyAsync(outs[c], h->stage + c * h->n, sizeof(double) * h->n, cudaMemcpyDeviceToHost, h->st),
                   "download");
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    if (pot && !want_pot) std::memset(pot, 0, sizeof(double) * h->n);
    return NEXT_OK;
}

int next_adaptive_dt(next_handle* h, double base_dt, double* dt_out) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (!dt_out) return fail(h, NEXT_ERR_INVALID_ARGUMENT, "NULL output");
    NB_TRY(launch_adaptive_dt(h->cur_bodies(), h->n, base_dt, h->partial, h->tickets + 1, h->dt_out, h->st), "adaptive dt");
    NB_TRY(cudaMemcpyAsync(h->h_dts, h->dt_out, sizeof(double), cudaMemcpyDeviceToHost, h->st), "dt");
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    *dt_out = h->h_dts[0];
    return NEXT_OK;
}

int next_direct_accel(next_handle* h, int64_t k, const int64_t* idx, double* ax, double* ay, double* az, double* pot) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (k < 0 || (k > 0 && !idx)) return fail(h, NEXT_ERR_INVALID_ARGUMENT, "bad sample");
    for (int64_t t = 0; t < k; ++t)
        if (idx[t] < 0 || idx[t] >= h->n) return fail(h, NEXT_ERR_INVALID_ARGUMENT, "sample index out of range");
    if (h->nsys != 1) return fail(h, NEXT_ERR_INVALID_ARGUMENT, "direct summation needs a single system");
    if (k == 0) return NEXT_OK;
    const int slices = direct_slices(h->n, k);
    if (k > h->direct_cap || slices > h->direct_slice_cap) {
        dfree(h->d_targets); dfree(h->d_targetpos); dfree(h->d_direct_partial); dfree(h->d_direct_out);
        cudaError_t e = cudaSuccess;
        auto A = [&](auto** q, size_t c) { if (e == cudaSuccess) e = dalloc(q, c); };
        A(&h->d_targets, k); A(&h->d_targetpos, k); A(&h->d_direct_partial, 4 * k * slices); A(&h->d_direct_out, 4 * k);
        if (e != cudaSuccess) return cuda_fail(h, e, "direct scratch");
        h->direct_cap = k;
        h->direct_slice_cap = slices;
    }
    NB_TRY(cudaMemcpyAsync(h->d_targets, idx, sizeof(int64_t) * k, cudaMemcpyHostToDevice, h->st), "sample");
    NB_TRY(launch_ids_to_positions(h->d_targets, h->inv, k, h->d_targetpos, h->st), "sample map");
    const double eps = h->P.physics == NEXT_PHYSICS_REFERENCE ? h->prm.eps : h->P.eps;
    NB_TRY(launch_direct(h->cur_bodies(), h->n, h->d_targetpos, k, eps, h->P.G, h->d_direct_partial, slices,
                         h->d_direct_out, h->st),
           "direct sum");
    std::vector<double> out(4 * k);
    NB_TRY(cudaMemcpyAsync(out.data(), h->d_direct_out, sizeof(double) * 4 * k, cudaMemcpyDeviceToHost, h->st), "direct out");
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    for (int64_t t = 0; t < k; ++t) {
        if (ax) ax[t] = out[4 * t];
        if (ay) ay[t] = out[4 * t + 1];
        if (az) az[t] = out[4 * t + 2];
        if (pot) pot[t] = out[4 * t + 3];
    }
    return NEXT_OK;
}

int next_diagnostics(next_handle* h, double* out8) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (!out8) return fail(h, NEXT_ERR_INVALID_ARGUMENT, "NULL output");
    const bool acc = h->P.physics == NEXT_PHYSICS_ACCURATE;
    if (acc && (!h->forces_valid || !h->pot_valid)) {
        rc = forces_checked(h, true);
        if (rc) return rc;
    }
    NB_TRY(launch_diagnostics(h->cur_bodies(), h->n, acc, h->partial, h->tickets + 2, h->diag, h->st), "diagnostics");
    NB_TRY(cudaMemcpyAsync(out8, h->diag, sizeof(double) * 8, cudaMemcpyDeviceToHost, h->st), "diagnostics");
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    return NEXT_OK;
}

int next_stats_get(next_handle* h, next_stats* s) {
    if (!h || !s) return NEXT_ERR_INVALID_ARGUMENT;
    std::memset(s, 0, sizeof(*s));
    s->n_bodies = h->n;
    s->n_systems = h->nsys;
    if (h->have_bodies) {
        int bits = 0;
        int rc = read_device_error(h, &bits);
        if (rc) return rc;
        rc = resolve_timers(h);
        if (rc) return rc;
        s->device_error = bits;
        s->n_internal = h->h_counts[0];
        s->n_nodes = h->h_counts[1];
        s->n_groups = h->h_counts[2];
        s->key_levels = h->sys.levels;
        s->recoveries = static_cast<int32_t>(h->recoveries);
        s->pp_interactions = static_cast<int64_t>(h->h_stats[0]);
        s->pc_interactions = static_cast<int64_t>(h->h_stats[1]);
        s->max_stack = static_cast<int64_t>(h->h_stats[2]);
    }
    s->steps = static_cast<int32_t>(h->timed_steps);
    s->ms_step = h->acc_step;
    s->ms_build = h->acc_build;
    s->ms_walk = h->acc_walk;
    s->ms_sort = h->acc_sort;
    s->ms_other = h->acc_other;
    s->walk_launches = h->timed_walks;
    return NEXT_OK;
}

int next_set_timing(next_handle* h, int on) {
    if (!h) return NEXT_ERR_INVALID_ARGUMENT;
    h->timing = on != 0;
    return NEXT_OK;
}

int next_reset_timers(next_handle* h) {
    if (!h) return NEXT_ERR_INVALID_ARGUMENT;
    if (h->st) cudaStreamSynchronize(h->st);
    h->ev_steps.clear();
    h->ev_used = 0;
    h->acc_step = h->acc_build = h->acc_walk = h->acc_sort = h->acc_other = 0;
    h->timed_steps = h->timed_walks = 0;
    NB_TRY(cudaMemsetAsync(h->stats, 0, sizeof(unsigned long long) * 4, h->st), "stats reset");
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    return NEXT_OK;
}

int next_sync(next_handle* h) {
    if (!h) return NEXT_ERR_INVALID_ARGUMENT;
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    return NEXT_OK;
}

int next_debug_keys(next_handle* h, uint64_t* keys, double* cube4) {
    int rc = check_ready(h);
    if (rc) return rc;
    Bodies b = h->cur_bodies();
    NB_TRY(launch_root_cubes(b, h->n, h->sys, h->d_offsets, h->partial, kReduceMax, h->tickets + 0, h->st), "root cube");
    NB_TRY(launch_keys(b, h->sysid, h->n, h->sys, h->keys, h->idx, h->st), "keys");
    std::vector<uint64_t> kw(h->n);
    std::vector<uint32_t> ids(h->n);
    NB_TRY(cudaMemcpyAsync(kw.data(), h->keys, sizeof(uint64_t) * h->n, cudaMemcpyDeviceToHost, h->st), "keys");
    NB_TRY(cudaMemcpyAsync(ids.data(), b.id, sizeof(uint32_t) * h->n, cudaMemcpyDeviceToHost, h->st), "ids");
    if (cube4)
        NB_TRY(cudaMemcpyAsync(cube4, h->cubes, sizeof(double) * 4, cudaMemcpyDeviceToHost, h->st), "cube");
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    if (keys)
        for (int64_t p = 0; p < h->n; ++p) keys[ids[p]] = kw[p];
    return NEXT_OK;
}

int next_debug_order(next_handle* h, int64_t* perm) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (!h->forces_valid) {
        rc = forces_checked(h, false);
        if (rc) return rc;
    }
    std::vector<uint32_t> ids(h->n);
    NB_TRY(cudaMemcpyAsync(ids.data(), h->cur_bodies().id, sizeof(uint32_t) * h->n, cudaMemcpyDeviceToHost, h->st), "ids");
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    for (int64_t p = 0; p < h->n; ++p) perm[p] = ids[p];
    return NEXT_OK;
}

int next_debug_tree(next_handle* h, double* rows, int64_t cap, int64_t* n_rows) {
    int rc = check_ready(h);
    if (rc) return rc;
    rc = forces_checked(h, false);
    if (rc) return rc;
    const int64_t nn = h->h_counts[1];
    std::vector<int2> link(nn);
    std::vector<int8_t> level(nn);
    std::vector<double4> com(nn);
    std::vector<double> q64(8 * nn);
    std::vector<uint32_t> ids(h->n);
    NB_TRY(cudaMemcpyAsync(link.data(), h->t.link, sizeof(int2) * nn, cudaMemcpyDeviceToHost, h->st), "tree");
    NB_TRY(cudaMemcpyAsync(level.data(), h->t.level, nn, cudaMemcpyDeviceToHost, h->st), "tree");
    NB_TRY(cudaMemcpyAsync(com.data(), h->t.com, sizeof(double4) * nn, cudaMemcpyDeviceToHost, h->st), "tree");
    NB_TRY(cudaMemcpyAsync(q64.data(), h->t.quad64, sizeof(double) * 8 * nn, cudaMemcpyDeviceToHost, h->st), "tree");
    NB_TRY(cudaMemcpyAsync(ids.data(), h->cur_bodies().id, sizeof(uint32_t) * h->n, cudaMemcpyDeviceToHost, h->st), "ids");
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    int64_t count = 0;
    std::vector<int> stackv;
    for (int r = h->nsys - 1; r >= 0; --r) stackv.push_back(r);
    while (!stackv.empty()) {
        const int nd = stackv.back();
        stackv.pop_back();
        if (count < cap && rows) {
            double* o = rows + 16 * count;
            const bool leaf = link[nd].y <= 0;
            const int cnt = leaf ? -link[nd].y : 0;
            o[0] = level[nd]; o[1] = com[nd].w; o[2] = com[nd].x; o[3] = com[nd].y; o[4] = com[nd].z;
            o[5] = q64[8 * nd + 6];
            for (int c = 0; c < 6; ++c) o[6 + c] = q64[8 * nd + c];
            o[12] = leaf ? 1.0 : 0.0;
            o[13] = (leaf && cnt == 1) ? static_cast<double>(ids[link[nd].x]) : -1.0;
            o[14] = 0.0;
            o[15] = leaf ? cnt : -1.0;
        }
        ++count;
        if (link[nd].y > 0)
            for (int k = link[nd].y - 1; k >= 0; --k) stackv.push_back(link[nd].x + k);
    }
    if (n_rows) *n_rows = count;
    return NEXT_OK;
}

int next_sort_pairs(next_handle* h, int64_t n, const uint64_t* keys_in, const uint32_t* vals_in, uint64_t* keys_out,
                    uint32_t* vals_out, int key_bits) {
    if (!h) return NEXT_ERR_INVALID_ARGUMENT;
    if (n < 0 || n >= (int64_t(1) << 30) || key_bits < 1 || key_bits > 64 || (n > 0 && (!keys_in || !vals_in)))
        return fail(h, NEXT_ERR_INVALID_ARGUMENT, "bad sort arguments");
    if (n == 0) return NEXT_OK;
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return cuda_fail(h, e, "set device");
    uint64_t *k0 = nullptr, *k1 = nullptr;
    uint32_t *v0 = nullptr, *v1 = nullptr, *scr = nullptr;
    auto A = [&](auto** q, size_t c) { if (e == cudaSuccess) e = dalloc(q, c); };
    A(&k0, n); A(&k1, n); A(&v0, n); A(&v1, n); A(&scr, sort_scratch_words(n));
    bool in_alt = false;
    // bits an earlier step left in the error word must not fail this sort
    if (e == cudaSuccess) e = cudaMemsetAsync(h->err, 0, sizeof(int), h->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(k0, keys_in, sizeof(uint64_t) * n, cudaMemcpyHostToDevice, h->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(v0, vals_in, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, h->st);
    if (e == cudaSuccess) e = radix_sort_pairs(k0, v0, k1, v1, n, key_bits, scr, h->err, &in_alt, h->st);
    if (e == cudaSuccess && keys_out)
        e = cudaMemcpyAsync(keys_out, in_alt ? k1 : k0, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess && vals_out)
        e = cudaMemcpyAsync(vals_out, in_alt ? v1 : v0, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->h_err, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    const int bits = e == cudaSuccess ? *h->h_err : 0;
    dfree(k0); dfree(k1); dfree(v0); dfree(v1); dfree(scr);
    if (e != cudaSuccess) return cuda_fail(h, e, "sort");
    if (bits & kErrSort) return fail(h, NEXT_ERR_DEVICE, "sort look-back timeout");
    if (bits) return fail(h, NEXT_ERR_DEVICE, "sort raised device error word " + std::to_string(bits));
    return NEXT_OK;
}

int next_fp32_peak(int device, double* tflops, double* sm_mhz_hint) {
    if (!tflops) return NEXT_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(device) != cudaSuccess) return NEXT_ERR_CUDA;
    int sms = 0, khz = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, device);
    float* out = nullptr;
    if (cudaMalloc(&out, sizeof(float)) != cudaSuccess) return NEXT_ERR_OUT_OF_MEMORY;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int blocks = sms * 8, iters = 4096;
    double best = 0.0;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(a, 0);
        launch_fma_peak(out, blocks, iters, 0);
        cudaEventRecord(b, 0);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        const double flops = 2.0 * 8.0 * 16.0 * iters * 256.0 * blocks;
        if (rep > 0 && ms > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    *tflops = best;
    if (sm_mhz_hint) *sm_mhz_hint = khz / 1000.0;
    return cudaGetLastError() == cudaSuccess ? NEXT_OK : NEXT_ERR_CUDA;
}

void* next_host_alloc(int64_t bytes) {
    void* p = nullptr;
    if (bytes <= 0 || cudaHostAlloc(&p, static_cast<size_t>(bytes), cudaHostAllocDefault) != cudaSuccess) return nullptr;
    return p;
}

void next_host_free(void* p) {
    if (p) cudaFreeHost(p);
}

int64_t next_kernel_launches(void) { return launches_so_far(); }

int next_autotune(next_handle* h, next_tune_result* out) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (!group_walk(h))
        return fail(h, NEXT_ERR_INVALID_ARGUMENT, "autotuning applies to the group walk (mixed or FP64-group precision)");
    struct Cand { int leaf, group, warps; };
    std::vector<Cand> cands;
    for (int g : {16, 24, 32})
        for (int l : {8, 12, 16, 24, 32})
            for (int w : {2, 4})
                if (l <= g) cands.push_back({l, g, w});
    // Small systems have fewer groups than the GPU has resident warps, and a
    // walk lasts as long as its slowest group: smaller groups (split over
    // more lane slices) put more warps to work there.
    if (h->n <= (int64_t(1) << 18))
        for (int l : {4, 8})
            for (int w : {2, 4}) cands.push_back({l, 8, w});
    const Params saved_P = h->P;
    const next_params saved_prm = h->prm;
    cudaEvent_t a, b;
    NB_TRY(cudaEventCreate(&a), "event");
    NB_TRY(cudaEventCreate(&b), "event");
    double best_ms = 1e300;
    Cand best = {saved_P.leaf_cap, saved_P.group_cap, saved_prm.walk_warps};
    int64_t best_stack = 0;
    int tried = 0;
    for (const Cand& c : cands) {
        h->P.leaf_cap = c.leaf;
        h->P.group_cap = c.group;
        h->prm.leaf_cap = c.leaf;
        h->prm.group_cap = c.group;
        h->prm.walk_warps = c.warps;
        drop_graphs(h);
        // first pass sizes the tree and the stack (with recovery), second is timed
        NB_TRY(cudaMemsetAsync(h->stats, 0, sizeof(unsigned long long) * 4, h->st), "stats");
        rc = forces_checked(h, false);
        if (rc) break;
        NB_TRY(cudaEventRecord(a, h->st), "event");
        rc = forces(h, false, nullptr);
        if (rc) break;
        NB_TRY(cudaEventRecord(b, h->st), "event");
        int bits = 0;
        rc = read_device_error(h, &bits);
        if (rc) break;
        if (bits) {
            rc = recover(h, bits);
            if (rc) break;
            continue;
        }
        float ms = 0.f;
        NB_TRY(cudaEventElapsedTime(&ms, a, b), "event time");
        ++tried;
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
            best_stack = static_cast<int64_t>(h->h_stats[2]);
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) {
        h->P = saved_P;
        h->prm = saved_prm;
        return rc;
    }
    h->P.leaf_cap = best.leaf;
    h->P.group_cap = best.group;
    h->prm.leaf_cap = best.leaf;
    h->prm.group_cap = best.group;
    h->prm.walk_warps = best.warps;
    // stack: 1.5x the deepest seen, in multiples of 64, at least 256
    int64_t st = ((best_stack * 3 / 2 + 63) / 64) * 64;
    h->prm.walk_stack = static_cast<int>(std::min<int64_t>(std::max<int64_t>(st, 256), 1 << 14));
    drop_graphs(h);
    rc = forces_checked(h, false);
    if (rc) return rc;
    NB_TRY(cudaMemsetAsync(h->stats, 0, sizeof(unsigned long long) * 4, h->st), "stats");
    if (out) {
        out->leaf_cap = best.leaf;
        out->group_cap = best.group;
        out->walk_warps = best.warps;
        out->walk_stack = h->prm.walk_stack;
        out->ms_force_phase = best_ms;
        out->candidates = tried;
    }
    return NEXT_OK;
}

int next_debug_softening(int device, int64_t k, const double* size, const double* mass, const double* dist,
                         double* out) {
    if (k < 0 || (k > 0 && (!size || !mass || !dist || !out))) return NEXT_ERR_INVALID_ARGUMENT;
    if (k == 0) return NEXT_OK;
    if (cudaSetDevice(device) != cudaSuccess) return NEXT_ERR_CUDA;
    double* d = nullptr;
    if (cudaMalloc(&d, sizeof(double) * 4 * k) != cudaSuccess) return NEXT_ERR_OUT_OF_MEMORY;
    cudaError_t e = cudaMemcpy(d, size, sizeof(double) * k, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + k, mass, sizeof(double) * k, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + 2 * k, dist, sizeof(double) * k, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_softening_eval(d, k, d + 3 * k, nullptr);
    if (e == cudaSuccess) e = cudaMemcpy(out, d + 3 * k, sizeof(double) * k, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? NEXT_OK : NEXT_ERR_CUDA;
}

int next_debug_fix_tree_capacity(next_handle* h, int64_t cap_internal) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (cap_internal < 1 || cap_internal >= (int64_t(1) << 31))
        return fail(h, NEXT_ERR_INVALID_ARGUMENT, "capacity out of range");
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    rc = alloc_tree(h, cap_internal);
    if (rc) return rc;
    h->fixed_tree_cap = true;     // the cached forces stay valid: they do not live in the tree
    return NEXT_OK;
}

int next_get_params(const next_handle* h, next_params* p) {
    if (!h || !p) return NEXT_ERR_INVALID_ARGUMENT;
    *p = h->prm;
    return NEXT_OK;
}

int next_dist_unique_id(unsigned char* id128) {
    if (!id128) return NEXT_ERR_INVALID_ARGUMENT;
    std::string why;
    return nccl_unique_id(id128, &why) ? NEXT_OK : NEXT_ERR_CUDA;
}

int next_dist_attach(next_handle* h, int rank, int world, const unsigned char* id128) {
    if (!h) return NEXT_ERR_INVALID_ARGUMENT;
    if (world < 1 || rank < 0 || rank >= world) return fail(h, NEXT_ERR_INVALID_ARGUMENT, "bad rank/world");
    if (h->nsys > 1) return fail(h, NEXT_ERR_INVALID_ARGUMENT, "sharding applies to a single system");
    h->io_ready = false;
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return cuda_fail(h, e, "set device");
    NB_TRY(cudaStreamSynchronize(h->st), "sync");
    drop_graphs(h);
    nccl_comm_destroy(h->comm);
    h->comm = nullptr;
    if (id128) {
        std::string why;
        if (!nccl_comm_init(&h->comm, rank, world, id128, &why)) return fail(h, NEXT_ERR_CUDA, why);
    }
    const bool resize = h->have_bodies && world != h->world;
    h->world = world;
    h->rank = rank;
    if (resize) {
        dfree(h->ax); dfree(h->ay); dfree(h->az); dfree(h->pot);
        const int64_t padded = ((h->cap_n + world - 1) / world) * world;
        auto A = [&](auto** q, size_t c) { if (e == cudaSuccess) e = dalloc(q, c); };
        A(&h->ax, padded); A(&h->ay, padded); A(&h->az, padded); A(&h->pot, padded);
        if (e != cudaSuccess) return cuda_fail(h, e, "force arrays");
    }
    set_share(h);
    h->forces_valid = false;
    return NEXT_OK;
}

int next_flush_l2(next_handle* h) {
    if (!h) return NEXT_ERR_INVALID_ARGUMENT;
    if (!h->flush) {
        h->flush_bytes = size_t(256) << 20;
        NB_TRY(cudaMalloc(&h->flush, h->flush_bytes), "flush buffer");
    }
    static unsigned char v = 0;
    NB_TRY(cudaMemsetAsync(h->flush, ++v, h->flush_bytes, h->st), "flush");
    return NEXT_OK;
}

}  // extern "C"
