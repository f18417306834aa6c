// Mixed-precision force walk: one warp per group of <= 32 Morton-contiguous
// target bodies, FP32 interactions, compensated accumulation.
//
// Traversal: a per-warp LIFO stack of node ids in shared memory; each round
// pops up to 32 nodes (one per lane) and applies the opening test
//     open  <=>  dmin(group box, COM)^2 < rcrit^2,   rcrit = l/theta + |COM - centre|
// to all of them at once.  __ballot_sync / warp scans then append
//   - accepted cells to the particle-cell (PC) list,
//   - children of opened cells to the stack,
//   - bodies of opened leaves to the particle-particle (PP) list,
// all held in shared memory.  Whenever a list holds 32 entries, the warp
// stages them (one per lane: FP64 COM/position minus the FP64 group centre,
// rounded to FP32 -- coordinates relative to the group keep FP32 exact
// enough near the group) and every lane runs the 32 interactions for its
// target from shared memory with FP32 FMA and rsqrt.  The 32-term partial
// is folded into the per-target sum with Kahan compensation.
//
// Scheduling: persistent blocks (SM count x resident blocks) pull groups
// from a global atomic work queue.  All waits are warp-synchronous; there
// are no inter-block waits.  Stack or list overflow raises an error bit and
// abandons the group.
//
// Roofline: FP32 pipe.  Algorithmic flops: 20 per PP, 56 per PC interaction.
#include "common.cuh"
#include "kernels.cuh"

namespace nb {

namespace {

// Compile-time knobs of the evaluation loop (unroll depth of a full batch and
// the minimum resident blocks the register allocation must allow).
#ifndef NB_WALK_UNROLL
#define NB_WALK_UNROLL 8
#endif
#ifndef NB_WALK_GENERIC_UNROLL
#define NB_WALK_GENERIC_UNROLL 1
#endif
#ifndef NB_WALK_FIXED
#define NB_WALK_FIXED 1
#endif
#ifndef NB_WALK_MIN_BLOCKS
#define NB_WALK_MIN_BLOCKS 6
#endif

constexpr int kWalkUnroll = NB_WALK_UNROLL;
constexpr int kWalkGenericUnroll = NB_WALK_GENERIC_UNROLL;
constexpr int kPcCap = 64;
constexpr int kPpChunk = 16;
constexpr int kPpCap = 32 + 32 * kPpChunk;

struct WarpLists {
    float4 stage[3 * 32];
    int pc[kPcCap];
    int pp[kPpCap];
};

__device__ __forceinline__ int warp_excl_scan(int v, int lane, int* total) {
    int inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    *total = __shfl_sync(0xffffffffu, inc, 31);
    return inc - v;
}

struct Target {
    float tx, ty, tz;
    float ax, ay, az, pot;       // running sums
    float cx, cy, cz, cp;        // Kahan compensation
};

__device__ __forceinline__ void kahan_add(float& s, float& c, float v) {
    const float y = v - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

// One body-cell interaction (monopole + traceless quadrupole) from a staged
// entry e[0] = (dx, dy, dz, G m) relative to the group centre, e[1] = G (Qxx Qyy
// Qzz Qxy), e[2] = G (Qxz Qyz - -).  56 algorithmic flops.
template <bool QUAD, bool POT>
__device__ __forceinline__ void pc_term(const float4* e, const Target& T, float eps2, float& sx, float& sy,
                                        float& sz, float& sp) {
    const float4 a = e[0];
    const float dx = a.x - T.tx, dy = a.y - T.ty, dz = a.z - T.tz;
    const float r2 = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, eps2)));
    const float rinv = rsqrtf(r2);
    const float rinv2 = rinv * rinv;
    const float rinv3 = rinv2 * rinv;
    if (QUAD) {
        const float4 b = e[1];
        const float4 c = e[2];
        const float qdx = fmaf(c.x, dz, fmaf(b.w, dy, b.x * dx));
        const float qdy = fmaf(c.y, dz, fmaf(b.y, dy, b.w * dx));
        const float qdz = fmaf(b.z, dz, fmaf(c.y, dy, c.x * dx));
        const float q = fmaf(dz, qdz, fmaf(dy, qdy, dx * qdx));
        // G m / r^3 + 2.5 q / r^7 = (G m + 2.5 q / r^4) / r^3
        const float cc = rinv3 * fmaf(q, (2.5f * rinv2) * rinv2, a.w);
        const float rinv5 = rinv3 * rinv2;
        sx = fmaf(cc, dx, fmaf(-rinv5, qdx, sx));
        sy = fmaf(cc, dy, fmaf(-rinv5, qdy, sy));
        sz = fmaf(cc, dz, fmaf(-rinv5, qdz, sz));
        if (POT) sp = fmaf(-0.5f * q, rinv5, fmaf(-a.w, rinv, sp));
    } else {
        const float mr3 = a.w * rinv3;
        sx = fmaf(mr3, dx, sx);
        sy = fmaf(mr3, dy, sy);
        sz = fmaf(mr3, dz, sz);
        if (POT) sp = fmaf(-a.w, rinv, sp);
    }
}

// One body-body interaction from a staged entry (dx, dy, dz, G m).  20 flops.
template <bool SOFT, bool POT>
__device__ __forceinline__ void pp_term(const float4* e, const Target& T, float eps2, float& sx, float& sy,
                                        float& sz, float& sp) {
    const float4 a = e[0];
    const float dx = a.x - T.tx, dy = a.y - T.ty, dz = a.z - T.tz;
    const float r2 = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, eps2)));
    float rinv = rsqrtf(r2);
    if (!SOFT) rinv = r2 > 0.f ? rinv : 0.f;     // the target itself, unsoftened
    const float mr = a.w * rinv;
    const float mr3 = mr * rinv * rinv;
    sx = fmaf(mr3, dx, sx);
    sy = fmaf(mr3, dy, sy);
    sz = fmaf(mr3, dz, sz);
    if (POT) sp -= r2 > eps2 ? mr : 0.f;          // no self term
}

// Entries [k0, k0 + N) of a staged batch (stride STRIDE float4 per entry),
// with a compile-time trip count so the loop unrolls into immediate offsets.
template <int N, int STRIDE, bool PC, bool F1, bool POT>
__device__ __forceinline__ void run_fixed(const float4* stage, int k0, const Target& T, float eps2, float& sx,
                                          float& sy, float& sz, float& sp) {
    const float4* e = stage + STRIDE * k0;
#pragma unroll kWalkUnroll
    for (int k = 0; k < N; ++k) {
        if (PC) pc_term<F1, POT>(e + STRIDE * k, T, eps2, sx, sy, sz, sp);
        else pp_term<F1, POT>(e + STRIDE * k, T, eps2, sx, sy, sz, sp);
    }
}

// Evaluate a staged batch of `count` entries for this lane's target: the
// lane's slice takes entries [slice*count/nslices, ...).  A full, unsplit
// batch (the common case) runs a loop with a compile-time trip count; split
// and partial batches a plain loop.  Both stay compact: instruction-cache
// misses cost more here than loop overhead.
template <int STRIDE, bool PC, bool F1, bool POT>
__device__ __forceinline__ void eval_batch(const float4* stage, int count, float eps2, bool active, int slice,
                                           int nslices, Target& T) {
    if (!active) return;
    float sx = 0.f, sy = 0.f, sz = 0.f, sp = 0.f;
    if (NB_WALK_FIXED && count == 32 && nslices == 1) {
        run_fixed<32, STRIDE, PC, F1, POT>(stage, 0, T, eps2, sx, sy, sz, sp);
    } else {
        const int chunk = (count + nslices - 1) / nslices;
        const int k0 = slice * chunk;
        const int k1 = min(count, k0 + chunk);
#pragma unroll kWalkGenericUnroll
        for (int k = k0; k < k1; ++k) {
            if (PC) pc_term<F1, POT>(stage + STRIDE * k, T, eps2, sx, sy, sz, sp);
            else pp_term<F1, POT>(stage + STRIDE * k, T, eps2, sx, sy, sz, sp);
        }
    }
    kahan_add(T.ax, T.cx, sx);
    kahan_add(T.ay, T.cy, sy);
    kahan_add(T.az, T.cz, sz);
    if (POT) kahan_add(T.pot, T.cp, sp);
}

// Stage up to 32 cells (one per lane) and evaluate them.
template <bool QUAD, bool POT>
__device__ __forceinline__ void eval_pc(WarpLists& L, const int* list, int count, const Tree& t, double gcx,
                                        double gcy, double gcz, float G, float eps2, bool active, int slice,
                                        int nslices, Target& T, int lane) {
    if (lane < count) {
        const int node = list[lane];
        const double4 c = t.com[node];
        L.stage[3 * lane + 0] = make_float4(static_cast<float>(c.x - gcx), static_cast<float>(c.y - gcy),
                                            static_cast<float>(c.z - gcz), static_cast<float>(G * c.w));
        if (QUAD) {
            L.stage[3 * lane + 1] = t.quad32[2 * node];
            L.stage[3 * lane + 2] = t.quad32[2 * node + 1];
        }
    }
    __syncwarp();
    eval_batch<3, true, QUAD, POT>(L.stage, count, eps2, active, slice, nslices, T);
    __syncwarp();
}

// Stage up to 32 bodies (one per lane) and evaluate them.
template <bool SOFT, bool POT>
__device__ __forceinline__ void eval_pp(WarpLists& L, const int* list, int count, const Bodies& bd, double gcx,
                                        double gcy, double gcz, float G, float eps2, bool active, int slice,
                                        int nslices, Target& T, int lane) {
    if (lane < count) {
        const int j = list[lane];
        L.stage[lane] = make_float4(static_cast<float>(bd.x[j] - gcx), static_cast<float>(bd.y[j] - gcy),
                                    static_cast<float>(bd.z[j] - gcz), static_cast<float>(G * bd.m[j]));
    }
    __syncwarp();
    eval_batch<1, false, SOFT, POT>(L.stage, count, eps2, active, slice, nslices, T);
    __syncwarp();
}

template <bool QUAD, bool SOFT, bool POT>
__global__ void __launch_bounds__(128, NB_WALK_MIN_BLOCKS)
walk_mixed_kernel(Bodies bd, int64_t nbodies, Tree t, float G, float eps2, int stack_cap, unsigned int* queue,
                  unsigned long long* stats, int* err, int64_t own_lo, int64_t own_hi) {
    if (*err & kErrAbort) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    WarpLists& L = reinterpret_cast<WarpLists*>(smem_raw)[w];
    int* stack = reinterpret_cast<int*>(smem_raw + sizeof(WarpLists) * nwarps) + w * stack_cap;
    const uint32_t lt = (1u << lane) - 1u;
    const int64_t ngroups = t.counts[2];
    const unsigned nnodes32 = static_cast<unsigned>(t.counts[1]);
    const unsigned nbodies32 = static_cast<unsigned>(nbodies);
    unsigned long long npp = 0, npc = 0;
    int max_sp = 0;

    for (;;) {
        int g = 0;
        if (lane == 0) g = static_cast<int>(atomicAdd(queue, 1u));
        g = __shfl_sync(0xffffffffu, g, 0);
        if (g >= ngroups) break;
        const int4 grp = t.groups[g];
        const int nt = grp.y;
        if (nt <= 0) continue;
        if (nt > 32 || grp.x < 0 || static_cast<int64_t>(grp.x) + nt > nbodies) {
            if (lane == 0) raise_error(err, kErrIndex);
            continue;
        }
        // sharded: only groups that hold bodies of this device's share
        if (static_cast<int64_t>(grp.x) + nt <= own_lo || grp.x >= own_hi) continue;
        const int64_t own_first = grp.x > own_lo ? grp.x : own_lo;
        const int64_t own_end = static_cast<int64_t>(grp.x) + nt < own_hi ? static_cast<int64_t>(grp.x) + nt : own_hi;
        const unsigned long long own_nt = static_cast<unsigned long long>(own_end - own_first);
        // Groups of at most 16 bodies are evaluated by 2, 4, ... warp slices,
        // each taking a share of every list batch; slices are summed at the end.
        int nslices = 1;
        while (nt * nslices * 2 <= 32) nslices *= 2;
        const int width = 32 / nslices;
        const int slice = lane / width;
        const int tl = lane % width;
        const bool active = tl < nt;
        const int i = grp.x + (active ? tl : 0);
        const double px = bd.x[i], py = bd.y[i], pz = bd.z[i];
        // group bounding box (FP64), centre and half extents
        double lox = px, hix = px, loy = py, hiy = py, loz = pz, hiz = pz;
        for (int o = 16; o > 0; o >>= 1) {
            lox = fmin(lox, __shfl_xor_sync(0xffffffffu, lox, o)); hix = fmax(hix, __shfl_xor_sync(0xffffffffu, hix, o));
            loy = fmin(loy, __shfl_xor_sync(0xffffffffu, loy, o)); hiy = fmax(hiy, __shfl_xor_sync(0xffffffffu, hiy, o));
            loz = fmin(loz, __shfl_xor_sync(0xffffffffu, loz, o)); hiz = fmax(hiz, __shfl_xor_sync(0xffffffffu, hiz, o));
        }
        const double gcx = 0.5 * (lox + hix), gcy = 0.5 * (loy + hiy), gcz = 0.5 * (loz + hiz);
        const float fgx = static_cast<float>(gcx), fgy = static_cast<float>(gcy), fgz = static_cast<float>(gcz);
        // half extents, padded for the FP32 rounding of the centre and of the COMs
        const float pad = 1e-6f * (fabsf(fgx) + fabsf(fgy) + fabsf(fgz)) + 1e-30f;
        const float hx = static_cast<float>(0.5 * (hix - lox)) * 1.000001f + pad;
        const float hy = static_cast<float>(0.5 * (hiy - loy)) * 1.000001f + pad;
        const float hz = static_cast<float>(0.5 * (hiz - loz)) * 1.000001f + pad;
        Target T;
        T.tx = static_cast<float>(px - gcx); T.ty = static_cast<float>(py - gcy); T.tz = static_cast<float>(pz - gcz);
        T.ax = T.ay = T.az = T.pot = 0.f;
        T.cx = T.cy = T.cz = T.cp = 0.f;

        int sp = 1, pc_n = 0, pp_n = 0;
        if (lane == 0) stack[0] = grp.z;
        bool failed = false;
        unsigned long long g_pp = 0, g_pc = 0;
        __syncwarp();
        while (sp > 0) {
            const int nb = sp < 32 ? sp : 32;
            sp -= nb;
            const int node = lane < nb ? stack[sp + lane] : -1;
            __syncwarp();
            bool valid = node >= 0;
            float4 box = make_float4(0.f, 0.f, 0.f, -1.f);
            int2 lk = make_int2(0, 0);
            if (valid) {
                // index guard: the node, its children or its bodies must lie inside their arrays
                const bool in_range = static_cast<unsigned>(node) < nnodes32;
                if (in_range) { box = __ldg(t.box + node); lk = __ldg(t.link + node); }
                const unsigned end = static_cast<unsigned>(lk.x) + static_cast<unsigned>(lk.y > 0 ? lk.y : -lk.y);
                const bool bad = !in_range || lk.x < 0 || lk.y > 8 || end > (lk.y > 0 ? nnodes32 : nbodies32);
                if (bad) raise_error(err, kErrIndex);
                valid = !bad && box.w >= 0.f;
            }
            const float dx = fmaxf(fabsf(box.x - fgx) - hx, 0.f);
            const float dy = fmaxf(fabsf(box.y - fgy) - hy, 0.f);
            const float dz = fmaxf(fabsf(box.z - fgz) - hz, 0.f);
            const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            const bool open = valid && d2 < box.w;
            const bool leaf = lk.y <= 0;
            const bool accept = valid && !open;
            const int push = (open && !leaf) ? lk.y : 0;
            int remaining = (open && leaf) ? -lk.y : 0;
            // accepted cells -> PC list
            const uint32_t am = __ballot_sync(0xffffffffu, accept);
            if (accept) L.pc[pc_n + __popc(am & lt)] = node;
            pc_n += __popc(am);
            // children of opened cells -> stack
            int total;
            const int off = warp_excl_scan(push, lane, &total);
            if (sp + total > stack_cap) { failed = true; break; }
            for (int k = 0; k < push; ++k) stack[sp + off + k] = lk.x + k;
            sp += total;
            if (sp > max_sp) max_sp = sp;
            __syncwarp();
            if (pc_n >= 32) {
                eval_pc<QUAD, POT>(L, L.pc, 32, t, gcx, gcy, gcz, G, eps2, active, slice, nslices, T, lane);
                g_pc += 32;
                pc_n -= 32;
                const int v = lane < pc_n ? L.pc[32 + lane] : 0;
                __syncwarp();
                if (lane < pc_n) L.pc[lane] = v;
                __syncwarp();
            }
            // bodies of opened leaves -> PP list (in chunks of kPpChunk per lane)
            int src = lk.x;
            while (__any_sync(0xffffffffu, remaining > 0)) {
                const int take = remaining < kPpChunk ? remaining : kPpChunk;
                int tot;
                const int o2 = warp_excl_scan(take, lane, &tot);
                for (int k = 0; k < take; ++k) L.pp[pp_n + o2 + k] = src + k;
                pp_n += tot;
                src += take;
                remaining -= take;
                __syncwarp();
                int head = 0;
                while (pp_n - head >= 32) {
                    eval_pp<SOFT, POT>(L, L.pp + head, 32, bd, gcx, gcy, gcz, G, eps2, active, slice, nslices, T, lane);
                    g_pp += 32;
                    head += 32;
                }
                if (head > 0) {
                    pp_n -= head;
                    const int v = lane < pp_n ? L.pp[head + lane] : 0;
                    __syncwarp();
                    if (lane < pp_n) L.pp[lane] = v;
                    __syncwarp();
                }
            }
        }
        if (failed) {
            if (lane == 0) raise_error(err, kErrStack);
            continue;
        }
        if (pc_n > 0) { eval_pc<QUAD, POT>(L, L.pc, pc_n, t, gcx, gcy, gcz, G, eps2, active, slice, nslices, T, lane); g_pc += pc_n; }
        if (pp_n > 0) { eval_pp<SOFT, POT>(L, L.pp, pp_n, bd, gcx, gcy, gcz, G, eps2, active, slice, nslices, T, lane); g_pp += pp_n; }
        double fx = static_cast<double>(T.ax) - static_cast<double>(T.cx);
        double fy = static_cast<double>(T.ay) - static_cast<double>(T.cy);
        double fz = static_cast<double>(T.az) - static_cast<double>(T.cz);
        double fp = POT ? static_cast<double>(T.pot) - static_cast<double>(T.cp) : 0.0;
        for (int o = width; o < 32; o <<= 1) {
            fx += __shfl_xor_sync(0xffffffffu, fx, o);
            fy += __shfl_xor_sync(0xffffffffu, fy, o);
            fz += __shfl_xor_sync(0xffffffffu, fz, o);
            if (POT) fp += __shfl_xor_sync(0xffffffffu, fp, o);
        }
        if (active && slice == 0 && i >= own_lo && i < own_hi) {
            bd.ax[i] = fx;
            bd.ay[i] = fy;
            bd.az[i] = fz;
            if (POT && bd.pot) bd.pot[i] = fp;
        }
        npp += g_pp * own_nt;
        npc += g_pc * own_nt;
    }
    if (lane == 0) {
        if (npp) atomicAdd(stats + 0, npp);
        if (npc) atomicAdd(stats + 1, npc);
        atomicMax(stats + 2, static_cast<unsigned long long>(max_sp));
    }
}

template <bool QUAD, bool SOFT, bool POT>
cudaError_t launch_variant(const Bodies& bd, int64_t nbodies, const Tree& t, const Params& P, int warps, int stack_cap,
                           unsigned int* queue, unsigned long long* stats, int* err, int sm_count,
                           cudaStream_t st) {
    auto kern = walk_mixed_kernel<QUAD, SOFT, POT>;
    const size_t smem = (sizeof(WarpLists) + sizeof(int) * stack_cap) * warps;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * warps, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    e = cudaMemsetAsync(queue, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return e;
    kern<<<per_sm * sm_count, 32 * warps, smem, st>>>(bd, nbodies, t, static_cast<float>(P.G),
                                                     static_cast<float>(P.eps * P.eps), stack_cap, queue, stats, err,
                                                     P.own_lo, P.own_hi);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace

size_t walk_mixed_smem(int warps, int stack_cap) { return (sizeof(WarpLists) + sizeof(int) * stack_cap) * warps; }

cudaError_t launch_walk_mixed(const Bodies& bd, int64_t nbodies, const Tree& t, const Params& P, bool potential, int warps,
                              int stack_cap, unsigned int* queue, unsigned long long* stats, int* err,
                              int sm_count, cudaStream_t st) {
    const bool soft = P.eps > 0.0;
    if (P.quad) {
        if (soft) return potential ? launch_variant<true, true, true>(bd, nbodies, t, P, warps, stack_cap, queue, stats, err, sm_count, st)
                                   : launch_variant<true, true, false>(bd, nbodies, t, P, warps, stack_cap, queue, stats, err, sm_count, st);
        return potential ? launch_variant<true, false, true>(bd, nbodies, t, P, warps, stack_cap, queue, stats, err, sm_count, st)
                         : launch_variant<true, false, false>(bd, nbodies, t, P, warps, stack_cap, queue, stats, err, sm_count, st);
    }
    if (soft) return potential ? launch_variant<false, true, true>(bd, nbodies, t, P, warps, stack_cap, queue, stats, err, sm_count, st)
                               : launch_variant<false, true, false>(bd, nbodies, t, P, warps, stack_cap, queue, stats, err, sm_count, st);
    return potential ? launch_variant<false, false, true>(bd, nbodies, t, P, warps, stack_cap, queue, stats, err, sm_count, st)
                     : launch_variant<false, false, false>(bd, nbodies, t, P, warps, stack_cap, queue, stats, err, sm_count, st);
}

}  // namespace nb
