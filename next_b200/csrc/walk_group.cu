// Group force walk: one warp per group of <= 32 Morton-contiguous target
// bodies, in two arithmetics over the same traversal:
//   * FP32-mixed (NEXT_PRECISION_MIXED): FP32 interactions, compensated
//     accumulation;
//   * FP64 (NEXT_PRECISION_FP64_GROUP): the same interaction lists -- same
//     tree, groups and opening decisions -- evaluated in FP64, so the two
//     differ in precision only.
//
// Traversal: a per-warp LIFO stack of node ids in shared memory; each round
// pops up to 32 nodes (one per lane) and applies the opening test
//     open  <=>  dmin(group box, COM)^2 < rcrit^2,   rcrit = l/theta + |COM - centre|
// to all of them at once.  __ballot_sync / warp scans then append
//   - accepted cells to the particle-cell (PC) list,
//   - children of opened cells to the stack,
//   - bodies of opened leaves to the particle-particle (PP) list,
// all held in shared memory.  Whenever a list holds kBatch (64) entries, the
// warp stages them (two per lane: FP64 COM/position minus the FP64 group
// centre, rounded to FP32 -- coordinates relative to the group keep FP32
// exact enough near the group) and every lane runs the kBatch interactions
// for its target from shared memory with packed FP32 FMA and rsqrt.  The
// batch's partial sum is folded into the per-target sum with Kahan
// compensation.  The FP64 arithmetic stages the same entries in FP64 and
// sums them in FP64.
//
// Scheduling: persistent blocks (SM count x resident blocks) pull groups
// from a global atomic work queue.  All waits are warp-synchronous; there
// are no inter-block waits.  Stack or list overflow raises an error bit and
// abandons the group.
//
// Roofline: FP32 pipe (FP64 pipe for the FP64 arithmetic).  Algorithmic
// flops: 20 per PP, 56 per PC interaction.
#include "common.cuh"
#include "kernels.cuh"

namespace nb {

namespace {

// Compile-time knobs of the walk: unroll depth of a full batch, the minimum
// resident blocks the register allocation must allow, and the traversal's
// form (fixed-trip list expansion loops, ballot-based scans of the children
// and body counts, one or two nodes per lane and round).  The defaults are
// the fastest measured at 1,048,576 bodies.
#ifndef NB_WALK_UNROLL
#define NB_WALK_UNROLL 4
#endif
#ifndef NB_WALK_GENERIC_UNROLL
#define NB_WALK_GENERIC_UNROLL 1
#endif
#ifndef NB_WALK_FIXED
#define NB_WALK_FIXED 1
#endif
#ifndef NB_WALK_PACKED
#define NB_WALK_PACKED 1
#endif
#ifndef NB_WALK_PARTIAL_FIXED
#define NB_WALK_PARTIAL_FIXED 1
#endif
#ifndef NB_WALK_EXPAND_UNROLLED
#define NB_WALK_EXPAND_UNROLLED 2
#endif
#ifndef NB_WALK_PP_UNROLL
#define NB_WALK_PP_UNROLL 4
#endif
#ifndef NB_WALK_BALLOT_SCAN
#define NB_WALK_BALLOT_SCAN 2
#endif
#ifndef NB_WALK_SKIP_EMPTY_PUSH
#define NB_WALK_SKIP_EMPTY_PUSH 1
#endif
#ifndef NB_WALK_GM_FROM_QUAD
#define NB_WALK_GM_FROM_QUAD 1
#endif
#ifndef NB_WALK_PC_FACTORED
#define NB_WALK_PC_FACTORED 1
#endif
#ifndef NB_WALK_MIN_BLOCKS
#define NB_WALK_MIN_BLOCKS 5
#endif
#ifndef NB_WALK64_MIN_BLOCKS
#define NB_WALK64_MIN_BLOCKS 4
#endif

constexpr int kWalkUnroll = NB_WALK_UNROLL;
constexpr int kWalkGenericUnroll = NB_WALK_GENERIC_UNROLL;
// Entries per evaluation batch (32 or 64): every lane stages kBatch / 32.
#ifndef NB_WALK_BATCH
#define NB_WALK_BATCH 64
#endif
constexpr int kBatch = NB_WALK_BATCH;
static_assert(kBatch == 32 || kBatch == 64, "evaluation batches of 32 or 64 entries");
// Nodes popped per lane in each traversal round (1 or 2).
#ifndef NB_WALK_POP_SLOTS
#define NB_WALK_POP_SLOTS 1
#endif
constexpr int kSlots = NB_WALK_POP_SLOTS;
static_assert(kSlots == 1 || kSlots == 2, "one or two nodes per lane and round");
constexpr int kPcCap = kBatch + 32 * kSlots;
constexpr int kPpChunk = 16;
static_assert(kPpChunk < 32, "PP chunk counts are scanned as 5-bit values");
constexpr int kPpCap = kBatch + 32 * kPpChunk;

// Per-warp shared lists; STAGE_BYTES hold one staged evaluation batch.
template <int STAGE_BYTES>
struct WarpListsT {
    alignas(16) unsigned char stage[STAGE_BYTES];
    double gc[4];                // FP64 group centre, read back at each staging
    int pc[kPcCap];
    int pp[kPpCap];
};

// Exclusive warp scan of values in [0, 2^BITS) from one ballot per bit: the
// ballots are independent of one another and use no shuffles, so the scan
// stays off the shared-memory pipe that the evaluation's broadcasts load.
template <int BITS>
__device__ __forceinline__ int warp_excl_scan_bits(int v, uint32_t lt, int* total) {
    int off = 0, tot = 0;
#pragma unroll
    for (int b = 0; b < BITS; ++b) {
        const uint32_t m = __ballot_sync(0xffffffffu, (v >> b) & 1);
        off += __popc(m & lt) << b;
        tot += __popc(m) << b;
    }
    *total = tot;
    return off;
}

__device__ __forceinline__ int warp_excl_scan(int v, int lane, int* total) {
    int inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    *total = __shfl_sync(0xffffffffu, inc, 31);
    return inc - v;
}

// The walk runs at its register cap (96 per thread: 5 blocks of 4 warps per
// SM; with batches of 64 entries the extra registers of 5 blocks beat the
// extra warps of 6).  The FP64 group centre is read back from shared memory
// at each staging rather than held in six registers across the evaluation
// loops; the volatile read keeps the compiler from hoisting it back.
__device__ __forceinline__ double vld(const double& v) { return *reinterpret_cast<const volatile double*>(&v); }

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
// entry e[0] = (dx, dy, dz, G m) relative to the group centre, e[1] = -G (Qxx
// Qyy Qzz Qxy), e[2] = -G (Qxz Qyz - -).  56 algorithmic flops.  With the
// negated Q, qd = -Q d and q = -d.Q.d, so
//   a = (G m + 2.5 q_true / r^4) / r^3 d - Q d / r^5 = rinv3 (G m - 2.5 q rinv4) d + rinv5 qd.
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
        const float cc = rinv3 * fmaf(q, (-2.5f * rinv2) * rinv2, a.w);
        const float rinv5 = rinv3 * rinv2;
        sx = fmaf(cc, dx, fmaf(rinv5, qdx, sx));
        sy = fmaf(cc, dy, fmaf(rinv5, qdy, sy));
        sz = fmaf(cc, dz, fmaf(rinv5, qdz, sz));
        if (POT) sp = fmaf(0.5f * q, rinv5, fmaf(-a.w, rinv, sp));
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
    if (NB_WALK_FIXED && count == kBatch && nslices == 1) {
        run_fixed<kBatch, STRIDE, PC, F1, POT>(stage, 0, T, eps2, sx, sy, sz, sp);
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

// ---- packed evaluation: two list entries per FP32 instruction --------------
// Blackwell's .f32x2 add/mul/fma do two FP32 operations per issued
// instruction at the FMA pipe's full FLOP rate, and this walk is bound by
// instruction issue, not by the FMA pipe.  Entries are staged in pairs,
// interleaved field by field, so one LDS.128 delivers a field of both.
typedef unsigned long long f2;

__device__ __forceinline__ f2 pk(float lo, float hi) {
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float2 upk(f2 v) {
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
    return r;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b) {
    f2 d;
    asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
    f2 d;
    asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
    f2 d;
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

struct PairAcc {
    f2 x, y, z;
};

// Two body-cell interactions.  e[0] = (x0 x1 y0 y1), e[1] = (z0 z1 m0 m1),
// e[2..4] = -G (Qxx, Qyy | Qzz, Qxy | Qxz, Qyz) of both cells.
template <bool QUAD>
__device__ __forceinline__ void pc_pair(const float4* e, f2 tx, f2 ty, f2 tz, f2 eps2, f2 neg25, PairAcc& s) {
    const float4 p0 = e[0], p1 = e[1];
    const f2 dx = sub2(pk(p0.x, p0.y), tx), dy = sub2(pk(p0.z, p0.w), ty), dz = sub2(pk(p1.x, p1.y), tz);
    const f2 m = pk(p1.z, p1.w);
    const f2 r2 = fma2(dz, dz, fma2(dy, dy, fma2(dx, dx, eps2)));
    const float2 r2s = upk(r2);
    const f2 rinv = pk(rsqrtf(r2s.x), rsqrtf(r2s.y));
    const f2 rinv2 = mul2(rinv, rinv);
    const f2 rinv3 = mul2(rinv2, rinv);
    if (QUAD) {
        const float4 a = e[2], b = e[3], c = e[4];
        const f2 qxx = pk(a.x, a.y), qyy = pk(a.z, a.w), qzz = pk(b.x, b.y), qxy = pk(b.z, b.w);
        const f2 qxz = pk(c.x, c.y), qyz = pk(c.z, c.w);
        const f2 qdx = fma2(qxz, dz, fma2(qxy, dy, mul2(qxx, dx)));
        const f2 qdy = fma2(qyz, dz, fma2(qyy, dy, mul2(qxy, dx)));
        const f2 qdz = fma2(qzz, dz, fma2(qyz, dy, mul2(qxz, dx)));
        const f2 q = fma2(dz, qdz, fma2(dy, qdy, mul2(dx, qdx)));
        if (NB_WALK_PC_FACTORED) {
            // r2 rinv5 = rinv3, so a = rinv5 (qd + (G m r2 - 2.5 q rinv2) d):
            // 12 packed operations after q instead of 13
            const f2 rinv5 = mul2(mul2(rinv2, rinv2), rinv);
            const f2 k = fma2(mul2(q, rinv2), neg25, mul2(m, r2));
            s.x = fma2(rinv5, fma2(dx, k, qdx), s.x);
            s.y = fma2(rinv5, fma2(dy, k, qdy), s.y);
            s.z = fma2(rinv5, fma2(dz, k, qdz), s.z);
        } else {
            const f2 cc = mul2(rinv3, fma2(q, mul2(mul2(neg25, rinv2), rinv2), m));
            const f2 rinv5 = mul2(rinv3, rinv2);
            s.x = fma2(cc, dx, fma2(rinv5, qdx, s.x));
            s.y = fma2(cc, dy, fma2(rinv5, qdy, s.y));
            s.z = fma2(cc, dz, fma2(rinv5, qdz, s.z));
        }
    } else {
        const f2 mr3 = mul2(m, rinv3);
        s.x = fma2(mr3, dx, s.x);
        s.y = fma2(mr3, dy, s.y);
        s.z = fma2(mr3, dz, s.z);
    }
}

// Two body-body interactions.  e[0] = (x0 x1 y0 y1), e[1] = (z0 z1 m0 m1).
__device__ __forceinline__ void pp_pair(const float4* e, f2 tx, f2 ty, f2 tz, f2 eps2, PairAcc& s) {
    const float4 p0 = e[0], p1 = e[1];
    const f2 dx = sub2(pk(p0.x, p0.y), tx), dy = sub2(pk(p0.z, p0.w), ty), dz = sub2(pk(p1.x, p1.y), tz);
    const f2 m = pk(p1.z, p1.w);
    const f2 r2 = fma2(dz, dz, fma2(dy, dy, fma2(dx, dx, eps2)));
    const float2 r2s = upk(r2);
    const f2 rinv = pk(rsqrtf(r2s.x), rsqrtf(r2s.y));
    const f2 mr3 = mul2(mul2(m, rinv), mul2(rinv, rinv));
    s.x = fma2(mr3, dx, s.x);
    s.y = fma2(mr3, dy, s.y);
    s.z = fma2(mr3, dz, s.z);
}

template <int NPAIRS, int STRIDE, bool PC, bool QUAD>
__device__ __forceinline__ void run_pairs_fixed(const float4* stage, int p0, f2 tx, f2 ty, f2 tz, f2 eps2, f2 neg25,
                                                PairAcc& s) {
    const float4* e = stage + STRIDE * p0;
#pragma unroll kWalkUnroll
    for (int p = 0; p < NPAIRS; ++p) {
        if (PC) pc_pair<QUAD>(e + STRIDE * p, tx, ty, tz, eps2, neg25, s);
        else pp_pair(e + STRIDE * p, tx, ty, tz, eps2, s);
    }
}

// Packed counterpart of eval_batch: pairs [slice*npairs/nslices, ...).
template <int STRIDE, bool PC, bool QUAD>
__device__ __forceinline__ void eval_batch_packed(const float4* stage, int count, float eps2, bool active, int slice,
                                                  int nslices, Target& T) {
    if (!active) return;
    const f2 tx = pk(T.tx, T.tx), ty = pk(T.ty, T.ty), tz = pk(T.tz, T.tz);
    const f2 e2 = pk(eps2, eps2), neg25 = pk(-2.5f, -2.5f);
    PairAcc s{0ull, 0ull, 0ull};
    const int npairs = (count + 1) >> 1;
    if (NB_WALK_FIXED && npairs == kBatch / 2 && nslices == 1) {
        run_pairs_fixed<kBatch / 2, STRIDE, PC, QUAD>(stage, 0, tx, ty, tz, e2, neg25, s);
    } else {
        const int chunk = (npairs + nslices - 1) / nslices;
        const int p0 = slice * chunk;
        const int p1 = min(npairs, p0 + chunk);
        int p = p0;
        // partial batches and slices: runs of 8 pairs with a compile-time
        // trip count, then the rest one pair at a time
        if (NB_WALK_PARTIAL_FIXED)
            for (; p + 8 <= p1; p += 8) run_pairs_fixed<8, STRIDE, PC, QUAD>(stage, p, tx, ty, tz, e2, neg25, s);
        for (; p < p1; ++p) {
            if (PC) pc_pair<QUAD>(stage + STRIDE * p, tx, ty, tz, e2, neg25, s);
            else pp_pair(stage + STRIDE * p, tx, ty, tz, e2, s);
        }
    }
    const float2 sx = upk(s.x), sy = upk(s.y), sz = upk(s.z);
    kahan_add(T.ax, T.cx, sx.x + sx.y);
    kahan_add(T.ay, T.cy, sy.x + sy.y);
    kahan_add(T.az, T.cz, sz.x + sz.y);
}

// Stage up to kBatch cells of `list` (entries lane, lane + 32, ...) as a
// packed batch: pairs of entries interleaved field by field, 5 float4 per
// pair; entries past `count` are zero-mass.  Positions are FP64 COM minus the
// FP64 group centre, rounded to FP32.
template <bool QUAD>
__device__ __forceinline__ void stage_pc_packed(float4* stage, const int* list, int count, const Tree& t, double gcx,
                                                double gcy, double gcz, float G, int lane) {
    // both of the lane's entries are loaded before either is stored (1 M
    // bodies: walk 2.720 -> 2.708 ms against storing each as it arrives)
    constexpr int kPer = kBatch / 32;
    float v[kPer][10];
#pragma unroll
    for (int it = 0; it < kPer; ++it) {
        const int e = lane + 32 * it;
#pragma unroll
        for (int k = 0; k < 10; ++k) v[it][k] = 0.f;
        if (e < count) {
            const int node = list[e];
            const double4 c = t.com[node];
            v[it][0] = static_cast<float>(c.x - gcx);
            v[it][1] = static_cast<float>(c.y - gcy);
            v[it][2] = static_cast<float>(c.z - gcz);
            if (QUAD) {
                const float4 q0 = t.quad32[2 * node], q1 = t.quad32[2 * node + 1];
                v[it][3] = NB_WALK_GM_FROM_QUAD ? q1.z : static_cast<float>(G * c.w);
                v[it][4] = q0.x; v[it][5] = q0.y; v[it][6] = q0.z; v[it][7] = q0.w; v[it][8] = q1.x; v[it][9] = q1.y;
            } else {
                v[it][3] = static_cast<float>(G * c.w);
            }
        }
    }
#pragma unroll
    for (int it = 0; it < kPer; ++it) {
        const int e = lane + 32 * it;
        float* f = reinterpret_cast<float*>(stage + 5 * (e >> 1)) + (e & 1);
#pragma unroll
        for (int k = 0; k < 10; ++k) f[2 * k] = v[it][k];
    }
}

// Stage up to kBatch bodies of `list` as a packed batch, 2 float4 per pair.
__device__ __forceinline__ void stage_pp_packed(float4* stage, const int* list, int count, const Bodies& bd,
                                                double gcx, double gcy, double gcz, float G, int lane) {
    constexpr int kPer = kBatch / 32;
    float v[kPer][4];
#pragma unroll
    for (int it = 0; it < kPer; ++it) {
        const int e = lane + 32 * it;
#pragma unroll
        for (int k = 0; k < 4; ++k) v[it][k] = 0.f;
        if (e < count) {
            const int j = list[e];
            v[it][0] = static_cast<float>(bd.x[j] - gcx);
            v[it][1] = static_cast<float>(bd.y[j] - gcy);
            v[it][2] = static_cast<float>(bd.z[j] - gcz);
            v[it][3] = static_cast<float>(G * bd.m[j]);
        }
    }
#pragma unroll
    for (int it = 0; it < kPer; ++it) {
        const int e = lane + 32 * it;
        float* f = reinterpret_cast<float*>(stage + 2 * (e >> 1)) + (e & 1);
#pragma unroll
        for (int k = 0; k < 4; ++k) f[2 * k] = v[it][k];
    }
}

// Stage up to 32 cells (one per lane) and evaluate them.  PACK stages them in
// pairs for the .f32x2 path (lanes past `count` stage zero-mass entries).
template <bool QUAD, bool POT, bool PACK>
__device__ __forceinline__ void eval_pc(float4* stage, const int* list, int count, const Tree& t, double gcx,
                                        double gcy, double gcz, float G, float eps2, bool active, int slice,
                                        int nslices, Target& T, int lane) {
    if (PACK) {
        stage_pc_packed<QUAD>(stage, list, count, t, gcx, gcy, gcz, G, lane);
        __syncwarp();
        eval_batch_packed<5, true, QUAD>(stage, count, eps2, active, slice, nslices, T);
        __syncwarp();
    } else {
        for (int e = lane; e < count; e += 32) {
            const int node = list[e];
            const double4 c = t.com[node];
            stage[3 * e + 0] = make_float4(static_cast<float>(c.x - gcx), static_cast<float>(c.y - gcy),
                                           static_cast<float>(c.z - gcz), static_cast<float>(G * c.w));
            if (QUAD) {
                stage[3 * e + 1] = t.quad32[2 * node];
                stage[3 * e + 2] = t.quad32[2 * node + 1];
            }
        }
        __syncwarp();
        eval_batch<3, true, QUAD, POT>(stage, count, eps2, active, slice, nslices, T);
        __syncwarp();
    }
}

// Stage up to 32 bodies (one per lane) and evaluate them.
template <bool SOFT, bool POT, bool PACK>
__device__ __forceinline__ void eval_pp(float4* stage, const int* list, int count, const Bodies& bd, double gcx,
                                        double gcy, double gcz, float G, float eps2, bool active, int slice,
                                        int nslices, Target& T, int lane) {
    if (PACK) {
        stage_pp_packed(stage, list, count, bd, gcx, gcy, gcz, G, lane);
        __syncwarp();
        eval_batch_packed<2, false, false>(stage, count, eps2, active, slice, nslices, T);
        __syncwarp();
    } else {
        for (int e = lane; e < count; e += 32) {
            const int j = list[e];
            stage[e] = make_float4(static_cast<float>(bd.x[j] - gcx), static_cast<float>(bd.y[j] - gcy),
                                   static_cast<float>(bd.z[j] - gcz), static_cast<float>(G * bd.m[j]));
        }
        __syncwarp();
        eval_batch<1, false, SOFT, POT>(stage, count, eps2, active, slice, nslices, T);
        __syncwarp();
    }
}

// ---- the two arithmetics of the walk -----------------------------------------
// Each provides the staging buffer size, the per-lane accumulator, the
// evaluation of a PC and a PP batch, and the final FP64 sums.

template <bool QUAD, bool SOFT, bool POT>
struct MixedArith {
    using Scalar = float;
    // softened forces without the potential take the packed two-entry path
    static constexpr bool kPack = NB_WALK_PACKED && SOFT && !POT;
    static constexpr int kStageBytes = 3 * kBatch * sizeof(float4);
    static constexpr int kMinBlocks = NB_WALK_MIN_BLOCKS;
    static constexpr bool kPot = POT;
    using Acc = Target;
    __device__ static void start(Acc& T, double px, double py, double pz, double gcx, double gcy, double gcz) {
        T.tx = static_cast<float>(px - gcx); T.ty = static_cast<float>(py - gcy); T.tz = static_cast<float>(pz - gcz);
        T.ax = T.ay = T.az = T.pot = 0.f;
        T.cx = T.cy = T.cz = T.cp = 0.f;
    }
    __device__ static void pc(unsigned char* stage, const int* list, int count, const Tree& t, const Bodies&,
                              double gcx, double gcy, double gcz, float G, float eps2, bool active, int slice,
                              int nslices, Acc& T, int lane) {
        eval_pc<QUAD, POT, kPack>(reinterpret_cast<float4*>(stage), list, count, t, gcx, gcy, gcz, G, eps2, active,
                                  slice, nslices, T, lane);
    }
    __device__ static void pp(unsigned char* stage, const int* list, int count, const Tree&, const Bodies& bd,
                              double gcx, double gcy, double gcz, float G, float eps2, bool active, int slice,
                              int nslices, Acc& T, int lane) {
        eval_pp<SOFT, POT, kPack>(reinterpret_cast<float4*>(stage), list, count, bd, gcx, gcy, gcz, G, eps2, active,
                                  slice, nslices, T, lane);
    }
    __device__ static void finish(const Acc& T, double& fx, double& fy, double& fz, double& fp) {
        fx = static_cast<double>(T.ax) - static_cast<double>(T.cx);
        fy = static_cast<double>(T.ay) - static_cast<double>(T.cy);
        fz = static_cast<double>(T.az) - static_cast<double>(T.cz);
        fp = POT ? static_cast<double>(T.pot) - static_cast<double>(T.cp) : 0.0;
    }
};

// FP64: entries staged as 10 (PC) or 4 (PP) doubles relative to the group
// centre, -G Q for the quadrupole; FP64 FMA and rsqrt, FP64 sums.
template <bool QUAD, bool SOFT, bool POT>
struct Fp64Arith {
    using Scalar = double;
    static constexpr int kStageBytes = kBatch * 10 * sizeof(double);
    static constexpr int kMinBlocks = NB_WALK64_MIN_BLOCKS;
    static constexpr bool kPot = POT;
    struct Acc {
        double tx, ty, tz, ax, ay, az, pot;
    };
    __device__ static void start(Acc& A, double px, double py, double pz, double gcx, double gcy, double gcz) {
        A.tx = px - gcx; A.ty = py - gcy; A.tz = pz - gcz;
        A.ax = A.ay = A.az = A.pot = 0.0;
    }
    // one body-cell term: a = rinv3 (G m - 2.5 q rinv4) d + rinv5 qd with the
    // negated Q staged (qd = -G Q d, q = -G d.Q.d), as the FP32 pc_term
    __device__ static void pc_term(const double* e, Acc& A, double eps2) {
        const double dx = e[0] - A.tx, dy = e[1] - A.ty, dz = e[2] - A.tz, m = e[3];
        const double r2 = fma(dz, dz, fma(dy, dy, fma(dx, dx, eps2)));
        const double rinv = rsqrt(r2);
        const double rinv2 = rinv * rinv;
        const double rinv3 = rinv2 * rinv;
        if (QUAD) {
            const double qdx = fma(e[8], dz, fma(e[7], dy, e[4] * dx));
            const double qdy = fma(e[9], dz, fma(e[5], dy, e[7] * dx));
            const double qdz = fma(e[6], dz, fma(e[9], dy, e[8] * dx));
            const double q = fma(dz, qdz, fma(dy, qdy, dx * qdx));
            const double cc = rinv3 * fma(q, (-2.5 * rinv2) * rinv2, m);
            const double rinv5 = rinv3 * rinv2;
            A.ax = fma(cc, dx, fma(rinv5, qdx, A.ax));
            A.ay = fma(cc, dy, fma(rinv5, qdy, A.ay));
            A.az = fma(cc, dz, fma(rinv5, qdz, A.az));
            if (POT) A.pot = fma(0.5 * q, rinv5, fma(-m, rinv, A.pot));
        } else {
            const double mr3 = m * rinv3;
            A.ax = fma(mr3, dx, A.ax);
            A.ay = fma(mr3, dy, A.ay);
            A.az = fma(mr3, dz, A.az);
            if (POT) A.pot = fma(-m, rinv, A.pot);
        }
    }
    __device__ static void pp_term(const double* e, Acc& A, double eps2) {
        const double dx = e[0] - A.tx, dy = e[1] - A.ty, dz = e[2] - A.tz;
        const double r2 = fma(dz, dz, fma(dy, dy, fma(dx, dx, eps2)));
        double rinv = rsqrt(r2);
        if (!SOFT) rinv = r2 > 0.0 ? rinv : 0.0;     // the target itself, unsoftened
        const double mr = e[3] * rinv;
        const double mr3 = mr * rinv * rinv;
        A.ax = fma(mr3, dx, A.ax);
        A.ay = fma(mr3, dy, A.ay);
        A.az = fma(mr3, dz, A.az);
        if (POT) A.pot -= r2 > eps2 ? mr : 0.0;        // no self term
    }
    template <int STRIDE, bool PC>
    __device__ static void run(const double* st, int count, double eps2, bool active, int slice, int nslices,
                               Acc& A) {
        if (!active) return;
        const int chunk = (count + nslices - 1) / nslices;
        const int k0 = slice * chunk;
        const int k1 = min(count, k0 + chunk);
#pragma unroll 4
        for (int k = k0; k < k1; ++k) {
            if (PC) pc_term(st + STRIDE * k, A, eps2);
            else pp_term(st + STRIDE * k, A, eps2);
        }
    }
    __device__ static void pc(unsigned char* stage, const int* list, int count, const Tree& t, const Bodies&,
                              double gcx, double gcy, double gcz, double G, double eps2, bool active, int slice,
                              int nslices, Acc& A, int lane) {
        double* st = reinterpret_cast<double*>(stage);
        for (int k = lane; k < count; k += 32) {
            const int node = list[k];
            const double4 c = t.com[node];
            double* e = st + 10 * k;
            e[0] = c.x - gcx; e[1] = c.y - gcy; e[2] = c.z - gcz; e[3] = G * c.w;
            if (QUAD) {
                const double* q = t.quad64 + 8 * static_cast<int64_t>(node);
#pragma unroll
                for (int f = 0; f < 6; ++f) e[4 + f] = -G * q[f];
            }
        }
        __syncwarp();
        run<10, true>(st, count, eps2, active, slice, nslices, A);
        __syncwarp();
    }
    __device__ static void pp(unsigned char* stage, const int* list, int count, const Tree&, const Bodies& bd,
                              double gcx, double gcy, double gcz, double G, double eps2, bool active, int slice,
                              int nslices, Acc& A, int lane) {
        double* st = reinterpret_cast<double*>(stage);
        for (int k = lane; k < count; k += 32) {
            const int j = list[k];
            double* e = st + 4 * k;
            e[0] = bd.x[j] - gcx; e[1] = bd.y[j] - gcy; e[2] = bd.z[j] - gcz; e[3] = G * bd.m[j];
        }
        __syncwarp();
        run<4, false>(st, count, eps2, active, slice, nslices, A);
        __syncwarp();
    }
    __device__ static void finish(const Acc& A, double& fx, double& fy, double& fz, double& fp) {
        fx = A.ax; fy = A.ay; fz = A.az; fp = POT ? A.pot : 0.0;
    }
};

template <class A>
__global__ void __launch_bounds__(128, A::kMinBlocks)
walk_group_kernel(Bodies bd, int64_t nbodies, Tree t, typename A::Scalar G, typename A::Scalar eps2, int stack_cap,
                  unsigned int* queue, unsigned long long* stats, int* err, int64_t own_lo, int64_t own_hi) {
    if (*err & kErrAbort) return;
    using WarpLists = WarpListsT<A::kStageBytes>;
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
        const unsigned own_nt = static_cast<unsigned>(own_end - own_first);
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
        typename A::Acc T;
        A::start(T, px, py, pz, gcx, gcy, gcz);

        int sp = 1, pc_n = 0, pp_n = 0;
        if (lane == 0) stack[0] = grp.z;
        bool failed = false;
        unsigned g_pp = 0, g_pc = 0;
        if (lane == 0) { L.gc[0] = gcx; L.gc[1] = gcy; L.gc[2] = gcz; }
        __syncwarp();
        while (sp > 0) {
            // pop up to 32 * kSlots nodes: slot k of lane l holds stack[sp + 32 k + l]
            const int nb = sp < 32 * kSlots ? sp : 32 * kSlots;
            sp -= nb;
            int node[kSlots];
#pragma unroll
            for (int k = 0; k < kSlots; ++k) node[k] = lane + 32 * k < nb ? stack[sp + 32 * k + lane] : -1;
            __syncwarp();
            float4 box[kSlots];
            int2 lk[kSlots];
            bool valid[kSlots];
#pragma unroll
            for (int k = 0; k < kSlots; ++k) {
                valid[k] = node[k] >= 0;
                box[k] = make_float4(0.f, 0.f, 0.f, -1.f);
                lk[k] = make_int2(0, 0);
                // index guard: the node, its children or its bodies must lie inside their arrays
                if (valid[k] && static_cast<unsigned>(node[k]) < nnodes32) {
                    box[k] = __ldg(t.box + node[k]);
                    lk[k] = __ldg(t.link + node[k]);
                }
            }
            int push[kSlots], rem[kSlots];
#pragma unroll
            for (int k = 0; k < kSlots; ++k) {
                if (valid[k]) {
                    const bool in_range = static_cast<unsigned>(node[k]) < nnodes32;
                    const unsigned end = static_cast<unsigned>(lk[k].x) +
                                         static_cast<unsigned>(lk[k].y > 0 ? lk[k].y : -lk[k].y);
                    const bool bad = !in_range || lk[k].x < 0 || lk[k].y > 8 ||
                                     end > (lk[k].y > 0 ? nnodes32 : nbodies32);
                    if (bad) raise_error(err, kErrIndex);
                    valid[k] = !bad && box[k].w >= 0.f;
                }
                const float dx = fmaxf(fabsf(box[k].x - fgx) - hx, 0.f);
                const float dy = fmaxf(fabsf(box[k].y - fgy) - hy, 0.f);
                const float dz = fmaxf(fabsf(box[k].z - fgz) - hz, 0.f);
                const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                const bool open = valid[k] && d2 < box[k].w;
                const bool leaf = lk[k].y <= 0;
                const bool accept = valid[k] && !open;
                push[k] = (open && !leaf) ? lk[k].y : 0;
                rem[k] = (open && leaf) ? -lk[k].y : 0;
                // accepted cells -> PC list
                const uint32_t am = __ballot_sync(0xffffffffu, accept);
                if (accept) L.pc[pc_n + __popc(am & lt)] = node[k];
                pc_n += __popc(am);
            }
            // children of opened cells -> stack
            int push_all = 0;
#pragma unroll
            for (int k = 0; k < kSlots; ++k) push_all += push[k];
            int total;
            const int off = NB_WALK_BALLOT_SCAN ? warp_excl_scan_bits<kSlots == 1 ? 4 : 5>(push_all, lt, &total)
                                                : warp_excl_scan(push_all, lane, &total);
            if (sp + total > stack_cap) { failed = true; break; }
            int o = off;
#pragma unroll
            for (int k = 0; k < kSlots; ++k) {
                if (NB_WALK_SKIP_EMPTY_PUSH && total == 0) break;   // warp-uniform
                if (NB_WALK_EXPAND_UNROLLED) {
#pragma unroll
                    for (int c = 0; c < 8; ++c)
                        if (c < push[k]) stack[sp + o + c] = lk[k].x + c;
                } else {
                    for (int c = 0; c < push[k]; ++c) stack[sp + o + c] = lk[k].x + c;
                }
                o += push[k];
            }
            sp += total;
            if (sp > max_sp) max_sp = sp;
            __syncwarp();
            if (pc_n >= kBatch) {
                A::pc(L.stage, L.pc, kBatch, t, bd, vld(L.gc[0]), vld(L.gc[1]), vld(L.gc[2]), G, eps2, active, slice,
                      nslices, T, lane);
                g_pc += kBatch;
                pc_n -= kBatch;               // < 32 * kSlots left over
#pragma unroll
                for (int e0 = 0; e0 < 32 * kSlots; e0 += 32) {
                    const int v = e0 + lane < pc_n ? L.pc[kBatch + e0 + lane] : 0;
                    __syncwarp();
                    if (e0 + lane < pc_n) L.pc[e0 + lane] = v;
                    __syncwarp();
                }
            }
            // bodies of opened leaves -> PP list (in chunks of kPpChunk per lane;
            // a lane drains its slot-0 leaf, then its slot-1 leaf)
            int remaining = rem[0];
            int src = lk[0].x;
            int rem2 = kSlots > 1 ? rem[kSlots - 1] : 0;
            int src2 = kSlots > 1 ? lk[kSlots - 1].x : 0;
            while (__any_sync(0xffffffffu, remaining > 0 || rem2 > 0)) {
                if (kSlots > 1 && remaining <= 0) { remaining = rem2; src = src2; rem2 = 0; }
                const int take = remaining < kPpChunk ? remaining : kPpChunk;
                int tot;
                const int o2 = NB_WALK_BALLOT_SCAN > 1 ? warp_excl_scan_bits<5>(take, lt, &tot)
                                                       : warp_excl_scan(take, lane, &tot);
                if (NB_WALK_EXPAND_UNROLLED > 1) {
                    for (int k0 = 0; k0 < take; k0 += NB_WALK_PP_UNROLL) {
#pragma unroll
                        for (int k = k0; k < k0 + NB_WALK_PP_UNROLL; ++k)
                            if (k < take) L.pp[pp_n + o2 + k] = src + k;
                    }
                } else {
                    for (int k = 0; k < take; ++k) L.pp[pp_n + o2 + k] = src + k;
                }
                pp_n += tot;
                src += take;
                remaining -= take;
                __syncwarp();
                int head = 0;
                while (pp_n - head >= kBatch) {
                    A::pp(L.stage, L.pp + head, kBatch, t, bd, vld(L.gc[0]), vld(L.gc[1]), vld(L.gc[2]), G, eps2,
                          active, slice, nslices, T, lane);
                    g_pp += kBatch;
                    head += kBatch;
                }
                if (head > 0) {
                    pp_n -= head;                 // < kBatch left over
#pragma unroll
                    for (int e0 = 0; e0 < kBatch; e0 += 32) {
                        const int v = e0 + lane < pp_n ? L.pp[head + e0 + lane] : 0;
                        __syncwarp();
                        if (e0 + lane < pp_n) L.pp[e0 + lane] = v;
                        __syncwarp();
                    }
                }
            }
        }
        if (failed) {
            if (lane == 0) raise_error(err, kErrStack);
            continue;
        }
        if (pc_n > 0) {
            A::pc(L.stage, L.pc, pc_n, t, bd, vld(L.gc[0]), vld(L.gc[1]), vld(L.gc[2]), G, eps2, active, slice,
                  nslices, T, lane);
            g_pc += pc_n;
        }
        if (pp_n > 0) {
            A::pp(L.stage, L.pp, pp_n, t, bd, vld(L.gc[0]), vld(L.gc[1]), vld(L.gc[2]), G, eps2, active, slice,
                  nslices, T, lane);
            g_pp += pp_n;
        }
        double fx, fy, fz, fp;
        A::finish(T, fx, fy, fz, fp);
        for (int o = width; o < 32; o <<= 1) {
            fx += __shfl_xor_sync(0xffffffffu, fx, o);
            fy += __shfl_xor_sync(0xffffffffu, fy, o);
            fz += __shfl_xor_sync(0xffffffffu, fz, o);
            if (A::kPot) fp += __shfl_xor_sync(0xffffffffu, fp, o);
        }
        if (active && slice == 0 && i >= own_lo && i < own_hi) {
            bd.ax[i] = fx;
            bd.ay[i] = fy;
            bd.az[i] = fz;
            if (A::kPot && bd.pot) bd.pot[i] = fp;
        }
        npp += static_cast<unsigned long long>(g_pp) * own_nt;
        npc += static_cast<unsigned long long>(g_pc) * own_nt;
    }
    if (lane == 0) {
        if (npp) atomicAdd(stats + 0, npp);
        if (npc) atomicAdd(stats + 1, npc);
        atomicMax(stats + 2, static_cast<unsigned long long>(max_sp));
    }
}

template <class A>
cudaError_t launch_variant(const Bodies& bd, int64_t nbodies, const Tree& t, const Params& P, int warps, int stack_cap,
                           unsigned int* queue, unsigned long long* stats, int* err, int sm_count,
                           cudaStream_t st) {
    auto kern = walk_group_kernel<A>;
    const size_t smem = (sizeof(WarpListsT<A::kStageBytes>) + sizeof(int) * stack_cap) * warps;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * warps, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    e = cudaMemsetAsync(queue, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return e;
    using S = typename A::Scalar;
    kern<<<per_sm * sm_count, 32 * warps, smem, st>>>(bd, nbodies, t, static_cast<S>(P.G),
                                                     static_cast<S>(P.eps * P.eps), stack_cap, queue, stats, err,
                                                     P.own_lo, P.own_hi);
    count_launches(1);
    return cudaGetLastError();
}

template <template <bool, bool, bool> class Arith>
cudaError_t launch_arith(const Bodies& bd, int64_t nbodies, const Tree& t, const Params& P, bool potential, int warps,
                         int stack_cap, unsigned int* queue, unsigned long long* stats, int* err, int sm_count,
                         cudaStream_t st) {
    const bool soft = P.eps > 0.0;
#define NB_WALK_CASE(Q, S, POT)                                                                                  \
    if (P.quad == Q && soft == S && potential == POT)                                                            \
        return launch_variant<Arith<Q, S, POT>>(bd, nbodies, t, P, warps, stack_cap, queue, stats, err, sm_count, st);
    NB_WALK_CASE(true, true, false)
    NB_WALK_CASE(true, true, true)
    NB_WALK_CASE(true, false, false)
    NB_WALK_CASE(true, false, true)
    NB_WALK_CASE(false, true, false)
    NB_WALK_CASE(false, true, true)
    NB_WALK_CASE(false, false, false)
    NB_WALK_CASE(false, false, true)
#undef NB_WALK_CASE
    return cudaErrorInvalidValue;
}

}  // namespace

size_t walk_group_smem(bool fp64, int warps, int stack_cap) {
    const size_t lists = fp64 ? sizeof(WarpListsT<Fp64Arith<true, true, false>::kStageBytes>)
                              : sizeof(WarpListsT<MixedArith<true, true, false>::kStageBytes>);
    return (lists + sizeof(int) * stack_cap) * warps;
}

cudaError_t launch_walk_group(const Bodies& bd, int64_t nbodies, const Tree& t, const Params& P, bool potential,
                              bool fp64, int warps, int stack_cap, unsigned int* queue, unsigned long long* stats,
                              int* err, int sm_count, cudaStream_t st) {
    if (fp64)
        return launch_arith<Fp64Arith>(bd, nbodies, t, P, potential, warps, stack_cap, queue, stats, err, sm_count, st);
    return launch_arith<MixedArith>(bd, nbodies, t, P, potential, warps, stack_cap, queue, stats, err, sm_count, st);
}

}  // namespace nb
