// Octree build from sorted octant keys, and the upward (moment) pass.
//
// A cell at level l is a run of sorted keys sharing their first l octant
// digits.  With d[s] = shared-prefix level of keys s-1 and s (-1 where a
// system starts), position s starts exactly the cells of levels > d[s]; the
// cell (l, s) holds more than B bodies iff the next B keys all share l
// digits with their predecessor, i.e. l <= min(d[s+1..s+B]).  So the
// internal cells (more than B bodies, above the deepest level) starting at s
// are the levels d[s]+1 .. min(min(d[s+1..s+B]), levels-1): counted per
// position, scanned, and materialised in one pass each -- no level-by-level
// loop.  For B = 1 this is exactly the tree the reference's one-body-per-
// leaf insertion builds (src/gravity/octree.h:69-87).
//
// Numbering: internal cells get a depth-first id q (position, then level);
// nodes are laid out sibling-contiguous (children of a node consecutive, in
// octant order, system roots first) for the walks.
//
// Child bounds: one thread per internal cell runs the eight lower-bound
// searches for the cell's end and child starts together.
//
// Upward pass, two launches and no per-level loop: one thread per leaf
// computes the leaf's moments and counts itself in at its parent; parents
// whose children are all leaves are then complete and go on a ready list.
// The second launch runs one thread per ready parent: it combines the
// children and climbs, an atomic arrival counter at each parent electing the
// last child's thread to combine all children in octant order
// (deterministic) and climb on.  With accurate physics a leaf's bodies and a
// cell's children are each read in one pass (moments about the first one,
// shifted to the centre of mass by the parallel-axis rule); the reference's
// physics keeps its own two-pass order for bit-exact moments.  The one-launch
// form (each leaf's thread climbing) is kept behind NB_UP_SPLIT=0.
//
// Built with -fmad=false: every FP64 + and * rounds separately, so the
// reference-mode moments repeat src/gravity/octree.h:92-127 bit for bit.
#include "common.cuh"
#include "kernels.cuh"

namespace nb {

namespace {

__global__ void dlev_kernel(const uint64_t* __restrict__ keys, int64_t n, int base, int levels,
                            int8_t* __restrict__ dlev) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    dlev[s] = static_cast<int8_t>(s == 0 ? -1 : shared_levels(keys[s - 1], keys[s], base, levels));
}

// Internal cells starting at each position; *deepest gets the deepest leaf
// level (one below the deepest internal cell) of the build, or
// kDepthOverfull if a cell at the last key level holds more than leaf_cap.
__global__ void nint_kernel(const int8_t* __restrict__ dlev, int64_t n, int leaf_cap, int levels,
                            int32_t* __restrict__ nint, unsigned long long* deepest) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    unsigned deep = 0;
    if (s < n) {
        int mb = -1;
        if (s + leaf_cap < n) {
            mb = 127;
            for (int j = 1; j <= leaf_cap; ++j) mb = min(mb, static_cast<int>(dlev[s + j]));
        }
        const int top = min(mb, levels - 1);
        const int c = max(0, top - static_cast<int>(dlev[s]));
        nint[s] = c;
        if (c > 0) deep = static_cast<unsigned>(top + 1);
        if (mb >= levels) deep = kDepthOverfull;
    }
    // block maximum, then one atomic per block, skipped when it cannot raise
    // the value (one hot address: unconditional atomics cost more than the pass)
    __shared__ unsigned warp_max[32];
    deep = __reduce_max_sync(0xffffffffu, deep);
    if ((threadIdx.x & 31) == 0) warp_max[threadIdx.x >> 5] = deep;
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned v = threadIdx.x < (blockDim.x >> 5) ? warp_max[threadIdx.x] : 0u;
        v = __reduce_max_sync(0xffffffffu, v);
        if (threadIdx.x == 0 && v > *reinterpret_cast<volatile unsigned long long*>(deepest))
            atomicMax(deepest, static_cast<unsigned long long>(v));
    }
}

// Walk groups from the children of one cell holding more than G bodies:
// the bodies of consecutive children of at most G bodies are cut into runs
// of G in key order (a child that does not fit tops the current run up to G
// and starts the next one with the rest of its bodies), so most groups fill
// a warp; a child of more than G bodies that is a leaf (deepest level) is
// cut into chunks of G.  emit(start, count) is called per group; returns
// the count.
template <typename F>
__device__ int pack_groups(const int32_t* b, int level, int levels, int leaf_cap, int group_cap, F emit) {
    int ng = 0, run_start = -1, run_cnt = 0;
    for (int c = 0; c < 8; ++c) {
        const int cnt = b[c + 1] - b[c];
        if (cnt == 0) continue;
        if (cnt <= group_cap) {
            if (run_start >= 0 && run_cnt + cnt <= group_cap) {
                run_cnt += cnt;
            } else if (run_start >= 0) {
                // top the run up to group_cap with the first bodies of this
                // child and go on with the rest of it: full warps
                const int take = group_cap - run_cnt;
                emit(run_start, group_cap); ++ng;
                run_start = b[c] + take; run_cnt = cnt - take;
            } else {
                run_start = b[c]; run_cnt = cnt;
            }
        } else {
            if (run_start >= 0) { emit(run_start, run_cnt); ++ng; run_start = -1; run_cnt = 0; }
            const bool leaf = !(cnt > leaf_cap && level + 1 < levels);
            if (leaf)
                for (int o = 0; o < cnt; o += group_cap) { emit(b[c] + o, min(group_cap, cnt - o)); ++ng; }
        }
    }
    if (run_start >= 0) { emit(run_start, run_cnt); ++ng; }
    return ng;
}

// Internal cell ids: position s starts the cells q = int_base[s] + k at
// levels dlev[s] + 1 + k.  Compacts them so the search kernel below runs one
// thread per cell rather than per position.
__global__ void cell_starts_kernel(const int8_t* __restrict__ dlev, const int32_t* __restrict__ int_base,
                                   int64_t n, Tree t, int* err) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int q0 = int_base[s];
    const int cnt = int_base[s + 1] - q0;
    if (cnt == 0) return;
    const int d = dlev[s];
    for (int k = 0; k < cnt; ++k) {
        const int64_t q = static_cast<int64_t>(q0) + k;
        if (q >= t.cap_int) { raise_error(err, kErrTree); return; }
        t.int_start[q] = static_cast<int32_t>(s);
        t.int_level[q] = static_cast<int8_t>(d + 1 + k);
    }
}

// Child boundaries of every internal cell (l, s): the cell ends at the first
// key above its prefix, and child c starts at the first key >= prefix | c at
// level l+1.  All eight are lower bounds over the same range [s, system end),
// run together with one shared step sequence (the range halves every step
// whatever the comparisons give), so a thread has eight independent loads in
// flight per step and no divergence.
#ifndef NB_INT_SCAN
#define NB_INT_SCAN 128
#endif
__global__ void __launch_bounds__(256)
internal_kernel(const uint64_t* __restrict__ keys, int64_t n, const int32_t* __restrict__ sysid,
                const int64_t* __restrict__ offsets, int base, int levels, int leaf_cap, int group_cap, Tree t,
                int* err) {
    if (*err & kErrAbort) return;
    const int64_t m = t.counts[0] < t.cap_int ? t.counts[0] : t.cap_int;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < m; q += (int64_t)gridDim.x * blockDim.x) {
        const int s = t.int_start[q];
        const int l = t.int_level[q];
        if (s < 0 || s >= n || l < 0 || l >= levels) { raise_error(err, kErrIndex); continue; }
        const int64_t hi = offsets ? offsets[(sysid ? sysid[s] : 0) + 1] : n;
        const uint64_t ks = keys[s];
        const int sh = base - 3 * l;                       // bits below level l's digits
        const uint64_t low = (sh >= 64) ? ~0ull : ((1ull << sh) - 1ull);
        const uint64_t prefix = ks & ~low;
        const int csh = sh - 3;
        uint64_t v[8];
        v[0] = (prefix | low) + 1ull;                      // end of the cell
#pragma unroll
        for (int c = 1; c < 8; ++c) v[c] = prefix | (static_cast<uint64_t>(c) << csh);
        // A small cell's end is the first p > s whose key shares fewer than l
        // digits with its predecessor (dlev[p] < l): found by reading dlev
        // forward, 16 positions per round trip, for up to NB_INT_SCAN
        // positions; the children's searches then run over the cell only.
        int64_t e = -1;
        if (NB_INT_SCAN > 0) {
            const int64_t lim = hi < static_cast<int64_t>(s) + 1 + NB_INT_SCAN ? hi : static_cast<int64_t>(s) + 1 + NB_INT_SCAN;
            for (int64_t p0 = static_cast<int64_t>(s) + 1; p0 < lim && e < 0; p0 += 16) {
                int dv[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) dv[j] = p0 + j < lim ? t.dlev[p0 + j] : 127;
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    if (e < 0 && dv[j] < l) e = p0 + j;
            }
            if (e < 0 && lim == hi) e = hi;
        }
        int64_t pos[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) pos[c] = s;
        int64_t len = (e >= 0 ? e : hi) - s;
        while (len > 1) {
            const int64_t half = len >> 1;
#pragma unroll
            for (int c = 0; c < 8; ++c) pos[c] = __ldg(keys + pos[c] + half) < v[c] ? pos[c] + half : pos[c];
            len -= half;
        }
        int32_t b[9];
        b[0] = s;
#pragma unroll
        for (int c = 1; c < 8; ++c) b[c] = static_cast<int32_t>(pos[c] + (__ldg(keys + pos[c]) < v[c] ? 1 : 0));
        b[8] = e >= 0 ? static_cast<int32_t>(e) : static_cast<int32_t>(pos[0] + (__ldg(keys + pos[0]) < v[0] ? 1 : 0));
        int nchild = 0;
        for (int c = 0; c < 8; ++c) nchild += b[c + 1] > b[c];
        int ngroups = 0;
        if (b[8] - b[0] > group_cap)
            ngroups = pack_groups(b, l, levels, leaf_cap, group_cap, [](int, int) {});
        for (int c = 0; c < 9; ++c) t.int_bounds[9 * q + c] = b[c];
        t.int_packed[q] = static_cast<int64_t>(nchild) | (static_cast<int64_t>(ngroups) << 32);
    }
}

__global__ void check_counts_kernel(int nsys, Tree t, int* err) {
    const int64_t m = t.counts[0];
    if (m > t.cap_int) { raise_error(err, kErrTree); t.counts[1] = nsys; t.counts[2] = nsys; return; }
    const int64_t packed = t.int_packed[m];
    const int64_t nodes = nsys + (packed & 0xffffffffll);
    const int64_t groups = nsys + (packed >> 32);
    if (nodes > t.cap_node || groups > t.cap_group) raise_error(err, kErrTree);
    t.counts[1] = nodes < t.cap_node ? nodes : t.cap_node;
    t.counts[2] = groups < t.cap_group ? groups : t.cap_group;
}

__global__ void roots_kernel(const int64_t* __restrict__ offsets, int64_t n, int nsys, int leaf_cap,
                             int group_cap, Tree t) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    const int64_t b = offsets ? offsets[s] : 0;
    const int64_t e = offsets ? offsets[s + 1] : n;
    const int cnt = static_cast<int>(e - b);
    if (cnt <= leaf_cap) {
        t.link[s] = make_int2(static_cast<int>(b), -cnt);
        t.parent[s] = -1;
        t.level[s] = 0;
    }
    t.groups[s] = make_int4(static_cast<int>(b), cnt <= group_cap ? cnt : 0, s, 0);
}

__global__ void children_kernel(const uint64_t* __restrict__ keys, const int8_t* __restrict__ dlev,
                                const int32_t* __restrict__ int_base, const int32_t* __restrict__ sysid,
                                int nsys, int levels, int leaf_cap, int group_cap, Tree t, int* err) {
    if (*err & kErrAbort) return;
    const int64_t m = t.counts[0];
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < m; q += (int64_t)gridDim.x * blockDim.x) {
        const int l = t.int_level[q];
        const int s = t.int_start[q];
        int32_t b[9];
        for (int c = 0; c < 9; ++c) b[c] = t.int_bounds[9 * q + c];
        const int64_t pk = t.int_packed[q], nx = t.int_packed[q + 1];
        const int fc = nsys + static_cast<int>(pk & 0xffffffffll);
        const int nc = static_cast<int>((nx & 0xffffffffll) - (pk & 0xffffffffll));
        const int fg = nsys + static_cast<int>(pk >> 32);
        const int sys = sysid ? sysid[s] : 0;
        if (l == 0) {
            t.int_node[q] = sys;
            t.link[sys] = make_int2(fc, nc);
            t.climb[q] = make_int4(sys, fc, nc, s);
            t.parent[sys] = -1;
            t.level[sys] = 0;
        }
        // every child's records are loaded before the first store (the tree's
        // arrays may alias as far as the compiler knows, so loads after a
        // store would each wait for it), and checked before any store
        int64_t q2c[8], p2c[8], n2c[8];
        bool bad = fc + nc > t.cap_node;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int cs = b[c], cnt = b[c + 1] - b[c];
            q2c[c] = -1; p2c[c] = 0; n2c[c] = 0;
            if (cnt > leaf_cap && l + 1 < levels) {
                const int64_t q2 = static_cast<int64_t>(int_base[cs]) + (l + 1 - dlev[cs] - 1);
                q2c[c] = q2;
                if (q2 <= q || q2 >= m) bad = true;
                else { p2c[c] = t.int_packed[q2]; n2c[c] = t.int_packed[q2 + 1]; }
            }
        }
        if (bad) { raise_error(err, kErrIndex); return; }
        int k = 0;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int cs = b[c], cnt = b[c + 1] - b[c];
            if (cnt == 0) continue;
            const int nid = fc + k++;
            t.parent[nid] = static_cast<int32_t>(q);
            t.level[nid] = static_cast<int8_t>(l + 1);
            if (q2c[c] >= 0) {
                const int64_t q2 = q2c[c];
                t.int_node[q2] = nid;
                const int fc2 = nsys + static_cast<int>(p2c[c] & 0xffffffffll);
                const int nc2 = static_cast<int>((n2c[c] & 0xffffffffll) - (p2c[c] & 0xffffffffll));
                t.link[nid] = make_int2(fc2, nc2);
                t.climb[q2] = make_int4(nid, fc2, nc2 | ((l + 1) << 8), cs);
            } else {
                t.link[nid] = make_int2(cs, -cnt);
            }
        }
        if (b[8] - b[0] > group_cap) {
            int g = fg;
            int4* groups = t.groups;
            const int64_t gcap = t.cap_group;
            pack_groups(b, l, levels, leaf_cap, group_cap, [&](int gs, int gc) {
                if (g < gcap) groups[g] = make_int4(gs, gc, sys, 0);
                ++g;
            });
        }
    }
}

// ---- moments ---------------------------------------------------------------

__device__ __forceinline__ double4 ldcg4(const double4* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = __ldcg(q), b = __ldcg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

struct Mom {
    double m, cx, cy, cz, q[6];
};

__device__ __forceinline__ void store_moments(Tree& t, int nid, const Mom& a, double half, double rcrit,
                                              double G, bool accurate) {
    t.com[nid] = make_double4(a.cx, a.cy, a.cz, a.m);
    double* q64 = t.quad64 + 8 * static_cast<int64_t>(nid);
    for (int c = 0; c < 6; ++c) q64[c] = a.q[c];
    q64[6] = half;
    q64[7] = rcrit;
    if (accurate) {
        const float r2 = a.m > 0.0 ? static_cast<float>(rcrit * rcrit) : -1.0f;
        t.box[nid] = make_float4(static_cast<float>(a.cx), static_cast<float>(a.cy), static_cast<float>(a.cz), r2);
        // stored negated (-G Q): the walk's quadrupole terms then need no negation
        t.quad32[2 * static_cast<int64_t>(nid)] =
            make_float4(static_cast<float>(-G * a.q[0]), static_cast<float>(-G * a.q[1]),
                        static_cast<float>(-G * a.q[2]), static_cast<float>(-G * a.q[3]));
        t.quad32[2 * static_cast<int64_t>(nid) + 1] =
            make_float4(static_cast<float>(-G * a.q[4]), static_cast<float>(-G * a.q[5]), static_cast<float>(G * a.m), 0.0f);
    }
}

// Reference rules (src/gravity/octree.h:104-126) over a list of (m, x, y, z)
// children in octant order; `size` is the cell's half-width.
template <typename Get>
__device__ Mom combine_ref(int count, double size, Get get) {
    Mom a{};
    double m = 0, cx = 0, cy = 0, cz = 0;
    for (int k = 0; k < count; ++k) {
        const double4 c = get(k);
        if (c.w == 0) continue;
        m += c.w;
        cx += c.x * c.w; cy += c.y * c.w; cz += c.z * c.w;
    }
    if (m > 0) { cx /= m; cy /= m; cz /= m; }
    for (int k = 0; k < count; ++k) {
        const double4 c = get(k);
        if (c.w == 0) continue;
        const double rx = c.x - cx, ry = c.y - cy, rz = c.z - cz;
        const double r2 = rx * rx + ry * ry + rz * rz + (size * size * 0.01);
        const double mc = c.w;
        a.q[0] += mc * (3.0 * rx * rx - r2);
        a.q[1] += mc * (3.0 * ry * ry - r2);
        a.q[2] += mc * (3.0 * rz * rz - r2);
        a.q[3] += mc * (3.0 * rx * ry);
        a.q[4] += mc * (3.0 * rx * rz);
        a.q[5] += mc * (3.0 * ry * rz);
    }
    a.m = m; a.cx = cx; a.cy = cy; a.cz = cz;
    return a;
}

// Geometric centre of the level-l cell holding `key` (the reference's child
// centre rule, src/gravity/octree.h:56-64).
__device__ double3 cell_centre(uint64_t key, int level, double4 cube, int base) {
    double cx = cube.x, cy = cube.y, cz = cube.z, h = cube.w;
    for (int l = 1; l <= level; ++l) {
        const int d = key_digit(key, l, base);
        const double hs = h * 0.5;
        cx = cx + ((d & 1) ? hs : -hs);
        cy = cy + ((d & 2) ? hs : -hs);
        cz = cz + ((d & 4) ? hs : -hs);
        h = hs;
    }
    return make_double3(cx, cy, cz);
}

__device__ double rcrit_of(const Mom& a, uint64_t key, int level, double4 cube, int base, double half,
                           double theta) {
    const double3 g = cell_centre(key, level, cube, base);
    double ox = a.cx - g.x, oy = a.cy - g.y, oz = a.cz - g.z;
    if (!(a.m > 0)) { ox = oy = oz = 0.0; }
    return 2.0 * half / theta + sqrt(ox * ox + oy * oy + oz * oz);
}

__device__ __forceinline__ int arrive_acq_rel(int32_t* counter) {
    int old;
    asm volatile("atom.add.acq_rel.gpu.s32 %0, [%1], 1;" : "=r"(old) : "l"(counter) : "memory");
    return old;
}

// Resident blocks the register allocation must allow: the one-launch pass
// (leaf moments and climb in one thread) at 4 per SM, the climb launch of the
// two-launch pass at 2 (no spills: each climbing thread's chain of round
// trips is the critical path there).
#ifndef NB_UP_MINB
#define NB_UP_MINB 4
#endif
#ifndef NB_UP_CLIMB_MINB
#define NB_UP_CLIMB_MINB 2
#endif
#ifndef NB_UP_LEAVES_MINB
#define NB_UP_LEAVES_MINB 3
#endif
// Children whose records a combining thread loads together (2: no spills
// at the climb launch's register cap; 4 and 8 spill and run slower).
#ifndef NB_UP_CHUNK
#define NB_UP_CHUNK 2
#endif
#ifndef NB_UP_SPLIT
#define NB_UP_SPLIT 1
#endif
#ifndef NB_UP_ONEPASS
#define NB_UP_ONEPASS 1
#endif
#ifndef NB_UP_ONEPASS_CLIMB
#define NB_UP_ONEPASS_CLIMB 1
#endif
// Moments of leaf n (bodies [first, first + cnt)), stored.
__device__ __forceinline__ void leaf_moments(const Bodies& bd, const uint64_t* __restrict__ keys,
                                             const int32_t* __restrict__ sysid, const double4* __restrict__ cubes,
                                             int base, const Params& P, Tree& t, bool accurate, int64_t n, int first,
                                             int cnt) {
    const int lvl = t.level[n];
    // an empty leaf can only be the root of an empty system (node id = system)
    const int sys = sysid ? (cnt > 0 ? sysid[first] : static_cast<int>(n)) : 0;
    const double4 cube = cubes[sys];
    const double half = ldexp(cube.w, -lvl);
    Mom a{};
    double rcrit = 0.0;
    if (!accurate) {
        if (cnt == 1) {
            a.m = bd.m[first]; a.cx = bd.x[first]; a.cy = bd.y[first]; a.cz = bd.z[first];
        } else if (cnt > 1) {
            a = combine_ref(cnt, half, [&](int k) {
                return make_double4(bd.x[first + k], bd.y[first + k], bd.z[first + k], bd.m[first + k]);
            });
        }
    } else if (NB_UP_ONEPASS) {
        // one pass over the leaf's bodies: mass, first and second moments
        // about its first body (all of cell size, so no cancellation),
        // then shifted to the centre of mass
        const uint64_t key = cnt > 0 ? keys[first] : 0ull;
        const double x0 = cnt > 0 ? bd.x[first] : 0.0, y0 = cnt > 0 ? bd.y[first] : 0.0,
                     z0 = cnt > 0 ? bd.z[first] : 0.0;
        double m = 0, sx = 0, sy = 0, sz = 0, sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
        for (int j = first; j < first + cnt; ++j) {
            const double mj = bd.m[j];
            const double dx = bd.x[j] - x0, dy = bd.y[j] - y0, dz = bd.z[j] - z0;
            const double mx = mj * dx, my = mj * dy, mz = mj * dz;
            m += mj; sx += mx; sy += my; sz += mz;
            sxx += mx * dx; syy += my * dy; szz += mz * dz;
            sxy += mx * dy; sxz += mx * dz; syz += my * dz;
        }
        double cx, cy, cz;
        if (m > 0) {
            const double ox = sx / m, oy = sy / m, oz = sz / m;
            cx = x0 + ox; cy = y0 + oy; cz = z0 + oz;
            // second moments about the centre of mass
            const double qxx = sxx - sx * ox, qyy = syy - sy * oy, qzz = szz - sz * oz;
            const double tr = qxx + qyy + qzz;
            a.q[0] = 3.0 * qxx - tr; a.q[1] = 3.0 * qyy - tr; a.q[2] = 3.0 * qzz - tr;
            a.q[3] = 3.0 * (sxy - sx * oy); a.q[4] = 3.0 * (sxz - sx * oz); a.q[5] = 3.0 * (syz - sy * oz);
        } else {
            const double3 g = cell_centre(key, lvl, cube, base);
            cx = g.x; cy = g.y; cz = g.z;
        }
        a.m = m; a.cx = cx; a.cy = cy; a.cz = cz;
        rcrit = rcrit_of(a, key, lvl, cube, base, half, P.theta);
    } else {
        double m = 0, cx = 0, cy = 0, cz = 0;
        for (int j = first; j < first + cnt; ++j) {
            const double mj = bd.m[j];
            m += mj; cx += mj * bd.x[j]; cy += mj * bd.y[j]; cz += mj * bd.z[j];
        }
        const uint64_t key = cnt > 0 ? keys[first] : 0ull;
        if (m > 0) { cx /= m; cy /= m; cz /= m; }
        else { const double3 g = cell_centre(key, lvl, cube, base); cx = g.x; cy = g.y; cz = g.z; }
        for (int j = first; j < first + cnt; ++j) {
            const double rx = bd.x[j] - cx, ry = bd.y[j] - cy, rz = bd.z[j] - cz;
            const double r2 = rx * rx + ry * ry + rz * rz;
            const double mj = bd.m[j];
            a.q[0] += mj * (3.0 * rx * rx - r2); a.q[1] += mj * (3.0 * ry * ry - r2);
            a.q[2] += mj * (3.0 * rz * rz - r2); a.q[3] += mj * (3.0 * rx * ry);
            a.q[4] += mj * (3.0 * rx * rz);      a.q[5] += mj * (3.0 * ry * rz);
        }
        a.m = m; a.cx = cx; a.cy = cy; a.cz = cz;
        rcrit = rcrit_of(a, key, lvl, cube, base, half, P.theta);
    }
    store_moments(t, static_cast<int>(n), a, half, rcrit, P.G, accurate);
}

// Moments of internal node rec.x from its children rec.y .. rec.y + nchild
// (all of them final), stored.
__device__ __forceinline__ void combine_children(const uint64_t* __restrict__ keys, const int32_t* __restrict__ sysid,
                                                 const double4* __restrict__ cubes, int base, const Params& P, Tree& t,
                                                 bool accurate, const int4 rec) {
    const int nid = rec.x;
    const int2 plk = make_int2(rec.y, rec.z & 0xff);
    const int pl = rec.z >> 8;
    const int ps = rec.w;
    const double4 pcube = cubes[sysid ? sysid[ps] : 0];
    const double phalf = ldexp(pcube.w, -pl);
    Mom p{};
    double prc = 0.0;
    if (!accurate) {
        p = combine_ref(plk.y, phalf, [&](int k) { return ldcg4(t.com + plk.x + k); });
    } else if (NB_UP_ONEPASS_CLIMB) {
        // one pass over the children: mass, first and second moments of
        // their centres of mass about the first child's, their own
        // quadrupoles; then shifted to the parent's centre of mass
        // (parallel axes)
        const double4 c0 = ldcg4(t.com + plk.x);
        double m = 0, sx = 0, sy = 0, sz = 0, sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
        double qs[6] = {0, 0, 0, 0, 0, 0};
        if (NB_UP_CHUNK > 1) {
            // the children's records in chunks whose loads are all in flight
            // together, summed in octant order as below
            for (int k0 = 0; k0 < plk.y; k0 += NB_UP_CHUNK) {
                double4 cc[NB_UP_CHUNK];
                double2 cq[NB_UP_CHUNK][3];
#pragma unroll
                for (int u = 0; u < NB_UP_CHUNK; ++u) {
                    if (k0 + u < plk.y) {
                        cc[u] = ldcg4(t.com + plk.x + k0 + u);
                        const double2* q2 = reinterpret_cast<const double2*>(t.quad64 + 8 * static_cast<int64_t>(plk.x + k0 + u));
#pragma unroll
                        for (int f = 0; f < 3; ++f) cq[u][f] = __ldcg(q2 + f);
                    }
                }
#pragma unroll
                for (int u = 0; u < NB_UP_CHUNK; ++u) {
                    if (k0 + u >= plk.y) break;
                    const double4 c = cc[u];
                    const double dx = c.x - c0.x, dy = c.y - c0.y, dz = c.z - c0.z;
                    const double mx = c.w * dx, my = c.w * dy, mz = c.w * dz;
                    m += c.w; sx += mx; sy += my; sz += mz;
                    sxx += mx * dx; syy += my * dy; szz += mz * dz;
                    sxy += mx * dy; sxz += mx * dz; syz += my * dz;
#pragma unroll
                    for (int f = 0; f < 3; ++f) { qs[2 * f] += cq[u][f].x; qs[2 * f + 1] += cq[u][f].y; }
                }
            }
        } else {
            for (int k = 0; k < plk.y; ++k) {
                const double4 c = ldcg4(t.com + plk.x + k);
                const double* cq = t.quad64 + 8 * static_cast<int64_t>(plk.x + k);
                const double dx = c.x - c0.x, dy = c.y - c0.y, dz = c.z - c0.z;
                const double mx = c.w * dx, my = c.w * dy, mz = c.w * dz;
                m += c.w; sx += mx; sy += my; sz += mz;
                sxx += mx * dx; syy += my * dy; szz += mz * dz;
                sxy += mx * dy; sxz += mx * dz; syz += my * dz;
#pragma unroll
                for (int f = 0; f < 6; ++f) qs[f] += __ldcg(cq + f);
            }
        }
        const uint64_t key = keys[ps];
        double cx, cy, cz;
        if (m > 0) {
            const double ox = sx / m, oy = sy / m, oz = sz / m;
            cx = c0.x + ox; cy = c0.y + oy; cz = c0.z + oz;
            const double qxx = sxx - sx * ox, qyy = syy - sy * oy, qzz = szz - sz * oz;
            const double tr = qxx + qyy + qzz;
            p.q[0] = qs[0] + (3.0 * qxx - tr); p.q[1] = qs[1] + (3.0 * qyy - tr);
            p.q[2] = qs[2] + (3.0 * qzz - tr); p.q[3] = qs[3] + 3.0 * (sxy - sx * oy);
            p.q[4] = qs[4] + 3.0 * (sxz - sx * oz); p.q[5] = qs[5] + 3.0 * (syz - sy * oz);
        } else {
            const double3 g = cell_centre(key, pl, pcube, base);
            cx = g.x; cy = g.y; cz = g.z;
            for (int f = 0; f < 6; ++f) p.q[f] = qs[f];
        }
        p.m = m; p.cx = cx; p.cy = cy; p.cz = cz;
        prc = rcrit_of(p, key, pl, pcube, base, phalf, P.theta);
    } else {
        double m = 0, cx = 0, cy = 0, cz = 0;
        for (int k = 0; k < plk.y; ++k) {
            const double4 c = ldcg4(t.com + plk.x + k);
            m += c.w; cx += c.w * c.x; cy += c.w * c.y; cz += c.w * c.z;
        }
        const uint64_t key = keys[ps];
        if (m > 0) { cx /= m; cy /= m; cz /= m; }
        else { const double3 g = cell_centre(key, pl, pcube, base); cx = g.x; cy = g.y; cz = g.z; }
        for (int k = 0; k < plk.y; ++k) {
            const double4 c = ldcg4(t.com + plk.x + k);
            const double* cq = t.quad64 + 8 * static_cast<int64_t>(plk.x + k);
            const double rx = c.x - cx, ry = c.y - cy, rz = c.z - cz;
            const double r2 = rx * rx + ry * ry + rz * rz;
            const double mk = c.w;
            p.q[0] += __ldcg(cq + 0) + mk * (3.0 * rx * rx - r2);
            p.q[1] += __ldcg(cq + 1) + mk * (3.0 * ry * ry - r2);
            p.q[2] += __ldcg(cq + 2) + mk * (3.0 * rz * rz - r2);
            p.q[3] += __ldcg(cq + 3) + mk * (3.0 * rx * ry);
            p.q[4] += __ldcg(cq + 4) + mk * (3.0 * rx * rz);
            p.q[5] += __ldcg(cq + 5) + mk * (3.0 * ry * rz);
        }
        p.m = m; p.cx = cx; p.cy = cy; p.cz = cz;
        prc = rcrit_of(p, key, pl, pcube, base, phalf, P.theta);
    }
    store_moments(t, nid, p, phalf, prc, P.G, accurate);
}

// A climb record is valid when it describes a node with 1-8 children inside
// the node array; false (and the index error raised) otherwise.
__device__ __forceinline__ bool climb_record_check(int64_t nodes, const int4& rec, int* err) {
    const int nc = rec.z & 0xff;
    if (rec.x < 0 || rec.x >= nodes || nc < 1 || nc > 8 || rec.y < 0 || static_cast<int64_t>(rec.y) + nc > nodes) {
        raise_error(err, kErrIndex);
        return false;
    }
    return true;
}

// From internal id q upward: arrive at each parent; the last child's thread
// combines the parent's children and goes on.  complete: q's children are
// all final already (no arrival at q itself).
__device__ __forceinline__ void climb_from(int q, bool complete, const uint64_t* __restrict__ keys,
                                          const int32_t* __restrict__ sysid, const double4* __restrict__ cubes,
                                          int base, const Params& P, Tree& t, bool accurate, int64_t nodes,
                                          int64_t ninternal, int* err) {
    int4 pre = q >= 0 && q < ninternal ? __ldg(t.climb + q) : make_int4(0, 0, 0, 0);
    while (q >= 0) {
        if (q >= ninternal) { raise_error(err, kErrIndex); break; }
        // the parent's record (written by the child-search pass, loaded the
        // level before) and the arrival both need only q
        int4 rec = pre;
        const bool ok = climb_record_check(nodes, rec, err);
        if (!complete) {
            // release this child's moments / acquire the siblings' ones
            const int old = arrive_acq_rel(t.counter + q);
            if (!ok || old != (rec.z & 0xff) - 1) break;
            t.counter[q] = 0;                  // re-armed for the next build
        } else if (!ok) {
            break;
        }
        complete = false;
        const int next_q = t.parent[rec.x];   // in flight beside the children's loads
        // the next level's record, loaded before this level's stores
        if (next_q >= 0 && next_q < ninternal) pre = __ldg(t.climb + next_q);
        combine_children(keys, sysid, cubes, base, P, t, accurate, rec);
        q = next_q;
    }
}

// One launch: one thread per leaf computes its moments and climbs.
__global__ void __launch_bounds__(256, NB_UP_MINB)
upward_kernel(Bodies bd, int64_t nbodies, const uint64_t* __restrict__ keys,
                              const int32_t* __restrict__ sysid, const double4* __restrict__ cubes, int base, Params P,
                              Tree t, int* err) {
    if (*err & kErrAbort) return;
    const bool accurate = P.physics == NEXT_PHYSICS_ACCURATE;
    const int64_t nodes = t.counts[1];
    const int64_t ninternal = t.counts[0];
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nodes;
         n += (int64_t)gridDim.x * blockDim.x) {
        const int2 lk = t.link[n];
        if (lk.y > 0) continue;                    // internal: filled by a climbing thread
        if (lk.x < 0 || static_cast<int64_t>(lk.x) - lk.y > nbodies) { raise_error(err, kErrIndex); continue; }
        leaf_moments(bd, keys, sysid, cubes, base, P, t, accurate, n, lk.x, -lk.y);
        climb_from(t.parent[n], false, keys, sysid, cubes, base, P, t, accurate, nodes, ninternal, err);
    }
}

// Two launches.  Leaves: one thread per leaf computes its moments and counts
// itself in at its parent (a plain atomic: the climb launch that reads the
// moments comes after this one); a parent all of whose children are leaves
// is complete when its last leaf arrives, and goes on the ready list.
template <bool ACCURATE>
__global__ void __launch_bounds__(256, NB_UP_LEAVES_MINB)
upward_leaves_kernel(Bodies bd, int64_t nbodies, const uint64_t* __restrict__ keys,
                     const int32_t* __restrict__ sysid, const double4* __restrict__ cubes, int base, Params P, Tree t,
                     int* err) {
    if (*err & kErrAbort) return;
    constexpr bool accurate = ACCURATE;
    const int64_t nodes = t.counts[1];
    const int64_t ninternal = t.counts[0];
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nodes;
         n += (int64_t)gridDim.x * blockDim.x) {
        const int2 lk = t.link[n];
        if (lk.y > 0) continue;
        if (lk.x < 0 || static_cast<int64_t>(lk.x) - lk.y > nbodies) { raise_error(err, kErrIndex); continue; }
        // the parent and its record before the moments' stores
        const int q = t.parent[n];
        const int4 rec = q >= 0 && q < ninternal ? __ldg(t.climb + q) : make_int4(0, 0, 0, 0);
        leaf_moments(bd, keys, sysid, cubes, base, P, t, accurate, n, lk.x, -lk.y);
        if (q < 0) continue;
        if (q >= ninternal) { raise_error(err, kErrIndex); continue; }
        if (!climb_record_check(nodes, rec, err)) continue;
        if (atomicAdd(t.counter + q, 1) == (rec.z & 0xff) - 1) {
            t.counter[q] = 0;
            const unsigned long long slot = atomicAdd(reinterpret_cast<unsigned long long*>(t.counts + 4), 1ull);
            if (slot < static_cast<unsigned long long>(t.cap_int)) t.ready[slot] = q;
            else raise_error(err, kErrIndex);
        }
    }
}

// Climb: one thread per ready parent combines its (leaf) children and
// climbs on as in the one-launch form; the parents' arrival counters already
// hold their leaf children.
template <bool ACCURATE>
__global__ void __launch_bounds__(256, NB_UP_CLIMB_MINB)
upward_climb_kernel(const uint64_t* __restrict__ keys, const int32_t* __restrict__ sysid,
                    const double4* __restrict__ cubes, int base, Params P, Tree t, int* err) {
    if (*err & kErrAbort) return;
    constexpr bool accurate = ACCURATE;
    const int64_t nodes = t.counts[1];
    const int64_t ninternal = t.counts[0];
    const int64_t nready = t.counts[4] < t.cap_int ? t.counts[4] : t.cap_int;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nready;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int q = t.ready[i];
        if (q < 0) { raise_error(err, kErrIndex); continue; }
        climb_from(q, true, keys, sysid, cubes, base, P, t, accurate, nodes, ninternal, err);
    }
}
}  // namespace

cudaError_t build_tree(const uint64_t* keys, int64_t n, const Bodies& bd, const int32_t* sysid,
                       const Systems& sys, const int64_t* d_offsets, const Params& P, Tree& t,
                       void* scan_tmp, int* err, cudaStream_t st) {
    const int threads = 256;
    const unsigned blocks = static_cast<unsigned>((n + threads - 1) / threads);
    const int leaf_cap = P.physics == NEXT_PHYSICS_REFERENCE ? 1 : P.leaf_cap;
    const int group_cap = P.group_cap < leaf_cap ? leaf_cap : P.group_cap;
    const int32_t* sid = sys.n > 1 ? sysid : nullptr;
    const int64_t* offs = sys.n > 1 ? d_offsets : nullptr;
    cudaError_t e0 = cudaMemsetAsync(t.counts + 3, 0, 2 * sizeof(int64_t), st);
    if (e0 != cudaSuccess) return e0;
    if (n > 0) {
        dlev_kernel<<<blocks, threads, 0, st>>>(keys, n, sys.base, sys.levels, t.dlev);
        nint_kernel<<<blocks, threads, 0, st>>>(t.dlev, n, leaf_cap, sys.levels, t.nint,
                                                reinterpret_cast<unsigned long long*>(t.counts + 3));
    }
    cudaError_t e = exclusive_scan<int32_t>(t.nint, t.nint, n, nullptr, static_cast<int32_t*>(scan_tmp),
                                            t.counts + 0, st);
    if (e != cudaSuccess) return e;
    if (n > 0) {
        cell_starts_kernel<<<blocks, threads, 0, st>>>(t.dlev, t.nint, n, t, err);
        const unsigned iblocks = static_cast<unsigned>((t.cap_int + threads - 1) / threads);
        internal_kernel<<<iblocks < 4096u ? (iblocks ? iblocks : 1u) : 4096u, threads, 0, st>>>(
            keys, n, sid, offs, sys.base, sys.levels, leaf_cap, group_cap, t, err);
    }
    e = exclusive_scan<int64_t>(t.int_packed, t.int_packed, t.cap_int, t.counts + 0,
                                static_cast<int64_t*>(scan_tmp), nullptr, st);
    if (e != cudaSuccess) return e;
    check_counts_kernel<<<1, 1, 0, st>>>(sys.n, t, err);
    e = cudaMemsetAsync(t.int_node, 0xff, sizeof(int32_t) * t.cap_int, st);
    if (e != cudaSuccess) return e;
    roots_kernel<<<(sys.n + 127) / 128, 128, 0, st>>>(offs, n, sys.n, leaf_cap, group_cap, t);
    const unsigned cblocks = static_cast<unsigned>((t.cap_int + threads - 1) / threads);
    children_kernel<<<cblocks < 4096u ? (cblocks ? cblocks : 1u) : 4096u, threads, 0, st>>>(
        keys, t.dlev, t.nint, sid, sys.n, sys.levels, leaf_cap, group_cap, t, err);
    const unsigned ublocks = static_cast<unsigned>((t.cap_node + threads - 1) / threads);
    Params Pu = P;
    const unsigned ugrid = ublocks < 8192u ? ublocks : 8192u;
    if (NB_UP_SPLIT) {
        const bool acc = P.physics == NEXT_PHYSICS_ACCURATE;
        if (acc)
            upward_leaves_kernel<true><<<ugrid, threads, 0, st>>>(bd, n, keys, sid, sys.cube, sys.base, Pu, t, err);
        else
            upward_leaves_kernel<false><<<ugrid, threads, 0, st>>>(bd, n, keys, sid, sys.cube, sys.base, Pu, t, err);
        const unsigned rblocks = static_cast<unsigned>((t.cap_int + threads - 1) / threads);
        const unsigned rgrid = rblocks < 8192u ? (rblocks ? rblocks : 1u) : 8192u;
        if (acc)
            upward_climb_kernel<true><<<rgrid, threads, 0, st>>>(keys, sid, sys.cube, sys.base, Pu, t, err);
        else
            upward_climb_kernel<false><<<rgrid, threads, 0, st>>>(keys, sid, sys.cube, sys.base, Pu, t, err);
        count_launches(1);
    } else {
        upward_kernel<<<ugrid, threads, 0, st>>>(bd, n, keys, sid, sys.cube, sys.base, Pu, t, err);
    }
    count_launches(n > 0 ? 9 : 5);
    return cudaGetLastError();
}

}  // namespace nb
