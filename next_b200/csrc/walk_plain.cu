// Plain FP64 force walk: one thread per target body, depth-first over the
// tree in octant order 0..7 -- the order bhAccel recurses
// (src/gravity/octree.h:176-178) -- with a per-level (next sibling, end)
// stack instead of recursion.  Reference physics repeats bhAccel's
// arithmetic (octree.h:134-173, softening.h:21-35) operation for operation;
// accurate physics uses Plummer softening, the full-width opening test and
// the corrected quadrupole.
//
// Also: the FP64 direct-summation kernel used to state force errors.
//
// Built with -fmad=false so each + and * rounds on its own, matching the
// reference's x86-64 build (no FMA contraction).  cbrt and pow come from
// CUDA's math library; they may differ from the host libm in the last bit.
#include "common.cuh"
#include "kernels.cuh"

namespace nb {

namespace {

__device__ __forceinline__ double dmax_like_std(double a, double b) { return (a < b) ? b : a; }

// nextSoftening: src/dt/softening.h:21-35.
__device__ __forceinline__ double next_softening(double size, double mass, double dist) {
    const double eps_size = size * 0.015;
    const double eps_mass = cbrt(mass) * 0.002;
    const double taper = 1.0 / (1.0 + dist * 10.0);
    const double eps = (eps_size + eps_mass) * taper;
    return dmax_like_std(eps, 1e-4);
}

// One accepted node in reference physics: src/gravity/octree.h:138-172.
__device__ __forceinline__ void ref_interact(double nm, double ncx, double ncy, double ncz, double size,
                                             const double* Q, double xi, double yi, double zi, double mi,
                                             int ti, double& ax, double& ay, double& az) {
    const double dx = ncx - xi, dy = ncy - yi, dz = ncz - zi;
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double dist = sqrt(r2 + 1e-20);
    double eps = next_softening(size, nm, dist);
    if (ti == 1) eps = dmax_like_std(eps, 2.0 * size / pow(nm / mi, 0.333333333));
    const double r2s = r2 + eps * eps;
    const double dinv = 1.0 / sqrt(r2s);
    const double inv3 = dinv * dinv * dinv;
    const double fac = 1.0 * nm * inv3;
    ax += dx * fac; ay += dy * fac; az += dz * fac;
    const double inv5 = inv3 * (dinv * dinv);
    const double inv7 = inv5 * (dinv * dinv);
    const double q = Q[0] * dx * dx + Q[1] * dy * dy + Q[2] * dz * dz +
                     2.0 * (Q[3] * dx * dy + Q[4] * dx * dz + Q[5] * dy * dz);
    const double qrx = 2.0 * (Q[0] * dx + Q[3] * dy + Q[4] * dz);
    const double qry = 2.0 * (Q[3] * dx + Q[1] * dy + Q[5] * dz);
    const double qrz = 2.0 * (Q[4] * dx + Q[5] * dy + Q[2] * dz);
    ax += 0.5 * (qrx * inv5 - 5.0 * q * inv7 * dx);
    ay += 0.5 * (qry * inv5 - 5.0 * q * inv7 * dy);
    az += 0.5 * (qrz * inv5 - 5.0 * q * inv7 * dz);
}

__device__ __forceinline__ void add_stats(unsigned long long* stats, unsigned long long pp, unsigned long long pc) {
    for (int o = 16; o > 0; o >>= 1) {
        pp += __shfl_xor_sync(0xffffffffu, pp, o);
        pc += __shfl_xor_sync(0xffffffffu, pc, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (pp) atomicAdd(stats + 0, pp);
        if (pc) atomicAdd(stats + 1, pc);
    }
}

template <bool ACCURATE>
__global__ void __launch_bounds__(128)
walk_plain_kernel(Bodies bd, const int32_t* __restrict__ sysid, int64_t n, Tree t, Params P,
                  unsigned long long* stats, int* err) {
    if (*err & kErrAbort) return;
    const int64_t nodes = t.counts[1];
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool active = i < n && i >= P.own_lo && i < P.own_hi;
    unsigned long long npp = 0, npc = 0;
    if (active) {
        const int root = sysid ? sysid[i] : 0;
        const double xi = bd.x[i], yi = bd.y[i], zi = bd.z[i], mi = bd.m[i];
        const int ti = bd.type[i];
        const double eps2 = P.eps * P.eps, G = P.G, theta = P.theta;
        double ax = 0.0, ay = 0.0, az = 0.0, pot = 0.0;
        int2 stack[kMaxLevel + 2];
        int sp = 0;
        int cur = root, end = root + 1;
        for (;;) {
            if (cur >= end) {
                if (sp == 0) break;
                --sp;
                cur = stack[sp].x;
                end = stack[sp].y;
                continue;
            }
            const int nd = cur++;
            if (nd < 0 || nd >= nodes) { raise_error(err, kErrIndex); break; }
            // the node's whole record in one round trip: centre of mass, link
            // and the 8 moment words (quadrupole, size, critical radius), all
            // issued before the first test uses any of them
            const double4 c = t.com[nd];
            const int2 lk = t.link[nd];
            const double2* q2 = reinterpret_cast<const double2*>(t.quad64 + 8 * static_cast<int64_t>(nd));
            const double2 qa = q2[0], qb = q2[1], qc = q2[2], qd = q2[3];
            const double q64[8] = {qa.x, qa.y, qb.x, qb.y, qc.x, qc.y, qd.x, qd.y};
            if (c.w == 0.0) continue;
            const bool leaf = lk.y <= 0;
            if (leaf ? (lk.x < 0 || static_cast<int64_t>(lk.x) - lk.y > n) : (sp >= kMaxLevel + 1)) {
                raise_error(err, leaf ? kErrIndex : kErrStack);
                break;
            }
            if (!ACCURATE) {
                const int cnt = -lk.y;
                if (leaf && cnt == 1 && lk.x == i) continue;          // own leaf (octree.h:135)
                const double size = q64[6];
                if (leaf && cnt > 1) {
                    // deepest-level bucket: its bodies act as one-body leaves of this size
                    const double Z[6] = {0, 0, 0, 0, 0, 0};
                    for (int j = lk.x; j < lk.x + cnt; ++j) {
                        if (j == i || bd.m[j] == 0.0) continue;
                        ref_interact(bd.m[j], bd.x[j], bd.y[j], bd.z[j], size, Z, xi, yi, zi, mi, ti, ax, ay, az);
                        ++npp;
                    }
                    continue;
                }
                const double dx = c.x - xi, dy = c.y - yi, dz = c.z - zi;
                const double r2 = dx * dx + dy * dy + dz * dz;
                const double dist = sqrt(r2 + 1e-20);
                if (leaf || (size / dist) < theta) {
                    const double Q[6] = {q64[0], q64[1], q64[2], q64[3], q64[4], q64[5]};
                    ref_interact(c.w, c.x, c.y, c.z, size, Q, xi, yi, zi, mi, ti, ax, ay, az);
                    if (leaf) ++npp; else ++npc;
                    continue;
                }
                stack[sp++] = make_int2(cur, end);
                cur = lk.x;
                end = lk.x + lk.y;
            } else {
                const double dx = c.x - xi, dy = c.y - yi, dz = c.z - zi;
                const double r2 = dx * dx + dy * dy + dz * dz;
                const double rc = q64[7];
                if (r2 < rc * rc) {
                    if (!leaf) {
                        stack[sp++] = make_int2(cur, end);
                        cur = lk.x;
                        end = lk.x + lk.y;
                        continue;
                    }
                    for (int j = lk.x; j < lk.x - lk.y; ++j) {
                        if (j == i) continue;
                        const double ex = bd.x[j] - xi, ey = bd.y[j] - yi, ez = bd.z[j] - zi;
                        const double e2 = ex * ex + ey * ey + ez * ez + eps2;
                        const double rinv = 1.0 / sqrt(e2);
                        const double mr3 = G * bd.m[j] * rinv * rinv * rinv;
                        ax += mr3 * ex; ay += mr3 * ey; az += mr3 * ez;
                        pot -= G * bd.m[j] * rinv;
                        ++npp;
                    }
                    continue;
                }
                const double r2s = r2 + eps2;
                const double rinv = 1.0 / sqrt(r2s);
                const double rinv2 = rinv * rinv;
                const double mr3 = G * c.w * rinv * rinv2;
                ax += mr3 * dx; ay += mr3 * dy; az += mr3 * dz;
                pot -= G * c.w * rinv;
                if (P.quad) {
                    const double qxx = q64[0], qyy = q64[1], qzz = q64[2];
                    const double qxy = q64[3], qxz = q64[4], qyz = q64[5];
                    const double qdx = qxx * dx + qxy * dy + qxz * dz;
                    const double qdy = qxy * dx + qyy * dy + qyz * dz;
                    const double qdz = qxz * dx + qyz * dy + qzz * dz;
                    const double q = dx * qdx + dy * qdy + dz * qdz;
                    const double rinv5 = rinv2 * rinv2 * rinv;
                    const double rinv7 = rinv5 * rinv2;
                    const double c7 = 2.5 * G * q * rinv7;
                    const double c5 = G * rinv5;
                    ax += c7 * dx - c5 * qdx;
                    ay += c7 * dy - c5 * qdy;
                    az += c7 * dz - c5 * qdz;
                    pot -= 0.5 * G * q * rinv5;
                }
                ++npc;
            }
        }
        bd.ax[i] = ax; bd.ay[i] = ay; bd.az[i] = az;
        if (bd.pot) bd.pot[i] = pot;
    }
    add_stats(stats, npp, npc);
}

// FP64 direct summation: block (x = 128 targets, y = source slice).
constexpr int kDirectThreads = 128;

__global__ void __launch_bounds__(kDirectThreads)
direct_kernel(const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
              const double* __restrict__ m, int64_t n, const int64_t* __restrict__ targets, int64_t k,
              double eps2, double G, double* __restrict__ partial) {
    __shared__ double4 src[kDirectThreads];
    const int64_t t = blockIdx.x * (int64_t)kDirectThreads + threadIdx.x;
    const int64_t slice = (n + gridDim.y - 1) / gridDim.y;
    const int64_t js = blockIdx.y * slice;
    const int64_t je = js + slice < n ? js + slice : n;
    const int64_t ti = t < k ? targets[t] : -1;
    const double xi = ti >= 0 ? x[ti] : 0.0, yi = ti >= 0 ? y[ti] : 0.0, zi = ti >= 0 ? z[ti] : 0.0;
    double ax = 0.0, ay = 0.0, az = 0.0, ph = 0.0;
    for (int64_t b = js; b < je; b += kDirectThreads) {
        const int64_t j = b + threadIdx.x;
        src[threadIdx.x] = j < je ? make_double4(x[j], y[j], z[j], m[j]) : make_double4(0, 0, 0, 0);
        __syncthreads();
        const int cnt = static_cast<int>(je - b < kDirectThreads ? je - b : kDirectThreads);
        for (int s = 0; s < cnt; ++s) {
            if (b + s == ti) continue;
            const double4 p = src[s];
            const double dx = p.x - xi, dy = p.y - yi, dz = p.z - zi;
            const double r2 = dx * dx + dy * dy + dz * dz + eps2;
            const double rinv = 1.0 / sqrt(r2);
            const double mr3 = G * p.w * rinv * rinv * rinv;
            ax += mr3 * dx; ay += mr3 * dy; az += mr3 * dz;
            ph -= G * p.w * rinv;
        }
        __syncthreads();
    }
    if (t < k) {
        double* o = partial + 4 * (blockIdx.y * k + t);
        o[0] = ax; o[1] = ay; o[2] = az; o[3] = ph;
    }
}

__global__ void direct_reduce_kernel(const double* __restrict__ partial, int64_t k, int slices,
                                     double* __restrict__ out) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= k) return;
    double s[4] = {0, 0, 0, 0};
    for (int sl = 0; sl < slices; ++sl)
        for (int c = 0; c < 4; ++c) s[c] += partial[4 * (sl * k + t) + c];
    for (int c = 0; c < 4; ++c) out[4 * t + c] = s[c];
}

// The device softening law on k (size, mass, dist) triples (test support).
__global__ void softening_kernel(const double* __restrict__ in, int64_t k, double* __restrict__ out) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < k) out[t] = next_softening(in[t], in[k + t], in[2 * k + t]);
}

}  // namespace

cudaError_t launch_softening_eval(const double* in, int64_t k, double* out, cudaStream_t st) {
    if (k <= 0) return cudaSuccess;
    softening_kernel<<<static_cast<unsigned>((k + 127) / 128), 128, 0, st>>>(in, k, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_walk_plain(const Bodies& bd, const int32_t* sysid, int64_t n, const Tree& t,
                              const Params& P, bool multi_system, unsigned long long* stats, int* err,
                              cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const unsigned blocks = static_cast<unsigned>((n + 127) / 128);
    const int32_t* sid = multi_system ? sysid : nullptr;
    if (P.physics == NEXT_PHYSICS_ACCURATE)
        walk_plain_kernel<true><<<blocks, 128, 0, st>>>(bd, sid, n, t, P, stats, err);
    else
        walk_plain_kernel<false><<<blocks, 128, 0, st>>>(bd, sid, n, t, P, stats, err);
    count_launches(1);
    return cudaGetLastError();
}

int direct_slices(int64_t n, int64_t k) {
    const int64_t tblocks = (k + kDirectThreads - 1) / kDirectThreads;
    int64_t slices = (4 * 148 + tblocks - 1) / (tblocks > 0 ? tblocks : 1);
    if (slices < 1) slices = 1;
    if (slices > 256) slices = 256;
    if (slices > n) slices = n > 0 ? n : 1;
    return static_cast<int>(slices);
}

cudaError_t launch_direct(const Bodies& bd, int64_t n, const int64_t* targets, int64_t k, double eps, double G,
                          double* partial, int slices, double* out, cudaStream_t st) {
    if (k <= 0) return cudaSuccess;
    dim3 grid(static_cast<unsigned>((k + kDirectThreads - 1) / kDirectThreads), static_cast<unsigned>(slices));
    direct_kernel<<<grid, kDirectThreads, 0, st>>>(bd.x, bd.y, bd.z, bd.m, n, targets, k, eps * eps, G, partial);
    direct_reduce_kernel<<<static_cast<unsigned>((k + 127) / 128), 128, 0, st>>>(partial, k, slices, out);
    count_launches(2);
    return cudaGetLastError();
}

}  // namespace nb
