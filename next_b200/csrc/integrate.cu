// KDK leapfrog updates, body reordering, the adaptive time step, FP64
// diagnostics, and the host<->device staging kernels.
//
// Built with -fmad=false: v += a*(dt/2) and x += v*dt round the product and
// the sum separately, as the reference's loops do (src/gravity/step.h:120-122,
// 143-145), so reference-mode trajectories match it bit for bit.
#include "box.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace nb {

namespace {

// Reorder of the body lanes into key order.  inv (original id -> position)
// is written here when inv_here is set; from NB_INV_SPLIT_N bodies up a launch
// of its own writes it instead: its scattered 4-byte stores, mixed into the
// reorder's gathers, slowed the reorder more than the extra launch costs
// (16.7 M bodies: 0.79 ms fused, 0.43 + 0.15 ms split).
#ifndef NB_INV_SPLIT_N
#define NB_INV_SPLIT_N 2097152
#endif
__global__ void gather_bodies_kernel(Bodies src, Bodies dst, const uint32_t* __restrict__ idx, int64_t n,
                                     uint32_t* __restrict__ inv, bool inv_here, int* err) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= n) return;
    const uint32_t j = idx[p];
    if (j >= n) { raise_error(err, kErrIndex); return; }
    // every lane's loads before any store: the lanes' pointers may alias as
    // far as the compiler knows, so interleaved copies would each wait for
    // the previous store
    const double x = src.x[j], y = src.y[j], z = src.z[j];
    const double vx = src.vx[j], vy = src.vy[j], vz = src.vz[j], m = src.m[j];
    const int type = src.type[j];
    const uint32_t id = src.id[j];
    dst.x[p] = x; dst.y[p] = y; dst.z[p] = z;
    dst.vx[p] = vx; dst.vy[p] = vy; dst.vz[p] = vz;
    dst.m[p] = m;
    dst.type[p] = type;
    dst.id[p] = id;
    if (inv_here) inv[id] = static_cast<uint32_t>(p);
}

// inv[id[p]] = p, the inverse of the reorder, for large systems.
__global__ void inv_scatter_kernel(const uint32_t* __restrict__ id, int64_t n, uint32_t* __restrict__ inv) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= n) return;
    const uint32_t k = id[p];
    if (k < n) inv[k] = static_cast<uint32_t>(p);
}

__global__ void kick_drift_kernel(Bodies b, int64_t n, const double* __restrict__ dts, const int* err) {
    if (*err & kErrAbort) return;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double dt = dts[0], half = dts[1];
    // all loads before the first store (the lanes may alias as far as the
    // compiler knows)
    const double vx0 = b.vx[i], vy0 = b.vy[i], vz0 = b.vz[i], ax = b.ax[i], ay = b.ay[i], az = b.az[i];
    const double x0 = b.x[i], y0 = b.y[i], z0 = b.z[i];
    const double vx = vx0 + ax * half, vy = vy0 + ay * half, vz = vz0 + az * half;
    b.vx[i] = vx; b.vy[i] = vy; b.vz[i] = vz;
    b.x[i] = x0 + vx * dt; b.y[i] = y0 + vy * dt; b.z[i] = z0 + vz * dt;
}

// The same kick-drift over a grid-stride loop that also boxes the drifted
// positions: the last block to finish folds the block boxes into the root
// cube the next build needs (one system), saving the build a pass over x, y, z.
#ifndef NB_KDB_BATCH
#define NB_KDB_BATCH 2
#endif
__global__ void __launch_bounds__(kBoxThreads)
kick_drift_box_kernel(Bodies b, int64_t n, const double* __restrict__ dts, const int* err, double* __restrict__ partial,
                      unsigned int* ticket, double4* cube) {
    if (*err & kErrAbort) return;
    const double dt = dts[0], half = dts[1];
    double lo[3] = {1e30, 1e30, 1e30}, hi[3] = {-1e30, -1e30, -1e30};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    if (NB_KDB_BATCH > 1) {
        // NB_KDB_BATCH bodies per thread and round, all their loads issued
        // before any store (the lanes' pointers may alias, so the compiler
        // would not hoist a later body's loads above an earlier one's stores)
        for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i0 < n; i0 += stride * NB_KDB_BATCH) {
            double vx[NB_KDB_BATCH], vy[NB_KDB_BATCH], vz[NB_KDB_BATCH], ax[NB_KDB_BATCH], ay[NB_KDB_BATCH],
                az[NB_KDB_BATCH], x[NB_KDB_BATCH], y[NB_KDB_BATCH], z[NB_KDB_BATCH];
#pragma unroll
            for (int u = 0; u < NB_KDB_BATCH; ++u) {
                const int64_t i = i0 + u * stride;
                if (i < n) {
                    vx[u] = b.vx[i]; vy[u] = b.vy[i]; vz[u] = b.vz[i];
                    ax[u] = b.ax[i]; ay[u] = b.ay[i]; az[u] = b.az[i];
                    x[u] = b.x[i]; y[u] = b.y[i]; z[u] = b.z[i];
                }
            }
#pragma unroll
            for (int u = 0; u < NB_KDB_BATCH; ++u) {
                const int64_t i = i0 + u * stride;
                if (i < n) {
                    const double wx = vx[u] + ax[u] * half, wy = vy[u] + ay[u] * half, wz = vz[u] + az[u] * half;
                    b.vx[i] = wx; b.vy[i] = wy; b.vz[i] = wz;
                    const double px = x[u] + wx * dt, py = y[u] + wy * dt, pz = z[u] + wz * dt;
                    b.x[i] = px; b.y[i] = py; b.z[i] = pz;
                    lo[0] = fmin(lo[0], px); hi[0] = fmax(hi[0], px);
                    lo[1] = fmin(lo[1], py); hi[1] = fmax(hi[1], py);
                    lo[2] = fmin(lo[2], pz); hi[2] = fmax(hi[2], pz);
                }
            }
        }
    } else {
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
            double vx = b.vx[i], vy = b.vy[i], vz = b.vz[i];
            vx += b.ax[i] * half; vy += b.ay[i] * half; vz += b.az[i] * half;
            b.vx[i] = vx; b.vy[i] = vy; b.vz[i] = vz;
            const double px = b.x[i] + vx * dt, py = b.y[i] + vy * dt, pz = b.z[i] + vz * dt;
            b.x[i] = px; b.y[i] = py; b.z[i] = pz;
            lo[0] = fmin(lo[0], px); hi[0] = fmax(hi[0], px);
            lo[1] = fmin(lo[1], py); hi[1] = fmax(hi[1], py);
            lo[2] = fmin(lo[2], pz); hi[2] = fmax(hi[2], pz);
        }
    }
    block_minmax3(lo, hi);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        for (int a = 0; a < 3; ++a) { partial[6 * blockIdx.x + a] = lo[a]; partial[6 * blockIdx.x + 3 + a] = hi[a]; }
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double l2[3] = {1e30, 1e30, 1e30}, h2[3] = {-1e30, -1e30, -1e30};
    for (int k = threadIdx.x; k < gridDim.x; k += blockDim.x)
        for (int a = 0; a < 3; ++a) {
            l2[a] = fmin(l2[a], __ldcg(partial + 6 * k + a));
            h2[a] = fmax(h2[a], __ldcg(partial + 6 * k + 3 + a));
        }
    block_minmax3(l2, h2);
    if (threadIdx.x == 0) {
        *cube = cube_from_box(l2, h2);
        *ticket = 0u;
    }
}

// The closing half-kick.  `done` (may be NULL) counts the kicks that ran:
// a graph-replayed step only reaches it if nothing earlier in the step
// raised an abort bit, so the count tells the host how many replayed steps
// completed before one failed.
__global__ void kick_kernel(Bodies b, int64_t n, const double* __restrict__ dts, const int* err,
                            unsigned int* done) {
    if (*err & kErrAbort) return;
    if (done && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(done, 1u);
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double half = dts[1];
    const double vx = b.vx[i], vy = b.vy[i], vz = b.vz[i], ax = b.ax[i], ay = b.ay[i], az = b.az[i];
    b.vx[i] = vx + ax * half; b.vy[i] = vy + ay * half; b.vz[i] = vz + az * half;
}

// computeAdaptiveDt (src/dt/adaptive.h:23-52): the largest squared speed is
// an exact max, so the order of the reduction does not change the result.
__global__ void __launch_bounds__(256)
adaptive_dt_kernel(const double* __restrict__ vx, const double* __restrict__ vy, const double* __restrict__ vz,
                   int64_t n, double base_dt, double* partial, unsigned int* ticket, double* out) {
    double mx = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double s2 = vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i];
        if (s2 > mx) mx = s2;
    }
    __shared__ double sm[8];
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = mx;
    __syncthreads();
    __shared__ bool last;
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b = fmax(b, sm[w]);
        partial[blockIdx.x] = b;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double v2 = 0.0;
    for (unsigned k = 0; k < gridDim.x; ++k) v2 = fmax(v2, __ldcg(partial + k));
    *ticket = 0u;
    double v = sqrt(v2);
    v = v < 1e4 ? v : 1e4;
    double dt;
    if (v < 1e-8) {
        dt = base_dt;
    } else {
        dt = base_dt / (1 + v);
        const double lo = base_dt * 0.01, hi = base_dt * 1.0;
        dt = (dt < lo) ? lo : dt;
        dt = (hi < dt) ? hi : dt;
    }
    out[0] = dt;
    out[1] = dt * 0.5;
}

// Kinetic energy, potential energy, momentum, angular momentum (FP64).
__global__ void __launch_bounds__(256)
diagnostics_kernel(Bodies b, int64_t n, bool have_pot, double* partial, unsigned int* ticket, double* out) {
    double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double m = b.m[i], vx = b.vx[i], vy = b.vy[i], vz = b.vz[i];
        const double x = b.x[i], y = b.y[i], z = b.z[i];
        s[0] += 0.5 * m * (vx * vx + vy * vy + vz * vz);
        if (have_pot) s[1] += 0.5 * m * b.pot[i];
        s[2] += m * vx; s[3] += m * vy; s[4] += m * vz;
        s[5] += m * (y * vz - z * vy);
        s[6] += m * (z * vx - x * vz);
        s[7] += m * (x * vy - y * vx);
    }
    __shared__ double sm[8][8];
    for (int c = 0; c < 8; ++c) {
        double v = s[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) sm[c][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    __shared__ bool last;
    if (threadIdx.x == 0) {
        for (int c = 0; c < 8; ++c) {
            double v = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += sm[c][w];
            partial[8 * blockIdx.x + c] = v;
        }
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    for (int c = 0; c < 8; ++c) {
        double v = 0.0;
        for (unsigned k = 0; k < gridDim.x; ++k) v += __ldcg(partial + 8 * k + c);
        out[c] = v;
    }
    *ticket = 0u;
}

// Upload support, one pass over the staged lanes: flags[1] = a non-finite
// value, flags[2] = a negative mass, and (compare) flags[0] = positions,
// masses or types differ from the bodies the handle holds (compared through
// inv: caller index -> working position).
__global__ void check_upload_kernel(const double* __restrict__ stage, const int* __restrict__ stype, Bodies b,
                                    const uint32_t* __restrict__ inv, int64_t n, bool compare, int* flags) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool finite = true;
    for (int c = 0; c < 7; ++c) finite &= isfinite(stage[c * n + i]);
    if (!finite) flags[1] = 1;
    if (stage[6 * n + i] < 0.0) flags[2] = 1;
    if (compare) {
        const uint32_t p = inv[i];
        const bool same = stage[i] == b.x[p] && stage[n + i] == b.y[p] && stage[2 * n + i] == b.z[p] &&
                          stage[6 * n + i] == b.m[p] && stype[i] == b.type[p];
        if (!same) flags[0] = 1;
    }
}

__global__ void load_velocities_kernel(const double* __restrict__ stage, Bodies b, const uint32_t* __restrict__ inv,
                                       int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t p = inv[i];
    b.vx[p] = stage[3 * n + i]; b.vy[p] = stage[4 * n + i]; b.vz[p] = stage[5 * n + i];
}

__global__ void load_all_kernel(const double* __restrict__ stage, const int* __restrict__ stype, Bodies b,
                                uint32_t* __restrict__ inv, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    b.x[i] = stage[i]; b.y[i] = stage[n + i]; b.z[i] = stage[2 * n + i];
    b.vx[i] = stage[3 * n + i]; b.vy[i] = stage[4 * n + i]; b.vz[i] = stage[5 * n + i];
    b.m[i] = stage[6 * n + i];
    b.type[i] = stype[i];
    b.id[i] = static_cast<uint32_t>(i);
    inv[i] = static_cast<uint32_t>(i);
    b.ax[i] = 0.0; b.ay[i] = 0.0; b.az[i] = 0.0;
}

// next_step_host's check that a call's inputs are the state the previous
// call returned: positions and velocities against that call's export,
// masses and types against its upload (all in caller order), bit for bit and
// finite.  flags[0] = 1 on any difference.
__global__ void same_as_last_kernel(const double* __restrict__ in, const int* __restrict__ type,
                                    const double* __restrict__ prev_out, const double* __restrict__ prev_in,
                                    const int* __restrict__ prev_type, int64_t n, int* flags) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool same = type[i] == prev_type[i];
    for (int c = 0; c < 6; ++c) {
        const double v = in[c * n + i];
        same &= isfinite(v) && __double_as_longlong(v) == __double_as_longlong(prev_out[c * n + i]);
    }
    const double m = in[6 * n + i];
    same &= isfinite(m) && __double_as_longlong(m) == __double_as_longlong(prev_in[6 * n + i]);
    if (!same) flags[0] = 1;
}

// Download support: gather `count` FP64 lanes into caller order.  The lane
// pointers travel by value in the launch, so no host-to-device copy of a
// pointer table precedes the gather.
struct LaneTable {
    const double* p[kMaxGatherLanes];
};

__global__ void gather_out_kernel(LaneTable lanes, int count, const uint32_t* __restrict__ inv, int64_t n,
                                  double* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t p = inv[i];
    double v[kMaxGatherLanes];
#pragma unroll
    for (int c = 0; c < kMaxGatherLanes; ++c)
        if (c < count) v[c] = lanes.p[c][p];
#pragma unroll
    for (int c = 0; c < kMaxGatherLanes; ++c)
        if (c < count) out[c * n + i] = v[c];
}

__global__ void ids_to_positions_kernel(const int64_t* __restrict__ ids, const uint32_t* __restrict__ inv, int64_t k,
                                        int64_t* __restrict__ pos) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < k) pos[t] = inv[ids[t]];
}

__global__ void set_dt_kernel(double* dts, double dt) {
    dts[0] = dt;
    dts[1] = dt * 0.5;
}

// FP32 FMA throughput probe: 8 independent chains per thread.
__global__ void __launch_bounds__(256) fma_peak_kernel(float* out, int iters, float a, float b) {
    float r[8];
    for (int k = 0; k < 8; ++k) r[k] = threadIdx.x * 1e-3f + k;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int k = 0; k < 8; ++k) r[k] = fmaf(r[k], a, b);
    }
    float s = 0.f;
    for (int k = 0; k < 8; ++k) s += r[k];
    if (s == 1.2345f) out[0] = s;   // keeps the chains live
}

inline unsigned grid_for(int64_t n, int threads) { return static_cast<unsigned>((n + threads - 1) / threads); }

}  // namespace

cudaError_t launch_gather_bodies(const Bodies& src, const Bodies& dst, const uint32_t* idx, int64_t n, uint32_t* inv,
                                 int* err, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const bool split = n >= NB_INV_SPLIT_N;
    gather_bodies_kernel<<<grid_for(n, 256), 256, 0, st>>>(src, dst, idx, n, inv, !split, err);
    count_launches(1);
    if (split) {
        inv_scatter_kernel<<<grid_for(n, 256), 256, 0, st>>>(dst.id, n, inv);
        count_launches(1);
    }
    return cudaGetLastError();
}

cudaError_t launch_kick_drift(const Bodies& b, int64_t n, const double* dts, const int* err, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    kick_drift_kernel<<<grid_for(n, 256), 256, 0, st>>>(b, n, dts, err);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_kick_drift_box(const Bodies& b, int64_t n, const double* dts, const int* err, double* partial,
                                  int partial_blocks, unsigned int* ticket, double4* cube, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    unsigned blocks = grid_for(n, kBoxThreads);
    if (blocks > static_cast<unsigned>(partial_blocks)) blocks = static_cast<unsigned>(partial_blocks);
    kick_drift_box_kernel<<<blocks, kBoxThreads, 0, st>>>(b, n, dts, err, partial, ticket, cube);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_kick(const Bodies& b, int64_t n, const double* dts, const int* err, cudaStream_t st,
                        unsigned int* done) {
    if (n <= 0) return cudaSuccess;
    kick_kernel<<<grid_for(n, 256), 256, 0, st>>>(b, n, dts, err, done);
    count_launches(1);
    return cudaGetLastError();
}

int reduce_blocks(int64_t n) {
    int64_t b = (n + 256 * 8 - 1) / (256 * 8);
    if (b < 1) b = 1;
    if (b > 1024) b = 1024;
    return static_cast<int>(b);
}

cudaError_t launch_adaptive_dt(const Bodies& b, int64_t n, double base_dt, double* partial, unsigned int* ticket,
                               double* out, cudaStream_t st) {
    adaptive_dt_kernel<<<reduce_blocks(n), 256, 0, st>>>(b.vx, b.vy, b.vz, n, base_dt, partial, ticket, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_diagnostics(const Bodies& b, int64_t n, bool have_pot, double* partial, unsigned int* ticket,
                               double* out, cudaStream_t st) {
    diagnostics_kernel<<<reduce_blocks(n), 256, 0, st>>>(b, n, have_pot, partial, ticket, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_check_upload(const double* stage, const int* stype, const Bodies& b, const uint32_t* inv, int64_t n,
                                bool compare, int* flags, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    check_upload_kernel<<<grid_for(n, 256), 256, 0, st>>>(stage, stype, b, inv, n, compare, flags);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_load_velocities(const double* stage, const Bodies& b, const uint32_t* inv, int64_t n,
                                   cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    load_velocities_kernel<<<grid_for(n, 256), 256, 0, st>>>(stage, b, inv, n);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_load_all(const double* stage, const int* stype, const Bodies& b, uint32_t* inv, int64_t n,
                            cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    load_all_kernel<<<grid_for(n, 256), 256, 0, st>>>(stage, stype, b, inv, n);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_same_as_last(const double* in, const int* type, const double* prev_out, const double* prev_in,
                                const int* prev_type, int64_t n, int* flags, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    same_as_last_kernel<<<grid_for(n, 256), 256, 0, st>>>(in, type, prev_out, prev_in, prev_type, n, flags);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_gather_out(const double* const* lanes, int count, const uint32_t* inv, int64_t n, double* out,
                              cudaStream_t st) {
    if (n <= 0 || count <= 0) return cudaSuccess;
    if (count > kMaxGatherLanes) return cudaErrorInvalidValue;
    LaneTable table{};
    for (int c = 0; c < count; ++c) table.p[c] = lanes[c];
    gather_out_kernel<<<grid_for(n, 256), 256, 0, st>>>(table, count, inv, n, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_ids_to_positions(const int64_t* ids, const uint32_t* inv, int64_t k, int64_t* pos,
                                    cudaStream_t st) {
    if (k <= 0) return cudaSuccess;
    ids_to_positions_kernel<<<grid_for(k, 256), 256, 0, st>>>(ids, inv, k, pos);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_set_dt(double* dts, double dt, cudaStream_t st) {
    set_dt_kernel<<<1, 1, 0, st>>>(dts, dt);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_fma_peak(float* out, int blocks, int iters, cudaStream_t st) {
    fma_peak_kernel<<<blocks, 256, 0, st>>>(out, iters, 0.9999999f, 1e-7f);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace nb
