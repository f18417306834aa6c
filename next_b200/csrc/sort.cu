// Stable LSD radix sort of (uint64 key, uint32 value) pairs: one histogram
// pass over the keys for all digits, then one "onesweep" pass per 8-bit
// digit.  A onesweep pass works on tiles of 256 x 15 pairs:
//   1. load the tile, count its digits per warp (ballot peer masks, kept in
//      shared memory for the ranking; one shared add per digit group) and
//      publish the per-digit tile counts in a status array (flag + count
//      packed in one 32-bit word);
//   2. read the statuses of the 8 preceding tiles (decoupled look-back),
//      and while those loads are in flight scan the counts and rank and
//      scatter the tile into shared memory in digit order;
//   3. finish the look-back, publish the inclusive counts, and write the
//      tile out, each digit run to its global offset,
// so a pass reads and writes every pair exactly once.  Tiles are numbered
// in the order blocks start (an atomic ticket), so every tile a block waits
// on is already running; each wait is still bounded and raises
// NEXT_DEVERR_SORT_TIMEOUT instead of spinning forever.
//
// Memory bound: per pass 12 B read + 12 B written per pair.
#include "common.cuh"
#include "kernels.cuh"

namespace nb {

namespace {

constexpr int kRadix = 256;
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = NB_SORT_ITEMS;
constexpr int kTile = kThreads * kItems;
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr uint32_t kCountMask = (1u << 30) - 1;
constexpr int kSpinLimit = 1 << 20;
constexpr int kLookWindow = 8;   // earlier tiles whose status one look-back step reads

// Digit mask of pass p for keys of key_bits significant bits: bits at and
// above key_bits take no part in the ordering.
__host__ __device__ __forceinline__ uint32_t pass_mask(int key_bits, int p) {
    const int left = key_bits - 8 * p;
    return left >= 8 ? 0xffu : (1u << left) - 1u;
}

__global__ void __launch_bounds__(kThreads)
histogram_kernel(const uint64_t* __restrict__ keys, int64_t n, int key_bits, uint32_t* __restrict__ hist) {
    const int passes = (key_bits + 7) / 8;
    __shared__ uint32_t local[8][kRadix];
    for (int i = threadIdx.x; i < 8 * kRadix; i += kThreads) (&local[0][0])[i] = 0;
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
        const uint64_t k = keys[i];
        for (int p = 0; p < passes; ++p) atomicAdd(&local[p][(k >> (8 * p)) & pass_mask(key_bits, p)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * kRadix; i += kThreads) {
        const uint32_t v = (&local[0][0])[i];
        if (v) atomicAdd(hist + i, v);
    }
}

// Exclusive scan of each pass's 256 digit counts (one block per pass).
__global__ void __launch_bounds__(kRadix) digit_offsets_kernel(const uint32_t* hist, uint32_t* offsets) {
    __shared__ uint32_t s[kRadix];
    const int p = blockIdx.x, t = threadIdx.x;
    s[t] = hist[p * kRadix + t];
    __syncthreads();
    for (int o = 1; o < kRadix; o <<= 1) {
        const uint32_t v = t >= o ? s[t - o] : 0u;
        __syncthreads();
        s[t] += v;
        __syncthreads();
    }
    offsets[p * kRadix + t] = s[t] - hist[p * kRadix + t];
}

template <int ITEMS>
struct SortSmemT {
    uint32_t warp_hist[kWarps][kRadix];
    uint32_t global_delta[kRadix];
    uint32_t warp_total[kWarps];
    uint64_t keys[kThreads * ITEMS];
    uint32_t vals[kThreads * ITEMS];
    uint32_t peers[ITEMS][kThreads];   // the count pass's peer masks, reused by the ranking
    int tile;
};
using SortSmem = SortSmemT<kItems>;

// Sorts of at most NB_SORT_SMALL_N pairs (the build's, not the allocation-
// free entry point's) use tiles of kThreads x NB_SORT_SMALL_ITEMS pairs: a
// few tiles make such a pass, so its time is about one tile's latency, which
// shorter tiles cut (16,384 pairs: sort 0.048 -> 0.039 ms).  At 1,048,576
// pairs the longer look-back chain of twice the tiles costs more than that
// (0.072 -> 0.079 ms), so larger sorts keep kTile.
#ifndef NB_SORT_SMALL_N
#define NB_SORT_SMALL_N 262144
#endif
#ifndef NB_SORT_SMALL_ITEMS
#define NB_SORT_SMALL_ITEMS 8
#endif
#ifndef NB_SORT_SMALL_MINB
#define NB_SORT_SMALL_MINB 4
#endif
constexpr int kSmallItems = NB_SORT_SMALL_ITEMS;

// Lanes of the warp whose 8-bit digit equals this lane's: eight ballots,
// one per digit bit (cheaper than a match-any on this part).  Written as one
// volatile block that is also ordered with memory accesses, so the compiler
// neither hoists the bit tests of all items nor keeps them in registers.
__device__ __forceinline__ uint32_t digit_peers(int dig) {
    uint32_t peers;
    asm volatile(
        "{\n\t.reg .pred p;\n\t.reg .u32 t, m, r;\n\t" "mov.u32 r, 0xffffffff;\n\t"
        "and.b32 t, %1, 1;\n\t" "setp.ne.u32 p, t, 0;\n\t" "vote.sync.ballot.b32 m, p, 0xffffffff;\n\t" "@!p not.b32 m, m;\n\t" "and.b32 r, r, m;\n\t"
        "and.b32 t, %1, 2;\n\t" "setp.ne.u32 p, t, 0;\n\t" "vote.sync.ballot.b32 m, p, 0xffffffff;\n\t" "@!p not.b32 m, m;\n\t" "and.b32 r, r, m;\n\t"
        "and.b32 t, %1, 4;\n\t" "setp.ne.u32 p, t, 0;\n\t" "vote.sync.ballot.b32 m, p, 0xffffffff;\n\t" "@!p not.b32 m, m;\n\t" "and.b32 r, r, m;\n\t"
        "and.b32 t, %1, 8;\n\t" "setp.ne.u32 p, t, 0;\n\t" "vote.sync.ballot.b32 m, p, 0xffffffff;\n\t" "@!p not.b32 m, m;\n\t" "and.b32 r, r, m;\n\t"
        "and.b32 t, %1, 16;\n\t" "setp.ne.u32 p, t, 0;\n\t" "vote.sync.ballot.b32 m, p, 0xffffffff;\n\t" "@!p not.b32 m, m;\n\t" "and.b32 r, r, m;\n\t"
        "and.b32 t, %1, 32;\n\t" "setp.ne.u32 p, t, 0;\n\t" "vote.sync.ballot.b32 m, p, 0xffffffff;\n\t" "@!p not.b32 m, m;\n\t" "and.b32 r, r, m;\n\t"
        "and.b32 t, %1, 64;\n\t" "setp.ne.u32 p, t, 0;\n\t" "vote.sync.ballot.b32 m, p, 0xffffffff;\n\t" "@!p not.b32 m, m;\n\t" "and.b32 r, r, m;\n\t"
        "and.b32 t, %1, 128;\n\t" "setp.ne.u32 p, t, 0;\n\t" "vote.sync.ballot.b32 m, p, 0xffffffff;\n\t" "@!p not.b32 m, m;\n\t" "and.b32 r, r, m;\n\t"
        "mov.u32 %0, r;\n\t}"
        : "=r"(peers) : "r"(dig) : "memory");
    return peers;
}

// Three resident blocks per SM (80 registers, 69 KB of shared memory with
// the stashed peer masks): the phases of one tile wait on memory and on
// earlier tiles, so occupancy matters as much as instruction count here.
#ifndef NB_SORT_MINB
#define NB_SORT_MINB 3
#endif
// Tile loads into registers: item k of lane l of warp w is pair
// tile_base + (w * kItems + k) * 32 + l; pairs past n are padding keys that
// rank after every real key of the tile and are never written out.
template <int ITEMS>
__device__ __forceinline__ void load_tile(const uint64_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                                          int64_t n, int tile, int w, int lane, uint64_t (&key)[ITEMS],
                                          uint32_t (&val)[ITEMS]) {
    const int64_t warp_base = static_cast<int64_t>(tile) * (kThreads * ITEMS) + static_cast<int64_t>(w) * ITEMS * 32;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const int64_t g = warp_base + k * 32 + lane;
        if (g < n) { key[k] = keys_in[g]; val[k] = vals_in[g]; }
        else { key[k] = ~0ull; val[k] = 0u; }
    }
}

// Persistent: a block takes tiles by ticket until none is left.  Once a
// tile's pairs sit ranked in shared memory, the block takes its next ticket
// and loads that tile into the registers the ranking has freed, so the load
// runs while this tile waits on its look-back and writes itself out.
template <int ITEMS, int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
onesweep_kernel(const uint64_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                uint64_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, int64_t n, int shift,
                uint32_t dmask, const uint32_t* __restrict__ digit_offsets, uint32_t* status, unsigned int* tile_ticket,
                int* err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmemT<ITEMS>& S = *reinterpret_cast<SortSmemT<ITEMS>*>(smem_raw);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int ntiles = static_cast<int>((n + (kThreads * ITEMS) - 1) / (kThreads * ITEMS));
    if (threadIdx.x == 0) S.tile = static_cast<int>(atomicAdd(tile_ticket, 1u));
    __syncthreads();
    int tile = S.tile;
    // Digits are re-extracted from the keys where needed: holding them (or
    // anything derived from them) across the passes costs more registers.
    uint64_t key[ITEMS];
    uint32_t val[ITEMS];
    if (tile < ntiles) load_tile(keys_in, vals_in, n, tile, w, lane, key, val);
    while (tile < ntiles) {
        const int64_t tile_base = static_cast<int64_t>(tile) * (kThreads * ITEMS);
        for (int i = threadIdx.x; i < kWarps * kRadix; i += kThreads) (&S.warp_hist[0][0])[i] = 0;
        __syncthreads();
        // Per-warp digit counts first (fire-and-forget shared adds by each digit's
        // lowest lane), so the tile's counts are published before the ranking.
        const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) {
            const int dk = static_cast<int>((key[k] >> shift) & dmask);
            const uint32_t peers = digit_peers(dk);
            S.peers[k][threadIdx.x] = peers;
            if ((peers & lt) == 0) atomicAdd(&S.warp_hist[w][dk], static_cast<uint32_t>(__popc(peers)));
        }
        __syncthreads();
        // Per digit d: exclusive prefix over warps and the tile count, published
        // at once; the first look-back window is read now and consumed after the
        // local scan and the ranking, which do not need it.
        const int d = threadIdx.x;
        uint32_t count = 0;
        for (int ww = 0; ww < kWarps; ++ww) {
            const uint32_t c = S.warp_hist[ww][d];
            S.warp_hist[ww][d] = count;
            count += c;
        }
        volatile uint32_t* vstat = status;
        if (tile == 0) vstat[d] = kFlagInc | count;
        else vstat[static_cast<int64_t>(tile) * kRadix + d] = kFlagAgg | count;
        uint32_t win[kLookWindow];
#pragma unroll
        for (int j = 0; j < kLookWindow; ++j)
            win[j] = tile - 1 - j >= 0 ? vstat[static_cast<int64_t>(tile - 1 - j) * kRadix + d]
                                       : static_cast<uint32_t>(kFlagInc);
        // Exclusive scan of the tile counts over digits: warp scans + warp totals.
        uint32_t inc = count;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += u;
        }
        if (lane == 31) S.warp_total[w] = inc;
        __syncthreads();
        uint32_t tile_start = inc - count;
        for (int ww = 0; ww < w; ++ww) tile_start += S.warp_total[ww];
        // warp_hist[w][d] becomes the first local slot of warp w's digit-d keys
        for (int ww = 0; ww < kWarps; ++ww) S.warp_hist[ww][d] += tile_start;
        __syncthreads();
        // Warp-level multisplit in item order (stable: item k of every lane
        // precedes item k+1, lanes in order within an item), scattering each key
        // to its local slot as it is ranked.
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) {
            const int dk = static_cast<int>((key[k] >> shift) & dmask);
            const uint32_t peers = S.peers[k][threadIdx.x];
            const uint32_t base = S.warp_hist[w][dk];
            const uint32_t pos = base + __popc(peers & lt);
            __syncwarp();
            if ((peers & lt) == 0) S.warp_hist[w][dk] = base + __popc(peers);
            S.keys[pos] = key[k];
            S.vals[pos] = val[k];
            __syncwarp();
        }
        // the tile is ranked in shared memory: take the next ticket and start
        // loading that tile into the registers it has freed
        if (threadIdx.x == 0) S.tile = static_cast<int>(atomicAdd(tile_ticket, 1u));
        __syncthreads();
        const int next = S.tile;
        if (next < ntiles) load_tile(keys_in, vals_in, n, next, w, lane, key, val);
        // Decoupled look-back for digit d over the earlier tiles, a window of
        // statuses per step: entries are taken in order, an entry without a
        // flag yet is re-read alone (bounded), the first inclusive one ends it.
        uint32_t excl = 0;
        if (tile > 0) {
            int pred = tile - 1;
            bool done = false, timed_out = false;
            while (!done) {
#pragma unroll
                for (int j = 0; j < kLookWindow; ++j) {
                    if (done) break;
                    uint32_t v = win[j];
                    int spins = 0;
                    while ((v & (kFlagAgg | kFlagInc)) == 0) {
                        if (++spins > kSpinLimit) { timed_out = true; break; }
                        v = vstat[static_cast<int64_t>(pred - j) * kRadix + d];
                    }
                    excl += v & kCountMask;
                    done = (v & kFlagInc) || timed_out || pred - j == 0;
                }
                if (done) break;
                pred -= kLookWindow;
#pragma unroll
                for (int j = 0; j < kLookWindow; ++j)
                    win[j] = pred - j >= 0 ? vstat[static_cast<int64_t>(pred - j) * kRadix + d]
                                           : static_cast<uint32_t>(kFlagInc);
            }
            if (timed_out) raise_error(err, kErrSort);
            vstat[static_cast<int64_t>(tile) * kRadix + d] = kFlagInc | ((excl + count) & kCountMask);
        }
        // global position of local slot i with digit d: global_delta[d] + i
        S.global_delta[d] = digit_offsets[d] + excl - tile_start;
        __syncthreads();
        const int64_t valid = n - tile_base < (kThreads * ITEMS) ? n - tile_base : (kThreads * ITEMS);
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) {
            const int i = k * kThreads + threadIdx.x;
            if (i < valid) {
                const uint64_t kk = S.keys[i];
                const int dd = static_cast<int>((kk >> shift) & dmask);
                const uint32_t gpos = S.global_delta[dd] + static_cast<uint32_t>(i);
                if (gpos >= n) { raise_error(err, kErrIndex); continue; }
                keys_out[gpos] = kk;
                vals_out[gpos] = S.vals[i];
            }
        }
        __syncthreads();          // shared memory is reused by the next tile
        tile = next;
    }
}

}  // namespace

// Pairs per tile of radix_sort_pairs for n pairs.
static int64_t tile_pairs(int64_t n) {
    return n <= NB_SORT_SMALL_N ? static_cast<int64_t>(kThreads) * kSmallItems : kTile;
}

// Scratch words for sorts of up to n pairs with either entry point: hist +
// offsets (8 x 256 each), tile tickets (8), status (8 x tiles x 256) for the
// larger of the two tile layouts any such sort can use.
size_t sort_scratch_words(int64_t n) {
    const int64_t small_n = n < NB_SORT_SMALL_N ? n : static_cast<int64_t>(NB_SORT_SMALL_N);
    const int64_t small_tile = static_cast<int64_t>(kThreads) * kSmallItems;
    const int64_t small_tiles = small_n > 0 ? (small_n + small_tile - 1) / small_tile : 0;
    const size_t small = static_cast<size_t>(2 * 8 * kRadix + 8 + 8 * small_tiles * kRadix);
    const size_t big = static_cast<size_t>(sort_scratch_words_for(n));
    return small > big ? small : big;
}

size_t sort_smem_bytes() { return sizeof(SortSmem); }

#ifndef NB_SORT_PERSISTENT
#define NB_SORT_PERSISTENT 1
#endif

// Blocks of one onesweep pass: every tile's own block, or (persistent) no
// more than fit on the device at once, each taking tiles until none is left.
template <int ITEMS, int MINB>
static unsigned onesweep_grid(int64_t tiles) {
    if (!NB_SORT_PERSISTENT) return static_cast<unsigned>(tiles);
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, onesweep_kernel<ITEMS, MINB>, kThreads,
                                                      sizeof(SortSmemT<ITEMS>)) != cudaSuccess ||
        per_sm < 1 || sms < 1)
        return static_cast<unsigned>(tiles);
    const int64_t resident = static_cast<int64_t>(per_sm) * sms;
    return static_cast<unsigned>(tiles < resident ? tiles : resident);
}

// One pass with tiles of kThreads x ITEMS pairs.
template <int ITEMS, int MINB>
static void launch_pass(int64_t n, const uint64_t* ki, const uint32_t* vi, uint64_t* ko, uint32_t* vo, int shift,
                        uint32_t dmask, const uint32_t* offs, uint32_t* status, unsigned int* ticket, int* err,
                        cudaStream_t st) {
    const int64_t tiles = (n + kThreads * ITEMS - 1) / (kThreads * ITEMS);
    onesweep_kernel<ITEMS, MINB><<<onesweep_grid<ITEMS, MINB>(tiles), kThreads, sizeof(SortSmemT<ITEMS>), st>>>(
        ki, vi, ko, vo, n, shift, dmask, offs, status, ticket, err);
}

cudaError_t sort_prepare() {
    cudaError_t e = cudaFuncSetAttribute(onesweep_kernel<kItems, NB_SORT_MINB>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(sizeof(SortSmemT<kItems>)));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(onesweep_kernel<kSmallItems, NB_SORT_SMALL_MINB>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(sizeof(SortSmemT<kSmallItems>)));
    return e;
}

// Sorts (keys, vals) of length n using (alt_keys, alt_vals) as the other
// half of the ping-pong.  The result lands in (keys, vals) when the number
// of passes is even, else in (alt_keys, alt_vals); *in_alt tells which.
// scratch holds sort_scratch_words(n) words.
cudaError_t radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* alt_keys, uint32_t* alt_vals,
                             int64_t n, int key_bits, uint32_t* scratch, int* err, bool* in_alt,
                             cudaStream_t st) {
    *in_alt = false;
    if (n <= 1) return cudaSuccess;
    const int passes = (key_bits + 7) / 8;
    const int64_t tiles = (n + tile_pairs(n) - 1) / tile_pairs(n);
    const bool small = tile_pairs(n) != kTile;
    uint32_t* hist = scratch;
    uint32_t* offsets = scratch + 8 * kRadix;
    unsigned int* tickets = scratch + 16 * kRadix;
    uint32_t* status = scratch + 16 * kRadix + 8;
    const size_t words = static_cast<size_t>(2 * 8 * kRadix + 8 + 8 * tiles * kRadix);
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(uint32_t) * words, st);
    if (e != cudaSuccess) return e;
    int hblocks = static_cast<int>((n + kThreads * 16 - 1) / (kThreads * 16));
    if (hblocks > 1184) hblocks = 1184;
    histogram_kernel<<<hblocks, kThreads, 0, st>>>(keys, n, key_bits, hist);
    digit_offsets_kernel<<<passes, kRadix, 0, st>>>(hist, offsets);
    uint64_t* src_k = keys; uint32_t* src_v = vals;
    uint64_t* dst_k = alt_keys; uint32_t* dst_v = alt_vals;
    for (int p = 0; p < passes; ++p) {
        uint32_t* pst = status + static_cast<int64_t>(p) * tiles * kRadix;
        if (small)
            launch_pass<kSmallItems, NB_SORT_SMALL_MINB>(n, src_k, src_v, dst_k, dst_v, 8 * p, pass_mask(key_bits, p),
                                                         offsets + p * kRadix, pst, tickets + p, err, st);
        else
            launch_pass<kItems, NB_SORT_MINB>(n, src_k, src_v, dst_k, dst_v, 8 * p, pass_mask(key_bits, p),
                                              offsets + p * kRadix, pst, tickets + p, err, st);
        uint64_t* tk = src_k; src_k = dst_k; dst_k = tk;
        uint32_t* tv = src_v; src_v = dst_v; dst_v = tv;
    }
    *in_alt = (passes & 1) != 0;
    count_launches(2 + passes);
    return cudaGetLastError();
}

}  // namespace nb

namespace nb {

static_assert(kSortTile == kTile, "tile size shared with the scratch-size formula");

// Sorts n pairs from (keys_in, vals_in) into (keys_out, vals_out), never
// writing the inputs: the passes alternate between the outputs and
// (alt_keys, alt_vals), starting on whichever side makes the last pass land
// in the outputs.  scratch holds sort_scratch_words(n) words, err one word.
cudaError_t radix_sort_pairs_to(const uint64_t* keys_in, const uint32_t* vals_in, uint64_t* keys_out,
                                uint32_t* vals_out, uint64_t* alt_keys, uint32_t* alt_vals, int64_t n, int key_bits,
                                uint32_t* scratch, int* err, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (n == 1) {
        cudaError_t e = cudaMemcpyAsync(keys_out, keys_in, sizeof(uint64_t), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(vals_out, vals_in, sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
        return e;
    }
    const int passes = (key_bits + 7) / 8;
    const int64_t tiles = (n + kTile - 1) / kTile;
    uint32_t* hist = scratch;
    uint32_t* offsets = scratch + 8 * kRadix;
    unsigned int* tickets = scratch + 16 * kRadix;
    uint32_t* status = scratch + 16 * kRadix + 8;
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(uint32_t) * static_cast<size_t>(sort_scratch_words_for(n)), st);
    if (e != cudaSuccess) return e;
    int hblocks = static_cast<int>((n + kThreads * 16 - 1) / (kThreads * 16));
    if (hblocks > 1184) hblocks = 1184;
    histogram_kernel<<<hblocks, kThreads, 0, st>>>(keys_in, n, key_bits, hist);
    digit_offsets_kernel<<<passes, kRadix, 0, st>>>(hist, offsets);
    const uint64_t* src_k = keys_in;
    const uint32_t* src_v = vals_in;
    for (int p = 0; p < passes; ++p) {
        const bool to_out = ((passes - 1 - p) & 1) == 0;
        uint64_t* dst_k = to_out ? keys_out : alt_keys;
        uint32_t* dst_v = to_out ? vals_out : alt_vals;
        launch_pass<kItems, NB_SORT_MINB>(n, src_k, src_v, dst_k, dst_v, 8 * p, pass_mask(key_bits, p),
                                          offsets + p * kRadix, status + static_cast<int64_t>(p) * tiles * kRadix,
                                          tickets + p, err, st);
        src_k = dst_k;
        src_v = dst_v;
    }
    count_launches(2 + passes);
    return cudaGetLastError();
}

}  // namespace nb
